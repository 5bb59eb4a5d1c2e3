"""Weighted counts (TermWeight IDF / PMI) on the device, through the C ABI,
against the oracle's restatement of the same semantics (oracle.StateW)."""
import numpy as np
import pytest

import oracle as O
import tomotopy_b200 as T
from tomotopy_b200._lib import TmtError

pytestmark = pytest.mark.gpu


def corpus(seed=1, V=700, D=130, mean=55):
    off, w = T.synth_corpus(V, 8, D, ("lognormal", np.log(mean), 1.0, 1, 20 * mean), seed=seed)
    off, w, rv, _ = T.prepare_ids(off, w, min_cf=2, rm_top=3)
    return O.Corpus(off, w, rv)


def weights(c, kind):
    if kind == "idf":
        return O.weights_idf(c)[0]
    if kind == "pmi":
        return O.weights_pmi(c)[0]
    return np.ones(len(c.words), np.float32)


def assert_same(eng, sw):
    z, nkw, nk, _ = eng.state()
    np.testing.assert_array_equal(z, sw.z)
    np.testing.assert_array_equal(eng.doc_topic(), sw.ndk)
    np.testing.assert_array_equal(nkw, sw.nkw)
    np.testing.assert_array_equal(nk, sw.nk)
    np.testing.assert_array_equal(eng.doc_weight_sums(), sw.doc_wlen[:sw.c.D])


@pytest.mark.parametrize("kind,K,groups", [("idf", 1, 1), ("idf", 7, 3), ("pmi", 20, 8), ("idf", 100, 8),
                                           ("pmi", 1000, 2), ("idf", 1100, 1)])
def test_weighted_sweeps_bitexact(kind, K, groups):
    """z, float n_dk / n_kw / n_k and the document weight sums equal the
    oracle's after the upload and after every train() call (the first sweeps
    run eagerly for the autotuner, the later ones as graph launches)."""
    c = corpus(seed=K)
    wt = weights(c, kind)
    alpha = np.float32(0.1) if K != 20 else (0.05 * (np.arange(K) + 1)).astype(np.float32)
    eng = T.Engine(K, c.V, alpha=alpha, eta=0.01, seed=7, optim_interval=0, sweep_groups=groups)
    eng.upload(c.doc_off, c.words, weights=wt)
    sw = O.StateW(c, K, alpha, 0.01, 7, wt)
    assert_same(eng, sw)
    step = 0
    for n in (1, 2, 3):
        eng.train(n)
        sw.doc_live_sweeps(n, start_step=step, groups=groups)
        step += n
        assert_same(eng, sw)


def test_unit_weights_equal_integer_counts():
    """With every weight 1 the weighted sweep is the integer sweep -- the
    integer sweep with long documents sampled in order, as weighted counts
    always are (splitting applies to integer counts only)."""
    c = corpus(seed=4)
    a = T.Engine(40, c.V, alpha=0.1, eta=0.01, seed=3, optim_interval=0)
    a.set_doc_split(2 ** 32 - 1)
    a.upload(c.doc_off, c.words)
    b = T.Engine(40, c.V, alpha=0.1, eta=0.01, seed=3, optim_interval=0)
    b.upload(c.doc_off, c.words, weights=np.ones(len(c.words), np.float32))
    a.train(5)
    b.train(5)
    za, nkwa, nka, _ = a.state()
    zb, nkwb, nkb, _ = b.state()
    np.testing.assert_array_equal(za, zb)
    np.testing.assert_array_equal(nkwa.astype(np.float32), nkwb)
    np.testing.assert_array_equal(a.doc_topic().astype(np.float32), b.doc_topic())


@pytest.mark.parametrize("kind", ["idf", "pmi"])
def test_weighted_ll_and_alpha_match_oracle(kind):
    c = corpus(seed=9)
    wt = weights(c, kind)
    K = 24
    eng = T.Engine(K, c.V, alpha=0.1, eta=0.01, seed=5, optim_interval=1)
    eng.upload(c.doc_off, c.words, weights=wt)
    sw = O.StateW(c, K, 0.1, 0.01, 5, wt)
    ld, lr = eng.ll()
    od, orr = sw.ll_f64()
    assert ld == pytest.approx(od, rel=1e-11, abs=1e-7)
    assert lr == pytest.approx(orr, rel=1e-11, abs=1e-7)
    for step in range(3):
        eng.train(1)
        sw.doc_live_sweeps(1, start_step=step, groups=8)
        sw.optimize_alpha()
        a_dev = eng.state()[3]
        np.testing.assert_allclose(a_dev, sw.alpha, rtol=2e-4)
        sw.alpha[:] = a_dev
        if not np.array_equal(eng.state()[0], sw.z):
            break
    ld, lr = eng.ll()
    od, orr = sw.ll_f64()
    assert (ld + lr) == pytest.approx(od + orr, rel=1e-6)


def test_weighted_rejects_bad_input_and_integer_reads():
    c = corpus(seed=2)
    eng = T.Engine(10, c.V, alpha=0.1, eta=0.01, seed=1)
    for bad in (-1.0, np.nan, np.inf, 1e6):
        wt = np.ones(len(c.words), np.float32)
        wt[np.flatnonzero(c.words < c.V)[3]] = bad
        with pytest.raises(ValueError):
            eng.upload(c.doc_off, c.words, weights=wt)
    eng.upload(c.doc_off, c.words, weights=np.full(len(c.words), 0.5, np.float32))
    from tomotopy_b200._lib import lib
    import ctypes as C
    nk = np.zeros(10, np.int32)
    assert lib.tmt_download_state(eng.h, None, None, nk.ctypes.data_as(C.c_void_p), None) != 0
    with pytest.raises(TmtError):
        eng.infer(c.doc_off[:3], c.words[:int(c.doc_off[2])], iters=5)
    # an integer-count corpus refuses the float reads
    e2 = T.Engine(10, c.V, alpha=0.1, eta=0.01, seed=1)
    e2.upload(c.doc_off, c.words)
    assert lib.tmt_download_counts_f32(e2.h, None, None, nk.ctypes.data_as(C.c_void_p), None) != 0


def _pmi_weights_of(words_sorted, V, vw):
    """PMI weights of one new document's tokens (sorted ids), as the host model
    computes them: max((float)log((float)tf / vw / len), 0)."""
    m = words_sorted < V
    tf = np.bincount(words_sorted[m].astype(np.int64), minlength=V)
    out = np.zeros(len(words_sorted), np.float32)
    q = (tf[words_sorted[m]].astype(np.float32) / vw[words_sorted[m]]) / np.float32(len(words_sorted))
    out[m] = np.maximum(np.log(q.astype(np.float64)).astype(np.float32), np.float32(0))
    return out


@pytest.mark.parametrize("kind,K", [("idf", 7), ("pmi", 20), ("idf", 100), ("pmi", 300), ("idf", 1000)])
def test_weighted_infer_matches_oracle(kind, K):
    """tmt_infer_batch_weighted: theta and z-driven FP64 ll equal the oracle's
    weighted per-document infer (theta bit-exact, ll to 1e-12)."""
    c = corpus(seed=K + 1)
    wt, vw = O.weights_idf(c) if kind == "idf" else O.weights_pmi(c)
    eng = T.Engine(K, c.V, alpha=0.1, eta=0.01, seed=3, optim_interval=0)
    eng.upload(c.doc_off, c.words, weights=wt)
    eng.train(15)
    _, nkw, nk, alpha = eng.state()
    off, w = T.synth_corpus(c.V + 20, 8, 40, ("lognormal", np.log(50), 1.0, 1, 500), seed=77)
    w = w.astype(np.uint32)
    ws = np.zeros(len(w), np.float32)
    docs = []
    for d in range(len(off) - 1):
        doc = np.sort(w[off[d]:off[d + 1]], kind="stable")
        if kind == "idf":
            dw = np.where(doc < c.V, vw[np.minimum(doc, c.V - 1)], 0).astype(np.float32)
        else:
            dw = _pmi_weights_of(doc, c.V, vw)
        w[off[d]:off[d + 1]] = doc
        ws[off[d]:off[d + 1]] = dw
        docs.append((doc, dw))
    theta, ll = eng.infer(off, w, iters=25, seed=9, weights=ws)
    for d, (doc, dw) in enumerate(docs):
        ol, _, _, ot = O.infer_doc_w(K, c.V, alpha, 0.01, nkw, nk, doc, dw, 25, 9, 0)
        np.testing.assert_array_equal(theta[d], ot)
        assert ll[d] == pytest.approx(ol, rel=1e-12, abs=1e-9)
    # a word whose tokens carry different weights in one document is rejected
    bad = ws.copy()
    d0 = next(d for d, (doc, _) in enumerate(docs) if len(doc) > 1 and doc[0] == doc[1] and doc[0] < c.V)
    bad[off[d0]] += 0.5
    with pytest.raises(ValueError):
        eng.infer(off, w, iters=5, seed=9, weights=bad)


@pytest.mark.parametrize("tw", ["idf", "pmi"])
def test_weighted_model_api(tw, tmp_path):
    """tomotopy's LDAModel(tw=IDF|PMI): train, save / load (tomotopy's layout
    with float counts and per-document word weights), continued training
    identical to the original's, infer and infer together."""
    import tomotopy_b200 as tp
    off, w = T.synth_corpus(1200, 10, 150, ("poisson", 70, 1, 700), seed=12)
    docs = [[f"w{x}" for x in w[off[d]:off[d + 1]]] for d in range(150)]
    mdl = tp.LDAModel(tw=tw, k=16, seed=5, min_cf=2)
    for d in docs:
        mdl.add_doc(d)
    mdl.train(40)
    assert mdl.tw == (tp.TermWeight.IDF if tw == "idf" else tp.TermWeight.PMI)
    ll0 = mdl.ll_per_word
    assert np.isfinite(ll0)
    assert mdl.get_count_by_topics().sum() == mdl.num_words       # token counts, not weights
    dist = mdl.get_topic_word_dist(2)
    assert abs(dist.sum() - 1) < 1e-3
    path = str(tmp_path / "w.bin")
    mdl.save(path)
    m2 = tp.LDAModel.load(path)
    assert m2.tw == mdl.tw
    np.testing.assert_array_equal(m2.docs[4].topics, mdl.docs[4].topics)
    assert m2.get_topic_words(3) == mdl.get_topic_words(3)
    np.testing.assert_allclose(m2.get_topic_word_dist(3), mdl.get_topic_word_dist(3), rtol=0, atol=0)
    # the loaded model divides its ll by the weight sum, as tomotopy's load does
    # (n_dk is recounted from Zs and weights on load, so its float sums may
    # differ from the trained rows in the last bits)
    assert m2.ll_per_word * m2._info().weighted_n == pytest.approx(ll0 * mdl.num_words, rel=1e-6)
    # inference reads only the frozen model: the loaded copy infers identically
    unseen = [mdl.make_doc(d) for d in docs[:6]]
    dists, lls = mdl.infer(unseen, iterations=20)
    for t in dists:
        assert abs(t.sum() - 1) < 1e-4
    t1, l1 = m2.infer(m2.make_doc(docs[2]), iterations=20)
    np.testing.assert_array_equal(t1, dists[2])
    assert l1 == lls[2]
    dists2, ll2 = mdl.infer(unseen, iterations=20, together=True)
    assert np.isfinite(ll2) and all(abs(t.sum() - 1) < 1e-4 for t in dists2)
    assert tp.LDAModel.loads(mdl.saves(full=False)).tw == mdl.tw
    m2.train(10)
    mdl.train(10)
    assert m2.global_step == mdl.global_step == 50
    assert m2.ll_per_word * m2._info().weighted_n == pytest.approx(mdl.ll_per_word * mdl.num_words, rel=0.02)


@pytest.mark.parametrize("kind", ["idf", "pmi"])
def test_weighted_ll_per_word_matches_reference_sampler(kind):
    """(d) for weighted counts: at the same iteration count the device's
    ll_per_word is within 1% of tomotopy's sequential sampler with the same
    weights (live float counts, clamped decrements), averaged over 5 seeds."""
    off, w = T.synth_corpus(5000, 20, 400, ("poisson", 500, 1, 10000), seed=21)
    off, w, Vr, _ = T.prepare_ids(off, w)
    c = O.Corpus(off, w, Vr)
    wt = weights(c, kind)
    K, iters = 20, 150
    gpu, ref = [], []
    for seed in (1, 2, 3, 4, 5):
        eng = T.Engine(K, Vr, alpha=0.1, eta=0.01, seed=seed, optim_interval=0)
        eng.upload(off, w, weights=wt)
        eng.train(iters)
        gpu.append(sum(eng.ll()) / c.N)
        st = O.StateW(c, K, 0.1, 0.01, seed, wt)
        st.gibbs_none(iters, seed)
        ref.append(sum(st.ll_f64()) / c.N)
    g, r = np.mean(gpu), np.mean(ref)
    assert abs(g - r) / abs(r) < 0.01, (gpu, ref)
