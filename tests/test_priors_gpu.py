"""Word priors (tomotopy's set_word_prior / etaByTopicWord) on the device,
through the C ABI, against the oracle's restatement (oracle.StateP): z0 from
the words' eta columns, every sweep's z and counts bit for bit, FP64 ll, and
per-document inference."""
import numpy as np
import pytest

import oracle as O
import tomotopy_b200 as T
from tomotopy_b200._lib import TmtError

pytestmark = pytest.mark.gpu


def corpus(seed=1, V=800, D=140, mean=60):
    off, w = T.synth_corpus(V, 8, D, ("lognormal", np.log(mean), 1.0, 1, 20 * mean), seed=seed)
    off, w, rv, _ = T.prepare_ids(off, w, min_cf=2, rm_top=2)
    return O.Corpus(off, w, rv)


def priors_for(c, K, seed):
    """A handful of words with priors: one pinned to a topic, one spread over
    two topics, one with a zero-free but uneven column."""
    rng = np.random.default_rng(seed)
    ids = rng.choice(np.arange(min(c.V, 200)), size=5, replace=False).astype(np.uint32)
    pr = np.zeros((len(ids), K), np.float32)
    pr[0, 0] = 1.0
    pr[1, min(1, K - 1)] = 0.5
    pr[1, K - 1] = 0.5
    pr[2] = rng.uniform(0.001, 0.2, K).astype(np.float32)
    pr[3] = 0.01
    pr[4, K // 2] = 2.0
    return ids, pr


@pytest.mark.parametrize("K,groups", [(5, 1), (20, 3), (100, 8), (1000, 2)])
def test_prior_sweeps_bitexact(K, groups):
    c = corpus(seed=K)
    ids, pr = priors_for(c, K, K)
    eng = T.Engine(K, c.V, alpha=0.1, eta=0.01, seed=11, optim_interval=0, sweep_groups=groups)
    eng.set_word_priors(ids, pr)
    eng.upload(c.doc_off, c.words)
    st = O.StateP(c, K, 0.1, 0.01, 11, ids, pr)

    def same():
        z, nkw, nk, _ = eng.state()
        np.testing.assert_array_equal(z, st.z)
        np.testing.assert_array_equal(nkw, st.nkw)
        np.testing.assert_array_equal(nk, st.nk)
        np.testing.assert_array_equal(eng.doc_topic(), st.ndk)

    same()
    step = 0
    for n in (1, 2, 3):
        eng.train(n)
        st.doc_live_sweeps(n, start_step=step, groups=groups)
        step += n
        same()
    # the pinned word never leaves its topic
    assert np.all(st.z[c.words == ids[0]] == 0)
    ld, lr = eng.ll()
    od, orr = st.ll_f64()
    assert ld == pytest.approx(od, rel=1e-11, abs=1e-7)
    assert lr == pytest.approx(orr, rel=1e-11, abs=1e-7)


@pytest.mark.parametrize("K", [7, 100, 300])
def test_prior_infer_matches_oracle(K):
    c = corpus(seed=K + 3)
    ids, pr = priors_for(c, K, K + 1)
    eng = T.Engine(K, c.V, alpha=0.1, eta=0.01, seed=2, optim_interval=0)
    eng.set_word_priors(ids, pr)
    eng.upload(c.doc_off, c.words)
    eng.train(12)
    st = O.StateP(c, K, 0.1, 0.01, 2, ids, pr)
    _, nkw, nk, alpha = eng.state()
    off, w = T.synth_corpus(c.V + 10, 8, 30, ("lognormal", np.log(40), 1.0, 1, 400), seed=31)
    w = w.astype(np.uint32)
    theta, ll = eng.infer(off, w, iters=20, seed=4)
    for d in range(len(off) - 1):
        doc = np.sort(w[off[d]:off[d + 1]], kind="stable")
        ol, _, _, ot = st.infer_doc(nkw, nk, alpha, doc, 20, 4, 0)
        np.testing.assert_array_equal(theta[d], ot)
        assert ll[d] == pytest.approx(ol, rel=1e-12, abs=1e-9)


def test_prior_validation():
    c = corpus(seed=5)
    eng = T.Engine(6, c.V, alpha=0.1, eta=0.01, seed=1)
    with pytest.raises(ValueError):
        eng.set_word_priors([c.V], np.ones((1, 6), np.float32))          # id out of range
    with pytest.raises(ValueError):
        eng.set_word_priors([3, 3], np.ones((2, 6), np.float32))         # twice
    bad = np.ones((1, 6), np.float32)
    bad[0, 2] = -0.1
    with pytest.raises(ValueError):
        eng.set_word_priors([3], bad)
    eng.set_word_priors([3], np.ones((1, 6), np.float32))
    eng.upload(c.doc_off, c.words)
    with pytest.raises(TmtError):
        eng.set_word_priors([4], np.ones((1, 6), np.float32))            # after the upload


def test_word_prior_model_api(tmp_path):
    """tomotopy's set_word_prior / get_word_prior on the LDAModel object: a word
    pinned to topic 0 never leaves it, a dict prior keeps eta for the other
    topics, the priors travel in the file (etaByWord), and a loaded model
    continues training exactly as the original."""
    import tomotopy_b200 as tp
    off, w = T.synth_corpus(900, 8, 120, ("poisson", 60, 1, 600), seed=21)
    docs = [[f"w{x}" for x in w[off[d]:off[d + 1]]] for d in range(120)]
    K = 10
    mdl = tp.LDAModel(k=K, seed=3, eta=0.02)
    for d in docs:
        mdl.add_doc(d)
    pin = [0.0] * K
    pin[0] = 1.0
    mdl.set_word_prior("w1", pin)
    mdl.set_word_prior("w2", {3: 0.5, 4: 0.5})
    mdl.set_word_prior("w1", [1.0] * K)            # ignored: the first prior of a word stays
    assert mdl.get_word_prior("w1") == pin
    assert mdl.get_word_prior("w2")[3] == 0.5 and mdl.get_word_prior("w2")[0] == pytest.approx(0.02)
    assert mdl.get_word_prior("w3") == []
    with pytest.raises(ValueError):
        mdl.set_word_prior("w4", [0.1] * (K - 1))
    with pytest.raises(ValueError):
        mdl.set_word_prior("w4", [-0.1] * K)
    mdl.train(30)
    with pytest.raises(RuntimeError):
        mdl.set_word_prior("w5", pin)
    assert mdl.get_word_prior("w3") == pytest.approx([0.02] * K)   # prepared: eta column
    w1 = mdl.vocabs.index("w1")
    for d in mdl.docs:
        for word, t in zip(d.words, d.topics):
            if word == w1:
                assert t == 0
    path = str(tmp_path / "p.bin")
    mdl.save(path)
    m2 = tp.LDAModel.load(path)
    assert m2.get_word_prior("w1") == pin
    assert m2.ll_per_word == pytest.approx(mdl.ll_per_word, rel=1e-12)
    m2.train(10)
    mdl.train(10)
    np.testing.assert_array_equal(m2.docs[5].topics, mdl.docs[5].topics)
    t, _ = mdl.infer(mdl.make_doc(["w1", "w1", "w2", "w7"]), iterations=20)
    assert abs(t.sum() - 1) < 1e-4
    ts, ll = mdl.infer([mdl.make_doc(["w1", "w1", "w2", "w7"]), mdl.make_doc(["w1", "w3"])], iterations=20,
                       together=True)
    assert np.isfinite(ll) and all(abs(x.sum() - 1) < 1e-4 for x in ts)


def test_prior_ll_per_word_matches_reference_sampler():
    """(d) with word priors: the device's ll_per_word within 1% of tomotopy's
    sequential sampler with the same etaByTopicWord, averaged over 5 seeds."""
    off, w = T.synth_corpus(5000, 20, 400, ("poisson", 500, 1, 10000), seed=22)
    off, w, Vr, _ = T.prepare_ids(off, w)
    c = O.Corpus(off, w, Vr)
    K, iters = 20, 150
    ids = np.arange(0, 40, 2, dtype=np.uint32)                 # 20 frequent words, one pinned per topic
    pr = np.full((len(ids), K), 0.0, np.float32)
    pr[np.arange(len(ids)), np.arange(len(ids)) % K] = 1.0
    gpu, ref = [], []
    for seed in (1, 2, 3, 4, 5):
        eng = T.Engine(K, Vr, alpha=0.1, eta=0.01, seed=seed, optim_interval=0)
        eng.set_word_priors(ids, pr)
        eng.upload(off, w)
        eng.train(iters)
        gpu.append(eng.ll_per_word())
        st = O.StateP(c, K, 0.1, 0.01, seed, ids, pr)
        st.gibbs_none(iters, seed)
        ref.append(sum(st.ll_f64()) / c.N)
    g, r = np.mean(gpu), np.mean(ref)
    assert abs(g - r) / abs(r) < 0.01, (gpu, ref)
