"""Per-document topic masks (the LLDA / PLDA label masks) and per-document
alphas (DMR) in the device sweep, against the oracle's restatement
(oracle.StateM): z and all counts bit for bit after every sweep, FP64 ll."""
import numpy as np
import pytest

import oracle as O
import tomotopy_b200 as T

pytestmark = pytest.mark.gpu


def corpus(seed=1, V=700, D=150, mean=50):
    off, w = T.synth_corpus(V, 8, D, ("lognormal", np.log(mean), 1.0, 1, 20 * mean), seed=seed)
    off, w, rv, _ = T.prepare_ids(off, w, min_cf=2)
    return O.Corpus(off, w, rv)


def masked_z0(c, K, mask, seed):
    """z0 inside each document's allowed topics (the caller's job, as LLDA's
    generator draws from the labelled topics)."""
    rng = np.random.default_rng(seed)
    z = np.full(len(c.words), 0xFFFF, np.uint16)
    for d in range(c.D):
        allowed = np.flatnonzero(mask[d])
        for i in range(int(c.doc_off[d]), int(c.doc_off[d + 1])):
            if c.words[i] < c.V:
                z[i] = rng.choice(allowed)
    return z


@pytest.mark.parametrize("K,groups,kind", [(8, 1, "mask"), (40, 4, "mask"), (130, 8, "alpha"), (1000, 2, "both"),
                                           (40, 3, "alpha")])
def test_masked_sweeps_bitexact(K, groups, kind):
    c = corpus(seed=K + groups)
    rng = np.random.default_rng(K)
    mask = rows = drow = None
    if kind in ("mask", "both"):
        mask = rng.random((c.D, K)) < 0.3
        mask[np.arange(c.D), rng.integers(0, K, c.D)] = True        # at least one topic per document
        mask[:5] = True                                               # some unlabelled documents
    if kind in ("alpha", "both"):
        rows = rng.uniform(0.01, 0.5, (6, K)).astype(np.float32)
        drow = rng.integers(0, 6, c.D).astype(np.uint32)
    z0 = masked_z0(c, K, mask if mask is not None else np.ones((c.D, K), bool), K)
    # with per-document alphas the optimiser must stay off even when scheduled
    eng = T.Engine(K, c.V, alpha=0.1, eta=0.01, seed=9, optim_interval=5 if rows is not None else 0,
                   sweep_groups=groups)
    eng.upload(c.doc_off, c.words, z0=z0)
    if mask is not None:
        eng.set_doc_topic_mask(mask)
    if rows is not None:
        eng.set_doc_alpha(rows, drow)
    st = O.StateM(c, K, 0.1, 0.01, 9, z0, mask=mask, alpha_rows=rows, doc_row=drow)
    step = 0
    for n in (1, 2, 4):
        eng.train(n)
        st.doc_live_sweeps(n, start_step=step, groups=groups)
        step += n
        z, nkw, nk, alpha = eng.state()
        np.testing.assert_array_equal(z, st.z)
        np.testing.assert_array_equal(nkw, st.nkw)
        np.testing.assert_array_equal(nk, st.nk)
        np.testing.assert_array_equal(eng.doc_topic(), st.ndk)
    if mask is not None:          # no token left its document's labels
        for d in range(c.D):
            zz = st.z[int(c.doc_off[d]):int(c.doc_off[d + 1])]
            zz = zz[zz != 0xFFFF]
            assert np.all(mask[d][zz])
    if rows is not None:          # the optimiser leaves alpha alone when documents carry their own
        np.testing.assert_array_equal(alpha, np.full(K, 0.1, np.float32))
    ld, lr = eng.ll()
    od, orr = st.ll_f64()
    assert ld == pytest.approx(od, rel=1e-11, abs=1e-7)
    assert lr == pytest.approx(orr, rel=1e-11, abs=1e-7)


def test_mask_and_alpha_validation():
    c = corpus(seed=2)
    eng = T.Engine(6, c.V, alpha=0.1, eta=0.01, seed=1)
    with pytest.raises(Exception):
        eng.set_doc_alpha(np.ones((1, 6), np.float32), np.zeros(c.D, np.uint32))   # before the upload
    eng.upload(c.doc_off, c.words)
    with pytest.raises(ValueError):
        eng.set_doc_alpha(np.zeros((1, 6), np.float32), np.zeros(c.D, np.uint32))  # alpha must be > 0
    with pytest.raises(ValueError):
        eng.set_doc_alpha(np.ones((2, 6), np.float32), np.full(c.D, 2, np.uint32))  # row out of range
    eng.set_doc_topic_mask(np.ones((c.D, 6), bool))
    eng.set_doc_topic_mask(None)
    eng.train(2)
