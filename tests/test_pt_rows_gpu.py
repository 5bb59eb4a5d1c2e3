"""The PT conditional (PTModel.hpp:13-24, 72-114, 206-235): documents share the
n_dk row of their pseudo-document.  After tmt_set_doc_rows every sweep's z, the
R shared rows, n_kw and n_k equal the oracle's restatement (oracle.StateR) bit
for bit; the log-likelihood and the alpha optimiser run over the rows; the
pseudo-documents can be re-assigned between sweeps (the rows are recounted
from z) and the shared rows cleared again."""
import numpy as np
import pytest

import oracle as O
import tomotopy_b200 as T
from tomotopy_b200._lib import TmtError

pytestmark = pytest.mark.gpu


def short_texts(D=700, V=1200, seed=31):
    """Short documents, the model's use case (lognormal(ln 14, 0.6) tokens)."""
    off, w = T.synth_corpus(V, 15, D, ("lognormal", float(np.log(14)), 0.6, 1, 80), seed=seed)
    off, w, V, _ = T.prepare_ids(off, w)
    return off, w, V


def assert_same(eng, st):
    z, nkw, nk, _ = eng.state()
    np.testing.assert_array_equal(z, st.z)
    np.testing.assert_array_equal(nk, st.nk)
    np.testing.assert_array_equal(nkw, st.nkw)
    np.testing.assert_array_equal(eng.doc_topic(), st.ndk)


@pytest.mark.parametrize("K,R,groups", [(10, 60, 1), (64, 90, 4), (300, 25, 2)])
def test_shared_rows_bitexact(K, R, groups):
    off, w, V = short_texts(seed=K)
    D = len(off) - 1
    rng = np.random.default_rng(K)
    rows = rng.integers(0, R, D).astype(np.uint32)
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=3, optim_interval=0, sweep_groups=groups)
    eng.upload(off, w)
    eng.set_doc_rows(rows, R)
    st = O.StateR(O.Corpus(off, w, V), K, 0.1, 0.01, 3, rows, R)
    assert_same(eng, st)
    step = 0
    for n in (1, 2, 2, 4):          # the tuner's sweeps (every variant) and graph sweeps after them
        eng.train(n)
        st.doc_live_sweeps(n, start_step=step, groups=groups)
        step += n
        assert_same(eng, st)
    ld, lr = eng.ll()
    od, orr = st.ll_f64()
    assert ld == pytest.approx(od, rel=1e-11) and lr == pytest.approx(orr, rel=1e-11)


def test_reassign_then_clear_rows():
    off, w, V = short_texts(seed=5)
    D, K = len(off) - 1, 40
    rng = np.random.default_rng(9)
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=4, optim_interval=0, sweep_groups=3)
    eng.upload(off, w)
    r1 = rng.integers(0, 50, D).astype(np.uint32)
    eng.set_doc_rows(r1, 50)
    st = O.StateR(O.Corpus(off, w, V), K, 0.1, 0.01, 4, r1, 50)
    eng.train(3)
    st.doc_live_sweeps(3, groups=3)
    assert_same(eng, st)
    # samplePseudoDoc moves documents between pseudo-documents (here: at random)
    r2 = rng.integers(0, 35, D).astype(np.uint32)
    eng.set_doc_rows(r2, 35)
    st.set_rows(r2, 35)
    assert_same(eng, st)
    eng.train(2)
    st.doc_live_sweeps(2, start_step=3, groups=3)
    assert_same(eng, st)
    # back to one row per document: the rows are recounted from z
    eng.set_doc_rows(None)
    plain = O.State(O.Corpus(off, w, V), K, 0.1, 0.01, 4, z0=st.z)
    np.testing.assert_array_equal(eng.doc_topic(), plain.ndk)
    eng.train(2)
    plain.doc_live_sweeps(2, start_step=5, groups=3)
    assert_same(eng, plain)


def test_rows_alpha_optimisation():
    """PTModel::optimizeParameters runs Minka's update over the pseudo-document
    rows; the device's alpha stays within 2e-4 of the oracle's."""
    off, w, V = short_texts(seed=8)
    D, K = len(off) - 1, 24
    rows = np.random.default_rng(2).integers(0, 70, D).astype(np.uint32)
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=6, optim_interval=0)
    eng.upload(off, w)
    eng.set_doc_rows(rows, 70)
    st = O.StateR(O.Corpus(off, w, V), K, 0.1, 0.01, 6, rows, 70)
    eng.train(2)
    st.doc_live_sweeps(2, groups=8)
    assert_same(eng, st)
    from tomotopy_b200._lib import lib
    from tomotopy_b200.engine import check
    check(lib.tmt_set_optim(eng.h, 1, 0), eng.h)
    eng.train(1)                     # one sweep, then the optimiser (optim_interval 1)
    st.doc_live_sweeps(1, start_step=2, groups=8)
    st.optimize_alpha()
    np.testing.assert_allclose(eng.state()[3], st.alpha, rtol=2e-4)


def test_rows_refuse_masks_and_bad_rows():
    off, w, V = short_texts(seed=12)
    D, K = len(off) - 1, 8
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=1, optim_interval=0)
    eng.upload(off, w)
    with pytest.raises((ValueError, TmtError)):
        eng.set_doc_rows(np.full(D, 5, np.uint32), 5)          # row 5 >= R
    eng.set_doc_rows(np.zeros(D, np.uint32), 1)
    with pytest.raises(TmtError):
        eng.set_doc_topic_mask(np.ones((D, K), bool))
