"""Weighted counts (TermWeight IDF / PMI) in the oracle, on the CPU.

The device restatement folds float n_kw / n_k states from integer deltas in
units of 2^-24 between document groups; with every weight 1 that is exact
integer arithmetic, so the weighted sweep must reproduce the integer sweep's
draws bit for bit."""
import numpy as np
import pytest

import oracle as O
import tomotopy_b200 as T


def small_corpus(seed=3, V=400, D=60, mean=40):
    off, w = T.synth_corpus(V, 6, D, ("poisson", mean, 1, 10 * mean), seed=seed)
    off, w, rv, _ = T.prepare_ids(off, w, min_cf=2, rm_top=2)
    return O.Corpus(off, w, rv)


def test_fixed_point_helpers():
    assert O.lib.orc_wq(1.0) == 1 << 24
    assert O.lib.orc_wq(0.0) == 0
    # round half to even on the 2^-24 grid (2^-25 is exactly half a unit)
    assert O.lib.orc_wq(2.0 ** -25) == 0
    assert O.lib.orc_wq(3 * 2.0 ** -25) == 2
    assert O.lib.orc_fold(np.float32(2.5), -(3 << 24)) == 0.0      # clamps at 0
    assert O.lib.orc_fold(np.float32(2.5), 1 << 23) == np.float32(3.0)


@pytest.mark.parametrize("K,groups", [(1, 1), (7, 3), (20, 8), (130, 2)])
def test_unit_weights_reproduce_integer_sweep(K, groups):
    c = small_corpus(seed=K)
    st = O.State(c, K, 0.1, 0.01, 11)
    sw = O.StateW(c, K, 0.1, 0.01, 11, np.ones(len(c.words), np.float32))
    np.testing.assert_array_equal(sw.ndk, st.ndk.astype(np.float32))
    np.testing.assert_array_equal(sw.nkw, st.nkw.astype(np.float32))
    st.doc_live_sweeps(3, groups=groups)
    sw.doc_live_sweeps(3, groups=groups)
    np.testing.assert_array_equal(sw.z, st.z)
    np.testing.assert_array_equal(sw.ndk, st.ndk.astype(np.float32))
    np.testing.assert_array_equal(sw.nkw, st.nkw.astype(np.float32))
    np.testing.assert_array_equal(sw.nk, st.nk.astype(np.float32))
    a, b = sw.ll_f64()
    a2, b2 = st.ll_f64()
    assert a == pytest.approx(a2, rel=1e-13) and b == pytest.approx(b2, rel=1e-13)


def test_term_weights():
    c = small_corpus(seed=5)
    wt, vw = O.weights_idf(c)
    df = np.zeros(c.V)
    for d in range(c.D):
        ws = c.words[c.doc_off[d]:c.doc_off[d + 1]]
        df[np.unique(ws[ws < c.V])] += 1
    np.testing.assert_allclose(vw, np.log(c.D / df), rtol=1e-6)
    assert np.all(wt[c.words >= c.V] == 0)
    wp, _ = O.weights_pmi(c)
    assert np.all(wp >= 0) and np.all(wp[c.words >= c.V] == 0)
    # PMI is a per-document weight: the same word can weigh differently in two documents
    w0 = c.words[c.doc_off[0]]
    per_doc = {float(wp[i]) for d in range(c.D) for i in range(c.doc_off[d], c.doc_off[d + 1]) if c.words[i] == w0}
    assert len(per_doc) > 1


def test_weighted_counts_invariants():
    """n_dk rows sum to the document weight sums; n_k and n_kw agree after folds."""
    c = small_corpus(seed=8)
    wt, _ = O.weights_pmi(c)
    sw = O.StateW(c, 12, 0.1, 0.01, 4, wt)
    sw.doc_live_sweeps(4, groups=4)
    np.testing.assert_allclose(sw.ndk.sum(1), sw.doc_wlen[:c.D], rtol=1e-4, atol=1e-3)
    np.testing.assert_allclose(sw.nkw.sum(0), sw.nk, rtol=1e-5, atol=1e-3)
    assert np.all(sw.ndk >= 0) and np.all(sw.nkw >= 0)
