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


def test_unit_weight_infer_equals_integer_infer():
    """The weighted inference restatement with every weight 1 and the model's
    counts as floats reproduces the integer restatement exactly."""
    c = small_corpus(seed=12)
    K = 9
    st = O.State(c, K, 0.1, 0.01, 3)
    st.doc_live_sweeps(4, groups=2)
    rng = np.random.default_rng(2)
    for _ in range(5):
        doc = np.sort(rng.integers(0, c.V + 3, 40).astype(np.uint32))
        ll, z, ndk, th = O.infer_doc(K, c.V, st.alpha, 0.01, st.nkw, st.nk, doc, 15, 7, 3)
        llw, zw, ndkw, thw = O.infer_doc_w(K, c.V, st.alpha, 0.01, st.nkw.astype(np.float32),
                                           st.nk.astype(np.float32), doc, np.ones(len(doc), np.float32), 15, 7, 3)
        np.testing.assert_array_equal(z, zw)
        np.testing.assert_array_equal(th, thw)
        np.testing.assert_array_equal(ndk.astype(np.float32), ndkw)
        assert ll == pytest.approx(llw, rel=1e-13)


def test_open_masks_and_global_alpha_rows_equal_plain_sweep():
    """Masks allowing every topic and per-document alpha rows equal to the
    model's alpha reproduce the plain doc-major sweep exactly."""
    c = small_corpus(seed=13)
    K = 11
    a = (0.05 * (1 + np.arange(K) % 3)).astype(np.float32)
    st = O.State(c, K, a, 0.01, 5)
    sm = O.StateM(c, K, a, 0.01, 5, st.z.copy(), mask=np.ones((c.D, K), bool),
                  alpha_rows=a[None, :].copy(), doc_row=np.zeros(c.D, np.uint32))
    st.doc_live_sweeps(3, groups=3)
    sm.doc_live_sweeps(3, groups=3)
    np.testing.assert_array_equal(st.z, sm.z)
    np.testing.assert_array_equal(st.nkw, sm.nkw)
    a1, _ = st.ll_f64()
    a2, _ = sm.ll_f64()
    assert a1 == pytest.approx(a2, rel=1e-12)
