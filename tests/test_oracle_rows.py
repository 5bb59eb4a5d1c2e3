"""The oracle's shared-row sweep (oracle.StateR, PT's pseudo-documents) with
one row per document is the per-document sweep, bit for bit; and with rows
shared, every row's counts stay the recount of its documents' z."""
import numpy as np

import oracle as O
import tomotopy_b200 as T


def corpus():
    off, w = T.synth_corpus(700, 9, 160, ("lognormal", float(np.log(20)), 0.7, 1, 120), seed=4)
    off, w, V, _ = T.prepare_ids(off, w)
    return off, w, V


def test_identity_rows_equal_documents():
    off, w, V = corpus()
    D = len(off) - 1
    a = O.State(O.Corpus(off, w, V), 12, 0.1, 0.01, 5)
    b = O.StateR(O.Corpus(off, w, V), 12, 0.1, 0.01, 5, np.arange(D), D)
    a.doc_live_sweeps(3, groups=3)
    b.doc_live_sweeps(3, groups=3)
    np.testing.assert_array_equal(a.z, b.z)
    np.testing.assert_array_equal(a.ndk, b.ndk)
    np.testing.assert_array_equal(a.nkw, b.nkw)
    assert a.ll_f64() == b.ll_f64()


def test_shared_rows_stay_consistent():
    off, w, V = corpus()
    D, K, R = len(off) - 1, 16, 20
    rows = np.random.default_rng(1).integers(0, R, D)
    st = O.StateR(O.Corpus(off, w, V), K, 0.1, 0.01, 6, rows, R)
    st.doc_live_sweeps(4, groups=2)
    ndk, nkw = st.ndk.copy(), st.nkw.copy()
    st.recount()
    np.testing.assert_array_equal(st.ndk, ndk)
    np.testing.assert_array_equal(st.nkw, nkw)
    assert st.ndk.sum() == st.c.N
