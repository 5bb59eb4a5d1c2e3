"""Corpus preparation on the device (tmt_prepare_corpus_device) against the
host tmt_prepare_corpus: the vocabulary order, realV, the re-numbered and
per-document sorted words, w_order, cf and df, all bit for bit."""
import ctypes as C

import numpy as np
import pytest

import tomotopy_b200 as T
from tomotopy_b200._lib import lib

pytestmark = pytest.mark.gpu


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def prepare(fn_device, off, w, nv, min_cf, min_df, rm_top):
    D = len(off) - 1
    N = len(w)
    out = np.zeros(max(N, 1), np.uint32)
    wo = np.zeros(max(N, 1), np.uint32)
    order = np.zeros(max(nv, 1), np.uint32)
    cf = np.zeros(max(nv, 1), np.uint64)
    df = np.zeros(max(nv, 1), np.uint64)
    rv = C.c_uint32()
    if fn_device:
        err = C.create_string_buffer(512)
        st = lib.tmt_prepare_corpus_device(0, D, _p(off), _p(w), nv, min_cf, min_df, rm_top, _p(out), _p(wo),
                                           _p(order), _p(cf), _p(df), C.byref(rv), err, len(err))
        assert st == 0, err.value.decode()
    else:
        st = lib.tmt_prepare_corpus(D, _p(off), _p(w), nv, min_cf, min_df, rm_top, _p(out), _p(wo), _p(order),
                                    _p(cf), _p(df), C.byref(rv))
        assert st == 0
    return out[:N], wo[:N], order[:nv], cf[:nv], df[:nv], rv.value


@pytest.mark.parametrize("seed,min_cf,min_df,rm_top", [(1, 0, 0, 0), (2, 3, 2, 5), (3, 0, 4, 0), (4, 2, 0, 10**6)])
def test_device_prepare_equals_host(seed, min_cf, min_df, rm_top):
    rng = np.random.default_rng(seed)
    D = 3000
    lens = np.concatenate([rng.integers(0, 40, D - 6), [0, 1, 31, 32, 33, 16384]])
    rng.shuffle(lens)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    nv = 5000
    # Zipf-like ids with gaps (ids that never occur) and heavy repeats within documents
    w = np.minimum(rng.zipf(1.3, int(off[-1])) - 1, nv - 1).astype(np.uint32)
    w[w % 7 == 3] = 0
    host = prepare(False, off, w, nv, min_cf, min_df, rm_top)
    dev = prepare(True, off, w, nv, min_cf, min_df, rm_top)
    for a, b in zip(host[:5], dev[:5]):
        np.testing.assert_array_equal(a, b)
    assert host[5] == dev[5]


def test_device_prepare_synthetic_corpus_and_limits():
    off, w = T.synth_corpus(20000, 50, 20000, ("lognormal", np.log(100), 1.2, 5, 5000), seed=9)
    nv = int(w.max()) + 1
    host = prepare(False, off, w, nv, 2, 0, 3)
    dev = prepare(True, off, w, nv, 2, 0, 3)
    for a, b in zip(host[:5], dev[:5]):
        np.testing.assert_array_equal(a, b)
    # a document longer than the on-chip sort is refused with a message
    off2 = np.array([0, 16385], np.uint64)
    w2 = np.zeros(16385, np.uint32)
    err = C.create_string_buffer(512)
    out = np.zeros(16385, np.uint32)
    order = np.zeros(1, np.uint32)
    rv = C.c_uint32()
    st = lib.tmt_prepare_corpus_device(0, 1, _p(off2), _p(w2), 1, 0, 0, 0, _p(out), None, _p(order), None, None,
                                       C.byref(rv), err, len(err))
    assert st != 0 and b"16384" in err.value
