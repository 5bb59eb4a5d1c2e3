"""The C-ABI library loads, exports every entry point include/*.h declares,
and its host-only functions (corpus preparation, synthetic corpus) agree
with the oracle.  No compute calls that need a GPU."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

import oracle as O
import tomotopy_b200 as T
from tomotopy_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(tmt_[a-z0-9_]+)\s*\(", txt):
            syms.add(m.group(1))
    return syms


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 10
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert declared_symbols() <= set(_lib.SIGNATURES) | {"tmt_status"}


def test_create_rejects_bad_arguments_without_gpu():
    # argument validation happens before any CUDA call (LDAModel ctor checks)
    for kw in [dict(K=0), dict(K=40000), dict(eta=0.0), dict(eta=-1.0), dict(alpha=0.0), dict(alpha=-0.1)]:
        args = dict(K=10, V=100, alpha=0.1, eta=0.01)
        args.update(kw)
        with pytest.raises(ValueError):
            T.Engine(**args)


def _oracle_prepare(doc_off, words, min_cf, min_df, rm_top):
    nv = int(words.max()) + 1
    cf = np.bincount(words, minlength=nv).astype(np.uint64)
    df = np.zeros(nv, np.uint64)
    for d in range(len(doc_off) - 1):
        df[np.unique(words[doc_off[d]:doc_off[d + 1]])] += 1
    order = np.zeros(nv, np.uint32)
    rv = O.lib.orc_remove_stopwords(nv, O._ptr(cf), O._ptr(df), min_cf, min_df, rm_top, O._ptr(order))
    w2 = order[words]
    for d in range(len(doc_off) - 1):
        b, e = int(doc_off[d]), int(doc_off[d + 1])
        seg = w2[b:e].copy()
        o = np.zeros(e - b, np.uint32)
        O.lib.orc_sort_doc(O._ptr(seg), e - b, O._ptr(o))
        w2[b:e] = seg
    return w2, rv, order


@pytest.mark.parametrize("min_cf,min_df,rm_top", [(0, 0, 0), (3, 0, 0), (0, 4, 0), (2, 2, 5), (0, 0, 50)])
def test_prepare_corpus_matches_oracle(min_cf, min_df, rm_top):
    off, w = T.synth_corpus(2000, 10, 200, ("poisson", 60, 1, 500), seed=3)
    off2, w2, rv, order = T.prepare_ids(off, w, min_cf, min_df, rm_top)
    ow, orv, oorder = _oracle_prepare(off, w, min_cf, min_df, rm_top)
    assert rv == orv
    np.testing.assert_array_equal(order, oorder)
    np.testing.assert_array_equal(w2, ow)


def test_synth_corpus_deterministic_across_threads():
    a = T.synth_corpus(3000, 20, 300, ("lognormal", np.log(50), 0.8, 5, 400), seed=11, threads=1)
    b = T.synth_corpus(3000, 20, 300, ("lognormal", np.log(50), 0.8, 5, 400), seed=11, threads=7)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    lens = np.diff(a[0].astype(np.int64))
    assert lens.min() >= 5 and lens.max() <= 400
    c = T.synth_corpus(3000, 20, 300, ("lognormal", np.log(50), 0.8, 5, 400), seed=12)
    assert not np.array_equal(a[1][:1000], c[1][:1000])


def test_synth_poisson_mean():
    off, w = T.synth_corpus(1000, 5, 2000, ("poisson", 150, 1, 10000), seed=5)
    lens = np.diff(off.astype(np.int64))
    assert abs(lens.mean() - 150) < 2.0
    assert abs(lens.var() - 150) < 25


def test_sparse_sampler_is_refused():
    """TMT_SAMPLER_SPARSE is not built: tmt_create says so (TMT_ERR_UNSUPPORTED)
    before touching a GPU, instead of running the dense sampler under that name."""
    lib = _lib.lib
    alpha = np.full(8, 0.1, np.float32)
    cfg = _lib.TmtConfig(K=8, V=100, alpha=alpha.ctypes.data_as(C.POINTER(C.c_float)), alpha_scalar=0.1, eta=0.01,
                      seed=1, optim_interval=0, burn_in=0, device=0, sampler=_lib.SAMPLER_SPARSE, hbm_budget=0,
                      sweep_groups=0)
    h = _lib._H()
    st = lib.tmt_create(C.byref(cfg), C.byref(h))
    try:
        assert st == -5
        assert b"sparse" in lib.tmt_last_error(h)
    finally:
        lib.tmt_destroy(h)


@pytest.mark.parametrize("length", [("poisson", 150, 1, 10000), ("lognormal", float(np.log(100)), 1.2, 5, 5000)])
def test_oracle_workload_equals_product_workload(length):
    """The CPU baseline builds the benchmark corpus without the engine
    (oracle.synth_corpus / oracle.prepare_ids); it must be the corpus the GPU
    arm samples, id for id."""
    a_off, a_w = T.synth_corpus(5000, 40, 700, length, seed=20261206, threads=3)
    b_off, b_w = O.synth_corpus(5000, 40, 700, length, seed=20261206, threads=5)
    np.testing.assert_array_equal(a_off, b_off)
    np.testing.assert_array_equal(a_w, b_w)
    pa = T.prepare_ids(a_off, a_w)
    pb = O.prepare_ids(b_off, b_w, threads=4)
    assert pa[2] == pb[2]
    np.testing.assert_array_equal(pa[1], pb[1])
    np.testing.assert_array_equal(pa[3], pb[3])
