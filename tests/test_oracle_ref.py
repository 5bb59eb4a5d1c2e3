"""Pins the oracle's restatements against tomotopy's own numeric primitives:
bit-exact against tests/golden/ref_primitives.npz (generated from
oracle/_ref, i.e. tomotopy's src/Utils/{math.h,LUT.hpp,sample.hpp,Utils.hpp}
compiled from the tomotopy tree) and, when oracle/_ref is built here, live."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_primitives.npz"))


def _aligned(src):
    raw = np.zeros(src.nbytes + 64, dtype=np.uint8)
    off = (-raw.ctypes.data) % 64
    a = raw[off:off + src.nbytes].view(src.dtype)
    a[:] = src
    return a


def test_lgamma_lut_bitexact():
    """lgammaT: math.h:119-153 + LUT.hpp:35-60."""
    xs = G["lut_x"]
    got = np.array([O.lib.orc_lgammaT(float(x)) for x in xs], dtype=np.float32)
    np.testing.assert_array_equal(got.view(np.uint32), G["lgammaT"].view(np.uint32))


def test_digamma_lut_bitexact():
    """digammaT: math.h:134-150 (table filled by digammaf, math.h:72-115)."""
    xs = G["lut_x"]
    got = np.array([O.lib.orc_digammaT(float(x)) for x in xs], dtype=np.float32)
    np.testing.assert_array_equal(got.view(np.uint32), G["digammaT"].view(np.uint32))
    xf = G["digammaf_x"]
    got = np.array([O.lib.orc_digammaf(float(x)) for x in xf], dtype=np.float32)
    np.testing.assert_array_equal(got.view(np.uint32), G["digammaf"].view(np.uint32))


def test_digamma_approx_close():
    """digammaApprox (math.h:170-176).  tomotopy evaluates it over Eigen float
    arrays; the scalar reference instantiation promotes to double, so the
    float restatement agrees to float rounding, not bitwise."""
    xs = G["digammaApprox_x"]
    got = np.array([O.lib.orc_digammaApprox(float(x)) for x in xs], dtype=np.float64)
    ref = G["digammaApprox"]
    np.testing.assert_allclose(got, ref, rtol=2e-6, atol=2e-6 * np.abs(ref).max() * 0 + 5e-6)


def test_prefix_sum_sse_bitexact():
    """prefixSum, SSE2 path (sample.hpp:62-86)."""
    lens, ins, outs = G["ps_len"], G["ps_in"], G["ps_out"]
    o = 0
    for n in lens:
        a = _aligned(ins[o:o + n].astype(np.float32))
        O.lib.orc_prefix_sum_sse(a.ctypes.data_as(C.c_void_p), int(n))
        np.testing.assert_array_equal(a.view(np.uint32), outs[o:o + n].view(np.uint32))
        o += n


def test_sample_acc_matches():
    """sampleFromDiscreteAcc (sample.hpp:133-189): strict <, K-1 fallback."""
    lens, cums, us, zs = G["sa_len"], G["sa_cum"], G["sa_u"], G["sa_z"]
    o = 0
    for n, u, z in zip(lens, us, zs):
        c = _aligned(cums[o:o + n].astype(np.float32))
        assert O.lib.orc_sample_acc(c.ctypes.data_as(C.c_void_p), int(n), float(u)) == z
        o += n


def test_shuffled_order_matches():
    """forShuffled (Utils.hpp:157-178), including the N % P == 0 fallback."""
    i = 0
    while f"sh{i}" in G:
        n, seed = int(G[f"sh{i}_n"]), int(G[f"sh{i}_seed"])
        out = np.zeros(n, dtype=np.uint64)
        O.lib.orc_shuffled_order(n, seed, out.ctypes.data_as(C.c_void_p))
        np.testing.assert_array_equal(out.astype(np.uint32), G[f"sh{i}"])
        i += 1
    assert i >= 5


def test_sort_and_write_order_matches():
    """sortAndWriteOrder (Utils.hpp:227-248): stable sort, order[old] = new."""
    i = 0
    while f"so{i}_in" in G:
        w = G[f"so{i}_in"].copy()
        o = np.zeros(len(w), dtype=np.uint32)
        O.lib.orc_sort_doc(w.ctypes.data_as(C.c_void_p), len(w), o.ctypes.data_as(C.c_void_p))
        np.testing.assert_array_equal(w, G[f"so{i}_w"])
        np.testing.assert_array_equal(o, G[f"so{i}_o"])
        i += 1


def test_remove_stopwords_matches():
    """removeStopwords' ordering rule (TopicModel.hpp:526-571)."""
    i = 0
    while f"rs{i}_args" in G:
        nv, mcf, mdf, rtop = (int(x) for x in G[f"rs{i}_args"])
        cf, df = G[f"rs{i}_cf"].copy(), G[f"rs{i}_df"].copy()
        order = np.zeros(nv, dtype=np.uint32)
        rv = O.lib.orc_remove_stopwords(nv, cf.ctypes.data_as(C.c_void_p), df.ctypes.data_as(C.c_void_p),
                                        mcf, mdf, rtop, order.ctypes.data_as(C.c_void_p))
        assert rv == int(G[f"rs{i}_rv"])
        np.testing.assert_array_equal(order, G[f"rs{i}_order"])
        i += 1


@pytest.mark.skipif(O.load_ref() is None, reason="oracle/_ref not built (no tomotopy tree here)")
def test_live_reference_spot_checks():
    r = O.load_ref()
    rng = np.random.default_rng(7)
    for x in rng.uniform(0, 2000, 2000).astype(np.float32):
        assert np.float32(O.lib.orc_lgammaT(float(x))) == np.float32(r.ref_lgammaT(float(x)))
        assert np.float32(O.lib.orc_digammaT(float(x))) == np.float32(r.ref_digammaT(float(x)))
