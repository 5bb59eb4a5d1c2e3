"""Generates tests/golden/ref_primitives.npz from tomotopy's own numeric
primitives (oracle/_ref/libtmtref.so, compiled from the tomotopy source tree
by oracle/Makefile).  Run here, where the tomotopy tree exists:
    make -C oracle && python tests/golden/make_golden.py
The fixture lets the oracle be pinned on machines without the tree."""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402


def aligned(n, dtype=np.float32, align=64):
    buf = np.zeros(n + align, dtype=np.uint8).view(np.uint8)
    raw = np.zeros(n * np.dtype(dtype).itemsize + align, dtype=np.uint8)
    off = (-raw.ctypes.data) % align
    return raw[off:off + n * np.dtype(dtype).itemsize].view(dtype)


def main():
    r = O.load_ref()
    if r is None:
        sys.exit("oracle/_ref/libtmtref.so is not built (needs the tomotopy tree)")
    rng = np.random.default_rng(20261203)
    # lgamma / digamma tables: the segment edges, each segment's interior,
    # the closed forms below 0.001 and above the last table point
    xs = np.concatenate([
        np.float32([0.0, 1e-6, 1e-4, 0.0009999, 0.001, 0.01, 0.1, 0.5, 0.999, 1.0, 1.0000001, 2.0, 3.0,
                    100.0, 100.99, 101.0, 101.01, 1100.0, 1100.75, 1100.875, 1101.0, 5000.0, 1e6, 1e9]),
        rng.uniform(0, 1, 400).astype(np.float32),
        rng.uniform(1, 101, 400).astype(np.float32),
        rng.uniform(101, 1101, 400).astype(np.float32),
        rng.uniform(1101, 1e7, 100).astype(np.float32),
        (np.arange(0, 5000, dtype=np.float32) + np.float32(0.1)),
        (np.arange(0, 3000, dtype=np.float32) + np.float32(0.01)),
    ]).astype(np.float32)
    lg = np.array([r.ref_lgammaT(float(x)) for x in xs], dtype=np.float32)
    dg = np.array([r.ref_digammaT(float(x)) for x in xs], dtype=np.float32)
    dgf_x = xs[(xs > 0) & (xs < 1e5)]
    dgf = np.array([r.ref_digammaf(float(x)) for x in dgf_x], dtype=np.float32)
    dga_x = xs[(xs > 0) & (xs < 1e7)]
    dga = np.array([r.ref_digammaApprox(float(x)) for x in dga_x], dtype=np.float64)
    # prefixSum (SSE order) on random non-negative vectors of many lengths
    ps_in, ps_out, ps_len = [], [], []
    for n in [1, 2, 3, 4, 5, 7, 8, 9, 20, 31, 32, 33, 100, 257, 1000, 1001]:
        for _ in range(3):
            a = aligned(n)
            a[:] = rng.exponential(1.0, n).astype(np.float32) * np.float32(rng.choice([1e-6, 1.0, 1e4]))
            ps_in.append(a.copy())
            r.ref_prefix_sum(a.ctypes.data_as(C.c_void_p), n)
            ps_out.append(a.copy())
            ps_len.append(n)
    # sampleFromDiscreteAcc: cumulative vectors (with flat runs) and u values
    sa_cum, sa_u, sa_z, sa_len = [], [], [], []
    for n in [1, 2, 8, 9, 31, 32, 33, 64, 100, 1000]:
        for _ in range(4):
            w = rng.exponential(1.0, n).astype(np.float32)
            w[rng.random(n) < 0.3] = 0
            c = aligned(n)
            c[:] = np.cumsum(w, dtype=np.float32)
            if c[-1] == 0:
                c[-1] = 1
            for u in np.concatenate([np.float32([0.0, 0.9999999]), rng.random(6).astype(np.float32)]):
                sa_cum.append(c.copy())
                sa_u.append(u)
                sa_z.append(r.ref_sample_acc(c.ctypes.data_as(C.c_void_p), n, float(u)))
                sa_len.append(n)
    # forShuffled orders
    sh = []
    for n, seed in [(1, 0), (7, 3), (100, 12345), (65537, 0), (65537 * 2, 0), (1000, 0xFFFFFFFF), (5000, 17)]:
        out = np.zeros(n, dtype=np.uint64)
        r.ref_shuffled_order(n, seed, out.ctypes.data_as(C.c_void_p))
        sh.append((n, seed, out))
    # sortAndWriteOrder on word lists with ties
    so_in, so_w, so_o = [], [], []
    for n in [0, 1, 5, 50, 300]:
        w = rng.integers(0, max(2, n // 3), n).astype(np.uint32)
        ww = w.copy()
        o = np.zeros(n, dtype=np.uint32)
        r.ref_sort_and_write_order(ww.ctypes.data_as(C.c_void_p), n, o.ctypes.data_as(C.c_void_p))
        so_in.append(w); so_w.append(ww); so_o.append(o)
    # removeStopwords vocabulary order
    rs = []
    for nv, mcf, mdf, rtop in [(50, 0, 0, 0), (50, 3, 0, 0), (50, 0, 2, 0), (50, 2, 2, 5), (200, 5, 3, 10),
                               (10, 100, 0, 0), (10, 0, 0, 10)]:
        cf = rng.integers(0, 20, nv).astype(np.uint64)
        df = np.minimum(cf, rng.integers(0, 10, nv)).astype(np.uint64)
        cf2, df2 = cf.copy(), df.copy()
        order = np.zeros(nv, dtype=np.uint32)
        rv = r.ref_remove_stopwords(nv, cf2.ctypes.data_as(C.c_void_p), df2.ctypes.data_as(C.c_void_p),
                                    mcf, mdf, rtop, order.ctypes.data_as(C.c_void_p))
        rs.append((nv, mcf, mdf, rtop, cf, df, order, rv))
    out = {
        "lut_x": xs, "lgammaT": lg, "digammaT": dg, "digammaf_x": dgf_x, "digammaf": dgf,
        "digammaApprox_x": dga_x, "digammaApprox": dga,
        "ps_len": np.array(ps_len), "ps_in": np.concatenate(ps_in), "ps_out": np.concatenate(ps_out),
        "sa_len": np.array(sa_len), "sa_cum": np.concatenate(sa_cum), "sa_u": np.array(sa_u, np.float32),
        "sa_z": np.array(sa_z, np.int64),
    }
    for i, (n, seed, o) in enumerate(sh):
        out[f"sh{i}_n"] = np.array(n); out[f"sh{i}_seed"] = np.array(seed, np.uint64); out[f"sh{i}"] = o.astype(np.uint32)
    for i in range(len(so_in)):
        out[f"so{i}_in"] = so_in[i]; out[f"so{i}_w"] = so_w[i]; out[f"so{i}_o"] = so_o[i]
    for i, (nv, mcf, mdf, rtop, cf, df, order, rv) in enumerate(rs):
        out[f"rs{i}_args"] = np.array([nv, mcf, mdf, rtop], np.uint64)
        out[f"rs{i}_cf"] = cf; out[f"rs{i}_df"] = df; out[f"rs{i}_order"] = order
        out[f"rs{i}_rv"] = np.array(rv, np.uint64)
    np.savez_compressed(os.path.join(HERE, "ref_primitives.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_primitives.npz"))


if __name__ == "__main__":
    main()
