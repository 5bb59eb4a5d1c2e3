"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Gates:
  (a) n_dk, n_kw, n_k recomputed from z equal the device counts after every sweep;
  (b) the same seed gives bit-identical z;
  (c) the device draws are exactly the oracle's (same float arithmetic and
      scan order), the float conditional is within 1e-5 relative of FP64,
      and a chi-square test on many i.i.d. draws accepts the FP64 conditional;
  (d) ll_per_word within 1% of the reference's sequential sampler at the same
      iteration count, averaged over seeds.
"""
import ctypes as C

import numpy as np
import pytest
from scipy import stats

import oracle as O
import tomotopy_b200 as T
from tomotopy_b200._lib import TmtError

pytestmark = pytest.mark.gpu

G = 8   # the engine's default number of document groups per sweep


def corpus(V=800, Tt=8, D=120, mean=60, seed=1, min_cf=0, rm_top=0, lognormal=False):
    if lognormal:
        off, w = T.synth_corpus(V, Tt, D, ("lognormal", np.log(mean), 1.0, 1, 20 * mean), seed=seed)
    else:
        off, w = T.synth_corpus(V, Tt, D, ("poisson", mean, 1, 10 * mean), seed=seed)
    off, w, rv, _ = T.prepare_ids(off, w, min_cf=min_cf, rm_top=rm_top)
    return off, w, rv


def oracle_state(off, w, V, K, alpha, eta, seed, z0=None):
    c = O.Corpus(off, w, V)
    return O.State(c, K, alpha, eta, seed, z0=z0)


def assert_same_state(eng, st):
    z, nkw, nk, _ = eng.state()
    np.testing.assert_array_equal(z, st.z)
    np.testing.assert_array_equal(nk, st.nk)
    np.testing.assert_array_equal(nkw, st.nkw)
    np.testing.assert_array_equal(eng.doc_topic(), st.ndk)


@pytest.mark.parametrize("K", [1, 7, 20, 100, 1000, 1100, 9000])
def test_init_and_counts_bitexact(K):
    off, w, V = corpus(min_cf=2)
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=42, optim_interval=0)
    eng.upload(off, w)
    st = oracle_state(off, w, V, K, 0.1, 0.01, 42)
    assert_same_state(eng, st)
    assert eng.info().N == st.c.N


def test_large_downloads_through_staging():
    """Downloads above 32 MB into pageable memory go through pinned staging
    buffers and threaded host copies: the counts (n_kw 80 MB, n_dk 36 MB here)
    equal the counts recomputed from z, and a download into pinned memory (one
    direct copy) gives the same bytes."""
    import torch
    from tomotopy_b200._lib import lib
    from tomotopy_b200.engine import _p, check
    K, V = 1000, 20000
    off, w = T.synth_corpus(V, 30, 9000, ("poisson", 20, 1, 200), seed=4)
    off, w, _, _ = T.prepare_ids(off, w)
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=3, optim_interval=0)
    eng.upload(off, w)
    eng.train(2)
    z, nkw, nk, _ = eng.state()
    ndk = eng.doc_topic()
    wi = w.astype(np.int64)
    ok = wi < V
    doc = np.repeat(np.arange(len(off) - 1), np.diff(off.astype(np.int64)))
    want_kw = np.zeros((V, K), np.int32)
    np.add.at(want_kw, (wi[ok], z[ok].astype(np.int64)), 1)
    want_dk = np.zeros((len(off) - 1, K), np.int32)
    np.add.at(want_dk, (doc[ok], z[ok].astype(np.int64)), 1)
    np.testing.assert_array_equal(nkw, want_kw)
    np.testing.assert_array_equal(ndk, want_dk)
    np.testing.assert_array_equal(nk, want_kw.sum(0))
    pz = torch.empty(len(z), dtype=torch.int16).pin_memory().numpy().view(np.uint16)
    pkw = torch.empty(V * K, dtype=torch.int32).pin_memory().numpy()
    nk2 = np.zeros(K, np.int32)
    a2 = np.zeros(K, np.float32)
    check(lib.tmt_download_state(eng.h, _p(pz), _p(pkw), _p(nk2), _p(a2)), eng.h)
    np.testing.assert_array_equal(pz, z)
    np.testing.assert_array_equal(pkw.reshape(V, K), nkw)
    # two handles staging at once from two threads (the process's staging
    # buffers serve one transfer at a time)
    import threading
    other = T.Engine(K, V, alpha=0.1, eta=0.01, seed=3, optim_interval=0)
    other.upload(off, w)
    other.train(2)
    got = {}
    ths = [threading.Thread(target=lambda k, e: got.__setitem__(k, e.state()), args=(k, e))
           for k, e in (("a", eng), ("b", other))]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    for k in ("a", "b"):
        np.testing.assert_array_equal(got[k][0], z)
        np.testing.assert_array_equal(got[k][1], nkw)
    other.close()
    # batched inference whose theta (9,000 x 1,000 floats, 36 MB) is staged
    # into pageable memory equals the same call into pinned memory
    th1, ll1 = eng.infer(off, w, iters=3, seed=2)
    pth = torch.empty((len(off) - 1) * K, dtype=torch.float32).pin_memory().numpy()
    pll = np.zeros(len(off) - 1, np.float64)
    check(lib.tmt_infer_batch(eng.h, _p(np.ascontiguousarray(w, dtype=np.uint32)),
                              _p(np.ascontiguousarray(off, dtype=np.uint64)), len(off) - 1, 3, 2, None,
                              _p(pth), _p(pll)), eng.h)
    np.testing.assert_array_equal(th1, pth.reshape(-1, K))
    np.testing.assert_array_equal(ll1, pll)
    # a destination in device memory takes one direct copy as well
    dkw = torch.zeros(V * K, dtype=torch.int32, device="cuda")
    check(lib.tmt_download_state(eng.h, None, C.c_void_p(dkw.data_ptr()), None, None), eng.h)
    np.testing.assert_array_equal(dkw.cpu().numpy().reshape(V, K), nkw)
    eng.close()


def test_pageable_uploads_through_staging():
    """Uploads above 32 MB from pageable memory go through the pinned staging
    buffers (words 34 MB, n_kw 36 MB here): the same corpus uploaded from
    pinned memory gives the same z and counts after a sweep, and counts set
    from pageable memory read back unchanged."""
    import torch
    from tomotopy_b200._lib import lib
    from tomotopy_b200.engine import _p, check
    K, V = 100, 90000
    off, w = T.synth_corpus(V, 40, 42000, ("poisson", 200, 1, 2000), seed=6)
    assert w.nbytes > (32 << 20)
    pw = torch.from_numpy(np.ascontiguousarray(w, dtype=np.uint32).view(np.int32)).pin_memory().numpy().view(np.uint32)
    a = T.Engine(K, V, alpha=0.1, eta=0.01, seed=5, optim_interval=0)
    b = T.Engine(K, V, alpha=0.1, eta=0.01, seed=5, optim_interval=0)
    a.upload(off, w)
    b.upload(off, pw)
    assert a.info().N == b.info().N == int(np.sum(w < V))
    a.train(1)
    b.train(1)
    za, kwa, ka, _ = a.state()
    zb, kwb, kb, _ = b.state()
    np.testing.assert_array_equal(za, zb)
    np.testing.assert_array_equal(kwa, kwb)
    np.testing.assert_array_equal(ka, kb)
    # weighted counts: 34 MB of token weights staged from pageable memory
    wts = (1.0 + (np.arange(len(w)) % 7) * 0.25).astype(np.float32)
    pwt = torch.from_numpy(wts).pin_memory().numpy()
    wa = T.Engine(K, V, alpha=0.1, eta=0.01, seed=5, optim_interval=0)
    wb = T.Engine(K, V, alpha=0.1, eta=0.01, seed=5, optim_interval=0)
    wa.upload(off, w, weights=wts)
    wb.upload(off, pw, weights=pwt)
    wa.train(1)
    wb.train(1)
    for x, y in zip(wa.state(), wb.state()):
        np.testing.assert_array_equal(x, y)
    wa.close()
    wb.close()
    # counts set from pageable memory (36 MB) come back unchanged
    kw2 = np.ascontiguousarray(kwa[::-1])
    check(lib.tmt_set_counts(b.h, _p(kw2), _p(ka)), b.h)
    _, kwc, _, _ = b.state()
    np.testing.assert_array_equal(kwc, kw2)
    a.close()
    b.close()


@pytest.mark.parametrize("K,groups", [(1, 1), (5, 1), (20, 1), (33, 3), (100, 1), (100, 4), (250, 1), (1000, 1),
                                      (1000, 2), (1100, 1), (3000, 1)])
def test_sweeps_bitexact(K, groups):
    """Every sweep's z and counts equal the oracle's doc-major sweep exactly:
    the autotuner's sweeps (every kernel variant, in the order 0, 1, .., n-1,
    n-1, .., 0) and the graph sweeps after them."""
    off, w, V = corpus(V=600, D=90, mean=50, seed=K, min_cf=2, rm_top=3)
    alpha = np.float32(0.1) if K != 20 else (0.05 * (np.arange(K) + 1)).astype(np.float32)
    eng = T.Engine(K, V, alpha=alpha, eta=0.01, seed=7, optim_interval=0, sweep_groups=groups)
    eng.upload(off, w)
    st = oracle_state(off, w, V, K, alpha, 0.01, 7)
    step = 0
    for n in (1, 2, 2, 5):
        eng.train(n)
        st.doc_live_sweeps(n, start_step=step, groups=groups)
        step += n
        assert_same_state(eng, st)
    # the tuner is done: each group runs the variant it timed fastest
    tm, var = eng.sweep_timings(), eng.sweep_variants()
    assert tm.shape[0] == len(var) and -1 not in var
    for g, v in enumerate(var):
        if tm[g].sum() > 0:
            assert v == int(np.argmin(tm[g])) and (tm[g] > 0).all()


@pytest.mark.parametrize("K,groups", [(24, 8), (300, 3)])
def test_graph_sweeps_identical_to_launches(K, groups):
    """Sweeps replayed as CUDA graphs (after the autotuner's eager sweeps) give
    the same z, counts, alpha and ll history as kernel-by-kernel launches,
    across train() calls, ll points, alpha optimisation and a seed change;
    and the graph sweeps equal the oracle's."""
    off, w, V = corpus(V=900, D=160, mean=60, seed=K, min_cf=2, lognormal=True)
    out = []
    for graphs in (True, False):
        eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=13, optim_interval=5, sweep_groups=groups)
        eng.set_graphs(graphs)
        eng.upload(off, w)
        lls = [eng.train(9, ll_every=3)]
        eng.train(4)
        lib_set_seed(eng, 99)
        lls.append(eng.train(6, ll_every=2))
        out.append((eng.state(), eng.doc_topic(), np.concatenate(lls), eng.info().kernel_launches))
    (sa, ndk_a, ll_a, la), (sb, ndk_b, ll_b, lb) = out
    for x, y in zip(sa, sb):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(ndk_a, ndk_b)
    np.testing.assert_array_equal(ll_a, ll_b)
    # a captured sweep counts its kernels, plus the sweep-counter kernels of the graph path
    assert la >= lb

    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=13, optim_interval=0, sweep_groups=groups)
    eng.upload(off, w)
    st = oracle_state(off, w, V, K, 0.1, 0.01, 13)
    eng.train(6)
    st.doc_live_sweeps(6, groups=groups)
    assert_same_state(eng, st)


def lib_set_seed(eng, seed):
    from tomotopy_b200._lib import lib, check
    check(lib.tmt_set_seed(eng.h, seed), eng.h)


def test_counts_invariant_after_every_sweep():
    off, w, V = corpus(V=1500, D=300, mean=80, seed=3, lognormal=True)
    K = 50
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=5, optim_interval=10)
    eng.upload(off, w)
    c = O.Corpus(off, w, V)
    for _ in range(12):
        eng.train(1)
        z, nkw, nk, alpha = eng.state()
        st = O.State(c, K, alpha, 0.01, 0, z0=z)   # recount from z
        np.testing.assert_array_equal(nkw, st.nkw)
        np.testing.assert_array_equal(nk, st.nk)
        np.testing.assert_array_equal(eng.doc_topic(), st.ndk)
        assert nk.sum() == c.N


def test_seed_determinism():
    off, w, V = corpus(V=1000, D=200, mean=70, seed=4)
    zs = []
    for seed in (11, 11, 12):
        eng = T.Engine(64, V, alpha=0.1, eta=0.01, seed=seed)
        eng.upload(off, w)
        eng.train(15)
        zs.append(eng.state()[0])
    np.testing.assert_array_equal(zs[0], zs[1])
    assert not np.array_equal(zs[0], zs[2])


@pytest.mark.parametrize("K", [20, 300])
def test_ll_fp64_matches_oracle(K):
    off, w, V = corpus(V=900, D=150, mean=70, seed=9, min_cf=2)
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=3, optim_interval=0)
    eng.upload(off, w)
    eng.train(3)
    st = oracle_state(off, w, V, K, 0.1, 0.01, 3)
    st.doc_live_sweeps(3, groups=G)
    ld, lr = eng.ll()
    od, orr = st.ll_f64()
    assert ld == pytest.approx(od, rel=1e-11, abs=1e-7)
    assert lr == pytest.approx(orr, rel=1e-11, abs=1e-7)
    # the reference's float-LUT likelihood agrees to the table's accuracy
    # (linear interpolation of lgamma, step 1/1024 below 1: ~1e-5 per term)
    lut = sum(st.ll_lut())
    assert (ld + lr) == pytest.approx(lut, rel=1e-4)


@pytest.mark.parametrize("asym", [False, True])
def test_alpha_optimisation_matches_oracle(asym):
    off, w, V = corpus(V=700, D=250, mean=60, seed=21)
    K = 16
    alpha = (0.02 * (np.arange(K) + 1)).astype(np.float32) if asym else np.float32(0.1)
    eng = T.Engine(K, V, alpha=alpha, eta=0.01, seed=8, optim_interval=1)
    eng.upload(off, w)
    st = oracle_state(off, w, V, K, alpha, 0.01, 8)
    for step in range(3):
        eng.train(1)
        st.doc_live_sweeps(1, start_step=step, groups=G)
        st.optimize_alpha()
        _, _, _, a_dev = eng.state()
        np.testing.assert_allclose(a_dev, st.alpha, rtol=2e-4)
        # keep the oracle on the device's alpha so later sweeps stay comparable
        st.alpha[:] = a_dev
        z = eng.state()[0]
        if not np.array_equal(z, st.z):
            break


def test_conditional_fp32_vs_fp64():
    """The float conditional the sampler uses is within 1e-5 relative of FP64."""
    off, w, V = corpus(V=500, D=60, mean=80, seed=2)
    K = 100
    st = oracle_state(off, w, V, K, 0.1, 0.01, 1)
    rng = np.random.default_rng(0)
    veta = np.float32(0.01) * np.float32(V)
    for _ in range(200):
        d = int(rng.integers(0, st.c.D))
        b, e = int(st.c.doc_off[d]), int(st.c.doc_off[d + 1])
        if e == b:
            continue
        i = int(rng.integers(b, e))
        v, zo = int(st.c.words[i]), int(st.z[i])
        row = st.ndk[d].copy()
        row[zo] -= 1
        p64 = np.zeros(K)
        O.lib.orc_conditional_f64(K, V, O._ptr(st.alpha), 0.01, O._ptr(np.ascontiguousarray(st.ndk[d])),
                                  O._ptr(np.ascontiguousarray(st.nkw[v])), O._ptr(st.nk), zo, O._ptr(p64))
        own = (np.arange(K) == zo).astype(np.int32)
        a32 = row.astype(np.float32) + st.alpha
        b32 = (st.nkw[v] - own).astype(np.float32) + np.float32(0.01)
        r32 = np.float32(1.0) / ((st.nk - own).astype(np.float32) + veta)
        w32 = (a32 * b32) * r32
        p32 = w32.astype(np.float64) / w32.astype(np.float64).sum()
        np.testing.assert_allclose(p32, p64, rtol=1e-5, atol=1e-12)


def test_chi_square_on_draws():
    """Identical documents with identical z0 give every first token the same
    start-of-sweep conditional; the device's draws across documents must fit
    the FP64 oracle's distribution."""
    rng = np.random.default_rng(1)
    K, V, D, L = 24, 300, 40000, 12
    doc = np.sort(rng.integers(0, V, L)).astype(np.uint32)
    z_doc = rng.integers(0, K, L).astype(np.uint16)
    off = np.arange(D + 1, dtype=np.uint64) * L
    words = np.tile(doc, D)
    z0 = np.tile(z_doc, D)
    # one document group: every first token sees the same start-of-sweep snapshot
    eng = T.Engine(K, V, alpha=0.3, eta=0.05, seed=99, optim_interval=0, sweep_groups=1)
    eng.upload(off, words, z0=z0)
    st = oracle_state(off, words, V, K, 0.3, 0.05, 99, z0=z0)
    p64 = np.zeros(K)
    v0, zo = int(doc[0]), int(z_doc[0])
    O.lib.orc_conditional_f64(K, V, O._ptr(st.alpha), 0.05, O._ptr(np.ascontiguousarray(st.ndk[0])),
                              O._ptr(np.ascontiguousarray(st.nkw[v0])), O._ptr(st.nk), zo, O._ptr(p64))
    eng.train(1)
    z = eng.state()[0]
    first = z[off[:-1].astype(np.int64)]
    obs = np.bincount(first, minlength=K).astype(np.float64)
    exp = p64 * D
    keep = exp >= 5
    obs_m = np.append(obs[keep], obs[~keep].sum())
    exp_m = np.append(exp[keep], exp[~keep].sum())
    if exp_m[-1] == 0:
        obs_m, exp_m = obs_m[:-1], exp_m[:-1]
    chi2, p = stats.chisquare(obs_m, exp_m)
    assert p > 1e-4, (chi2, p)


def test_chi_square_mid_document_k1000():
    """K = 1000, a token deep inside a long document: each test document is
    3,000 tokens of an anchor word whose word prior allows only topic zo
    (so every anchor draw is zo again, exactly) followed by one token of its
    own word, whose other occurrences (in background documents) give every
    test word the same column.  With one document group every test token
    draws from the same start-of-sweep conditional, with n_dk[zo] = 3,000
    live counts before it and n_kw[zo, v] = 1 (the own-topic case); the
    draws across 20,000 documents must fit the FP64 conditional."""
    rng = np.random.default_rng(11)
    K, zo, La, Dt, eta, alpha = 1000, 517, 3000, 20000, 0.01, 0.1
    V = 1 + Dt
    pattern = np.repeat(np.sort(rng.choice(np.delete(np.arange(K), zo), 30, replace=False)), 8)   # 240 tokens
    docs_w, docs_z = [], []
    for d in range(Dt):                     # test documents: anchors, then the document's word
        docs_w.append(np.concatenate([np.zeros(La, np.uint32), [1 + d]]).astype(np.uint32))
        docs_z.append(np.full(La + 1, zo, np.uint16))
    for d in range(Dt):                     # background: the word with the shared topic pattern
        docs_w.append(np.full(len(pattern), 1 + d, np.uint32))
        docs_z.append(pattern.astype(np.uint16))
    lens = np.array([len(x) for x in docs_w])
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    words = np.concatenate(docs_w)
    z0 = np.concatenate(docs_z)
    prior = np.zeros(K, np.float32)
    prior[zo] = 1.0
    eng = T.Engine(K, V, alpha=alpha, eta=eta, seed=123, optim_interval=0, sweep_groups=1)
    eng.set_word_priors([0], prior[None, :])
    eng.upload(off, words, z0=z0)
    # FP64 conditional of a test token from the start-of-sweep counts
    nk = np.bincount(z0.astype(np.int64), minlength=K).astype(np.float64)
    col = np.bincount(pattern, minlength=K).astype(np.float64)
    col[zo] += 1
    own = (np.arange(K) == zo).astype(np.float64)
    esum = (V - 1) * eta + prior.astype(np.float64)
    A = np.full(K, alpha)
    A[zo] += La
    w64 = A * (col - own + eta) / (nk - own + esum)
    p64 = w64 / w64.sum()
    eng.train(1)
    z = eng.state()[0]
    anchors_ok = np.all(z[np.concatenate([np.arange(off[d], off[d] + La) for d in range(0, Dt, 997)]).astype(np.int64)] == zo)
    assert anchors_ok, "an anchor token left its only allowed topic"
    draws = z[(off[1:Dt + 1] - 1).astype(np.int64)].astype(np.int64)
    obs = np.bincount(draws, minlength=K).astype(np.float64)
    exp = p64 * Dt
    keep = exp >= 5
    obs_m = np.append(obs[keep], obs[~keep].sum())
    exp_m = np.append(exp[keep], exp[~keep].sum())
    chi2, p = stats.chisquare(obs_m, exp_m)
    assert p > 1e-4, (chi2, p, int(keep.sum()))


def test_full_config1_two_sweeps_bitexact():
    """The k=20 benchmark corpus in full (V=10k, D=1,000 Poisson(1500)
    documents, 1.5M tokens): z and every count after two sweeps equal the
    oracle's restatement bit for bit."""
    import bench
    off, w, V = bench.make_corpus(bench.WORKLOADS["c1"])
    eng = T.Engine(20, V, alpha=0.1, eta=0.01, seed=7, optim_interval=0)
    eng.upload(off, w)
    st = oracle_state(off, w, V, 20, 0.1, 0.01, 7)
    assert_same_state(eng, st)
    eng.train(2)
    st.doc_live_sweeps(2, groups=G)
    assert_same_state(eng, st)


@pytest.mark.parametrize("K,V,Tt,D,mean,iters", [(20, 5000, 20, 400, 500, 200), (100, 8000, 50, 1500, 200, 150)])
def test_ll_per_word_matches_reference_train(K, V, Tt, D, mean, iters):
    """(d) At the same iteration count, the device's ll_per_word is within 1%
    of tomotopy's train() -- its default ParallelScheme::PARTITION on every
    host thread, restated in the oracle -- averaged over 5 seeds."""
    import os
    off, w = T.synth_corpus(V, Tt, D, ("poisson", mean, 1, 20 * mean), seed=K + 1)
    off, w, Vr, _ = T.prepare_ids(off, w)
    c = O.Corpus(off, w, Vr)
    cf = np.bincount(w[w < Vr], minlength=Vr).astype(np.uint64)
    gpu, ref = [], []
    for seed in (1, 2, 3, 4, 5):
        eng = T.Engine(K, Vr, alpha=0.1, eta=0.01, seed=seed, optim_interval=0)
        eng.upload(off, w)
        eng.train(iters)
        gpu.append(eng.ll_per_word())
        st = O.State(c, K, 0.1, 0.01, seed)
        p = O.Partition(st, os.cpu_count() or 1, vocab_cf=cf, seed=seed)
        p.train(iters)
        p.close()
        ref.append(st.ll_per_word())
    g, r = np.mean(gpu), np.mean(ref)
    assert abs(g - r) / abs(r) < 0.01, (gpu, ref)


def test_edge_cases():
    # empty corpus, empty docs, docs whose words are all removed
    eng = T.Engine(5, 10, alpha=0.1, eta=0.01, seed=1)
    eng.upload(np.zeros(1, np.uint64), np.zeros(0, np.uint32))
    eng.train(3)
    assert eng.info().global_step == 3
    assert eng.ll() == (0.0, 0.0)
    off = np.array([0, 0, 3, 3, 5, 6], dtype=np.uint64)
    words = np.array([1, 1, 9, 11, 12, 2], dtype=np.uint32)     # V=10: 11, 12 are skipped
    eng = T.Engine(3, 10, alpha=0.1, eta=0.01, seed=2, optim_interval=0)
    eng.upload(off, words)
    st = oracle_state(off, words, 10, 3, 0.1, 0.01, 2)
    assert_same_state(eng, st)
    eng.train(4)
    st.doc_live_sweeps(4, groups=G)
    assert_same_state(eng, st)
    z = eng.state()[0]
    assert z[3] == 0xFFFF and z[4] == 0xFFFF
    assert eng.info().N == 4


def test_bad_inputs_raise():
    eng = T.Engine(4, 10, alpha=0.1, eta=0.01, seed=1)
    with pytest.raises(TmtError):
        eng.train(1)                       # before upload: TMT_ERR_STATE
    with pytest.raises(ValueError):
        eng.upload(np.array([0, 2], np.uint64), np.array([1, 2], np.uint32), z0=np.array([0, 9], np.uint16))
    with pytest.raises(ValueError):
        eng.upload(np.array([0, 2, 1], np.uint64), np.array([1, 2], np.uint32))
    small = T.Engine(4, 10, alpha=0.1, eta=0.01, seed=1, hbm_budget=1024)
    with pytest.raises(TmtError) as e:
        small.upload(np.array([0, 300], np.uint64), np.ones(300, np.uint32))
    assert e.value.status == -3
