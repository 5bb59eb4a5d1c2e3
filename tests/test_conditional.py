"""Gate (c) on the sweep kernel's own arithmetic: the topic probabilities
that its blocked two-pass draw implies -- the float lane totals (fma chain,
own topic added last), the lane scan and the pass-2 prefix sums, restated
bit for bit by the oracle (orc_draw_intervals / orc_blocked_draw; the GPU
tests check the oracle's sweep against the kernel z for z) -- against the
FP64 conditional of getZLikelihoods (LDAModel.hpp:273-285).

The bound: |p_device_k - p64_k| <= 1e-5 * max(p64_k, 0.1) for every topic,
i.e. 1e-5 relative for every topic holding at least a tenth of the mass and
1e-6 of the total below that.  Any float32 CDF draw resolves a topic only to
a few 2^-24 of the total (tomotopy's own prefix-sum draw measures ~2.4e-6
absolute on the same tokens), so a per-topic relative bound on the smallest
topics would test float32 itself rather than the kernel."""
import numpy as np
import pytest

import oracle as O
import tomotopy_b200 as T

TOL_REL, P_FLOOR = 1e-5, 0.1


def check_token(ndk_row, nkw_col, nk, alpha, eta, V, zo):
    p_dev, p_ref, p64 = O.implied_conditionals(ndk_row, nkw_col, nk, alpha, eta, V, zo)
    assert abs(p_dev.sum() - 1) < 1e-12
    err = np.abs(p_dev - p64)
    bound = TOL_REL * np.maximum(p64, P_FLOOR)
    assert (err <= bound).all(), (int(np.argmax(err / bound)), float(err.max()), float((err / bound).max()))
    return err, np.abs(p_ref - p64)


@pytest.fixture(scope="module")
def trained_k1000():
    """A K=1000 state after 20 PARTITION sweeps (the restated reference
    scheme) over 2,000 documents of the k=1000 benchmark configuration's
    generator: realistic documents and word columns."""
    off, w = T.synth_corpus(100000, 1000, 2000, ("lognormal", float(np.log(100)), 1.2, 5, 5000), seed=20261206)
    off, w, V, _ = T.prepare_ids(off, w)
    c = O.Corpus(off, w, V)
    st = O.State(c, 1000, 0.1, 0.01, 1)
    p = O.Partition(st, 4, seed=1)
    p.train(20)
    p.close()
    return c, st


def test_implied_conditional_realistic_k1000(trained_k1000):
    c, st = trained_k1000
    rng = np.random.default_rng(0)
    worst_dev = worst_ref = 0.0
    n = 0
    while n < 400:
        d = int(rng.integers(0, c.D))
        b, e = int(c.doc_off[d]), int(c.doc_off[d + 1])
        if e == b:
            continue
        i = int(rng.integers(b, e))
        v = int(c.words[i])
        if v >= c.V:
            continue
        ed, er = check_token(st.ndk[d], st.nkw[v], st.nk, st.alpha, 0.01, c.V, int(st.z[i]))
        worst_dev, worst_ref = max(worst_dev, ed.max()), max(worst_ref, er.max())
        n += 1
    # the device's draw resolves topics at least as finely as tomotopy's
    assert worst_dev <= worst_ref, (worst_dev, worst_ref)


@pytest.mark.parametrize("eta", [0.01, 0.001])
@pytest.mark.parametrize("n_own", [500, 5000, 50000])
def test_implied_conditional_own_topic_dominates(eta, n_own):
    """The case a subtract-and-add own-topic correction cancels in: a long
    document almost entirely in topic zo, the token the only one of its word
    in zo (n_kw[zo, v] = 1), K = 1000.  The old correction
    (s - A*phi_zo + A*phi_own) reached 3.9e-6 absolute error here."""
    rng = np.random.default_rng(n_own + int(1e6 * eta))
    K, V, zo = 1000, 100000, 517
    nk = rng.integers(5000, 50000, K).astype(np.int32)
    col = np.zeros(K, np.int32)
    col[rng.integers(0, K, 40)] = rng.integers(1, 200, 40)
    col[zo] = 1
    row = np.zeros(K, np.int32)
    row[zo] = n_own + 1
    row[rng.integers(0, K, 20)] += 1
    alpha = np.full(K, 0.1, np.float32)
    check_token(row, col, nk, alpha, eta, V, zo)


@pytest.mark.parametrize("K", [1, 5, 20, 33, 100, 250, 1000, 3000])
def test_implied_conditional_shapes(K):
    """Every lane layout: partial blocks of four, lanes without topics,
    pass 2 over more than 32 topics per lane (K > 4096 not needed: 3000
    gives 24 per lane)."""
    rng = np.random.default_rng(K)
    V = 5000
    for _ in range(30):
        nk = rng.integers(50, 5000, K).astype(np.int32)
        col = rng.integers(0, 30, K).astype(np.int32)
        zo = int(rng.integers(0, K))
        col[zo] = max(col[zo], 1)
        nk = np.maximum(nk, col + 1)
        row = rng.integers(0, 20, K).astype(np.int32)
        row[zo] += 1
        alpha = rng.uniform(0.01, 1.0, K).astype(np.float32)
        check_token(row, col, nk, alpha, 0.01, V, zo)


def test_draw_falls_in_its_interval():
    """orc_blocked_draw (the kernel's draw restated) returns, for r = u *
    total, the topic whose implied interval holds r: the widths above are
    the draw's."""
    rng = np.random.default_rng(3)
    for K in (7, 100, 1000):
        V = 3000
        nk = rng.integers(100, 9000, K).astype(np.int32)
        col = rng.integers(0, 40, K).astype(np.int32)
        zo = int(rng.integers(0, K))
        col[zo] = max(col[zo], 1)
        row = rng.integers(0, 30, K).astype(np.int32)
        row[zo] += 1
        A, phi, phi_own, _, _ = O.token_factors(row, col, nk, np.full(K, 0.1, np.float32), 0.01, V, zo)
        w = np.zeros(K)
        start = np.zeros(K)
        total = O.lib.orc_draw_intervals(O._ptr(A), O._ptr(phi), K, zo, float(phi_own), O._ptr(w), O._ptr(start))
        for u in rng.random(3000).astype(np.float32):
            k = O.lib.orc_blocked_draw(O._ptr(A), O._ptr(phi), K, zo, float(phi_own), float(u))
            r = float(np.float32(u) * np.float32(total))
            assert start[k] <= r < start[k] + w[k], (K, k, r, start[k], w[k])
