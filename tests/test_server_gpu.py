"""Served inference (continuous batching over resident models): every
document's result equals tmt_infer_batch's for the same model, words, seed
and key, whether it ran alone or among others; admission respects the token
budget; waits are bounded."""
import time

import numpy as np
import pytest

import tomotopy_b200 as T
from tomotopy_b200._lib import TmtError

pytestmark = pytest.mark.gpu


def model(K, V=600, D=120, seed=1):
    off, w = T.synth_corpus(V, 8, D, ("poisson", 70, 1, 700), seed=seed)
    off, w, Vr, order = T.prepare_ids(off, w)
    eng = T.Engine(K, Vr, alpha=0.1, eta=0.01, seed=seed, optim_interval=0)
    eng.upload(off, w)
    eng.train(15)
    return eng


def docs(V, n, seed, lo=3, hi=400):
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi, n)
    return [rng.integers(0, V + 3, L).astype(np.uint32) for L in lens]


def drain(srv, n, timeout_s=120):
    out = {}
    t0 = time.time()
    while len(out) < n and time.time() - t0 < timeout_s:
        r = srv.poll(wait_ms=200)
        if r is not None:
            out[r[0]] = r
    assert len(out) == n
    return out


def batch_ref(eng, ds, iters, seed, keys):
    off = np.concatenate([[0], np.cumsum([len(d) for d in ds])]).astype(np.uint64)
    w = np.concatenate(ds).astype(np.uint32) if ds else np.zeros(0, np.uint32)
    return eng.infer(off, w, iters=iters, seed=seed, doc_keys=np.asarray(keys, np.uint64))


def test_served_equals_batch_alone_and_mixed():
    eng = model(40)
    ds = docs(eng.V, 60, seed=3)
    keys = np.arange(100, 160, dtype=np.uint64)
    theta, ll = batch_ref(eng, ds, 30, 7, keys)
    srv = T.Server(max_slots=16, token_budget=4000, step_token_sweeps=500, max_doc_len=1000)
    mid = srv.add_engine_model(eng)
    # alone: one request at a time
    for i in (0, 5, 33):
        rid = srv.submit(mid, ds[i], iters=30, seed=7, key=int(keys[i]))
        r = srv.poll(wait_ms=30000)
        assert r is not None and r[0] == rid
        np.testing.assert_array_equal(r[2], theta[i])
        assert r[3] == ll[i]
    # mixed: all at once (more than the slots; they queue and join as slots free up)
    ids = {srv.submit(mid, d, iters=30, seed=7, key=int(k)): i for i, (d, k) in enumerate(zip(ds, keys))}
    res = drain(srv, len(ds))
    for rid, (r_id, m, th, l, lat) in res.items():
        i = ids[rid]
        np.testing.assert_array_equal(th, theta[i])
        assert l == ll[i]
        assert lat > 0
    st = srv.stats()
    assert st.completed == len(ds) + 3
    assert st.mean_active > 1.5          # documents overlapped on the device
    srv.close()


def test_two_resident_models_interleaved():
    e1, e2 = model(24, seed=2), model(130, V=800, seed=4)
    d1, d2 = docs(e1.V, 30, seed=5), docs(e2.V, 30, seed=6)
    t1, l1 = batch_ref(e1, d1, 20, 3, np.zeros(30))
    t2, l2 = batch_ref(e2, d2, 20, 3, np.zeros(30))
    srv = T.Server(max_slots=8, token_budget=3000, step_token_sweeps=300, max_doc_len=1000)
    m1, m2 = srv.add_engine_model(e1), srv.add_engine_model(e2)
    ids = {}
    for i in range(30):
        ids[srv.submit(m1, d1[i], iters=20, seed=3)] = (m1, i)
        ids[srv.submit(m2, d2[i], iters=20, seed=3)] = (m2, i)
    res = drain(srv, 60)
    for rid, r in res.items():
        m, i = ids[rid]
        assert r[1] == m
        if m == m1:
            np.testing.assert_array_equal(r[2], t1[i]); assert r[3] == l1[i]
        else:
            np.testing.assert_array_equal(r[2], t2[i]); assert r[3] == l2[i]
    srv.close()


def test_admission_by_token_budget_and_bounded_waits():
    eng = model(16)
    srv = T.Server(max_slots=64, token_budget=300, step_token_sweeps=200, max_doc_len=300)
    mid = srv.add_engine_model(eng)
    t0 = time.time()
    assert srv.poll(wait_ms=50) is None          # nothing submitted: times out
    assert time.time() - t0 < 5
    ds = [np.full(100, i % eng.V, np.uint32) for i in range(12)]
    for d in ds:
        srv.submit(mid, d, iters=10, seed=1)
    drain(srv, 12)
    st = srv.stats()
    assert st.tokens_in_flight_max <= 300
    with pytest.raises(ValueError):
        srv.submit(mid, np.zeros(301, np.uint32), iters=10)
    srv.close()


def test_batch_submit_and_poll():
    e1, e2 = model(24, seed=2), model(130, V=800, seed=4)
    d1, d2 = docs(e1.V, 40, seed=8), docs(e2.V, 40, seed=9)
    k1 = np.arange(40, dtype=np.uint64) * 3
    t1, l1 = batch_ref(e1, d1, 20, 3, k1)
    t2, l2 = batch_ref(e2, d2, 20, 3, np.zeros(40))
    srv = T.Server(max_slots=8, token_budget=3000, step_token_sweeps=300, max_doc_len=1000)
    m1, m2 = srv.add_engine_model(e1), srv.add_engine_model(e2)
    allds = d1 + d2
    off = np.concatenate([[0], np.cumsum([len(d) for d in allds])]).astype(np.uint64)
    w = np.concatenate(allds).astype(np.uint32)
    mids = np.array([m1] * 40 + [m2] * 40, np.uint32)
    keys = np.concatenate([k1, np.zeros(40, np.uint64)])
    rids = srv.submit_batch(mids, off, w, iters=20, seed=3, keys=keys)
    assert len(set(rids.tolist())) == 80
    where = {int(r): i for i, r in enumerate(rids)}
    got = 0
    t0 = time.time()
    while got < 80 and time.time() - t0 < 60:
        r = srv.poll_batch(max_n=7, wait_ms=2000)
        if r is None:
            continue
        rid, mid, th, ll, lat = r
        assert len(rid) <= 7
        for j in range(len(rid)):
            i = where[int(rid[j])]
            if i < 40:
                assert mid[j] == m1
                np.testing.assert_array_equal(th[j, :24], t1[i]); assert ll[j] == l1[i]
            else:
                assert mid[j] == m2
                np.testing.assert_array_equal(th[j, :130], t2[i - 40]); assert ll[j] == l2[i - 40]
            assert lat[j] > 0
        got += len(rid)
    assert got == 80
    assert srv.poll_batch(max_n=4, wait_ms=20) is None
    st = srv.stats()
    assert st.kernel_ms > 0 and st.busy_ms >= st.kernel_ms * 0.5 and st.token_sweeps > 0
    srv.close()


def test_served_model_with_word_priors():
    """A resident model with word priors: served results equal tmt_infer_batch
    on the engine holding the same priors; priors are refused once the model
    has served a request."""
    off, w = T.synth_corpus(600, 8, 120, ("poisson", 70, 1, 700), seed=5)
    off, w, Vr, _ = T.prepare_ids(off, w)
    K = 24
    ids = np.array([0, 3, 7], np.uint32)
    pr = np.full((3, K), 0.01, np.float32)
    pr[0, :] = 0.0
    pr[0, 2] = 1.0
    pr[1, 5:9] = 0.3
    eng = T.Engine(K, Vr, alpha=0.1, eta=0.01, seed=5, optim_interval=0)
    eng.set_word_priors(ids, pr)
    eng.upload(off, w)
    eng.train(10)
    ds = docs(eng.V, 20, seed=8)
    keys = np.arange(20, dtype=np.uint64)
    theta, ll = batch_ref(eng, ds, 25, 3, keys)
    srv = T.Server(max_slots=8, token_budget=4000, step_token_sweeps=300, max_doc_len=1000)
    mid = srv.add_engine_model(eng)
    rids = [srv.submit(mid, d, iters=25, seed=3, key=int(k)) for d, k in zip(ds, keys)]
    out = drain(srv, len(rids))
    for i, rid in enumerate(rids):
        np.testing.assert_array_equal(out[rid][2], theta[i])
        assert out[rid][3] == ll[i]
    with pytest.raises(TmtError):
        srv.set_model_priors(mid, ids, pr)
    srv.close()


def test_served_weighted_model():
    """A resident model with weighted counts (TermWeight IDF): served results,
    one by one and in a batch, equal tmt_infer_batch_weighted on the engine."""
    import oracle as O
    off, w = T.synth_corpus(600, 8, 150, ("poisson", 70, 1, 700), seed=6)
    off, w, Vr, _ = T.prepare_ids(off, w, min_cf=1)      # every kept word occurs: finite IDF
    c = O.Corpus(off, w, Vr)
    wt, vw = O.weights_idf(c)
    K = 16
    eng = T.Engine(K, Vr, alpha=0.1, eta=0.01, seed=6, optim_interval=0)
    eng.upload(off, w, weights=wt)
    eng.train(10)
    ds = docs(eng.V, 24, seed=9)
    wts = [np.where(d < Vr, vw[np.minimum(d, Vr - 1)], 0).astype(np.float32) for d in ds]
    keys = np.arange(24, dtype=np.uint64)
    doff = np.concatenate([[0], np.cumsum([len(d) for d in ds])]).astype(np.uint64)
    theta, ll = eng.infer(doff, np.concatenate(ds), iters=20, seed=2, doc_keys=keys, weights=np.concatenate(wts))
    srv = T.Server(max_slots=8, token_budget=4000, step_token_sweeps=300, max_doc_len=1000)
    mid = srv.add_engine_model(eng)
    rids = [srv.submit(mid, d, iters=20, seed=2, key=int(k), weights=x) for d, x, k in zip(ds[:12], wts[:12], keys)]
    rids += list(srv.submit_batch(mid, doff[12:] - doff[12], np.concatenate(ds[12:]), iters=20, seed=2,
                                  keys=keys[12:], weights=np.concatenate(wts[12:])))
    out = drain(srv, len(rids))
    for i, rid in enumerate(rids):
        np.testing.assert_array_equal(out[int(rid)][2], theta[i])
        assert out[int(rid)][3] == ll[i]
    with pytest.raises(ValueError):
        srv.submit(mid, ds[0], iters=5)                 # a weighted model takes weighted requests only
    srv.close()
