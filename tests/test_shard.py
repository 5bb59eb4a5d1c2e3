"""A corpus sharded across processes (tmt_upload_shard), host side: the
shard planner against the single-corpus grouping, and two gloo ranks that run
the oracle's doc-major sweep on their own documents, group by group, summing
their count deltas through the product's allreduce callback -- the result must
equal one process sweeping the whole corpus, bit for bit."""
import ctypes as C
import os
import socket
import sys

import numpy as np
import pytest

import tomotopy_b200 as T
from tomotopy_b200 import shard

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "oracle"))
import oracle as O  # noqa: E402


def corpus(D=120, V=300, seed=3):
    off, w = T.synth_corpus(V, 8, D, ("lognormal", float(np.log(40)), 1.0, 1, 400), seed=seed)
    # a few words outside the vocabulary and an empty document
    w = w.copy()
    w[::97] = V + 5
    lens = np.diff(off.astype(np.int64))
    lens[7] = 0
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    return off, w[:int(off[-1])], V


def single_groups(lens, G):
    """The grouping of one corpus (restated): longest first, equal-token cuts."""
    order = np.argsort(-lens.astype(np.int64), kind="stable")
    total = int(lens.sum())
    prefix = np.concatenate([[0], np.cumsum(lens[order])[:-1]]).astype(np.int64)
    bounds = [0] + [int(np.sum(prefix * G < g * total)) for g in range(1, G)] + [len(lens)]
    return order, bounds


@pytest.mark.parametrize("G", [1, 3, 8])
def test_plan_matches_single_corpus(G):
    off, w, V = corpus()
    lens = np.diff(off.astype(np.int64)).astype(np.uint64)
    order, bounds = single_groups(lens, G)
    lo, lb, gb, toff = shard.plan(lens, G, 0, len(lens))
    np.testing.assert_array_equal(lo, order)
    np.testing.assert_array_equal(lb, bounds)
    np.testing.assert_array_equal(gb, bounds)
    assert toff == 0
    # three uneven shards: together they hold every document once, in its global group
    cuts = [0, 17, 80, len(lens)]
    seen = {}
    for r in range(3):
        b, e = cuts[r], cuts[r + 1]
        lo, lb, gb, toff = shard.plan(lens, G, b, e - b)
        np.testing.assert_array_equal(gb, bounds)
        assert toff == int(lens[:b].sum())
        for g in range(G):
            for d in lo[lb[g]:lb[g + 1]]:
                seen[int(d) + b] = g
        # within the shard, global order is kept
        pos = {int(d): i for i, d in enumerate(order)}
        glob = [int(d) + b for d in lo]
        assert glob == sorted(glob, key=lambda x: pos[x])
    want = {int(order[p]): g for g in range(G) for p in range(bounds[g], bounds[g + 1])}
    assert seen == want


@pytest.mark.parametrize("case", ["ties", "zipf", "huge"])
def test_plan_order_is_stable_longest_first(case):
    """The planner sorts by counting (lengths up to 4D + 65536) or by a
    comparison sort (longer documents); both give numpy's stable order."""
    rng = np.random.default_rng(5)
    if case == "ties":
        lens = rng.integers(0, 6, 5000).astype(np.uint64)
    elif case == "zipf":
        lens = np.minimum(rng.zipf(1.3, 20000), 10 ** 5).astype(np.uint64)
    else:
        lens = rng.integers(0, 3, 3000).astype(np.uint64)
        lens[[5, 17, 2900]] = [10 ** 7, 3 * 10 ** 6, 10 ** 7]
    for G in (1, 5, 8):
        order, bounds = single_groups(lens, G)
        lo, lb, gb, toff = shard.plan(lens, G, 0, len(lens))
        np.testing.assert_array_equal(lo, order)
        np.testing.assert_array_equal(lb, bounds)


def test_plan_rejects_bad_shards():
    lens = np.array([3, 4, 5], np.uint64)
    with pytest.raises(Exception):
        shard.plan(lens, 2, 2, 5)


SPLIT_MIN = 60    # split threshold override: documents of 60+ tokens are split


def _rank(rank, world, port, G, iters, out_q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        off, w, V = corpus()
        K = 11
        lens = np.diff(off.astype(np.int64)).astype(np.uint64)
        D = len(lens)
        cuts = [0, 47, D]
        b, e = cuts[rank], cuts[rank + 1]
        lo, lb, gb, _ = shard.plan(lens, G, b, e - b)
        c = O.Corpus(off, w, V)
        st = O.State(c, K, 0.1, 0.01, seed=5)          # z0 keyed by the global token index
        ar = shard.make_allreduce(memory="host")
        # long documents are split by the rule of the GLOBAL group (its tokens
        # over all ranks), so every rank splits the same documents; a low
        # threshold here makes this small corpus split some
        order_all, _ = single_groups(lens, G)
        gtok = [int(lens[order_all[gb[g]:gb[g + 1]].astype(np.int64)].sum()) for g in range(G)]
        for it in range(iters):
            for g in range(G):
                if gb[g] == gb[g + 1]:
                    continue
                mine = (lo[lb[g]:lb[g + 1]].astype(np.uint64) + np.uint64(b)).copy()
                delta = np.zeros(V * K + K, np.int32)
                dk = delta[:V * K].reshape(V, K)
                dn = delta[V * K:]
                if len(mine):
                    sp = O.SweepSpec(K=K, V=V, alpha=st.alpha.ctypes.data, eta=st.eta, seed=st.seed, iter=it,
                                     doc_off=c.doc_off.ctypes.data, words=c.words.ctypes.data,
                                     ndk=st.ndk.ctypes.data, nkw=st.nkw.ctypes.data, nk=st.nk.ctypes.data,
                                     nkw_next=dk.ctypes.data, nk_next=dn.ctypes.data, z=st.z.ctypes.data,
                                     split_len=O.split_len_of(gtok[g], K, SPLIT_MIN), slices=O.SPLIT_SLICES,
                                     step=O.SPLIT_STEP)
                    O.lib.orc_sweep_docs(C.byref(sp), O._ptr(mine), len(mine))
                assert ar(None, delta.ctypes.data_as(C.c_void_p), len(delta), 0, None) == 0
                st.nkw = st.nkw + dk
                st.nk = st.nk + dn
        ref = O.State(c, K, 0.1, 0.01, seed=5)
        ref.doc_live_sweeps(iters, groups=G, split_min=SPLIT_MIN)
        own = np.zeros(len(w), bool)
        own[int(off[b]):int(off[e])] = True
        ok = (np.array_equal(st.z[own], ref.z[own]) and np.array_equal(st.ndk[b:e], ref.ndk[b:e])
              and np.array_equal(st.nkw, ref.nkw) and np.array_equal(st.nk, ref.nk))
        x = np.array([1.5 * (rank + 1)] * 3, np.float64)    # the f64 path of the callback
        assert ar(None, x.ctypes.data_as(C.c_void_p), 3, 1, None) == 0
        ok = ok and np.allclose(x, 4.5)
        out_q.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("G", [1, 4])
def test_two_gloo_ranks_equal_one_process(G):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, G, 3, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=240) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert res == {0: True, 1: True}


def test_sharded_prepare_equals_whole_corpus():
    off, w = T.synth_corpus(500, 6, 90, ("lognormal", float(np.log(30)), 1.0, 1, 200), seed=8)
    nv = int(w.max()) + 1
    whole = T.prepare_ids(off, w)
    cuts = [0, 31, 90]
    shards = []
    for b, e in zip(cuts[:-1], cuts[1:]):
        shards.append(((off[b:e + 1] - off[b]).astype(np.uint64), w[int(off[b]):int(off[e])]))
    counts = []
    for so, sw in shards:       # each shard's counts, then their sum handed to both
        cf = np.zeros(nv, np.uint64)
        df = np.zeros(nv, np.uint64)
        T._lib.check(T._lib.lib.tmt_corpus_counts(len(so) - 1, shard._p(so), shard._p(np.ascontiguousarray(sw)),
                                                  nv, shard._p(cf), shard._p(df)), None, "counts")
        counts.append((cf, df))
    tot_cf = sum(c[0] for c in counts)
    tot_df = sum(c[1] for c in counts)

    def summed(cf, df):
        cf[:] = tot_cf
        df[:] = tot_df

    outs = [shard.prepare_ids(so, sw, nv, summed) for so, sw in shards]
    assert all(o[2] == whole[2] for o in outs)
    np.testing.assert_array_equal(outs[0][3], whole[3])
    np.testing.assert_array_equal(np.concatenate([o[1] for o in outs]), whole[1])
