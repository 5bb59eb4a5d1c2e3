"""A corpus sharded across ranks, on the device: two ShardedEngine ranks on
one GPU, each driven by its own host thread, exchange their count deltas
through a host-side allreduce (copy out, sum, copy back; the threads meet at a
barrier, no kernel waits on another).  z, n_dk and every count must equal one
engine holding the whole corpus, bit for bit."""
import threading

import numpy as np
import pytest

import tomotopy_b200 as T
from tomotopy_b200 import shard
from tomotopy_b200._lib import ALLREDUCE_FN, TMT_I32

pytestmark = pytest.mark.gpu


def corpus(D=400, V=900, seed=12):
    off, w = T.synth_corpus(V, 10, D, ("lognormal", float(np.log(60)), 1.1, 1, 800), seed=seed)
    off, w, V, _ = T.prepare_ids(off, w)
    w = w.copy()
    w[::211] = V + 3                      # words outside the vocabulary
    return off, w, V


class HostAllreduce:
    """allreduce for `world` ranks living in one process (one thread each)."""

    def __init__(self, world):
        import torch
        self.torch = torch
        self.world = world
        self.bar = threading.Barrier(world, timeout=120)
        self.bufs = [None] * world
        self.calls = 0

    def fn(self, rank):
        torch = self.torch

        def cb(user, buf, count, dtype, stream):
            try:
                torch.cuda.ExternalStream(int(stream)).synchronize()
                typestr = "<i4" if dtype == TMT_I32 else "<f8"
                t = torch.as_tensor(shard._DeviceView(buf, count, typestr), device="cuda")
                self.bufs[rank] = t.cpu()
                self.bar.wait()
                total = sum(self.bufs)
                self.bar.wait()
                t.copy_(total.to("cuda"))
                torch.cuda.synchronize()
                if rank == 0:
                    self.calls += 1
                return 0
            except Exception:
                return -1
        return ALLREDUCE_FN(cb)


def run_sharded(off, w, V, K, cuts, iters, groups, optim, ll=True, split=None):
    world = len(cuts) - 1
    lens = np.diff(off.astype(np.int64)).astype(np.uint64)
    har = HostAllreduce(world)
    engines, out, errs = [], [None] * world, []

    def rank_main(r):
        try:
            b, e = cuts[r], cuts[r + 1]
            loff = (off[b:e + 1] - off[b]).astype(np.uint64)
            lw = w[int(off[b]):int(off[e])]
            eng = shard.ShardedEngine(K, V, alpha=0.1, eta=0.01, seed=9, optim_interval=optim,
                                      sweep_groups=groups)
            engines.append(eng)
            if split:
                eng.set_doc_split(*split)
            eng.upload_shard(loff, lw, lens, b, r, world, allreduce=har.fn(r))
            eng.train(iters)
            z, nkw, nk, alpha = eng.state()
            ndk = eng.doc_topic()
            lld = eng.ll() if ll else None
            out[r] = (z, nkw, nk, alpha, ndk, lld)
        except Exception as ex:       # surfaced below
            errs.append(ex)
            har.bar.abort()

    ts = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=600)
    assert not errs, errs
    for eng in engines:
        eng.close()
    return out, har.calls


def run_single(off, w, V, K, iters, groups, optim, split=None):
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=9, optim_interval=optim, sweep_groups=groups)
    if split:
        eng.set_doc_split(*split)
    eng.upload(off, w)
    eng.train(iters)
    z, nkw, nk, alpha = eng.state()
    res = (z, nkw, nk, alpha, eng.doc_topic(), eng.ll())
    eng.close()
    return res


@pytest.mark.parametrize("K,groups,cuts,split", [(24, 4, [0, 150, 400], None), (130, 1, [0, 250, 400], None),
                                                 (40, 8, [0, 90, 260, 400], None),
                                                 (24, 3, [0, 150, 400], (50, 8))])
def test_sharded_equals_one_gpu(K, groups, cuts, split):
    """split: a low threshold, so many documents are split; the split of
    each group follows the global group, so every rank splits alike."""
    off, w, V = corpus()
    iters = 4
    ref = run_single(off, w, V, K, iters, groups, 0, split)
    out, calls = run_sharded(off, w, V, K, cuts, iters, groups, 0, split=split)
    z = np.concatenate([o[0] for o in out])
    np.testing.assert_array_equal(z, ref[0])
    for o in out:
        np.testing.assert_array_equal(o[1], ref[1])       # n_kw replicas
        np.testing.assert_array_equal(o[2], ref[2])
    np.testing.assert_array_equal(np.concatenate([o[4] for o in out]), ref[4])
    for o in out:            # LLDocs summed over ranks (FP64 sums in another order), LLRest replicated
        assert o[5][0] == pytest.approx(ref[5][0], rel=1e-12)
        assert o[5][1] == ref[5][1]
        assert o[5] == out[0][5]
    assert calls >= 2 + iters * 1                          # counts at upload, then per group


def test_sharded_alpha_optimisation():
    off, w, V = corpus()
    K, iters = 30, 6
    ref = run_single(off, w, V, K, iters, 2, 2)
    out, _ = run_sharded(off, w, V, K, [0, 200, 400], iters, 2, 2, ll=False)
    for o in out:
        np.testing.assert_allclose(o[3], ref[3], rtol=1e-6)   # alpha: FP64 sums reduced in another order
        np.testing.assert_array_equal(o[3], out[0][3])       # identical on every rank
    z = np.concatenate([o[0] for o in out])
    assert np.mean(z == ref[0]) > 0.99
