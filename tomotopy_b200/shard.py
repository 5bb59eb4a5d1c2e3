"""A corpus sharded across GPUs, one process per GPU (tomotopy's COPY_MERGE
scheme, LDAModel.hpp:555-570, with the workers on different devices).

Rank r holds the contiguous global documents [doc_begin, doc_begin + D) and a
replica of n_kw / n_k.  The engine cuts its document groups over the global
longest-first order, samples this rank's documents of each group, and after
each group sums the ranks' integer count deltas through `allreduce`
(torch.distributed: NCCL between GPUs, gloo for host buffers).  Draws are
keyed by the global token index, so the result equals one GPU holding the
whole corpus, bit for bit.
"""
import ctypes as C

import numpy as np

from ._lib import lib, check, ALLREDUCE_FN, TmtShard, TMT_I32
from .engine import Engine, _p


class _DeviceView:
    """Zero-copy view of device memory for torch.as_tensor."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def make_allreduce(group=None, memory="device"):
    """An allreduce callback for the engine: in-place SUM over the process
    group of `count` int32 (dtype 0) or float64 (dtype 1) values.  memory =
    "device": the buffer is device memory and the collective is ordered on the
    engine's stream (NCCL); "host": the buffer is host memory (gloo)."""
    import torch
    import torch.distributed as dist

    def cb(user, buf, count, dtype, stream):
        try:
            if count == 0:
                return 0
            if memory == "host":
                ct = C.c_int32 if dtype == TMT_I32 else C.c_double
                arr = np.ctypeslib.as_array(C.cast(buf, C.POINTER(ct)), shape=(int(count),))
                dist.all_reduce(torch.from_numpy(arr), group=group)
                return 0
            typestr = "<i4" if dtype == TMT_I32 else "<f8"
            t = torch.as_tensor(_DeviceView(buf, count, typestr), device="cuda")
            with torch.cuda.stream(torch.cuda.ExternalStream(int(stream or 0))):
                dist.all_reduce(t, group=group)
            return 0
        except Exception:           # the engine turns a nonzero status into an error
            return -1

    return ALLREDUCE_FN(cb)


def prepare_ids(doc_off, words, n_vocab, sum_counts, min_cf=0, min_df=0, rm_top=0):
    """engine.prepare_ids for one shard of a corpus split across processes:
    sum_counts(cf, df) sums the shards' (cf, df) arrays (uint64, n_vocab) in
    place, so every shard gets one vocabulary order.  Returns (doc_off, words,
    realV, order)."""
    doc_off = np.ascontiguousarray(doc_off, dtype=np.uint64)
    words = np.ascontiguousarray(words, dtype=np.uint32)
    D = len(doc_off) - 1
    cf = np.zeros(max(n_vocab, 1), np.uint64)
    df = np.zeros(max(n_vocab, 1), np.uint64)
    check(lib.tmt_corpus_counts(D, _p(doc_off), _p(words), n_vocab, _p(cf), _p(df)), None, "tmt_corpus_counts")
    sum_counts(cf, df)
    out = np.zeros(max(len(words), 1), np.uint32)
    order = np.zeros(max(n_vocab, 1), np.uint32)
    rv = C.c_uint32()
    check(lib.tmt_prepare_corpus_counted(D, _p(doc_off), _p(words), n_vocab, _p(cf), _p(df), min_cf, min_df, rm_top,
                                         _p(out), None, _p(order), C.byref(rv)), None, "tmt_prepare_corpus_counted")
    return doc_off, out[:len(words)], int(rv.value), order[:n_vocab]


def plan(doc_len_global, groups, doc_begin, D_local):
    """tmt_plan_shard: (local_order, local_bounds, global_bounds, token_offset)."""
    lens = np.ascontiguousarray(doc_len_global, dtype=np.uint64)
    G = max(1, int(groups))
    order = np.zeros(max(int(D_local), 1), np.uint32)
    lb = np.zeros(G + 1, np.uint64)
    gb = np.zeros(G + 1, np.uint64)
    off = C.c_uint64()
    check(lib.tmt_plan_shard(_p(lens), len(lens), G, int(doc_begin), int(D_local), _p(order), _p(lb), _p(gb),
                             C.byref(off)), None, "tmt_plan_shard")
    return order[:int(D_local)], lb, gb, int(off.value)


class ShardedEngine(Engine):
    """An Engine holding one rank's documents of a corpus split across
    processes.  train(), ll() and anything that optimises alpha are
    collective: every rank calls them in the same order."""

    def upload_shard(self, doc_off, words, doc_len_global, doc_begin, rank, world, group=None, z0=None,
                     memory="device", allreduce=None):
        """doc_off / words: this rank's documents (doc_off from 0);
        doc_len_global: every rank's document lengths, rank order; allreduce:
        an ALLREDUCE_FN to use instead of torch.distributed over `group`."""
        self._doc_off = np.ascontiguousarray(doc_off, dtype=np.uint64)
        self._words = np.ascontiguousarray(words, dtype=np.uint32)
        self._lens = np.ascontiguousarray(doc_len_global, dtype=np.uint64)
        zz = np.ascontiguousarray(z0, dtype=np.uint16) if z0 is not None else None
        self.D = len(self._doc_off) - 1
        self.n_all = int(self._doc_off[-1]) if self.D >= 0 else 0
        if allreduce is not None:
            self._ar = allreduce
        else:
            self._ar = make_allreduce(group, memory) if world > 1 else ALLREDUCE_FN()
        sh = TmtShard(rank=int(rank), world=int(world), D_global=len(self._lens), doc_begin=int(doc_begin),
                      doc_len_global=self._lens.ctypes.data_as(C.c_void_p), allreduce=self._ar, user=None)
        check(lib.tmt_upload_shard(self.h, _p(self._words), _p(self._doc_off), self.D, _p(zz), C.byref(sh)), self.h)
