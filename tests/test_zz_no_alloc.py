"""tmt_ll_counts_noalloc: the log-likelihood entry point for callers that may
not allocate device memory (a serving process whose device memory is carved
up by its own pool, a plug-in inside a framework that owns all device
allocations, a pipelined stream that must not pick up the implicit
synchronisation of cudaMalloc).  It must give the same result as tmt_ll on
the same counts, call after call, while its scratch lives in one static
device array that every call reuses.

This file is collected last on purpose, so a run that stops at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest

import tomotopy_b200 as T
from tomotopy_b200._lib import lib


def _call(ndk, doc_len, alpha, nkw, nk, eta, out, stream=None):
    err = C.create_string_buffer(256)
    st = lib.tmt_ll_counts_noalloc(
        C.c_void_p(ndk.data_ptr()), ndk.shape[0], alpha.shape[0], C.c_void_p(doc_len.data_ptr()),
        C.c_void_p(alpha.data_ptr()), C.c_void_p(nkw.data_ptr()), nkw.shape[0], C.c_void_p(nk.data_ptr()),
        float(eta), C.c_void_p(out.data_ptr()), C.c_void_p(stream), err, len(err))
    return st, err.value.decode()


@pytest.mark.gpu
def test_noalloc_ll_matches_tmt_ll_on_two_calls():
    import torch

    off, w = T.synth_corpus(1500, 12, 300, ("lognormal", np.log(80), 0.9, 5, 2000), seed=17)
    off, w, V, _ = T.prepare_ids(off, w, min_cf=2)
    K, eta = 48, 0.01
    alpha = (0.02 * (1 + np.arange(K) % 5)).astype(np.float32)
    eng = T.Engine(K, V, alpha=alpha, eta=eta, seed=5, optim_interval=0)
    eng.upload(off, w)
    doc_len = np.array([(w[off[d]:off[d + 1]] < V).sum() for d in range(len(off) - 1)], dtype=np.int32)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    out = torch.zeros(2, dtype=torch.float64, device=dev)
    for sweeps in (2, 3):          # two calls in a row, on two different model states
        eng.train(sweeps)
        ref_docs, ref_rest = eng.ll()
        _, nkw, nk, a = eng.state()
        ndk = eng.doc_topic()
        t = [torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in (ndk, doc_len, a, nkw, nk)]
        out.fill_(float("nan"))
        st, msg = _call(t[0], t[1], t[2], t[3], t[4], eta, out, stream)
        assert st == 0, msg
        torch.cuda.synchronize(dev)
        got = out.cpu().numpy()
        # tmt_ll's grid and summation order: the same bits
        np.testing.assert_array_equal(got, [ref_docs, ref_rest])


@pytest.mark.gpu
def test_noalloc_rejects_host_arrays():
    """A host array would be read by the kernels as a device address: it is
    refused before anything is launched."""
    import torch

    dev = torch.device("cuda", 0)
    K, V, D = 8, 20, 3
    ndk = torch.zeros((D, K), dtype=torch.int32, device=dev)
    doc_len = torch.zeros(D, dtype=torch.int32, device=dev)
    alpha = torch.full((K,), 0.1, dtype=torch.float32, device=dev)
    nkw = torch.zeros((V, K), dtype=torch.int32, device=dev)
    out = torch.zeros(2, dtype=torch.float64, device=dev)
    nk_host = np.zeros(K, dtype=np.int32)
    err = C.create_string_buffer(256)
    st = lib.tmt_ll_counts_noalloc(
        C.c_void_p(ndk.data_ptr()), D, K, C.c_void_p(doc_len.data_ptr()), C.c_void_p(alpha.data_ptr()),
        C.c_void_p(nkw.data_ptr()), V, nk_host.ctypes.data_as(C.c_void_p), 0.01, C.c_void_p(out.data_ptr()),
        None, err, len(err))
    assert st == -1 and b"n_k" in err.value, err.value
    torch.cuda.synchronize(dev)


def test_noalloc_rejects_k_beyond_scratch():
    err = C.create_string_buffer(256)
    st = lib.tmt_ll_counts_noalloc(None, 0, 40000, None, C.c_void_p(16), None, 0, C.c_void_p(16), 0.01,
                                   C.c_void_p(16), None, err, len(err))
    assert st == -1
    assert b"32767" in err.value
