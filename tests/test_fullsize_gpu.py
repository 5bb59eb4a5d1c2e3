"""The training sweep at the benchmark's full size (K=1000, V=100,000,
D=1,000,000 documents, ~204M tokens; the seeded synthetic LDA corpus the
bench times), checked through properties that do not depend on the size,
since the oracle's sequential sweep cannot finish there:

- n_kw and n_k equal the counts recounted from the downloaded z
  (tomotopy's mergeState invariant, LDAModel.hpp:552-604);
- every word's n_kw row sums to that word's token count, whatever z is;
- n_k sums to the number of valid tokens N;
- the FP64 log-likelihood (getLLDocs + getLLRest, LDAModel.hpp:616-668) is
  finite and rises from the first sweep to the third, as collapsed Gibbs
  sampling from a random start does on data drawn from the model.

The recount runs on the device with torch bincount: it is the checker, not
the path under test."""
import math

import numpy as np
import pytest

import tomotopy_b200 as T

V_GEN, TOPICS, D, K = 100000, 1000, 1000000, 1000
LENGTH = ("lognormal", float(np.log(100)), 1.2, 5, 5000)
SEED = 20261206


@pytest.mark.gpu
def test_full_size_counts_match_z_and_ll_rises():
    import torch

    off, words = T.synth_corpus(V_GEN, TOPICS, D, LENGTH, seed=SEED)
    off, words, V, _ = T.prepare_ids(off, words)
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=1, optim_interval=0)
    eng.upload(off, words)
    N = eng.info().N
    assert N > 150_000_000

    eng.train(1)
    ll1 = sum(eng.ll())
    eng.train(2)
    ll3 = sum(eng.ll())
    assert math.isfinite(ll1) and math.isfinite(ll3)
    assert ll3 > ll1

    z, nkw, nk, _ = eng.state()
    eng.close()
    assert nkw.shape == (V, K)
    assert int(nk.astype(np.int64).sum()) == N

    dev = torch.device("cuda", 0)
    w = torch.from_numpy(words.astype(np.int64)).to(dev)
    zt = torch.from_numpy(z.astype(np.int32)).to(dev).long()
    valid = w < V
    assert int(valid.sum()) == N
    w, zt = w[valid], zt[valid]
    assert int(zt.max()) < K
    cf = torch.bincount(w, minlength=V)
    rec_nk = torch.bincount(zt, minlength=K)
    rec_nkw = torch.bincount(w * K + zt, minlength=V * K).view(V, K)
    del w, zt

    nkw_d = torch.from_numpy(nkw).to(dev)
    assert torch.equal(nkw_d.long().sum(dim=1), cf)
    assert torch.equal(torch.from_numpy(nk).to(dev).long(), rec_nk)
    assert torch.equal(nkw_d.long(), rec_nkw)
