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
  sampling from a random start does on data drawn from the model;
- the same seed gives the same z, another seed another z;
- with TermWeight IDF token weights (LDAModel.hpp:1093-1122), n_k and n_kw
  each sum to the total weight of the corpus;
- inference of unseen documents (LDAModel::_infer, LDAModel.hpp:920-953)
  against the full model gives a document the same theta and ll whatever
  batch it comes in, and theta rows sum to 1.

The recount runs on the device with torch bincount: it is the checker, not
the path under test."""
import math

import numpy as np
import pytest

import tomotopy_b200 as T

V_GEN, TOPICS, D, K = 100000, 1000, 1000000, 1000
LENGTH = ("lognormal", float(np.log(100)), 1.2, 5, 5000)
SEED = 20261206


@pytest.fixture(scope="module")
def corpus():
    off, words = T.synth_corpus(V_GEN, TOPICS, D, LENGTH, seed=SEED)
    return T.prepare_ids(off, words)      # (doc_off, words, V, vocabulary order)


@pytest.mark.gpu
def test_full_size_counts_match_z_and_ll_rises(corpus):
    import torch

    off, words, V, _ = corpus
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


@pytest.mark.gpu
def test_full_size_same_seed_same_z(corpus):
    off, words, V, _ = corpus
    zs = []
    for seed in (7, 7, 8):
        eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=seed, optim_interval=0)
        eng.upload(off, words)
        eng.train(2)
        zs.append(eng.state()[0])
        eng.close()
    assert np.array_equal(zs[0], zs[1])
    assert not np.array_equal(zs[0], zs[2])


def _idf(off, words, V):
    """(float)log(D / df(w)) per token, df over documents (LDAModel.hpp:1093-1122);
    each prepared document holds its words sorted, so a run start is a new word."""
    o = off.astype(np.int64)
    first = np.ones(len(words), bool)
    first[1:] = words[1:] != words[:-1]
    first[o[:-1][np.diff(o) > 0]] = True
    ok = words < V
    df = np.bincount(words[first & ok], minlength=V)[:V]
    idf = np.log((len(off) - 1) / np.maximum(df, 1).astype(np.float64)).astype(np.float32)
    return np.where(ok, idf[np.minimum(words, V - 1)], np.float32(0)).astype(np.float32)


@pytest.mark.gpu
def test_full_size_idf_counts_sum_to_total_weight(corpus):
    off, words, V, _ = corpus
    wts = _idf(off, words, V)
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=3, optim_interval=0)
    eng.upload(off, words, weights=wts)
    eng.train(2)
    _, nkw, nk, _ = eng.state()
    eng.close()
    total = float(wts.astype(np.float64).sum())
    assert float(nk.astype(np.float64).sum()) == pytest.approx(total, rel=1e-3)
    assert float(nkw.astype(np.float64).sum()) == pytest.approx(total, rel=1e-3)
    assert (nk >= 0).all() and (nkw >= 0).all()


@pytest.mark.gpu
def test_full_size_infer_is_batch_independent(corpus):
    off, words, V, order = corpus
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=5, optim_interval=0)
    eng.upload(off, words)
    eng.train(2)
    noff, nw = T.synth_corpus(V_GEN, TOPICS, 4000, LENGTH, seed=SEED + 1)
    # generator ids -> the model's vocabulary; words it never saw become out-of-vocabulary
    nw = np.where(nw < len(order), order[np.minimum(nw, len(order) - 1)], V + 5).astype(np.uint32)
    theta, ll = eng.infer(noff, nw, iters=20, seed=9)
    assert np.isfinite(ll).all()
    np.testing.assert_allclose(theta.sum(axis=1), 1.0, atol=1e-4)
    t2, l2 = eng.infer(noff[:1001], nw[:int(noff[1000])], iters=20, seed=9)
    np.testing.assert_array_equal(t2, theta[:1000])
    np.testing.assert_array_equal(l2, ll[:1000])
    for d in (0, 1234, 3999):
        a, b = int(noff[d]), int(noff[d + 1])
        t1, l1 = eng.infer(np.array([0, b - a], np.uint64), nw[a:b], iters=20, seed=9)
        np.testing.assert_array_equal(t1[0], theta[d])
        assert l1[0] == ll[d]
    eng.close()
