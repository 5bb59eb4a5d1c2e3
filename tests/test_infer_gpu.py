"""Inference (tomotopy's LDAModel.infer, together=False) on the device,
checked against the oracle's restatement document by document: theta
bit-exact, FP64 log-likelihood to 1e-12 relative."""
import numpy as np
import pytest

import oracle as O
import tomotopy_b200 as T

pytestmark = pytest.mark.gpu


def trained(K, V=900, D=150, seed=3, sweeps=20, alpha=0.1):
    off, w = T.synth_corpus(V, 10, D, ("poisson", 80, 1, 800), seed=seed)
    off, w, Vr, order = T.prepare_ids(off, w, min_cf=2)
    eng = T.Engine(K, Vr, alpha=alpha, eta=0.01, seed=seed, optim_interval=0)
    eng.upload(off, w)
    eng.train(sweeps)
    return eng, Vr, order


def new_docs(order, n, seed, V_out):
    off, w = T.synth_corpus(len(order), 10, n, ("lognormal", np.log(60), 1.0, 1, 600), seed=seed)
    w = np.where(w < len(order), order[np.minimum(w, len(order) - 1)], V_out + 5).astype(np.uint32)
    return off, w


def oracle_infer(eng, off, w, iters, seed, keys=None):
    _, nkw, nk, alpha = eng.state()
    th, lls = [], []
    for d in range(len(off) - 1):
        doc = np.sort(w[off[d]:off[d + 1]], kind="stable")
        key = int(keys[d]) if keys is not None else 0
        ll, _, _, theta = O.infer_doc(eng.K, eng.V, alpha, 0.01, nkw, nk, doc, iters, seed, key)
        th.append(theta)
        lls.append(ll)
    return np.array(th), np.array(lls)


@pytest.mark.parametrize("K", [7, 20, 100, 300, 1000])
def test_infer_matches_oracle(K):
    eng, V, order = trained(K)
    off, w = new_docs(order, 60, seed=11, V_out=V)
    theta, ll = eng.infer(off, w, iters=30, seed=5)
    ot, ol = oracle_infer(eng, off, w, 30, 5)
    np.testing.assert_array_equal(theta, ot)
    np.testing.assert_allclose(ll, ol, rtol=1e-12, atol=1e-9)


def test_infer_edge_documents_and_keys():
    K = 24
    eng, V, order = trained(K, V=400, D=80)
    docs = [
        np.zeros(0, np.uint32),                                  # empty
        np.full(5, V + 3, np.uint32),                            # every word outside the vocabulary
        np.full(100, 7, np.uint32),                              # one word, a run longer than a warp
        np.array([5, 1, 5, 2, 1, 5, V + 1, 0], np.uint32),       # unsorted, repeats, one unknown
        np.arange(min(V, 300), dtype=np.uint32)[::-1].copy(),    # many distinct words
    ]
    off = np.concatenate([[0], np.cumsum([len(x) for x in docs])]).astype(np.uint64)
    w = np.concatenate(docs).astype(np.uint32)
    keys = np.array([3, 9, 27, 81, 243], np.uint64)
    theta, ll = eng.infer(off, w, iters=40, seed=2, doc_keys=keys)
    ot, ol = oracle_infer(eng, off, w, 40, 2, keys)
    np.testing.assert_array_equal(theta, ot)
    np.testing.assert_allclose(ll, ol, rtol=1e-12, atol=1e-9)
    _, _, _, alpha = eng.state()
    np.testing.assert_allclose(theta[0], alpha / alpha.sum(), rtol=1e-6)
    assert ll[0] == 0.0 and ll[1] == 0.0


def test_infer_is_batch_independent_and_leaves_model_unchanged():
    K = 50
    eng, V, order = trained(K)
    before = eng.state()
    off, w = new_docs(order, 40, seed=21, V_out=V)
    theta, ll = eng.infer(off, w, iters=25, seed=9)
    # the same documents one at a time and reversed: identical results
    for d in (0, 17, 39):
        t1, l1 = eng.infer(np.array([0, off[d + 1] - off[d]], np.uint64), w[off[d]:off[d + 1]], iters=25, seed=9)
        np.testing.assert_array_equal(t1[0], theta[d])
        assert l1[0] == ll[d]
    after = eng.state()
    for a, b in zip(before, after):
        np.testing.assert_array_equal(a, b)
