"""Long documents sampled by a block in slices (k_sweep_doc phase 1): z and
every count equal the oracle's restatement (orc_sweep_docs) bit for bit --
a document of at least split_len tokens is cut into 8 contiguous slices
sampled side by side, each with a private copy of the document's row that
takes in the other slices' changes every `step` positions -- for the
engine's rule and for set thresholds and steps, with word priors and with
per-document masks / alphas, and the split never depends on timing."""
import numpy as np
import pytest

import oracle as O
import tomotopy_b200 as T

pytestmark = pytest.mark.gpu


def long_corpus(V=1500, D=90, seed=21):
    """Lognormal lengths up to 3,000 tokens, a few words outside the vocabulary."""
    off, w = T.synth_corpus(V, 12, D, ("lognormal", float(np.log(250)), 1.0, 1, 3000), seed=seed)
    off, w, V, _ = T.prepare_ids(off, w)
    w = w.copy()
    w[::173] = V + 2
    return off, w, V


def assert_same(eng, st):
    z, nkw, nk, _ = eng.state()
    np.testing.assert_array_equal(z, st.z)
    np.testing.assert_array_equal(nk, st.nk)
    np.testing.assert_array_equal(nkw, st.nkw)
    np.testing.assert_array_equal(eng.doc_topic(), st.ndk)


@pytest.mark.parametrize("K", [1, 7, 20, 100, 300, 512])
@pytest.mark.parametrize("groups", [1, 3])
def test_split_rule_bitexact(K, groups):
    off, w, V = long_corpus()
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=4, optim_interval=0, sweep_groups=groups)
    eng.upload(off, w)
    lens = np.diff(off.astype(np.int64))
    # a small corpus: every group's threshold is the rule's floor, 8 stale windows
    assert sum(eng.doc_split()) == int(np.sum(lens >= O.split_len_of(0, K))) > 0
    st = O.State(O.Corpus(off, w, V), K, 0.1, 0.01, 4)
    for step in range(3):
        eng.train(1)
        st.doc_live_sweeps(1, start_step=step, groups=groups)
        assert_same(eng, st)


@pytest.mark.parametrize("min_tokens,step", [(40, 4), (100, 16), (1, 32), (700, 1)])
def test_split_settings_bitexact(min_tokens, step):
    off, w, V = long_corpus(seed=22)
    K = 50
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=5, optim_interval=0, sweep_groups=2)
    eng.set_doc_split(min_tokens, step)
    eng.upload(off, w)
    st = O.State(O.Corpus(off, w, V), K, 0.1, 0.01, 5)
    eng.train(3)
    st.doc_live_sweeps(3, groups=2, split_min=min_tokens, split_step=step)
    assert_same(eng, st)


def test_no_split_above_k512_and_when_disabled():
    off, w, V = long_corpus(seed=23)
    eng = T.Engine(513, V, alpha=0.1, eta=0.01, seed=6, optim_interval=0)
    eng.upload(off, w)
    assert sum(eng.doc_split()) == 0
    eng2 = T.Engine(64, V, alpha=0.1, eta=0.01, seed=6, optim_interval=0)
    eng2.set_doc_split(2 ** 32 - 1)
    eng2.upload(off, w)
    assert sum(eng2.doc_split()) == 0
    st = O.State(O.Corpus(off, w, V), 64, 0.1, 0.01, 6)
    eng2.train(2)
    st.doc_live_sweeps(2, groups=8, split_min=2 ** 32 - 1)
    assert_same(eng2, st)


def test_split_with_word_priors_bitexact():
    off, w, V = long_corpus(seed=24)
    K = 40
    rng = np.random.default_rng(2)
    ids = np.sort(rng.choice(V, 25, replace=False)).astype(np.uint32)
    pri = rng.uniform(0, 0.5, (len(ids), K)).astype(np.float32)
    pri[pri < 0.15] = 0
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=8, optim_interval=0, sweep_groups=2)
    eng.set_word_priors(ids, pri)
    eng.set_doc_split(60, 8)
    eng.upload(off, w)
    st = O.StateP(O.Corpus(off, w, V), K, 0.1, 0.01, 8, ids, pri)
    assert_same(eng, st)
    eng.train(3)
    st.doc_live_sweeps(3, groups=2, split_min=60, split_step=8)
    assert_same(eng, st)


def test_split_with_masks_and_doc_alphas_bitexact():
    off, w, V = long_corpus(seed=25)
    K = 30
    D = len(off) - 1
    rng = np.random.default_rng(3)
    mask = rng.random((D, K)) < 0.5
    mask[np.arange(D), rng.integers(0, K, D)] = True
    # z0 inside each document's labels
    z0 = np.zeros(len(w), np.uint16)
    for d in range(D):
        allowed = np.flatnonzero(mask[d])
        z0[off[d]:off[d + 1]] = rng.choice(allowed, int(off[d + 1] - off[d]))
    rows = rng.uniform(0.05, 0.5, (4, K)).astype(np.float32)
    doc_row = rng.integers(0, 4, D).astype(np.uint32)
    eng = T.Engine(K, V, alpha=0.1, eta=0.01, seed=9, optim_interval=0, sweep_groups=3)
    eng.set_doc_split(80, 16)
    eng.upload(off, w, z0=z0)
    eng.set_doc_topic_mask(mask)
    eng.set_doc_alpha(rows, doc_row)
    st = O.StateM(O.Corpus(off, w, V), K, 0.1, 0.01, 9, z0, mask=mask, alpha_rows=rows, doc_row=doc_row)
    eng.train(3)
    st.doc_live_sweeps(3, groups=3, split_min=80, split_step=16)
    assert_same(eng, st)
    z = eng.state()[0]
    ok = w < V
    doc = np.repeat(np.arange(D), np.diff(off.astype(np.int64)))
    assert mask[doc[ok], z[ok].astype(np.int64)].all()


def test_split_graphs_identical_to_launches():
    """Captured sweeps carry the split launches unchanged."""
    off, w, V = long_corpus(seed=26)
    res = []
    for graphs in (True, False):
        eng = T.Engine(20, V, alpha=0.1, eta=0.01, seed=10, optim_interval=5)
        eng.set_graphs(graphs)
        eng.upload(off, w)
        eng.train(14)
        res.append(eng.state()[0])
    np.testing.assert_array_equal(res[0], res[1])
