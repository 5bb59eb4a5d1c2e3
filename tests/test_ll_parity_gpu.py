"""Gate (d) at the benchmark configurations: at the same iteration count,
the device sampler's ll_per_word is within 1% of tomotopy's train() --
ParallelScheme::PARTITION on all host threads with the model defaults
(optim_interval 10, burn_in 0; LDAModel.hpp:210, 436-539, TopicModel.hpp:684-760)
-- averaged over seeds 1..5.  tomotopy's side is the oracle's restatement of
PARTITION, computed once (it is deterministic for a thread count) and kept in
tests/golden/ll_partition.json by tests/golden/make_ll_parity.py:
  c1   the k=20 configuration: V=10k, D=1,000 Poisson(1500) documents, 200 iterations
  c2   the k=100 configuration: V=50k, D=100,000 lognormal(ln 200, 0.8) documents, 500 iterations
  c3s  the k=1000 configuration's generator, first 100,000 documents, 50 iterations"""
import json
import os

import numpy as np
import pytest

import bench

with open(bench.PARITY_FILE) as f:
    REF = json.load(f)["runs"]


@pytest.mark.gpu
@pytest.mark.parametrize("key", sorted(REF))
def test_ll_per_word_within_1pct_of_partition(key):
    r = REF[key]
    run = key.split("/")[0]
    corpus = bench.parity_corpus(run)
    assert corpus[4] == r["corpus_sha1"], "the corpus generator changed: regenerate the fixture"
    g = bench.gpu_parity(run, r["optim_interval"], corpus=corpus)
    cmp = bench.parity_compare(r, g)
    assert cmp["rel_gap"] < 0.01, cmp


def test_fixture_is_complete():
    """Every recorded run holds 5 seeds with one value per 10 iterations."""
    assert REF
    for key, r in REF.items():
        assert sorted(r["ll_per_word"]) == ["1", "2", "3", "4", "5"], key
        for c in r["ll_per_word"].values():
            assert len(c) == r["iters"] // 10 and all(np.isfinite(c)) and all(x < 0 for x in c), key
