"""Host-side helpers of the engine binding (no GPU)."""
import numpy as np

from tomotopy_b200.engine import pack_topic_mask


def test_pack_topic_mask_bit_layout():
    rng = np.random.default_rng(1)
    for K in (1, 20, 32, 33, 70, 1000):
        m = rng.random((5, K)) < 0.4
        words = pack_topic_mask(m, K)
        assert words.dtype == np.uint32 and words.shape == (5, (K + 31) // 32)
        for d in range(5):
            for k in range(K):
                assert bool((words[d, k >> 5] >> (k & 31)) & 1) == bool(m[d, k])
            # no bits beyond K
            for k in range(K, words.shape[1] * 32):
                assert not (words[d, k >> 5] >> (k & 31)) & 1


def test_bench_idf_weights_match_oracle():
    """bench.py --tw idf computes TermWeight IDF per token from the prepared
    corpus's sorted runs; the oracle counts document frequencies directly."""
    import os
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import bench
    import oracle as O
    import tomotopy_b200 as T
    off, w = T.synth_corpus(3000, 12, 400, ("lognormal", float(np.log(80)), 1.0, 1, 900), seed=11)
    off, w, V, _ = T.prepare_ids(off, w, min_cf=3)    # drops rare words: ids >= V at each document's end
    o = off.astype(np.int64)
    w = np.delete(w, np.arange(o[5], o[6]))          # an empty document
    lens = np.diff(o)
    lens[5] = 0
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    got = bench.idf_weights(off, w, V)
    want, _ = O.weights_idf(O.Corpus(off, w, V))
    assert np.array_equal(got, want)
    assert np.any(w >= V)
