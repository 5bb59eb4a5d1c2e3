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
