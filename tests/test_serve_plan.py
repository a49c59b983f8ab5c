"""Host-side logic of the serving loop (no GPU): the request plan follows the
serving mix, and request texts are windows of the pooled class texts."""
import numpy as np

from psacak_b200 import serve


def test_request_plan_mix_and_lengths():
    plan = serve.request_plan(4000, seed=9, lo=4 << 10, hi=64 << 20)
    lens = np.array([n for n, _, _ in plan])
    assert lens.min() >= 4 << 10 and lens.max() <= 64 << 20
    # log-uniform: the median is near the geometric mean of the bounds
    assert abs(np.log2(np.median(lens)) - 0.5 * (12 + 26)) < 0.5
    counts = {c: sum(1 for _, k, _ in plan if k == c) for c in serve.CLASSES}
    assert all(900 < v < 1100 for v in counts.values()), counts
    assert serve.request_plan(50, seed=9) == serve.request_plan(50, seed=9)


def test_pool_windows():
    pool = serve.TextPool(1 << 16, seed=3, copies=2)
    for c in serve.CLASSES:
        t = pool.text(5000, c, 12345)
        assert t.size == 5000 and t.dtype == (np.uint8 if serve.width_of(c) == 1 else np.uint32)
        full = pool.texts[c][12345 % 2]
        off = (12345 >> 8) % ((1 << 16) - 5000 + 1)
        assert np.array_equal(t, full[off:off + 5000])
    acgt = pool.text(1 << 16, "acgt_iid", 7)
    assert set(np.unique(acgt).tolist()) <= set(b"ACGT")
    assert pool.text(1 << 16, "u32_iid", 7).max() < (1 << 16)
