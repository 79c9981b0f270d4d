"""The batched solver's bucket plan (zolo_batch_plan, host only): every member in exactly one
bucket, padded sizes covering their members, the optimized split never predicted slower than
the fixed size ladder, and the latency / padding trade-off moving the split the right way."""
import math

import numpy as np

import zolo_svd_b200 as zb


def config4_sizes(seed=1004, count=512):
    rng = np.random.default_rng(seed)
    m, n = [], []
    for _ in range(count):
        nn = int(round(math.exp(rng.uniform(math.log(64), math.log(1024)))))
        mm = int(round(nn * (1 + rng.uniform(0, 1))))
        rng.uniform(2, 14)
        m.append(mm)
        n.append(nn)
    return np.array(m), np.array(n)


def check_cover(m, n, bucket, pads):
    assert len(bucket) == len(n)
    seen = np.zeros(len(pads), dtype=int)
    for i, b in enumerate(bucket):
        mb, nb = pads[b]
        assert nb % 32 == 0 and mb % 32 == 0
        assert nb >= n[i] and mb >= m[i] + nb - n[i]  # the member fits with its identity padding
        seen[b] += 1
    assert np.all(seen > 0)


def test_plan_covers_config4_and_beats_ladder():
    m, n = config4_sizes()
    bucket, pads, pred = zb.batch_plan(m, n)
    check_cover(m, n, bucket, pads)
    lb, lpads, lpred = zb.batch_plan(m, n, mode=1)
    check_cover(m, n, lb, lpads)
    assert pred <= lpred * (1 + 1e-12)


def test_same_size_members_share_one_bucket():
    m = np.full(300, 700)
    n = np.full(300, 500)
    bucket, pads, _ = zb.batch_plan(m, n)
    assert set(bucket.tolist()) == {0} and pads == [(736, 512)]  # 700 + 12 identity rows, to 32


def test_max_batch_splits_buckets():
    m = np.full(10, 64)
    n = np.full(10, 64)
    bucket, pads, _ = zb.batch_plan(m, n, max_batch=4)
    assert len(pads) == 3 and np.bincount(bucket).max() <= 4


def test_latency_versus_padding_tradeoff():
    rng = np.random.default_rng(3)
    n = rng.integers(40, 900, 200)
    m = n + rng.integers(0, 300, 200)
    high_latency = [50.0, 5.0, 25.0, 384.0, 4]
    no_latency = [0.0, 0.0, 25.0, 384.0, 4]
    _, p_hi, _ = zb.batch_plan(m, n, high_latency)
    _, p_lo, _ = zb.batch_plan(m, n, no_latency)
    assert len(p_hi) < len(p_lo)
    # without latency every distinct padded n is its own bucket (padding only costs)
    assert len(p_lo) == len(set(((n + 31) // 32 * 32).tolist())) or len(p_lo) >= len(p_hi)


def test_empty_and_bad_input():
    bucket, pads, pred = zb.batch_plan([], [])
    assert pads == [] and pred == 0.0
    import pytest
    with pytest.raises(zb.ZoloError):
        zb.batch_plan([5], [10])  # m < n
