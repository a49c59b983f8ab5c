"""Short strings sorted in one CTA's shared memory (prefix doubling with a
block-wide radix sort), singly and as batches, compared with the oracle."""
import numpy as np
import pytest

import oracle_lib as o
import psacak_b200 as pk
from psacak_b200 import synth

pytestmark = pytest.mark.gpu
SMALL_MAX = 8192


@pytest.fixture(scope="module")
def ctx():
    c = pk.Context(0)
    yield c
    c.close()


def edge_texts():
    rng = np.random.default_rng(41)
    ts = [b"ab", b"ba", b"aaaa", b"mississippi", b"\xff" * 8192, b"\xff\x00" * 4096, b"\x00" * 8191 + b"\x01",
          bytes(range(255, -1, -1)) * 32, b"ab" * 4096, b"abc" * 2731]
    ts = [np.frombuffer(t, np.uint8) for t in ts]
    ts += [rng.integers(0, 256, SMALL_MAX).astype(np.uint8), rng.integers(0, 2, SMALL_MAX).astype(np.uint8),
           synth.genome(SMALL_MAX, seed=3), synth.genome(SMALL_MAX - 1, seed=4), synth.genome(SMALL_MAX + 1, seed=5)]
    return ts


def test_edge_cases_single(ctx):
    for t in edge_texts():
        assert (ctx.psacak(t) == o.psacak8(t)).all(), (t.size, bytes(t[:8]))


def test_random_lengths_and_alphabets(ctx):
    rng = np.random.default_rng(42)
    for _ in range(400):
        n = int(rng.integers(2, SMALL_MAX + 1))
        k = int(rng.choice([1, 2, 3, 4, 20, 255, 256]))
        t = rng.integers(0, k, n).astype(np.uint8)
        if rng.random() < 0.3:  # long repeats: many doubling rounds
            p = rng.integers(1, 50)
            t = np.resize(t[:p], n)
        assert (ctx.psacak(t) == o.psacak8(t)).all(), (n, k)


def test_small_u32_levels(ctx):
    rng = np.random.default_rng(43)
    for _ in range(100):
        n = int(rng.integers(4, SMALL_MAX + 1))
        k = int(rng.choice([2, 7, 300, 5000, 1 << 31]))
        t = rng.integers(0, k, n, dtype=np.uint64).astype(np.uint32)
        assert (ctx.psacak32(t) == o.psacak32(t)).all(), (n, k)


def test_batch_of_small_and_large_texts(ctx):
    rng = np.random.default_rng(44)
    lens = np.concatenate([rng.integers(0, SMALL_MAX + 1, 700), rng.integers(SMALL_MAX, 200_000, 30)])
    rng.shuffle(lens)
    texts = [synth.genome(int(k), seed=1000 + i) if k else np.zeros(0, np.uint8) for i, k in enumerate(lens)]
    got = ctx.psacak_batch(texts)
    for t, sa in zip(texts, got):
        assert (sa == o.psacak8(t)).all(), t.size
    # the concatenated build alone (no direct finisher) gives the same arrays
    sched = {"engine": pk.ENGINE_BUCKET, "inner_engine": pk.ENGINE_DOUBLING}
    got0 = ctx.psacak_batch(texts, sched)
    for a, b in zip(got, got0):
        assert (a == b).all()


def test_batch_of_only_small_texts(ctx):
    rng = np.random.default_rng(45)
    texts = [rng.integers(0, int(rng.choice([2, 4, 256])), int(rng.integers(1, 3000))).astype(np.uint8)
             for _ in range(3000)]
    got = ctx.psacak_batch(texts)
    for t, sa in zip(texts, got):
        assert (sa == o.psacak8(t)).all(), t.size
