"""Prefix doubling of a whole string (sort_by_doubling) on the GPU against the
oracle, on inputs that reach each of its paths:

* the packed first round at its extremes: one distinct symbol (16 symbols
  packed, the cap), bytes (7 packed), integer names of ~2^21 values (2);
* group-ordered rounds (work lists of 2^20 items or more, at most 16 items
  per group on average): groups of at most 64 items sorted in shared
  memory beside groups of 65 and more gathered, radix-sorted and put back,
  with repeats of exactly 64 and 65 copies at the boundary;
* full rounds over lists whose groups are large (periodic texts).

Byte texts take finish_below = "always" (prefix doubling from the text),
integer texts the library default (prefix doubling below 2^30 symbols).
Every suffix array is compared with the oracle's element by element.
"""
import numpy as np
import pytest

import oracle_lib as o
import psacak_b200 as pk
from psacak_b200 import synth

pytestmark = pytest.mark.gpu
ALWAYS = 0xFFFFFFFF
BYTES_BY_DOUBLING = {"engine": pk.ENGINE_BUCKET, "inner_engine": pk.ENGINE_DOUBLING, "tile_items": 16,
                     "finish_below": ALWAYS, "inner_finish_below": 1 << 30}


@pytest.fixture(scope="module")
def ctx():
    c = pk.Context(0)
    yield c
    c.close()


def paired_with_repeats(rng, alphabet, dtype, copies):
    """A random region and its copy (2^20 suffix pairs that stay unresolved
    for many rounds: small groups), then a 300-symbol block repeated
    `copies[k]` times for each k (groups of exactly that many items once the
    prefixes exceed the block), then random symbols."""
    region = rng.integers(0, alphabet, 1 << 20).astype(dtype)
    parts = [region, region.copy()]
    for k in copies:
        block = rng.integers(0, alphabet, 300).astype(dtype)
        parts.append(np.tile(block, k))
    parts.append(rng.integers(0, alphabet, 200_000).astype(dtype))
    return np.concatenate(parts)


def direct(trace):
    """The build sorted the input directly (one level, no LMS recursion)."""
    return len(trace) == 1 and trace[0]["n_lms"] == 0


def profiled(ctx, build):
    """Runs build() with the kernel profiler on; returns the launched classes."""
    ctx.profile_reset()
    ctx.profile(True)
    try:
        out = build()
    finally:
        ctx.profile(False)
    return out, {s["name"]: s["launches"] for s in ctx.profile_stats() if s["launches"]}


@pytest.mark.parametrize("copies", [(64, 65), (3, 100, 400)])
def test_bytes_group_ordered_rounds_with_large_groups(ctx, copies):
    rng = np.random.default_rng(sum(copies))
    t = paired_with_repeats(rng, 4, np.uint8, copies) + ord("A")
    sa, cls = profiled(ctx, lambda: ctx.psacak(t, BYTES_BY_DOUBLING))
    assert direct(ctx.trace())
    # group-ordered rounds ran, and some of their groups took the radix sort
    assert cls.get("double_seg_keys", 0) > 0 and cls.get("seg_gather", 0) > 0, cls
    assert (sa == o.psacak8(t)).all()


@pytest.mark.parametrize("copies", [(64, 65), (3, 100, 400)])
def test_integers_group_ordered_rounds_with_large_groups(ctx, copies):
    rng = np.random.default_rng(100 + sum(copies))
    t = paired_with_repeats(rng, 1 << 20, np.uint32, copies)
    sa, cls = profiled(ctx, lambda: ctx.psacak32(t))
    assert direct(ctx.trace())
    assert cls.get("double_seg_keys", 0) > 0 and cls.get("seg_gather", 0) > 0, cls
    assert (sa == o.psacak32(t)).all()


def test_one_symbol(ctx):
    """One distinct name: the first round packs 16 symbols; every later round
    has a single group of every unresolved suffix."""
    t = np.full(3_000_000, 7, np.uint32)
    sa = ctx.psacak32(t)
    assert direct(ctx.trace())
    assert (sa == np.arange(t.size - 1, -1, -1, dtype=np.uint32)).all()
    b = np.full(2_000_000, ord("a"), np.uint8)
    assert (ctx.psacak(b, BYTES_BY_DOUBLING) == np.arange(b.size - 1, -1, -1, dtype=np.uint32)).all()


def test_periodic(ctx):
    """Period 2 and a 1,000-symbol period: large groups in every round."""
    ab = np.frombuffer(b"ab" * 1_200_000, np.uint8)
    assert (ctx.psacak(ab, BYTES_BY_DOUBLING) == o.psacak8(ab)).all()
    rng = np.random.default_rng(9)
    t = np.tile(rng.integers(0, 1 << 16, 1000).astype(np.uint32), 2000)
    assert (ctx.psacak32(t) == o.psacak32(t)).all()


def test_wide_names(ctx):
    """Integer symbols over 2^32: ~n distinct names, 2 packed in the first
    round; and a genome-like byte text of 3 MiB."""
    rng = np.random.default_rng(11)
    t = rng.integers(0, 1 << 32, 2_500_000, dtype=np.uint64).astype(np.uint32)
    assert (ctx.psacak32(t) == o.psacak32(t)).all()
    g = synth.genome(3 << 20, seed=12)
    assert (ctx.psacak(g, BYTES_BY_DOUBLING) == o.psacak8(g)).all()
