"""GPU builds through the C ABI compared with the CPU oracle.

Suffix arrays are integer permutations: every comparison here is exact.
"""
import json
import os

import numpy as np
import pytest

import oracle_lib as o
import psacak_b200 as pk
from psacak_b200 import synth

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
ENGINES = [pk.ENGINE_BUCKET, pk.ENGINE_DOUBLING]


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def ctx():
    c = pk.Context(0)
    yield c
    c.close()


def sched(engine):
    return {"engine": engine, "inner_engine": pk.ENGINE_DOUBLING}


@pytest.mark.parametrize("engine", ENGINES)
def test_mississippi(ctx, engine):
    assert ctx.psacak(b"mississippi", sched(engine)).tolist() == [10, 7, 4, 1, 0, 9, 8, 6, 3, 5, 2]


@pytest.mark.parametrize("engine", ENGINES)
def test_reference_tables(ctx, engine):
    for case in load("reference_vectors.json")["tables"]:
        t = case["text"]
        assert ctx.psacak(np.array(t, np.uint8), sched(engine)).tolist() == case["sa"], t
        assert ctx.psacak32(np.array(t, np.uint32)).tolist() == case["sa"], t


@pytest.mark.parametrize("engine", ENGINES)
def test_edge_cases(ctx, engine):
    cases = [b"", b"a", b"ab", b"ba", b"aaa", b"aaaa", b"abab", b"\xff\xff\xff\xff\xfe\xff",
             bytes(range(255, -1, -1)), b"\x00" * 1000, b"ab" * 500, bytes([255]) * 77 + b"\x00",
             b"\x00" * 70000, b"A" * 131073, bytes(range(256)) * 300]
    for t in cases:
        a = np.frombuffer(t, np.uint8)
        assert (ctx.psacak(a, sched(engine)) == o.psacak8(a)).all(), t[:20]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_runs_of_every_length(ctx, seed):
    """Runs of one character of every length around the chain scan's direct
    depths and its in-scan measuring cap (1..12), plus runs of hundreds to
    tens of thousands (measured after the scan), mixed in random order, so
    that bucket parts hold seeds of every depth and deep cells."""
    rng = np.random.default_rng(seed)
    pieces = []
    for _ in range(3000):
        c = rng.integers(0, 4)
        k = int(rng.integers(1, 13)) if rng.random() < 0.97 else int(rng.integers(100, 20000))
        pieces.append(np.full(k, [65, 67, 71, 84][c], np.uint8))
        if rng.random() < 0.3:
            pieces.append(rng.integers(65, 69, int(rng.integers(1, 4))).astype(np.uint8))
    t = np.concatenate(pieces)
    want = o.psacak8(t)
    for engine in ENGINES:
        assert (ctx.psacak(t, sched(engine)) == want).all(), engine


@pytest.mark.parametrize("engine", ENGINES)
def test_random_small_u8(ctx, engine):
    rng = np.random.default_rng(20)
    for _ in range(300):
        n = int(rng.integers(0, 3000))
        k = int(rng.choice([1, 2, 3, 4, 5, 16, 255, 256]))
        t = rng.integers(0, k, n).astype(np.uint8)
        got = ctx.psacak(t, sched(engine))
        assert (got == o.psacak8(t)).all(), (n, k)


def test_random_small_u32(ctx):
    rng = np.random.default_rng(21)
    for _ in range(300):
        n = int(rng.integers(0, 3000))
        k = int(rng.choice([1, 2, 7, 100, 5000, 1 << 20, 1 << 32]))
        t = rng.integers(0, k, n, dtype=np.uint64).astype(np.uint32)
        assert (ctx.psacak32(t) == o.psacak32(t)).all(), (n, k)


@pytest.mark.parametrize("engine", ENGINES)
def test_synthetic_traces(ctx, engine):
    from golden.make_golden import make_input
    for case in load("synthetic_traces.json"):
        t = make_input(case["generator"], case["n"], case["seed"])
        if case["generator"] == "zipf32":
            sa = ctx.psacak32(t, {})  # explicit zero schedule: recursion all the way down, as the oracle's trace
        else:
            sa = ctx.psacak(t, sched(engine))
        assert o.hash_u32(sa) == case["sa_hash"], case["name"]
        assert ctx.trace() == case["levels"], case["name"]


@pytest.mark.parametrize("engine", ENGINES)
def test_config1_8mib_acgt(ctx, engine):
    t = synth.iid(8 << 20, b"ACGT", seed=1)
    sa = ctx.psacak(t, sched(engine))
    assert (sa == o.psacak8(t)).all()


def test_genome_16mib(ctx):
    t = synth.genome(16 << 20, seed=2)
    sa = ctx.psacak(t)
    assert (sa == o.psacak8(t)).all()


def test_zipf32_4m(ctx):
    t = synth.zipf32(4 << 20, seed=3)
    sa = ctx.psacak32(t)
    assert (sa == o.psacak32(t)).all()


SCHEDULES = [dict(engine=e, inner_engine=pk.ENGINE_DOUBLING, tile_items=t, finish_below=f)
             for e in (pk.ENGINE_BUCKET, pk.ENGINE_DOUBLING) for t in (8, 12, 16) for f in (0, 1 << 14)]


def test_every_schedule_gives_the_same_sa(ctx):
    rng = np.random.default_rng(23)
    texts = [synth.genome(300_000, seed=5), rng.integers(0, 3, 50_000).astype(np.uint8),
             np.frombuffer(b"abracadabra" * 3000, np.uint8)]
    for t in texts:
        want = o.psacak8(t)
        for sc in SCHEDULES:
            assert (ctx.psacak(t, sc) == want).all(), sc
    sym = synth.zipf32(200_000, alphabet=1 << 16, seed=6)
    want = o.psacak32(sym)
    for sc in SCHEDULES:
        assert (ctx.psacak32(sym, sc) == want).all(), sc


@pytest.mark.parametrize("finish", [1 << 12, 1 << 16, 1 << 22])
def test_byte_texts_sorted_directly_by_prefix_doubling(ctx, finish):
    """Byte texts shorter than finish_below skip the induced scans and are
    sorted by prefix doubling from their bytes; the SA is the same."""
    rng = np.random.default_rng(finish)
    texts = [np.frombuffer(b"mississippi", np.uint8), np.frombuffer(b"aaaa", np.uint8),
             rng.integers(65, 69, 3000).astype(np.uint8), synth.genome(40_000, seed=3),
             np.full(5000, 0, np.uint8), rng.integers(0, 256, 60_000).astype(np.uint8)]
    for t in texts:
        sc = {"engine": pk.ENGINE_BUCKET, "inner_engine": pk.ENGINE_DOUBLING, "finish_below": finish}
        assert (ctx.psacak(t, sc) == o.psacak8(t)).all(), (finish, t.size)


def test_init_and_shutdown_of_the_default_context():
    """psacak_init creates the thread's default context up front; after
    psacak_shutdown the next call creates a new one and builds the same SA."""
    t = synth.genome(200_000, seed=31)
    want = o.psacak8(t)
    pk.init(0)
    assert (pk.psacak(t) == want).all()
    import ctypes
    sa = np.empty(t.size, np.uint32)
    assert pk.lib().psacak8(ctypes.c_void_p(t.ctypes.data), t.size, ctypes.c_void_p(sa.ctypes.data)) == 0
    assert (sa == want).all()
    pk.shutdown()
    sa[:] = 0
    assert pk.lib().psacak8(ctypes.c_void_p(t.ctypes.data), t.size, ctypes.c_void_p(sa.ctypes.data)) == 0
    assert (sa == want).all()
    assert (pk.psacak(t) == want).all()
    bad = pk.lib().psacak_init(1 << 20)
    assert bad == -1
