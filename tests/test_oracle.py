"""The CPU oracle pinned against the reference's own known answers.

The oracle (oracle/psacak_oracle.cpp) restates the reference's serial path;
these tests pin it to the reference's golden vectors (src/lib.rs:12-15,
src/psacak8.rs:508-524, src/psacak32.rs:826-842), to a naive sort on random
inputs (the reference's quickcheck_sacak8/32, src/psacak8.rs:531-534,
src/psacak32.rs:849-852) and to the committed level traces.
"""
import json
import os

import numpy as np
import pytest

import oracle_lib as o

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def naive(seq):
    return np.array(sorted(range(len(seq)), key=lambda i: seq[i:]), dtype=np.uint32)


def test_mississippi():
    v = load("reference_vectors.json")["mississippi"]
    sa = o.psacak8(b"mississippi")
    assert sa.tolist() == [10, 7, 4, 1, 0, 9, 8, 6, 3, 5, 2] == v["sa"]
    # the sentinel-prefixed form of src/lib.rs:37-42
    assert [11] + sa.tolist() == v["sa_with_sentinel"]


@pytest.mark.parametrize("idx", range(11))
def test_reference_tables(idx):
    case = load("reference_vectors.json")["tables"][idx]
    t = case["text"]
    assert o.psacak8(np.array(t, np.uint8)).tolist() == case["sa"]
    assert o.psacak32(np.array(t, np.uint32)).tolist() == case["sa"]


def test_random_u8_vs_naive():
    rng = np.random.default_rng(7)
    for _ in range(1500):
        n = int(rng.integers(0, 200))
        k = int(rng.choice([1, 2, 3, 4, 16, 256]))
        t = rng.integers(0, k, n).astype(np.uint8)
        assert (o.psacak8(t) == naive(t.tolist())).all()


def test_random_u32_vs_naive():
    rng = np.random.default_rng(8)
    for _ in range(1500):
        n = int(rng.integers(0, 200))
        k = int(rng.choice([1, 2, 5, 50, 1 << 20, 1 << 32]))
        t = rng.integers(0, k, n, dtype=np.uint64).astype(np.uint32)
        assert (o.psacak32(t) == naive(t.tolist())).all()


@pytest.mark.parametrize("text", [
    b"", b"a", b"ab", b"ba", b"aaa", b"aaaa", b"abab", b"\xff\xff\xff\xff\xfe\xff",
    bytes(range(255, -1, -1)), b"\x00" * 1000, b"ab" * 500, bytes([255]) * 77 + b"\x00",
])
def test_edge_cases(text):
    assert (o.psacak8(np.frombuffer(text, np.uint8)) == naive(text)).all()


def test_translate_sample_matches_restatement():
    rng = np.random.default_rng(9)
    for _ in range(200):
        n = int(rng.integers(1, 100))
        t = rng.integers(0, int(rng.integers(1, 40)), n).astype(np.uint32)
        got = o.translate_sample(t)
        vals = sorted(set(t.tolist()))
        if len(vals) >= n:
            assert got is None
            continue
        cnt = {v: int((t == v).sum()) for v in vals}
        head, acc = {}, 0
        for v in vals:
            head[v] = acc
            acc += cnt[v]
        # types right to left (src/common.rs:72-97)
        s = [False] * n
        for i in range(n - 2, -1, -1):
            s[i] = t[i] < t[i + 1] or (t[i] == t[i + 1] and s[i + 1])
        want = [head[v] + cnt[v] - 1 if s[i] else head[v] for i, v in enumerate(t.tolist())]
        assert got.tolist() == want


def test_checker_detects_errors():
    rng = np.random.default_rng(10)
    t = rng.integers(0, 4, 5000).astype(np.uint8)
    sa = o.psacak8(t)
    assert o.check_sa8(t, sa)
    bad = sa.copy()
    bad[10], bad[11] = bad[11], bad[10]
    assert not o.check_sa8(t, bad)
    bad = sa.copy()
    bad[5] = bad[6]
    assert not o.check_sa8(t, bad)


def test_medium_random_checked():
    rng = np.random.default_rng(11)
    for n, k in [(131071, 4), (131072, 4), (262145, 2), (65537, 200)]:
        t = rng.integers(0, k, n).astype(np.uint8)
        assert o.check_sa8(t, o.psacak8(t))
        t32 = rng.integers(0, 1000, n // 2).astype(np.uint32)
        assert o.check_sa32(t32, o.psacak32(t32))


def test_synthetic_traces_pinned():
    from golden.make_golden import make_input
    for case in load("synthetic_traces.json"):
        if case["n"] > (1 << 19):
            continue  # the larger cases are checked by the GPU suite
        t = make_input(case["generator"], case["n"], case["seed"])
        if case["generator"] == "zipf32":
            sa, tr = o.psacak32(t, trace=True)
        else:
            sa, tr = o.psacak8(t, trace=True)
        assert tr == case["levels"]
        assert o.hash_u32(sa) == case["sa_hash"]


@pytest.mark.parametrize("threads", [1, 3, 8])
def test_pipelined_scans_equal_serial(threads):
    """The all-core CPU baseline -- the restatement of the reference's
    pipelined induced scans, its chunked parallel naming and the prefetching
    u32 scans of the inner levels -- builds the same suffix array as the
    serial restatement: texts of several 128Ki blocks (their reduced strings
    pass 2 x 64Ki symbols and 2^16 LMS substrings, so the inner levels and
    the naming run in parallel too), with repeats, runs and an all-equal
    stretch that sends writes far beyond the next block."""
    from psacak_b200 import synth
    rng = np.random.default_rng(threads)
    texts = [synth.genome(3 << 20, seed=threads),
             rng.integers(65, 69, 600_000).astype(np.uint8),
             np.concatenate([np.full(300_000, 65, np.uint8), rng.integers(65, 70, 400_000).astype(np.uint8)]),
             np.repeat(rng.integers(0, 256, 40_000).astype(np.uint8), rng.integers(1, 20, 40_000))]
    for t in texts:
        assert (o.psacak8_par(t, threads) == o.psacak8(t)).all()


def _naive_lcp(t, sa):
    out = [0] * len(sa)
    for i in range(1, len(sa)):
        a, b, h = int(sa[i - 1]), int(sa[i]), 0
        while a + h < len(t) and b + h < len(t) and t[a + h] == t[b + h]:
            h += 1
        out[i] = h
    return out


def test_lcp_and_bwt_restatements_match_definitions():
    """Kasai's LCP and the divbwt-convention BWT of the oracle against their
    definitions: direct suffix comparison, and the sorted rotations of
    text + sentinel with the sentinel's character left out."""
    rng = np.random.default_rng(11)
    cases = [b"mississippi", b"a", b"aaaa", b"abab", b"banana"] + [
        bytes(rng.integers(97, 97 + int(rng.integers(1, 5)), int(rng.integers(1, 60))).astype(np.uint8))
        for _ in range(300)]
    for t in cases:
        a = np.frombuffer(t, np.uint8)
        sa = o.psacak8(a)
        assert o.lcp(a, sa).tolist() == _naive_lcp(t, sa), t
        # rotations of t + sentinel (sentinel below every byte), sorted
        u = list(t) + [-1]
        rot = sorted(range(len(u)), key=lambda r: u[r:] + u[:r])
        full = [u[r - 1] for r in rot]
        primary = full.index(-1)
        want = [c for c in full if c != -1]
        got, p = o.bwt(a, sa)
        assert got.tolist() == want and p == primary, t
    u32 = rng.integers(0, 7, 500).astype(np.uint32)
    sa = o.psacak32(u32)
    assert o.lcp(u32, sa).tolist() == _naive_lcp(u32.tolist(), sa)
