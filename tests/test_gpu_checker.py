"""The device suffix-array checks (psacak_check_sa8_dev, psacak_check_sa32_dev
and the allocation-free psacak_check_sa8_noalloc) against the oracle's check
on correct and corrupted suffix arrays.

The bench's full-size `verified` flags rest on these checks, so each is
pinned here case by case: for every corruption the device verdict must equal
the oracle's (oracle_check_sa8/32, the same Burkhardt-Kaerkkaeinen test
restated on the CPU, itself checked against the naive definition in
tests/test_oracle.py).  Corruptions: a duplicated entry, an out-of-range
entry, an adjacent swap in the middle of the array, a swap of two suffixes
that start with the same symbol, the last suffix (position n-1) moved, and a
shuffled stretch.  The reference's own check is the CLI's quadratic
comparison of adjacent suffixes (src/bin/psacak.rs:73-80).
"""
import numpy as np
import pytest

import oracle_lib as o
import psacak_b200 as pk
from psacak_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def corruptions(text, sa, rng, count):
    """(name, corrupted copy of sa) pairs."""
    n = sa.size
    out = []
    for r in range(count):
        kind = r % 6
        s = sa.copy()
        if kind == 0:  # a duplicated entry
            j, k = rng.choice(n, 2, replace=False)
            s[j] = s[k]
            out.append(("duplicate", s))
        elif kind == 1:  # an entry outside [0, n)
            j = int(rng.integers(0, n))
            s[j] = np.uint32(n + int(rng.integers(0, 3))) if r % 4 else np.uint32(0xFFFFFFFF)
            out.append(("out of range", s))
        elif kind == 2:  # an adjacent swap in the middle
            j = int(rng.integers(n // 4, 3 * n // 4))
            s[j], s[j + 1] = s[j + 1], s[j]
            out.append(("adjacent swap", s))
        elif kind == 3:  # two suffixes with the same first symbol swapped
            first = text[sa.astype(np.int64)]
            j = int(rng.integers(0, n - 1))
            same = np.flatnonzero(first == first[j])
            same = same[same != j]
            k = int(rng.choice(same)) if same.size else (j + 1)
            s[j], s[k] = s[k], s[j]
            out.append(("same-symbol swap", s))
        elif kind == 4:  # the last suffix moved by a few slots
            i = int(np.flatnonzero(sa == n - 1)[0])
            d = int(rng.integers(1, 5)) * (1 if i < n // 2 else -1)
            s = np.insert(np.delete(s, i), i + d, np.uint32(n - 1))
            out.append(("last position moved", s))
        else:  # a shuffled stretch
            j = int(rng.integers(0, n - 8))
            seg = s[j:j + 8].copy()
            rng.shuffle(seg)
            if np.array_equal(seg, s[j:j + 8]):
                seg = seg[::-1].copy()
            s[j:j + 8] = seg
            out.append(("shuffled stretch", s))
    return out


@pytest.fixture(scope="module")
def ctx():
    c = pk.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("kind", ["genome", "runs", "acgt"])
def test_check_sa8_dev_matches_oracle_on_corruptions(ctx, kind):
    rng = np.random.default_rng({"genome": 1, "runs": 2, "acgt": 3}[kind])
    if kind == "genome":
        text = synth.genome(200_000, seed=61)
    elif kind == "runs":
        text = np.repeat(rng.integers(65, 68, 4000).astype(np.uint8), rng.integers(1, 40, 4000))
    else:
        text = synth.iid(50_000, b"ACGT", seed=62)
    sa = o.psacak8(text)
    stream = torch.cuda.current_stream().cuda_stream
    dt = torch.from_numpy(text).cuda()
    cases = [("correct", sa)] + corruptions(text, sa, rng, 48)
    for name, s in cases:
        want = o.check_sa8(text, s)
        assert want == (name == "correct"), name
        ds = torch.from_numpy(s.view(np.int32)).cuda()
        assert ctx.check_sa8_dev(dt.data_ptr(), text.size, ds.data_ptr(), stream) == want, name
        assert pk.check_sa8_noalloc(dt.data_ptr(), text.size, ds.data_ptr(), stream) == want, name


@pytest.mark.parametrize("kind", ["zipf", "small_alphabet"])
def test_check_sa32_dev_matches_oracle_on_corruptions(ctx, kind):
    rng = np.random.default_rng({"zipf": 4, "small_alphabet": 5}[kind])
    if kind == "zipf":
        text = synth.zipf32(150_000, alphabet=1 << 16, seed=63)
    else:
        text = rng.integers(0, 3, 60_000).astype(np.uint32) * np.uint32(1 << 30)
    sa = o.psacak32(text)
    stream = torch.cuda.current_stream().cuda_stream
    dt = torch.from_numpy(text.view(np.int32)).cuda()
    cases = [("correct", sa)] + corruptions(text, sa, rng, 48)
    for name, s in cases:
        want = o.check_sa32(text, s)
        assert want == (name == "correct"), name
        ds = torch.from_numpy(s.view(np.int32)).cuda()
        assert ctx.check_sa32_dev(dt.data_ptr(), text.size, ds.data_ptr(), stream) == want, name


def test_checks_on_tiny_inputs(ctx):
    stream = torch.cuda.current_stream().cuda_stream
    for t in (b"a", b"ab", b"ba", b"aaa", b"mississippi"):
        text = np.frombuffer(t, np.uint8).copy()
        sa = o.psacak8(text)
        dt = torch.from_numpy(text).cuda()
        for s in [sa] + ([sa[::-1].copy()] if sa.size > 1 else []):
            want = o.check_sa8(text, s)
            ds = torch.from_numpy(np.ascontiguousarray(s).view(np.int32)).cuda()
            assert ctx.check_sa8_dev(dt.data_ptr(), text.size, ds.data_ptr(), stream) == want, t
            d32 = torch.from_numpy(text.astype(np.uint32).view(np.int32)).cuda()
            assert ctx.check_sa32_dev(d32.data_ptr(), text.size, ds.data_ptr(), stream) == o.check_sa32(
                text.astype(np.uint32), s), t
