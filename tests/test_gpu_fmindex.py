"""FM-index on the device (psacak_fm_build_dev / psacak_fm_count_dev) over the
BWT of psacak_bwt8_dev: the suffix-array range of every pattern must equal
the oracle's binary search on the suffix array (oracle_sa_range8); patterns
that do not occur must give empty ranges.  Patterns: substrings of the text
of lengths 1..64 at random positions (present), random strings (mostly
absent), bytes that never occur, the empty pattern, the whole text, and
texts whose lengths straddle the 256-byte blocks and 64 KiB superblocks of
the rank checkpoints."""
import numpy as np
import pytest

import oracle_lib as o
import psacak_b200 as pk
from psacak_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    c = pk.Context(0)
    yield c
    c.close()


def _patterns(text, rng, count):
    pats = []
    n = text.size
    for i in range(count):
        kind = i % 4
        if kind < 2 and n > 0:
            m = int(rng.integers(1, 65))
            p = int(rng.integers(0, max(n - m, 0) + 1))
            pats.append(text[p:p + m].tobytes())
        elif kind == 2:
            pats.append(rng.choice(np.frombuffer(b"ACGTN", np.uint8), int(rng.integers(1, 12))).tobytes())
        else:
            pats.append(bytes(rng.integers(0, 256, int(rng.integers(1, 4))).astype(np.uint8)))
    pats += [b"", text.tobytes(), b"\x00", b"\xff\xfe"]
    return pats


def _search(ctx, text, pats):
    n = text.size
    stream = torch.cuda.current_stream().cuda_stream
    dt = torch.from_numpy(text).cuda()
    ds = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    if n:
        ctx.psacak8_dev(dt.data_ptr(), n, ds.data_ptr(), stream)
    db = torch.empty(max(n, 1), dtype=torch.uint8, device="cuda")
    primary = ctx.bwt8_dev(dt.data_ptr(), n, ds.data_ptr(), db.data_ptr(), stream) if n else 0
    fm = torch.empty(pk.fm_bytes(n), dtype=torch.uint8, device="cuda")
    ctx.fm_build_dev(db.data_ptr(), n, primary, fm.data_ptr(), stream)
    off = np.zeros(len(pats) + 1, np.uint64)
    off[1:] = np.cumsum([len(p) for p in pats])
    buf = np.frombuffer(b"".join(pats) or b"\0", np.uint8).copy()
    dp = torch.from_numpy(buf).cuda()
    doff = torch.from_numpy(off.view(np.int64)).cuda()
    dr = torch.zeros(2 * len(pats), dtype=torch.int32, device="cuda")
    ctx.fm_count_dev(fm.data_ptr(), db.data_ptr(), dp.data_ptr(), doff.data_ptr(), len(pats), dr.data_ptr(), stream)
    torch.cuda.synchronize()
    sa = ds.cpu().numpy().view(np.uint32)[:n]
    return sa, dr.cpu().numpy().view(np.uint32).reshape(-1, 2)


def _compare(text, sa, pats, ranges):
    for p, (lo, hi) in zip(pats, ranges):
        want = o.sa_range8(text, sa, p)
        if want[1] > want[0]:
            assert (int(lo), int(hi)) == want, (p[:20], len(p), (lo, hi), want)
        else:
            assert hi == lo, (p[:20], (lo, hi))


@pytest.mark.parametrize("n", [1, 2, 255, 256, 257, 4096, 65535, 65536, 65537, 300_001])
def test_fm_ranges_match_oracle_at_checkpoint_edges(ctx, n):
    rng = np.random.default_rng(n)
    text = synth.genome(n, seed=n) if n > 3 else np.frombuffer(b"abca"[:n], np.uint8).copy()
    pats = _patterns(text, rng, 400)
    sa, ranges = _search(ctx, text, pats)
    assert np.array_equal(sa, o.psacak8(text))
    _compare(text, sa, pats, ranges)


@pytest.mark.parametrize("kind", ["bytes", "runs", "mississippi"])
def test_fm_ranges_match_oracle_on_alphabets(ctx, kind):
    rng = np.random.default_rng(7)
    if kind == "bytes":
        text = rng.integers(0, 256, 200_000).astype(np.uint8)
    elif kind == "runs":
        text = np.repeat(rng.integers(65, 68, 3000).astype(np.uint8), rng.integers(1, 200, 3000))
    else:
        text = np.frombuffer(b"mississippi" * 1000, np.uint8).copy()
    pats = _patterns(text, rng, 600)
    if kind == "runs":
        pats += [b"A" * k for k in (1, 50, 150, 199, 400)]
    sa, ranges = _search(ctx, text, pats)
    _compare(text, sa, pats, ranges)


def test_fm_count_of_every_substring_occurrence(ctx):
    # counts (hi - lo) add up: every length-3 substring of the text occurs
    # hi - lo times, and those counts sum to n - 2
    text = synth.iid(50_000, b"ACG", seed=9)
    pats = sorted({text[i:i + 3].tobytes() for i in range(text.size - 2)})
    sa, ranges = _search(ctx, text, pats)
    assert int((ranges[:, 1] - ranges[:, 0]).astype(np.int64).sum()) == text.size - 2
    _compare(text, sa, pats, ranges)
