"""Stage-by-stage GPU parity: the radix sort and scan primitives against
numpy, L/S typing against a direct restatement of the reference's typing
(src/common.rs:43-68, :101-117), and the level-0 reduced string against the
oracle's (naming + translate, src/naming.rs:51-93, :263-274)."""
import numpy as np
import pytest

import oracle_lib as o
import psacak_b200 as pk
from psacak_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def st():
    c = pk.Context(0)
    yield pk.Stages(c)
    c.close()


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host_types(t):
    """S flags (True = S) and LMS flags, as the reference computes them."""
    t = np.asarray(t).astype(np.int64)
    n = t.size
    s = np.zeros(n, bool)
    if n == 0:
        return s, s.copy()
    change = np.flatnonzero(t[:-1] != t[1:])
    nxt_idx = np.searchsorted(change, np.arange(n))
    has = nxt_idx < change.size
    q = np.where(has, change[np.minimum(nxt_idx, max(change.size - 1, 0))] if change.size else 0, n - 1)
    s = np.zeros(n, bool)
    ok = q < n - 1
    s[ok] = t[q[ok]] < t[q[ok] + 1]
    lms = np.zeros(n, bool)
    lms[1:] = s[1:] & ~s[:-1]
    return s, lms


def unpack(words, n):
    b = np.unpackbits(words.view(np.uint8), bitorder="little")
    return b[:n].astype(bool)


@pytest.mark.parametrize("n,b0,b1", [(1, 0, 8), (100, 0, 8), (5000, 0, 20), (70000, 0, 40), (1_000_003, 0, 58),
                                     (3_000_000, 8, 24), (262144, 0, 64)])
def test_radix_sort_u64(st, n, b0, b1):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 2**63, n, dtype=np.int64).astype(np.uint64)
    if n > 10:
        keys[: n // 3] &= np.uint64(0xFFFF)  # many ties in the low bits
    vals = np.arange(n, dtype=np.uint32)
    mask = np.uint64(((1 << (b1 - b0)) - 1) << b0) if b1 - b0 < 64 else np.uint64(2**64 - 1)
    order = np.argsort(keys & mask, kind="stable")
    dk, dv = dev(keys.view(np.int64)), dev(vals.view(np.int32))
    st.radix_sort_u64(dk.data_ptr(), dv.data_ptr(), n, b0, b1)
    got_v = dv.cpu().numpy().view(np.uint32)
    assert (got_v == vals[order]).all()
    assert (dk.cpu().numpy().view(np.uint64) == keys[order]).all()


@pytest.mark.parametrize("n", [3071, 3072, 300_001])
def test_radix_sort_u64_unaligned(st, n):
    """Arrays that are not 16-byte aligned take the plain-load path of the
    radix pass instead of the bulk copies."""
    rng = np.random.default_rng(n + 5)
    keys = rng.integers(0, 2**40, n + 1, dtype=np.int64).astype(np.uint64)
    vals = np.arange(n + 1, dtype=np.uint32)
    order = np.argsort(keys[1:], kind="stable")
    dk, dv = dev(keys.view(np.int64)), dev(vals.view(np.int32))
    st.radix_sort_u64(dk[1:].data_ptr(), dv[1:].data_ptr(), n, 0, 40)
    assert (dv[1:].cpu().numpy().view(np.uint32) == vals[1:][order]).all()
    assert (dk[1:].cpu().numpy().view(np.uint64) == keys[1:][order]).all()


@pytest.mark.parametrize("n", [1, 7, 4096, 4097, 1_000_000, 5_000_001])
def test_radix_sort_u32(st, n):
    rng = np.random.default_rng(n + 1)
    keys = rng.integers(0, 1000, n).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    order = np.argsort(keys, kind="stable")
    dk, dv = dev(keys.view(np.int32)), dev(vals.view(np.int32))
    st.radix_sort_u32(dk.data_ptr(), dv.data_ptr(), n, 0, 32)
    assert (dv.cpu().numpy().view(np.uint32) == vals[order]).all()


@pytest.mark.parametrize("n", [1, 2047, 2048, 2049, 1_000_000, 10_000_019])
def test_exclusive_sum(st, n):
    rng = np.random.default_rng(n + 2)
    a = rng.integers(0, 3, n).astype(np.uint32)
    want = np.concatenate([[0], np.cumsum(a)[:-1]]).astype(np.uint32)
    din, dout = dev(a.view(np.int32)), torch.empty(n, dtype=torch.int32, device="cuda")
    st.exclusive_sum(din.data_ptr(), dout.data_ptr(), n)
    assert (dout.cpu().numpy().view(np.uint32) == want).all()


def _types_case(st, t, width):
    n = t.size
    nw = (n + 31) // 32 + 1
    dt = dev(t.view(np.int32) if width == 4 else t)
    ty = torch.zeros(nw, dtype=torch.int32, device="cuda")
    lm = torch.zeros(nw, dtype=torch.int32, device="cuda")
    st.types(dt.data_ptr(), n, width, ty.data_ptr(), lm.data_ptr())
    s, l = host_types(t)
    gs = unpack(ty.cpu().numpy(), n)
    gl = unpack(lm.cpu().numpy(), n)
    assert (gs == s).all(), np.flatnonzero(gs != s)[:10]
    assert (gl == l).all(), np.flatnonzero(gl != l)[:10]


@pytest.mark.parametrize("n,k", [(5, 2), (33, 2), (8191, 3), (8193, 3), (100_000, 4), (1_000_001, 2), (70_000, 1)])
def test_types_u8(st, n, k):
    rng = np.random.default_rng(n * 7 + k)
    _types_case(st, rng.integers(0, k, n).astype(np.uint8), 1)


def test_types_long_runs(st):
    t = np.concatenate([np.full(20000, 5), np.full(9000, 2), np.full(30000, 7), [1], np.full(17000, 7)]).astype(np.uint8)
    _types_case(st, t, 1)
    _types_case(st, synth.genome(3 << 20, seed=5), 1)


@pytest.mark.parametrize("n,k", [(100, 5), (8192 * 3 + 5, 1000), (1_000_000, 50000)])
def test_types_u32(st, n, k):
    rng = np.random.default_rng(n + k)
    _types_case(st, rng.integers(0, k, n).astype(np.uint32), 4)


@pytest.mark.parametrize("engine", [pk.ENGINE_BUCKET, pk.ENGINE_DOUBLING])
@pytest.mark.parametrize("gen,n", [("iid3", 2676), ("iid4", 100_000), ("genome", 1 << 20), ("iid256", 300_000),
                                   ("runs", 200_000)])
def test_reduced_string_level0(st, gen, n, engine):
    if gen == "genome":
        t = synth.genome(n, seed=9)
    elif gen == "runs":
        rng = np.random.default_rng(3)
        t = np.repeat(rng.integers(0, 3, n // 50).astype(np.uint8), rng.integers(1, 100, n // 50))[:n]
        n = t.size
    else:
        k = int(gen[3:])
        t = np.random.default_rng(n).integers(0, k, n).astype(np.uint8)
    want, wk = o.reduced8(t)
    dt = dev(t)
    dr = torch.zeros(max(want.size, 1), dtype=torch.int32, device="cuda")
    n1, k = st.reduced8(dt.data_ptr(), n, dr.data_ptr(), want.size,
                        {"engine": engine, "inner_engine": pk.ENGINE_DOUBLING})
    assert (n1, k) == (want.size, wk)
    assert (dr.cpu().numpy().view(np.uint32)[:n1] == want).all()
