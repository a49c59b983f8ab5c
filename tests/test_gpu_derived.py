"""Inverse SA, BWT and LCP on the GPU (psacak_isa_dev, psacak_bwt8_dev,
psacak_lcp8_dev / psacak_lcp32_dev, through the C ABI) against the CPU
restatements (Kasai's LCP; the divbwt-convention BWT).  Exact equality."""
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


def _texts():
    rng = np.random.default_rng(5)
    runs = np.repeat(rng.integers(65, 69, 30000).astype(np.uint8), rng.integers(1, 40, 30000))
    return [np.frombuffer(b"mississippi", np.uint8), np.frombuffer(b"a", np.uint8), np.frombuffer(b"ab" * 700, np.uint8),
            np.full(200_000, 65, np.uint8), rng.integers(65, 69, 300_001).astype(np.uint8), runs,
            synth.genome(4 << 20, seed=9), rng.integers(0, 256, 100_000).astype(np.uint8)]


def test_derived_u8(ctx):
    for t in _texts():
        n = t.size
        dt = torch.from_numpy(t.copy()).cuda()
        ds = torch.empty(n, dtype=torch.int32, device="cuda")
        ctx.psacak8_dev(dt.data_ptr(), n, ds.data_ptr())
        sa = ds.cpu().numpy().view(np.uint32)
        assert (sa == o.psacak8(t)).all()
        isa = torch.empty(n, dtype=torch.int32, device="cuda")
        ctx.isa_dev(ds.data_ptr(), n, isa.data_ptr())
        want_isa = np.empty(n, np.uint32)
        want_isa[sa] = np.arange(n, dtype=np.uint32)
        assert (isa.cpu().numpy().view(np.uint32) == want_isa).all()
        bwt = torch.empty(n, dtype=torch.uint8, device="cuda")
        primary = ctx.bwt8_dev(dt.data_ptr(), n, ds.data_ptr(), bwt.data_ptr())
        want_bwt, want_primary = o.bwt(t, sa)
        assert primary == want_primary and (bwt.cpu().numpy() == want_bwt).all()
        lcp = torch.empty(n, dtype=torch.int32, device="cuda")
        ctx.lcp8_dev(dt.data_ptr(), n, ds.data_ptr(), lcp.data_ptr())
        assert (lcp.cpu().numpy().view(np.uint32) == o.lcp(t, sa)).all(), n


def test_lcp_u32(ctx):
    rng = np.random.default_rng(6)
    for t in [synth.zipf32(1 << 20, 1 << 12, 1.1, 0.1, 100, 5000, seed=7),
              rng.integers(0, 3, 200_000).astype(np.uint32)]:
        t = np.ascontiguousarray(t, dtype=np.uint32)
        n = t.size
        sa = o.psacak32(t)
        dt = torch.from_numpy(t.view(np.int32).copy()).cuda()
        ds = torch.from_numpy(sa.view(np.int32).copy()).cuda()
        lcp = torch.empty(n, dtype=torch.int32, device="cuda")
        ctx.lcp32_dev(dt.data_ptr(), n, ds.data_ptr(), lcp.data_ptr())
        assert (lcp.cpu().numpy().view(np.uint32) == o.lcp(t, sa)).all()


def test_lcp_run_heavy_texts_finish_quickly(ctx):
    """Long runs of one character: the single irreducible position of a run
    has a PLCP about the run's length, compared by a whole CTA rather than
    one thread; mixed with periodic stretches whose irreducible positions
    cross the per-thread limit by various amounts."""
    import time
    rng = np.random.default_rng(8)
    texts = [np.concatenate([np.full(8 << 20, 65, np.uint8), rng.integers(65, 69, 1000).astype(np.uint8)]),
             np.concatenate([rng.integers(65, 69, 5000).astype(np.uint8), np.full(3_000_017, 67, np.uint8),
                             np.tile(np.frombuffer(b"ACGTTGCA", np.uint8), 200_000),
                             np.full(16383, 71, np.uint8), np.full(16385, 84, np.uint8)]),
             np.tile(synth.iid(5000, b"ACGT", seed=3), 300)]
    for t in texts:
        n = t.size
        sa = o.psacak8(t)
        dt = torch.from_numpy(t.copy()).cuda()
        ds = torch.from_numpy(sa.view(np.int32).copy()).cuda()
        lcp = torch.empty(n, dtype=torch.int32, device="cuda")
        ctx.lcp8_dev(dt.data_ptr(), n, ds.data_ptr(), lcp.data_ptr())  # warm-up
        t0 = time.perf_counter()
        ctx.lcp8_dev(dt.data_ptr(), n, ds.data_ptr(), lcp.data_ptr())
        secs = time.perf_counter() - t0
        assert (lcp.cpu().numpy().view(np.uint32) == o.lcp(t, sa)).all(), n
        assert secs < 0.5, (n, secs)
