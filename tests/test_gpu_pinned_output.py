"""Host-pointer builds into pinned output memory.

With a pinned destination the byte-level build sends every bucket part of
the final suffix array to the host as soon as the scans have finished it,
while the rest of the build runs; the result must be the same array that a
pageable destination receives after the build."""
import numpy as np
import pytest
import torch

import oracle_lib as o
import psacak_b200 as pk
from psacak_b200 import synth

pytestmark = pytest.mark.gpu


def pinned_u32(n):
    return torch.empty(max(n, 1), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)[:n]


def texts():
    rng = np.random.default_rng(31)
    return [synth.genome(3_000_000, seed=7), synth.iid(1 << 20, b"ACGT", seed=8),
            rng.integers(0, 256, 500_000).astype(np.uint8), rng.integers(0, 2, 300_000).astype(np.uint8),
            np.full(200_000, 65, np.uint8), np.frombuffer(b"mississippi", np.uint8),
            np.frombuffer(b"ab" * 70_000, np.uint8)]


def test_pinned_output_equals_oracle():
    for t in texts():
        want = o.psacak8(t)
        for sched in (None, {"engine": pk.ENGINE_BUCKET, "inner_engine": pk.ENGINE_DOUBLING},
                      {"engine": pk.ENGINE_DOUBLING, "inner_engine": pk.ENGINE_DOUBLING}):
            suf = pinned_u32(t.size)
            suf[:] = 0xDEADBEEF
            if sched is None:
                pk.psacak_inplace(t, suf)
            else:
                with pk.Context(0) as ctx:
                    import ctypes
                    rc = pk.lib().psacak8_ctx(ctx.handle, ctypes.c_void_p(t.ctypes.data), t.size,
                                              ctypes.c_void_p(suf.ctypes.data), pk._sched_ptr(sched))
                    pk._raise(rc)
            assert (suf == want).all(), (t.size, sched)


def test_pinned_and_pageable_agree_back_to_back():
    t = synth.genome(8 << 20, seed=9)
    a = pinned_u32(t.size)
    pk.psacak_inplace(t, a)
    b = pk.psacak(t)
    c = pinned_u32(t.size)
    pk.psacak_inplace(t, c)
    assert (a == b).all() and (b == c).all()
    assert (b == o.psacak8(t)).all()


def test_pageable_buffers_go_through_the_staging_ring():
    """Pageable text and SA buffers larger than the two 64 MiB staging slots
    (several chunks each way, a chunk boundary inside the buffers) give the
    same array as pinned buffers, and the array passes the device check."""
    t = synth.genome(150_000_000, seed=11)
    page = np.empty(t.size, np.uint32)
    pk.psacak_inplace(np.array(t), page)
    pin = pinned_u32(t.size)
    pk.psacak_inplace(t, pin)
    assert (page == pin).all()
    with pk.Context(0) as ctx:
        dt = torch.from_numpy(t).cuda()
        ds = torch.from_numpy(page.view(np.int32)).cuda()
        assert ctx.check_sa8_dev(dt.data_ptr(), t.size, ds.data_ptr())


def test_batch_with_pageable_and_pinned_buffers():
    rng = np.random.default_rng(12)
    lens = rng.integers(0, 1_500_000, 200)
    lens[::17] = 0
    texts = [synth.genome(int(k), seed=100 + i) if k else np.zeros(0, np.uint8) for i, k in enumerate(lens)]
    with pk.Context(0) as ctx:
        got = ctx.psacak_batch(texts)  # pageable numpy buffers: staged
        import ctypes
        n = len(texts)
        pins = [torch.empty(max(int(k), 1), dtype=torch.uint8, pin_memory=True).numpy()[:int(k)] for k in lens]
        for p, tx in zip(pins, texts):
            p[:] = tx
        outs = [pinned_u32(int(k)) for k in lens]
        tp = (ctypes.c_void_p * n)(*[p.ctypes.data for p in pins])
        sp = (ctypes.c_void_p * n)(*[o_.ctypes.data for o_ in outs])
        ln = (ctypes.c_uint64 * n)(*[int(k) for k in lens])
        pk._raise(pk.lib().psacak8_batch(ctx.handle, tp, ln, n, sp, None))
    for i in range(n):
        assert (got[i] == outs[i]).all(), i
    for i in (1, 5, 50, 199):
        assert (got[i] == o.psacak8(texts[i])).all(), i


def test_pageable_output_drained_during_the_scans():
    """Pageable outputs of 32M symbols and more are drained by a host thread
    while the final scans run; many small bucket parts (random bytes: 512
    parts) and a single bucket (one byte value) both arrive intact."""
    rng = np.random.default_rng(13)
    for t in (rng.integers(0, 256, 40_000_000).astype(np.uint8), np.full(34_000_000, 7, np.uint8)):
        page = np.empty(t.size, np.uint32)
        pk.psacak_inplace(t, page)
        pin = pinned_u32(t.size)
        pk.psacak_inplace(t, pin)
        assert (page == pin).all()
        with pk.Context(0) as ctx:
            dt = torch.from_numpy(t).cuda()
            ds = torch.from_numpy(page.view(np.int32)).cuda()
            assert ctx.check_sa8_dev(dt.data_ptr(), t.size, ds.data_ptr())
