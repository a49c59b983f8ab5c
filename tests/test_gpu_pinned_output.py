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
