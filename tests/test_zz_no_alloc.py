"""psacak_check_sa8_noalloc: the suffix-array check for callers that cannot
allocate device memory (a serving loop where cudaMalloc would synchronise the
device, or a host process that owns the memory budget).  It must agree with
the allocating check, psacak_check_sa8_dev, on correct and corrupted suffix
arrays, on two calls in a row (its fixed scratch keeps the previous call's
contents), and refuse sizes above its fixed maximum.

Collected last on purpose (file name), so a run stopping at the first failure
has run every other test first.
"""
import ctypes

import numpy as np
import pytest

import psacak_b200 as pk
from psacak_b200 import synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _noalloc(d_text, n, d_sa, stream):
    ok = ctypes.c_int(-1)
    rc = pk.lib().psacak_check_sa8_noalloc(ctypes.c_void_p(d_text), n, ctypes.c_void_p(d_sa), ctypes.byref(ok),
                                           ctypes.c_void_p(stream))
    return rc, ok.value


@pytest.mark.parametrize("n", [1, 11, 100_000, pk.NOALLOC_CHECK_MAX])
def test_noalloc_check_matches_allocating_check(n):
    text = synth.genome(n, seed=31) if n > 11 else np.frombuffer(b"mississippi"[:n], np.uint8).copy()
    with pk.Context(0) as ctx:
        stream = torch.cuda.current_stream()
        dt = torch.from_numpy(text).cuda()
        ds = torch.empty(n, dtype=torch.int32, device="cuda")
        ctx.psacak8_dev(dt.data_ptr(), n, ds.data_ptr(), stream.cuda_stream)
        bad = ds.clone()
        if n >= 2:
            bad[[0, 1]] = bad[[1, 0]]
        for sa in (ds, bad):
            want = ctx.check_sa8_dev(dt.data_ptr(), n, sa.data_ptr(), stream.cuda_stream)
            for _ in range(2):  # two calls in a row share the same scratch
                rc, ok = _noalloc(dt.data_ptr(), n, sa.data_ptr(), stream.cuda_stream)
                assert rc == pk.PSACAK_OK
                assert bool(ok) == want
        assert ctx.check_sa8_dev(dt.data_ptr(), n, ds.data_ptr(), stream.cuda_stream)
        if n >= 2:
            assert not ctx.check_sa8_dev(dt.data_ptr(), n, bad.data_ptr(), stream.cuda_stream)


def test_noalloc_check_allocates_no_device_memory():
    n = pk.NOALLOC_CHECK_MAX
    text = synth.genome(n, seed=32)
    stream = torch.cuda.current_stream()
    with pk.Context(0) as ctx:
        dt = torch.from_numpy(text).cuda()
        ds = torch.empty(n, dtype=torch.int32, device="cuda")
        ctx.psacak8_dev(dt.data_ptr(), n, ds.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        # the first call loads the library's module and looks up the array
        assert _noalloc(dt.data_ptr(), n, ds.data_ptr(), stream.cuda_stream) == (pk.PSACAK_OK, 1)
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        for _ in range(4):
            assert _noalloc(dt.data_ptr(), n, ds.data_ptr(), stream.cuda_stream) == (pk.PSACAK_OK, 1)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0


def test_noalloc_check_rejects_oversize():
    n = pk.NOALLOC_CHECK_MAX + 1
    dt = torch.zeros(n, dtype=torch.uint8, device="cuda")
    ds = torch.zeros(n, dtype=torch.int32, device="cuda")
    rc, _ = _noalloc(dt.data_ptr(), n, ds.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == pk.PSACAK_EINVAL
    assert b"exceeds" in pk.lib().psacak_last_error_string()
