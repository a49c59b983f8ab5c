"""The C-ABI library loads and exports every entry point its header
declares; argument checks that need no GPU return the documented status."""
import ctypes
import os
import re

import numpy as np
import pytest

import psacak_b200 as pk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(psacak\w*)\s*\(", src, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("psacak8", "psacak32", "psacak8_dev", "psacak32_dev", "psacak8_batch",
                     "psacak_ctx_create", "psacak_ctx_destroy", "psacak_last_error_string"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(pk.library_path())
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_version():
    assert pk.lib().psacak_version().decode().count(".") == 2


def test_null_context_is_einval():
    lib = pk.lib()
    t = np.zeros(4, np.uint8)
    sa = np.zeros(4, np.uint32)
    rc = lib.psacak8_ctx(None, t.ctypes.data, 4, sa.ctypes.data, None)
    assert rc == pk.PSACAK_EINVAL
    assert b"context" in lib.psacak_last_error_string()


def test_length_limits_are_einval():
    lib = pk.lib()
    rc = lib.psacak8(ctypes.c_void_p(1), 0xFFFFFFFF, ctypes.c_void_p(1))
    assert rc == pk.PSACAK_EINVAL
    rc = lib.psacak32(ctypes.c_void_p(1), 0x80000000, ctypes.c_void_p(1))
    assert rc == pk.PSACAK_EINVAL
    rc = lib.psacak8(None, 10, None)
    assert rc == pk.PSACAK_EINVAL


def test_python_limits_raise():
    with pytest.raises(ValueError):
        pk.psacak_inplace(b"abc", np.zeros(2, np.uint32))
    with pytest.raises(TypeError):
        pk.psacak_inplace(b"abc", np.zeros(3, np.int64))


def test_init_rejects_bad_devices_and_shutdown_without_context():
    lib = pk.lib()
    assert lib.psacak_init(-1) == pk.PSACAK_EINVAL
    assert lib.psacak_shutdown() == 0


def test_failure_path_entry_points_reject_null_context():
    lib = pk.lib()
    assert lib.psacak_cancel(None) == pk.PSACAK_EINVAL
    dl = pk._debug_lib()
    assert dl.psacak_debug_set_limits(None, 0, 0) == pk.PSACAK_EINVAL
    assert dl.psacak_debug_stalled_scan(None, None, None, 0) == pk.PSACAK_EINVAL
