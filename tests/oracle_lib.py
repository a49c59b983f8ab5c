"""ctypes binding of the CPU oracle (oracle/libpsacak_oracle.so).

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg load this module.  The product path never does.
"""
import ctypes
import os

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_LIB_PATH = os.path.join(_ROOT, "oracle", "libpsacak_oracle.so")


class OracleLevel(ctypes.Structure):
    _fields_ = [
        ("level", ctypes.c_uint32),
        ("width", ctypes.c_uint32),
        ("m", ctypes.c_uint64),
        ("n_lms", ctypes.c_uint64),
        ("k", ctypes.c_uint64),
        ("hash", ctypes.c_uint64),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", os.path.join(_ROOT, "oracle")])
        _lib = ctypes.CDLL(_LIB_PATH)
        p, u64, u32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32
        _lib.oracle_psacak8.argtypes = [p, u64, p, p, u32, p]
        _lib.oracle_psacak32.argtypes = [p, u64, p, p, u32, p]
        _lib.oracle_psacak8_par.argtypes = [p, u64, p, u32]
        _lib.oracle_lcp8.argtypes = [p, u64, p, p]
        _lib.oracle_lcp32.argtypes = [p, u64, p, p]
        _lib.oracle_bwt8.argtypes = [p, u64, p, p]
        _lib.oracle_bwt8.restype = u64
        _lib.oracle_sa_range8.argtypes = [p, u64, p, p, u64, p, p]
        _lib.oracle_saca_tiny8.argtypes = [p, u64, p]
        _lib.oracle_saca_tiny32.argtypes = [p, u64, p]
        _lib.oracle_translate_sample.argtypes = [p, u64, p]
        _lib.oracle_check_sa8.argtypes = [p, u64, p]
        _lib.oracle_check_sa32.argtypes = [p, u64, p]
        _lib.oracle_hash_u32.argtypes = [p, u64]
        _lib.oracle_hash_u32.restype = u64
        _lib.oracle_reduced8.argtypes = [p, u64, p, u64, p]
        _lib.oracle_reduced8.restype = u64
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a.size else ctypes.c_void_p(0)


def _levels(buf, count):
    return [dict(level=l.level, width=l.width, m=l.m, n_lms=l.n_lms, k=l.k, hash=l.hash)
            for l in buf[:count]]


def psacak8(text, trace=False):
    t = np.ascontiguousarray(np.frombuffer(bytes(text), dtype=np.uint8) if isinstance(text, (bytes, bytearray)) else text, dtype=np.uint8)
    sa = np.zeros(t.size, dtype=np.uint32)
    buf = (OracleLevel * 64)()
    cnt = ctypes.c_uint32(0)
    rc = lib().oracle_psacak8(_ptr(t), t.size, _ptr(sa), buf, 64, ctypes.byref(cnt))
    if rc != 0:
        raise ValueError("oracle_psacak8 rejected the input")
    return (sa, _levels(buf, min(cnt.value, 64))) if trace else sa


def psacak8_par(text, threads):
    """The reference's pipelined induced scans (fetch / induce / flush) on
    `threads` threads; equal to psacak8."""
    t = np.ascontiguousarray(np.frombuffer(bytes(text), dtype=np.uint8) if isinstance(text, (bytes, bytearray)) else text, dtype=np.uint8)
    sa = np.zeros(t.size, dtype=np.uint32)
    if lib().oracle_psacak8_par(_ptr(t), t.size, _ptr(sa), threads) != 0:
        raise ValueError("oracle_psacak8_par rejected the input")
    return sa


def lcp(text, sa):
    """LCP array (Kasai et al.) of `text` (u8 or u32) with suffix array `sa`."""
    t = np.ascontiguousarray(text)
    s = np.ascontiguousarray(sa, dtype=np.uint32)
    out = np.zeros(s.size, dtype=np.uint32)
    if t.dtype == np.uint8:
        lib().oracle_lcp8(_ptr(t), t.size, _ptr(s), _ptr(out))
    else:
        t = np.ascontiguousarray(t, dtype=np.uint32)
        lib().oracle_lcp32(_ptr(t), t.size, _ptr(s), _ptr(out))
    return out


def bwt(text, sa):
    """(BWT bytes, primary index) in libdivsufsort's divbwt convention."""
    t = np.ascontiguousarray(text, dtype=np.uint8)
    s = np.ascontiguousarray(sa, dtype=np.uint32)
    out = np.zeros(t.size, dtype=np.uint8)
    primary = lib().oracle_bwt8(_ptr(t), t.size, _ptr(s), _ptr(out))
    return out, int(primary)


def psacak32(text, trace=False):
    t = np.ascontiguousarray(text, dtype=np.uint32)
    sa = np.zeros(t.size, dtype=np.uint32)
    buf = (OracleLevel * 64)()
    cnt = ctypes.c_uint32(0)
    rc = lib().oracle_psacak32(_ptr(t), t.size, _ptr(sa), buf, 64, ctypes.byref(cnt))
    if rc != 0:
        raise ValueError("oracle_psacak32 rejected the input")
    return (sa, _levels(buf, min(cnt.value, 64))) if trace else sa


def saca_tiny8(text):
    t = np.ascontiguousarray(text, dtype=np.uint8)
    sa = np.zeros(t.size, dtype=np.uint32)
    lib().oracle_saca_tiny8(_ptr(t), t.size, _ptr(sa))
    return sa


def saca_tiny32(text):
    t = np.ascontiguousarray(text, dtype=np.uint32)
    sa = np.zeros(t.size, dtype=np.uint32)
    lib().oracle_saca_tiny32(_ptr(t), t.size, _ptr(sa))
    return sa


def translate_sample(text):
    t = np.ascontiguousarray(text, dtype=np.uint32)
    out = np.zeros(t.size, dtype=np.uint32)
    ok = lib().oracle_translate_sample(_ptr(t), t.size, _ptr(out))
    return out if ok else None


def check_sa8(text, sa):
    t = np.ascontiguousarray(text, dtype=np.uint8)
    s = np.ascontiguousarray(sa, dtype=np.uint32)
    assert s.size == t.size
    return bool(lib().oracle_check_sa8(_ptr(t), t.size, _ptr(s)))


def check_sa32(text, sa):
    t = np.ascontiguousarray(text, dtype=np.uint32)
    s = np.ascontiguousarray(sa, dtype=np.uint32)
    assert s.size == t.size
    return bool(lib().oracle_check_sa32(_ptr(t), t.size, _ptr(s)))


def hash_u32(v):
    a = np.ascontiguousarray(v, dtype=np.uint32)
    return int(lib().oracle_hash_u32(_ptr(a), a.size))


def reduced8(text):
    t = np.ascontiguousarray(text, dtype=np.uint8)
    out = np.zeros(max(t.size // 2, 1), dtype=np.uint32)
    k = ctypes.c_uint64(0)
    n1 = lib().oracle_reduced8(_ptr(t), t.size, _ptr(out), out.size, ctypes.byref(k))
    return out[:n1].copy(), int(k.value)


def sa_range8(text, sa, pattern):
    """[lo, hi) of suffix-array indices whose suffixes start with `pattern`."""
    t = np.ascontiguousarray(text, dtype=np.uint8)
    s = np.ascontiguousarray(sa, dtype=np.uint32)
    pt = np.frombuffer(bytes(pattern), np.uint8).copy() if not isinstance(pattern, np.ndarray) else \
        np.ascontiguousarray(pattern, dtype=np.uint8)
    lo, hi = ctypes.c_uint64(0), ctypes.c_uint64(0)
    lib().oracle_sa_range8(_ptr(t), t.size, _ptr(s), _ptr(pt), pt.size, ctypes.byref(lo), ctypes.byref(hi))
    return int(lo.value), int(hi.value)
