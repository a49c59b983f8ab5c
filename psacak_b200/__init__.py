"""psacak_b200 -- pSACAK suffix-array construction on an NVIDIA B200.

Python mirror of hucsmn/psacak's public API (src/lib.rs):

* ``psacak(text) -> numpy.ndarray[uint32]``        (src/lib.rs:64)
* ``psacak_inplace(text, suf)``                   (src/lib.rs:77)
* ``psacak32(symbols) -> numpy.ndarray[uint32]``  (integer alphabet; the
  reference's translate_sample + psacak32 path, src/psacak32.rs:873-943)

Like the reference, the suffix array excludes the sentinel position, and the
same length limits apply (``len < 2**32 - 1`` for bytes, ``<= 2**31 - 1``
for integer symbols).  Where the reference panics, these functions raise
``ValueError``.  Every call runs on the GPU through the C ABI in
``lib/libpsacak_b200.so``; there is no CPU fallback, and importing the
functions without the built library raises ``ImportError`` on first use.
"""
import ctypes
import os
import threading

import numpy as np

__all__ = [
    "psacak", "psacak_inplace", "psacak32", "Context", "Schedule", "PsacakError",
    "ENGINE_AUTO", "ENGINE_BUCKET", "ENGINE_DOUBLING", "lib", "library_path",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "libpsacak_b200.so")

PSACAK_OK = 0
PSACAK_EINVAL = -1
PSACAK_ENOMEM = -2
PSACAK_ECUDA = -3
PSACAK_ETIMEOUT = -4
PSACAK_EINTERNAL = -5
PSACAK_ECANCELED = -6

ENGINE_AUTO = 0
ENGINE_BUCKET = 1
ENGINE_DOUBLING = 2

_ERRNAMES = {
    PSACAK_EINVAL: "EINVAL", PSACAK_ENOMEM: "ENOMEM", PSACAK_ECUDA: "ECUDA",
    PSACAK_ETIMEOUT: "ETIMEOUT", PSACAK_EINTERNAL: "EINTERNAL", PSACAK_ECANCELED: "ECANCELED",
}


class PsacakError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (_ERRNAMES.get(code, "E?"), code, msg))
        self.code = code


class Schedule(ctypes.Structure):
    """Tunables of one build (psacak_schedule).  Every schedule yields the
    same suffix array; only the speed differs."""
    _fields_ = [
        ("engine", ctypes.c_uint32),
        ("inner_engine", ctypes.c_uint32),
        ("scan_ctas_per_sm", ctypes.c_uint32),
        ("batch_chunk_mib", ctypes.c_uint32),
        ("tile_items", ctypes.c_uint32),
        ("finish_below", ctypes.c_uint32),
        ("inner_finish_below", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32 * 1),
    ]


class KernelStat(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 32),
        ("launches", ctypes.c_uint64),
        ("items", ctypes.c_uint64),
        ("bytes", ctypes.c_uint64),
        ("ms", ctypes.c_double),
    ]


class LevelInfo(ctypes.Structure):
    _fields_ = [
        ("level", ctypes.c_uint32),
        ("width", ctypes.c_uint32),
        ("m", ctypes.c_uint64),
        ("n_lms", ctypes.c_uint64),
        ("k", ctypes.c_uint64),
        ("hash", ctypes.c_uint64),
    ]


_lib = None
_lib_lock = threading.Lock()


def library_path():
    return _LIB_PATH


def lib():
    """Loads lib/libpsacak_b200.so (raises ImportError if it is not built)."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(_LIB_PATH):
            raise ImportError("psacak_b200: %s is not built; run `python -m psacak_b200.build`" % _LIB_PATH)
        L = ctypes.CDLL(_LIB_PATH)
        p, u64, u32, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int
        pp = ctypes.POINTER(ctypes.c_void_p)
        L.psacak_ctx_create.argtypes = [i32, pp]
        L.psacak_ctx_destroy.argtypes = [p]
        L.psacak_last_error_string.restype = ctypes.c_char_p
        L.psacak_version.restype = ctypes.c_char_p
        L.psacak8.argtypes = [p, u64, p]
        L.psacak_init.argtypes = [i32]
        L.psacak32.argtypes = [p, u64, p]
        L.psacak8_ctx.argtypes = [p, p, u64, p, p]
        L.psacak32_ctx.argtypes = [p, p, u64, p, p]
        L.psacak8_dev.argtypes = [p, p, u64, p, p, p]
        L.psacak32_dev.argtypes = [p, p, u64, p, p, p]
        L.psacak8_batch.argtypes = [p, p, p, u32, p, p]
        L.psacak8_batch_dev.argtypes = [p, p, p, u32, p, p, p]
        L.psacak8_batch_dev.restype = i32
        L.psacak_get_trace.argtypes = [p, p, u32, ctypes.POINTER(u32)]
        L.psacak_cancel.argtypes = [p]
        L.psacak_check_sa8_dev.argtypes = [p, p, u64, p, ctypes.POINTER(i32), p]
        L.psacak_check_sa32_dev.argtypes = [p, p, u64, p, ctypes.POINTER(i32), p]
        L.psacak_profile_enable.argtypes = [p, i32]
        L.psacak_profile_reset.argtypes = [p]
        L.psacak_profile_get.argtypes = [p, p, u32, ctypes.POINTER(u32)]
        L.psacak_check_sa8_noalloc.argtypes = [p, u64, p, ctypes.POINTER(i32), p]
        L.psacak_check_sa8_noalloc.restype = i32
        L.psacak_kernel_launches.argtypes = [p]
        L.psacak_kernel_launches.restype = u64
        L.psacak_round_trips.argtypes = [p]
        L.psacak_round_trips.restype = u64
        L.psacak_isa_dev.argtypes = [p, p, u64, p, p]
        L.psacak_bwt8_dev.argtypes = [p, p, u64, p, p, ctypes.POINTER(u64), p]
        L.psacak_lcp8_dev.argtypes = [p, p, u64, p, p, p]
        L.psacak_lcp32_dev.argtypes = [p, p, u64, p, p, p]
        L.psacak_fm_bytes.argtypes = [u64]
        L.psacak_fm_bytes.restype = u64
        L.psacak_fm_build_dev.argtypes = [p, p, u64, u64, p, p]
        L.psacak_fm_count_dev.argtypes = [p, p, p, p, p, u32, p, p]
        for f in (L.psacak_isa_dev, L.psacak_bwt8_dev, L.psacak_lcp8_dev, L.psacak_lcp32_dev,
                  L.psacak_fm_build_dev, L.psacak_fm_count_dev):
            f.restype = i32
        for name in ("psacak8", "psacak32", "psacak8_ctx", "psacak32_ctx", "psacak8_dev", "psacak32_dev",
                     "psacak8_batch", "psacak_get_trace", "psacak_check_sa8_dev", "psacak_check_sa32_dev",
                     "psacak_ctx_create", "psacak_ctx_destroy", "psacak_profile_enable", "psacak_profile_reset",
                     "psacak_profile_get", "psacak_cancel"):
            getattr(L, name).restype = i32
        _lib = L
        return L


def _raise(rc):
    if rc != PSACAK_OK:
        msg = lib().psacak_last_error_string()
        raise PsacakError(rc, msg.decode() if msg else "")


def _as_u8(text):
    if isinstance(text, (bytes, bytearray, memoryview)):
        return np.frombuffer(bytes(text), dtype=np.uint8)
    a = np.ascontiguousarray(text)
    if a.dtype != np.uint8:
        raise TypeError("psacak expects bytes or a uint8 array, got %s" % a.dtype)
    return a.reshape(-1)


def _vp(a):
    return ctypes.c_void_p(a.ctypes.data) if a.size else ctypes.c_void_p(0)


class Context:
    """A builder context on one CUDA device (psacak_ctx).  It owns a stream,
    a cached device workspace and the trace of its last build."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        _raise(lib().psacak_ctx_create(int(device), ctypes.byref(h)))
        self._h = h
        self.device = int(device)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().psacak_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- host-pointer builds -------------------------------------------------
    def psacak(self, text, schedule=None):
        t = _as_u8(text)
        if t.size >= 0xFFFFFFFF:
            raise ValueError("text length must be below 2**32 - 1")
        suf = np.empty(t.size, dtype=np.uint32)
        _raise(lib().psacak8_ctx(self._h, _vp(t), t.size, _vp(suf), _sched_ptr(schedule)))
        return suf

    def psacak32(self, symbols, schedule=None):
        t = np.ascontiguousarray(symbols, dtype=np.uint32).reshape(-1)
        if t.size > 0x7FFFFFFF:
            raise ValueError("symbol string length must be at most 2**31 - 1")
        suf = np.empty(t.size, dtype=np.uint32)
        _raise(lib().psacak32_ctx(self._h, _vp(t), t.size, _vp(suf), _sched_ptr(schedule)))
        return suf

    def psacak_batch(self, texts, schedule=None):
        arrs = [_as_u8(t) for t in texts]
        sas = [np.empty(a.size, dtype=np.uint32) for a in arrs]
        n = len(arrs)
        tp = (ctypes.c_void_p * n)(*[a.ctypes.data if a.size else 0 for a in arrs])
        sp = (ctypes.c_void_p * n)(*[s.ctypes.data if s.size else 0 for s in sas])
        lens = (ctypes.c_uint64 * n)(*[a.size for a in arrs])
        _raise(lib().psacak8_batch(self._h, tp, lens, n, sp, _sched_ptr(schedule)))
        return sas

    # -- device-pointer builds (integer pointers, e.g. torch data_ptr()) ----
    def psacak8_dev(self, d_text, n, d_sa, stream=0, schedule=None):
        _raise(lib().psacak8_dev(self._h, ctypes.c_void_p(d_text), n, ctypes.c_void_p(d_sa),
                                 ctypes.c_void_p(stream), _sched_ptr(schedule)))

    def psacak32_dev(self, d_text, n, d_sa, stream=0, schedule=None):
        _raise(lib().psacak32_dev(self._h, ctypes.c_void_p(d_text), n, ctypes.c_void_p(d_sa),
                                  ctypes.c_void_p(stream), _sched_ptr(schedule)))

    def psacak8_batch_dev(self, d_texts, offsets, d_sas, stream=0, schedule=None):
        """Texts packed in device memory; `offsets` (len = texts + 1) host ints."""
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        _raise(lib().psacak8_batch_dev(self._h, ctypes.c_void_p(d_texts), _vp(off), off.size - 1,
                                       ctypes.c_void_p(d_sas), ctypes.c_void_p(stream), _sched_ptr(schedule)))

    def isa_dev(self, d_sa, n, d_isa, stream=0):
        """Inverse suffix array: d_isa[d_sa[i]] = i (device pointers)."""
        _raise(lib().psacak_isa_dev(self._h, ctypes.c_void_p(d_sa), n, ctypes.c_void_p(d_isa),
                                    ctypes.c_void_p(stream)))

    def bwt8_dev(self, d_text, n, d_sa, d_bwt, stream=0):
        """BWT of text + sentinel without the sentinel character (divbwt
        convention) into d_bwt (n bytes); returns the primary index."""
        primary = ctypes.c_uint64(0)
        _raise(lib().psacak_bwt8_dev(self._h, ctypes.c_void_p(d_text), n, ctypes.c_void_p(d_sa),
                                     ctypes.c_void_p(d_bwt), ctypes.byref(primary), ctypes.c_void_p(stream)))
        return int(primary.value)

    def lcp8_dev(self, d_text, n, d_sa, d_lcp, stream=0):
        """LCP array of a byte text and its suffix array (device pointers)."""
        _raise(lib().psacak_lcp8_dev(self._h, ctypes.c_void_p(d_text), n, ctypes.c_void_p(d_sa),
                                     ctypes.c_void_p(d_lcp), ctypes.c_void_p(stream)))

    def lcp32_dev(self, d_text, n, d_sa, d_lcp, stream=0):
        """LCP array of a u32 text and its suffix array (device pointers)."""
        _raise(lib().psacak_lcp32_dev(self._h, ctypes.c_void_p(d_text), n, ctypes.c_void_p(d_sa),
                                      ctypes.c_void_p(d_lcp), ctypes.c_void_p(stream)))

    def fm_build_dev(self, d_bwt, n, primary, d_fm, stream=0):
        """FM-index of the BWT (divbwt convention) into d_fm, a device buffer
        of fm_bytes(n) bytes."""
        _raise(lib().psacak_fm_build_dev(self._h, ctypes.c_void_p(d_bwt), n, primary, ctypes.c_void_p(d_fm),
                                         ctypes.c_void_p(stream)))

    def fm_count_dev(self, d_fm, d_bwt, d_patterns, d_offsets, n_patterns, d_ranges, stream=0):
        """Backward search: suffix-array ranges [lo, hi) of the patterns
        (device pointers; offsets are n_patterns + 1 device uint64)."""
        _raise(lib().psacak_fm_count_dev(self._h, ctypes.c_void_p(d_fm), ctypes.c_void_p(d_bwt),
                                         ctypes.c_void_p(d_patterns), ctypes.c_void_p(d_offsets), n_patterns,
                                         ctypes.c_void_p(d_ranges), ctypes.c_void_p(stream)))

    def check_sa8_dev(self, d_text, n, d_sa, stream=0):
        ok = ctypes.c_int(0)
        _raise(lib().psacak_check_sa8_dev(self._h, ctypes.c_void_p(d_text), n, ctypes.c_void_p(d_sa),
                                          ctypes.byref(ok), ctypes.c_void_p(stream)))
        return bool(ok.value)

    def check_sa32_dev(self, d_text, n, d_sa, stream=0):
        ok = ctypes.c_int(0)
        _raise(lib().psacak_check_sa32_dev(self._h, ctypes.c_void_p(d_text), n, ctypes.c_void_p(d_sa),
                                           ctypes.byref(ok), ctypes.c_void_p(stream)))
        return bool(ok.value)

    def trace(self):
        buf = (LevelInfo * 128)()
        cnt = ctypes.c_uint32(0)
        _raise(lib().psacak_get_trace(self._h, buf, 128, ctypes.byref(cnt)))
        return [dict(level=l.level, width=l.width, m=l.m, n_lms=l.n_lms, k=l.k, hash=l.hash)
                for l in buf[:min(cnt.value, 128)]]

    def cancel(self):
        """Asks the build running on this context (or the next one) to stop;
        that build raises PsacakError with code PSACAK_ECANCELED.  Safe to
        call from another thread (psacak_cancel)."""
        _raise(lib().psacak_cancel(self._h))

    def kernel_launches(self):
        return int(lib().psacak_kernel_launches(self._h))

    def round_trips(self):
        """Host round trips (device counts read back mid-build) so far."""
        return int(lib().psacak_round_trips(self._h))

    def profile(self, on=True):
        _raise(lib().psacak_profile_enable(self._h, 1 if on else 0))

    def profile_reset(self):
        _raise(lib().psacak_profile_reset(self._h))

    def profile_stats(self):
        buf = (KernelStat * 128)()
        cnt = ctypes.c_uint32(0)
        _raise(lib().psacak_profile_get(self._h, buf, 128, ctypes.byref(cnt)))
        return [dict(name=s.name.decode(), launches=s.launches, items=s.items, bytes=s.bytes, ms=s.ms)
                for s in buf[:min(cnt.value, 128)]]


def _sched_ptr(schedule):
    if schedule is None:
        return None
    if isinstance(schedule, dict):
        s = Schedule()
        for k, v in schedule.items():
            setattr(s, k, int(v))
        schedule = s
    return ctypes.byref(schedule)


def fm_bytes(n):
    """Bytes of the FM-index of an n-byte text (psacak_fm_bytes)."""
    return int(lib().psacak_fm_bytes(n))


NOALLOC_CHECK_MAX = 1 << 21


def check_sa8_noalloc(d_text, n, d_sa, stream=0):
    """Suffix-array check for callers that may not allocate device memory:
    uses a fixed scratch array inside the library (n <= NOALLOC_CHECK_MAX);
    calls overlapping on the GPU race.  Device pointers as ints."""
    ok = ctypes.c_int(0)
    _raise(lib().psacak_check_sa8_noalloc(ctypes.c_void_p(d_text), n, ctypes.c_void_p(d_sa), ctypes.byref(ok),
                                          ctypes.c_void_p(stream)))
    return bool(ok.value)


_default = threading.local()


def _ctx():
    c = getattr(_default, "ctx", None)
    if c is None:
        c = Context(0)
        _default.ctx = c
    return c


def init(device=0):
    """Creates the calling thread's default C-ABI context on `device` now
    (psacak_init) and makes the Python default context use that device too."""
    _raise(lib().psacak_init(int(device)))
    c = getattr(_default, "ctx", None)
    if c is not None:
        c.close()
    _default.ctx = Context(int(device))


def shutdown():
    """Releases the calling thread's default contexts (psacak_shutdown); the
    next build creates new ones."""
    c = getattr(_default, "ctx", None)
    if c is not None:
        c.close()
        _default.ctx = None
    _raise(lib().psacak_shutdown())


def psacak(text):
    """Suffix array of a byte string (src/lib.rs:64), sentinel excluded."""
    return _ctx().psacak(text)


def psacak_inplace(text, suf):
    """Writes the suffix array of `text` into suf[:len(text)] (src/lib.rs:77)."""
    t = _as_u8(text)
    if not isinstance(suf, np.ndarray) or suf.dtype != np.uint32:
        raise TypeError("suf must be a numpy uint32 array")
    if t.size > suf.size:
        raise ValueError("the suffix array is shorter than the text")
    if t.size >= 0xFFFFFFFF:
        raise ValueError("text length must be below 2**32 - 1")
    if suf.flags["C_CONTIGUOUS"]:
        # write straight into the caller's buffer (only suf[:len(text)] changes)
        _raise(lib().psacak8_ctx(_ctx().handle, _vp(t), t.size, _vp(suf), None))
    else:
        suf[:t.size] = _ctx().psacak(t)


def psacak32(symbols):
    """Suffix array of an integer-alphabet string (uint32 symbols)."""
    return _ctx().psacak32(symbols)


# -- internal stages (include/psacak_b200_debug.h) ---------------------------
def _debug_lib():
    L = lib()
    if not getattr(L, "_debug_bound", False):
        p, u64, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int
        L.psacak_debug_radix_sort_u64.argtypes = [p, p, p, u64, i32, i32]
        L.psacak_debug_radix_sort_u32.argtypes = [p, p, p, u64, i32, i32]
        L.psacak_debug_exclusive_sum.argtypes = [p, p, p, u64]
        L.psacak_debug_types.argtypes = [p, p, u64, i32, p, p]
        L.psacak_debug_reduced8.argtypes = [p, p, u64, p, u64, ctypes.POINTER(u64), ctypes.POINTER(u64), p]
        L.psacak_debug_set_limits.argtypes = [p, ctypes.c_uint32, u64]
        L.psacak_debug_stalled_scan.argtypes = [p, p, p, u64]
        for name in ("psacak_debug_radix_sort_u64", "psacak_debug_radix_sort_u32", "psacak_debug_exclusive_sum",
                     "psacak_debug_types", "psacak_debug_reduced8", "psacak_debug_set_limits",
                     "psacak_debug_stalled_scan"):
            getattr(L, name).restype = i32
        L._debug_bound = True
    return L


class Stages:
    """Stage-level entry points on device pointers (ints), for tests/tuning."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.L = _debug_lib()

    def radix_sort_u64(self, d_keys, d_vals, n, b0, b1):
        _raise(self.L.psacak_debug_radix_sort_u64(self.ctx.handle, d_keys, d_vals, n, b0, b1))

    def radix_sort_u32(self, d_keys, d_vals, n, b0, b1):
        _raise(self.L.psacak_debug_radix_sort_u32(self.ctx.handle, d_keys, d_vals, n, b0, b1))

    def exclusive_sum(self, d_in, d_out, n):
        _raise(self.L.psacak_debug_exclusive_sum(self.ctx.handle, d_in, d_out, n))

    def types(self, d_text, n, width, d_types, d_lms):
        _raise(self.L.psacak_debug_types(self.ctx.handle, d_text, n, width, d_types, d_lms))

    def set_limits(self, spin_limit=0, workspace_cap=0):
        """Failure-path limits of the context: polls per bounded device wait
        (0 = compiled limits) and most workspace bytes per build (0 = none)."""
        _raise(self.L.psacak_debug_set_limits(self.ctx.handle, spin_limit, workspace_cap))

    def stalled_scan(self, d_in, d_out, n):
        """The look-back scan without its first tile: returns the status code
        (PSACAK_ETIMEOUT once the waits run out) instead of raising."""
        return int(self.L.psacak_debug_stalled_scan(self.ctx.handle, d_in, d_out, n))

    def reduced8(self, d_text, n, d_red, cap, schedule=None):
        n1 = ctypes.c_uint64(0)
        k = ctypes.c_uint64(0)
        _raise(self.L.psacak_debug_reduced8(self.ctx.handle, d_text, n, d_red, cap, ctypes.byref(n1),
                                            ctypes.byref(k), _sched_ptr(schedule)))
        return int(n1.value), int(k.value)
