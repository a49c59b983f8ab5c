"""Seeded synthetic inputs (ctypes over lib/libpsacak_synth.so).

The generators stand in for the reference's benchmark corpus; every input
is reproducible from its seed (xoshiro256** seeded by splitmix64).
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "libpsacak_synth.so")
_lib = None


class GenomeStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in
                ("n_bases", "n_nrun", "n_copied", "n_mutated", "n_segments")]


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            from . import build as _b
            _b.build_synth()
        L = ctypes.CDLL(_LIB_PATH)
        p, u64, u32, d = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double
        L.psacak_synth_iid.argtypes = [p, u64, p, u32, u64]
        L.psacak_synth_genome.argtypes = [p, u64, u64, p]
        L.psacak_synth_markov2.argtypes = [p, u64, u64]
        L.psacak_synth_loguniform.argtypes = [p, u64, u64, u64, u64]
        L.psacak_synth_zipf32.argtypes = [p, u64, u32, d, d, u32, u32, u64]
        L.psacak_synth_zipf32.restype = ctypes.c_int
        L.psacak_synth_hash2.argtypes = [u64, u64]
        L.psacak_synth_hash2.restype = u64
        _lib = L
    return _lib


def _vp(a):
    return ctypes.c_void_p(a.ctypes.data)


def iid(n, alphabet=b"ACGT", seed=1, out=None):
    """i.i.d. uniform bytes over `alphabet`."""
    out = np.empty(n, dtype=np.uint8) if out is None else out
    alpha = np.frombuffer(bytes(alphabet), dtype=np.uint8).copy()
    _load().psacak_synth_iid(_vp(out), n, _vp(alpha), alpha.size, seed)
    return out


def genome(n, seed=2, out=None, stats=False):
    """Order-3 Markov ACGT with ~5% N runs and ~30% mutated copies."""
    out = np.empty(n, dtype=np.uint8) if out is None else out
    st = GenomeStats()
    _load().psacak_synth_genome(_vp(out), n, seed, ctypes.byref(st))
    if stats:
        return out, {k: getattr(st, k) for k, _ in GenomeStats._fields_}
    return out


def markov2(n, seed, out=None):
    """Order-2 Markov ACGT."""
    out = np.empty(n, dtype=np.uint8) if out is None else out
    _load().psacak_synth_markov2(_vp(out), n, seed)
    return out


def loguniform(count, lo, hi, seed):
    out = np.empty(count, dtype=np.uint64)
    _load().psacak_synth_loguniform(_vp(out), count, lo, hi, seed)
    return out


def zipf32(n, alphabet=1 << 20, s=1.1, repeat_frac=0.10, rep_min=1000, rep_max=100000,
           seed=3, out=None):
    """u32 Zipf(s) symbols with planted exact repeats."""
    out = np.empty(n, dtype=np.uint32) if out is None else out
    rc = _load().psacak_synth_zipf32(_vp(out), n, alphabet, s, repeat_frac, rep_min, rep_max, seed)
    if rc != 0:
        raise MemoryError("psacak_synth_zipf32 failed")
    return out


def hash2(seed, i):
    return int(_load().psacak_synth_hash2(seed, i))
