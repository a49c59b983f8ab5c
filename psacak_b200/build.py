"""Builds the native libraries of psacak_b200 in-tree.

lib/libpsacak_b200.so  -- the CUDA builder (sm_100a) and its C ABI
lib/libpsacak_synth.so -- host-only synthetic-input generators
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
OBJ = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")

CU_SOURCES = ["prims.cu", "level.cu", "induce_doubling.cu", "induce_bucket.cu", "api.cu", "noalloc.cu", "batch.cu", "selector.cu", "gen.cu", "derived.cu", "hostio.cu", "small.cu", "fmindex.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-I", INCLUDE,
]


def nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "psacak_b200.h"))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, extra, verbose):
    obj = os.path.join(OBJ, src.replace(".cu", ".o"))
    deps = [os.path.join(CSRC, src)] + _headers()
    if not _stale(obj, deps):
        return obj, None
    cmd = [nvcc()] + NVCC_FLAGS + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
    return obj, (r.stderr if verbose else None)


def build_cuda(verbose=False, extra=None):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    extra = list(extra or [])
    if verbose:
        extra += ["-Xptxas", "-v"]
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        results = list(ex.map(lambda s: _compile(s, extra, verbose), CU_SOURCES))
    objs = [r[0] for r in results]
    for _, log in results:
        if log:
            sys.stderr.write(log)
    out = os.path.join(LIB, "libpsacak_b200.so")
    if _stale(out, objs):
        cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", out] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    return out


def build_synth():
    os.makedirs(LIB, exist_ok=True)
    src = os.path.join(CSRC, "synth.c")
    out = os.path.join(LIB, "libpsacak_synth.so")
    if _stale(out, [src]):
        subprocess.check_call(["gcc", "-O3", "-march=x86-64-v2", "-fPIC", "-shared", "-o", out, src, "-lm"])
    return out


def build_all(verbose=False):
    build_synth()
    return build_cuda(verbose=verbose)


if __name__ == "__main__":
    print(build_all(verbose="-v" in sys.argv))
