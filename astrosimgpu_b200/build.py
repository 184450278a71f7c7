"""Build the engine library in-tree with nvcc for sm_100a.

Produces ``astrosimgpu_b200/libasg_b200.so`` (CUDA kernels, the C ABI of
``include/asg_b200.h`` and the host-side config / builder / serving code)
and the command-line driver ``astrosimgpu_b200/astrosim_b200``.  Objects go
to ``astrosimgpu_b200/_build/``; a source is recompiled when it or a header
is newer than its object.

Device code is compiled with ``-fmad=false`` so that no multiply-add is
contracted: the FP64 arithmetic of the step then matches the host build
operation for operation.  Host code is compiled with ``-ffp-contract=off``
for the same reason.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libasg_b200.so")
CLI = os.path.join(HERE, "astrosim_b200")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
NVCC_FLAGS = COMMON + ARCH + ["-lineinfo", "-fmad=false", "--expt-relaxed-constexpr",
                              "-Xcompiler", "-fPIC,-ffp-contract=off,-fopenmp",
                              "-Xptxas", "-warn-spills"]


def _sources():
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(p for p in glob.glob(os.path.join(CSRC, "*.cpp"))
                 if not p.endswith("main.cpp"))
    return cu + cpp


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp"))
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose):
    obj = os.path.join(OUT_DIR, os.path.basename(src) + ".o")
    if not _stale(obj, [src] + _headers()):
        return obj
    cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "cu"] + NVCC_FLAGS + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr.strip():
        print(res.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False) -> str:
    """Compile every source and link the shared library; returns its path."""
    os.makedirs(OUT_DIR, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-Xcompiler", "-fopenmp", "-lcudart", "-lgomp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    main = os.path.join(CSRC, "main.cpp")
    if os.path.exists(main) and _stale(CLI, [main, LIB] + _headers()):
        cmd = [NVCC, "-x", "cu"] + NVCC_FLAGS + [main, "-o", CLI, "-L" + HERE, "-lasg_b200",
                                                 "-Xlinker", "-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"CLI build failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
