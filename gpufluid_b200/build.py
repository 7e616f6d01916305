"""Build libgfb200.so in-tree with nvcc for sm_100a.

    python -m gpufluid_b200.build [--verbose] [--bounds-check]

Every translation unit is compiled to an object (in parallel) and the objects
are linked into one shared library.  The library is written for B200 only:
the single target is compute_100a / sm_100a.

FMA contraction is decided per translation unit.  The stages that are checked
bit-for-bit against the CPU oracle (binning, forces/divergence, Jacobi and
GS-RB sweeps, projection, G2P, region compaction, the mesher, the
allocation-free Jacobi) are compiled with -fmad=false, so every product and
sum rounds separately in the reference's float32 operation order.  The
shared-memory PCG, the coarse-correction set-up and the adjoint kernels are
checked against tolerances (an FP64 solve, FP64 gradients), so they are
compiled with contraction on.
Kernels in a bit-exact unit that are themselves tolerance-checked (P2G, whose
float atomics already reorder the sums) use explicit fused multiply-adds.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgfb200.so")
OBJ = os.path.join(HERE, "_build")
# the bounds-checked variant: every instrumented index is checked (GF_IN)
LIB_CHECKED = os.path.join(HERE, "libgfb200_checked.so")
OBJ_CHECKED = os.path.join(HERE, "_build_checked")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
          "--expt-relaxed-constexpr"]
# translation units whose results are compared within a tolerance only
FMA_UNITS = {"pcg_smem.cu", "adjoint.cu", "coarse.cu"}


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def unit_flags(src: str) -> list:
    fma = "true" if os.path.basename(src) in FMA_UNITS else "false"
    return [*COMMON, f"-fmad={fma}"]


def needs_build(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [
        os.path.join(HERE, "..", "include", "gfb200.h"), os.path.abspath(__file__)]
    return any(os.path.getmtime(p) > t for p in deps)


def _env():
    env = dict(os.environ)
    env["CC"] = "gcc"
    env["CXX"] = "g++"
    return env


def _compile(src: str, verbose: bool, objdir: str, extra: list):
    obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
    cmd = [NVCC, *unit_flags(src), *extra, *(["-Xptxas", "-v"] if verbose else []), "-c", "-o",
           obj, src]
    r = subprocess.run(cmd, capture_output=True, text=True, env=_env())
    return obj, r


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    """Build libgfb200.so, or with ``checked`` the bounds-checked
    libgfb200_checked.so (-DGF_BOUNDS_CHECK)."""
    lib, objdir = (LIB_CHECKED, OBJ_CHECKED) if checked else (LIB, OBJ)
    extra = ["-DGF_BOUNDS_CHECK"] if checked else []
    if not force and not needs_build(lib):
        return lib
    os.makedirs(objdir, exist_ok=True)
    srcs = sources()
    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose, objdir, extra), srcs))
    errs = [r.stdout + r.stderr for _, r in results if r.returncode != 0]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    if verbose:
        for _, r in results:
            sys.stdout.write(r.stdout + r.stderr)
    cmd = [NVCC, *ARCH, "-shared", "-o", lib, *(o for o, _ in results)]
    r = subprocess.run(cmd, capture_output=True, text=True, env=_env())
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    return lib


if __name__ == "__main__":
    print(build(force=True, verbose="--verbose" in sys.argv,
                checked="--bounds-check" in sys.argv))
