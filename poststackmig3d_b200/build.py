"""Build recipe for the native parts of poststackmig3d_b200 (in-tree, no JIT cache).

    python -m poststackmig3d_b200.build [--force] [--debug-bounds]

produces
    poststackmig3d_b200/lib/libpsm_cuda.so   sm_100a kernels + C ABI (include/psm.h)
    poststackmig3d_b200/lib/libpsm_host.so   C++ host surface (include/psm_host.h)
    poststackmig3d_b200/bin/poststackmig     the config.txt-driven migration binary
nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
BIN = os.path.join(PKG, "bin")
INC = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# translation units of libpsm_cuda.so, compiled in parallel and linked into one library
CUDA_SRC = [os.path.join(CSRC, "psm_cuda.cu"), os.path.join(CSRC, "psm_limbs.cu")]
CUDA_HDR = [os.path.join(CSRC, h) for h in ("psm_kernels.cuh", "psm_adjoint.cuh",
                                             "psm_segy.cuh", "psm_vrms.cuh")] + \
    [os.path.join(INC, "psm.h")]
CUDA_DEPS = CUDA_SRC + CUDA_HDR
# Flush-to-zero: the reference's -ffast-math build runs with FTZ/DAZ set (GCC links
# crtfastmath), and without it every rsqrt carries a subnormal fix-up.  Divisions and square
# roots that must round like the reference use the explicit __f*_rn intrinsics.
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-ftz=true"]
HOST_SRC = [os.path.join(CSRC, "host", f) for f in
            ("config.cpp", "segy.cpp", "velocity.cpp", "driver.cpp", "host_abi.cpp")]
HOST_DEPS = HOST_SRC + [os.path.join(CSRC, "host", "host.hpp"),
                        os.path.join(INC, "psm_host.h"), os.path.join(INC, "psm.h")]
MAIN_SRC = os.path.join(CSRC, "host", "main.cpp")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_cuda(force: bool = False, extra=()) -> str:
    """Each translation unit compiles to an object under _build/ (in parallel, only when it
    or a header changed), then nvcc links the objects into lib/libpsm_cuda.so."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libpsm_cuda.so")
    if not force and not extra and not _stale(out, CUDA_DEPS):
        return out  # newer than every source (the objects need not be present)
    obj_dir = os.path.join(PKG, "_build", "debug" if extra else "release")
    os.makedirs(obj_dir, exist_ok=True)
    objs = [os.path.join(obj_dir, os.path.basename(s)[:-3] + ".o") for s in CUDA_SRC]
    todo = [(s, o) for s, o in zip(CUDA_SRC, objs)
            if force or _stale(o, [s] + CUDA_HDR)]
    with ThreadPoolExecutor(max_workers=len(CUDA_SRC)) as ex:
        list(ex.map(lambda so: _run([NVCC, *ARCH, *NVCC_FLAGS, "-Xcompiler", "-fPIC,-fopenmp",
                                     f"-I{INC}", *extra, "-c", "-o", so[1], so[0]]), todo))
    if force or todo or _stale(out, objs):
        _run([NVCC, *ARCH, "-shared", "-o", out, *objs, "-lgomp"])
    return out


def build_host(force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    out = os.path.join(LIB, "libpsm_host.so")
    if all(os.path.exists(s) for s in HOST_SRC):
        if force or _stale(out, HOST_DEPS + [os.path.join(LIB, "libpsm_cuda.so")]):
            _run([CXX, "-std=c++17", "-O2", "-fPIC", "-shared", "-fopenmp", f"-I{INC}",
                  "-o", out, *HOST_SRC, f"-L{LIB}", "-lpsm_cuda", "-Wl,-rpath,$ORIGIN"])
        exe = os.path.join(BIN, "poststackmig")
        if force or _stale(exe, [MAIN_SRC, out]):
            _run([CXX, "-std=c++17", "-O2", f"-I{INC}", "-o", exe, MAIN_SRC, f"-L{LIB}",
                  "-lpsm_host", "-lpsm_cuda", "-Wl,-rpath,$ORIGIN/../lib"])
    return out


def build(force: bool = False, debug_bounds: bool = False) -> None:
    """debug_bounds: the forward kernel checks that every sample index it reads lies inside
    its staged window and reports PSM_ERR_DEVICE instead of reading outside it (slower;
    for validation runs)."""
    build_cuda(force, ["-DPSM_DEBUG_BOUNDS"] if debug_bounds else ())
    build_host(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, debug_bounds="--debug-bounds" in sys.argv)
