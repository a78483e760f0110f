"""Build recipe for the native libraries of pi-compute_b200 (in-tree, no JIT cache).

  libpigpu.so   CUDA kernels + the C ABI declared in include/pi_b200.h (sm_100a only)
  libpib200.so  C++17 host library: B200Multiplier (a pi::Multiplier over the C ABI),
                binary splitting and the pi engine, linked to libgmp.so.10 and libpigpu.so
  pi_b200       command-line program mirroring the reference's pi_compute flags

Run `python pi-compute_b200/build.py` (or __graft_entry__.build()). Objects are rebuilt only
when a source or header is newer than the target.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
INCLUDE = os.path.join(ROOT, "include")
GMP_SO = "/usr/lib/x86_64-linux-gnu/libgmp.so.10"

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", shutil.which("g++") or "g++")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-Xptxas", "-O3"] + ARCH

LIBPIGPU = os.path.join(HERE, "libpigpu.so")
LIBPIB200 = os.path.join(HERE, "libpib200.so")
PI_B200 = os.path.join(HERE, "pi_b200")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_gpu(verbose_ptxas: bool = False) -> str:
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
                 + glob.glob(os.path.join(INCLUDE, "*.h")))
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs, jobs = [], []
    for src in cu:
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if _newer(obj, [src] + hdr):
            extra = ["-Xptxas", "-v"] if verbose_ptxas else []
            jobs.append([NVCC, *NVCC_FLAGS, *extra, "-I", INCLUDE, "-c", src, "-o", obj])
    # translation units compile independently: run them side by side
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, j) for j in jobs]:
            f.result()
    if _newer(LIBPIGPU, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIBPIGPU, *objs, "-lcudart"])
    return LIBPIGPU


def build_host() -> str:
    srcs = sorted(glob.glob(os.path.join(HOST, "*.cpp")))
    if not srcs:
        return ""
    lib_srcs = [s for s in srcs if os.path.basename(s) != "main.cpp"]
    hdr = sorted(glob.glob(os.path.join(HOST, "*.h")) + glob.glob(os.path.join(INCLUDE, "*.h")))
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "include")
    cuda_lib = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "lib64")
    flags = ["-O3", "-std=c++17", "-fPIC", "-pthread", "-Wall", "-I", HOST, "-I", INCLUDE, "-I", cuda_inc]
    rpath = ["-Wl,-rpath,$ORIGIN", "-Wl,-rpath," + os.path.dirname(GMP_SO)]
    if _newer(LIBPIB200, lib_srcs + hdr + [LIBPIGPU]):
        # -Bsymbolic: the library's own classes (pi::BinarySplitting, pi::PiEngine, ...) always bind to
        # their definitions here, even in a process that also loads another library with classes of the
        # same names (the test shim that runs the reference's own sources with B200Multiplier).
        _run([CXX, *flags, "-shared", "-Wl,-Bsymbolic", "-o", LIBPIB200, *lib_srcs, LIBPIGPU, GMP_SO, "-L", cuda_lib,
              "-lcudart", *rpath])
    main = os.path.join(HOST, "main.cpp")
    if os.path.exists(main) and _newer(PI_B200, [main, LIBPIB200] + hdr):
        _run([CXX, *flags, "-o", PI_B200, main, LIBPIB200, LIBPIGPU, GMP_SO, "-L", cuda_lib, "-lcudart", *rpath])
    return LIBPIB200


def build_all(verbose_ptxas: bool = False) -> None:
    build_gpu(verbose_ptxas)
    build_host()


if __name__ == "__main__":
    build_all(verbose_ptxas="-v" in sys.argv)
