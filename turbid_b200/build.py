"""Build recipe for libturbid_gpu.so (nvcc, sm_100a) -- built in-tree.

    python -m turbid_b200.build        # or turbid_b200.build.build()

The library is written next to this file so that it travels with the
repository snapshot; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libturbid_gpu.so")
BUILD_DIR = os.path.join(HERE, "_build")

CU_SOURCES = ["api.cu", "fft.cu", "gemm.cu", "fields.cu", "islice.cu"]
DRIVER_SRC = os.path.join(HERE, "host", "channelflat_gpu.cc")
DRIVER = os.path.join(HERE, "channelflat_gpu")
# the reference's solver-layer library (include/solver_channel_flat.h)
PSLIB_SRC = os.path.join(HERE, "host", "pseudospectral.cc")
PSLIB = os.path.join(HERE, "libpseudospectral.so")
# the reference's own main program, compiled unchanged against PSLIB when a
# reference source tree is at hand (built here, not committed; it travels with
# the other built files)
REFERENCE = os.environ.get("TURBID_REFERENCE", "/root/reference")
REF_MAIN = os.path.join(HERE, "channelflat")
INCLUDE = os.path.join(HERE, "..", "include")
CC_SOURCES = ["setup.cc"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, sources) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile every CUDA/C++ source of the product into libturbid_gpu.so."""
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES + CC_SOURCES]
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "turbid_gpu.h"))
    if not force and _newer(LIB, srcs + headers):
        build_driver(verbose=verbose)
        build_pseudospectral(verbose=verbose)
        return LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-lineinfo", "--expt-relaxed-constexpr"]
    objs = [os.path.join(BUILD_DIR, os.path.basename(s) + ".o") for s in srcs]

    def compile_one(src_obj):
        src, obj = src_obj
        if not force and _newer(obj, [src] + headers):
            return
        cmd = [nvcc, "-c", src, "-o", obj] + ARCH + common
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    # translation units compile in parallel (the transform kernels dominate)
    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 1)) as pool:
        list(pool.map(compile_one, zip(srcs, objs)))
    cmd = [nvcc, "-shared", "-o", LIB] + objs + ARCH + ["-Xcompiler", "-fPIC"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    build_driver(verbose=verbose, force=True)
    build_pseudospectral(verbose=verbose, force=True)
    return LIB


def build_driver(verbose: bool = False, force: bool = False) -> str:
    """The C++ main program over the plugin classes (include/turbid_plugin.hpp)."""
    deps = [DRIVER_SRC, LIB, os.path.join(INCLUDE, "turbid_plugin.hpp"), os.path.join(INCLUDE, "turbid_gpu.h")]
    if not force and _newer(DRIVER, deps):
        return DRIVER
    cxx = shutil.which("g++") or "c++"
    cmd = [cxx, "-O2", "-std=c++17", "-Wall", "-I", INCLUDE, DRIVER_SRC, "-L", HERE, "-lturbid_gpu",
           "-Wl,-rpath,$ORIGIN", "-o", DRIVER]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return DRIVER


def build_pseudospectral(verbose: bool = False, force: bool = False) -> str:
    """libpseudospectral.so (FlatChannelSolver of the reference's solver layer
    over the plugin classes) and, when the reference's main/channelflat.cc is
    at hand, that main program linked against it unchanged."""
    hdrs = [os.path.join(INCLUDE, h) for h in ("turbid_plugin.hpp", "turbid_gpu.h", "system.h",
                                               "solver_channel_flat.h")]
    cxx = shutil.which("g++") or "c++"
    if force or not _newer(PSLIB, [PSLIB_SRC, LIB] + hdrs):
        cmd = [cxx, "-O2", "-std=c++17", "-Wall", "-fPIC", "-shared", "-I", INCLUDE, PSLIB_SRC, "-L", HERE,
               "-lturbid_gpu", "-Wl,-rpath,$ORIGIN", "-o", PSLIB]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    main_src = os.path.join(REFERENCE, "main", "channelflat.cc")
    if os.path.isfile(main_src) and (force or not _newer(REF_MAIN, [main_src, PSLIB] + hdrs)):
        cmd = [cxx, "-O2", "-std=c++17", "-I", INCLUDE, main_src, "-L", HERE, "-lpseudospectral",
               "-Wl,-rpath,$ORIGIN", "-o", REF_MAIN]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return PSLIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
