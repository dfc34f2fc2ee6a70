"""Build recipe of the native libraries (in-tree, so they travel with the repo).

* ``_lib/libnkgpu.so``  - the CUDA PageRank library behind include/nkgpu.h,
  compiled for sm_100a only.
* ``_lib/libnkgen.so``  - host-side synthetic graph generators and the
  NetworkitBinaryGraph file decoder (C++/OpenMP), used by the benchmarks and
  tests to make their inputs and by :mod:`networkit_b200.graphio`.
* ``_cypagerank*.so``   - the Cython ``PageRank`` class (``_cypagerank.pyx``
  with the declarations of ``_nkgpu.pxd``), compiled against include/nkgpu.h
  and linked to ``_lib/libnkgpu.so``.

``python -m networkit_b200.build`` rebuilds whatever is out of date.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "_lib")
INCLUDE = os.path.join(ROOT, "include")

GPU_LIB = os.path.join(LIBDIR, "libnkgpu.so")
GEN_LIB = os.path.join(LIBDIR, "libnkgen.so")

GPU_SOURCES = ["nkgpu.cu", "noalloc.cu", "ppr.cu", "adjoint.cu", "batch.cu", "centrality.cu",
               "local.cu", "part.cu", "nkbg.cu"]
GPU_HEADERS = ["common.cuh", "sweep.cuh", "refine.cuh", "graph.hpp", "host.hpp"]
GEN_SOURCES = ["graphgen.cpp", "graphio.cpp"]
# Restatements of the reference's generators: compiled as the reference is
# (baseline x86-64, no floating-point contraction) so that they round alike.
GEN_EXACT_SOURCES = ["refgen.cpp"]
GEN_HEADERS = ["nkgen.hpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _host_cxx() -> str:
    # The system g++ ships libgomp; an inherited CXX may not.
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def _stale(target, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_gpu(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in GPU_SOURCES]
    deps = srcs + [os.path.join(CSRC, h) for h in GPU_HEADERS] + [os.path.join(INCLUDE, "nkgpu.h"),
                                                                  __file__]
    if not force and not _stale(GPU_LIB, deps):
        return GPU_LIB
    os.makedirs(LIBDIR, exist_ok=True)
    cmd = [_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-ccbin", _host_cxx(),
           "-I" + INCLUDE, "-I" + CSRC, "-o", GPU_LIB + ".tmp", *srcs]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(GPU_LIB + ".tmp", GPU_LIB)
    return GPU_LIB


def build_gen(force: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in GEN_SOURCES]
    exact = [os.path.join(CSRC, s) for s in GEN_EXACT_SOURCES]
    deps = srcs + exact + [os.path.join(CSRC, h) for h in GEN_HEADERS] + [
        os.path.join(INCLUDE, "nkgio.h"), __file__]
    if not force and not _stale(GEN_LIB, deps):
        return GEN_LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs = []
    for src in exact:
        obj = os.path.join(LIBDIR, os.path.basename(src) + ".o")
        subprocess.run([_host_cxx(), "-std=c++17", "-O3", "-ffp-contract=off", "-fopenmp", "-fPIC",
                        "-c", "-o", obj, src], check=True)
        objs.append(obj)
    cmd = [_host_cxx(), "-std=c++17", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared",
           "-I", INCLUDE,
           "-o", GEN_LIB + ".tmp", *srcs, *objs]
    subprocess.run(cmd, check=True)
    os.replace(GEN_LIB + ".tmp", GEN_LIB)
    return GEN_LIB


def cython_target() -> str:
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    return os.path.join(PKG, "_cypagerank" + suffix)


def build_cython(force: bool = False) -> str:
    """Cythonize ``_cypagerank.pyx`` and link it to libnkgpu.so (found at run
    time through an ``$ORIGIN/_lib`` rpath)."""
    pyx = os.path.join(PKG, "_cypagerank.pyx")
    pxd = os.path.join(PKG, "_nkgpu.pxd")
    target = cython_target()
    if not force and not _stale(target, [pyx, pxd, GPU_LIB, os.path.join(INCLUDE, "nkgpu.h"),
                                         __file__]):
        return target
    os.makedirs(LIBDIR, exist_ok=True)
    c_file = os.path.join(LIBDIR, "_cypagerank.c")
    subprocess.run([sys.executable, "-m", "cython", "-3", "-I", ROOT, "-o", c_file, pyx],
                   check=True)
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else (shutil.which("gcc") or "gcc")
    cmd = [cc, "-O2", "-fPIC", "-shared", "-I", sysconfig.get_paths()["include"], "-I", INCLUDE,
           "-o", target + ".tmp", c_file, "-L", LIBDIR, "-l:libnkgpu.so",
           "-Wl,-rpath,$ORIGIN/_lib"]
    subprocess.run(cmd, check=True)
    os.replace(target + ".tmp", target)
    return target


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_gen(force)
    build_gpu(force, verbose)
    build_cython(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
