"""In-tree build of the B200 ISDF library.

Produces, next to this file:
  libisdf_b200.so                  C-ABI (include/isdf_b200.h), CUDA kernels for sm_100a
  mp_isdf.cpython-*.so             pybind11 drop-in module `mp_isdf` over the C-ABI

Run ``python -m mp_isdf_b200.build`` (or ``__graft_entry__.build()``).  nvcc
cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
import sysconfig
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
                     "--expt-relaxed-constexpr", "-I", str(ROOT / "include"), "-I", str(CSRC)]
CU_SOURCES = ["context.cu", "linalg.cu", "select_sketch.cu", "select_pairqr.cu", "fit.cu",
              "capi.cu", "profile.cu", "qrcp_sketch.cu", "project_tc.cu",
              "adjoint.cu", "noalloc.cu", "gram_tiles.cu", "metric.cu", "rbrp.cu", "jk.cu"]
LIB = PKG / "libisdf_b200.so"
EXT_SUFFIX = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
PYMOD = PKG / f"mp_isdf{EXT_SUFFIX}"


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "isdf_b200.h"]


def _compile(src: str, verbose: bool) -> Path:
    obj = BUILD / (Path(src).stem + ".o")
    if _newer(obj, [CSRC / src, *_headers()]):
        cmd = [NVCC, *NVCC_FLAGS, "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return obj


def build_library(verbose=False) -> Path:
    BUILD.mkdir(exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), CU_SOURCES))
    if _newer(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [NVCC, *ARCH, "-shared", "-o", str(tmp), *map(str, objs)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


def build_pymodule(verbose=False) -> Path:
    import pybind11
    src = CSRC / "pybind_mp_isdf.cpp"
    if _newer(PYMOD, [src, LIB, ROOT / "include" / "isdf_b200.h"]):
        inc = sysconfig.get_paths()["include"]
        tmp = PYMOD.with_name(PYMOD.name + ".tmp")
        cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
               "-I", pybind11.get_include(), "-I", inc, "-I", str(ROOT / "include"),
               str(src), "-o", str(tmp), "-L", str(PKG), "-lisdf_b200",
               "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, PYMOD)
    return PYMOD


def build(verbose=False):
    build_library(verbose)
    build_pymodule(verbose)
    return LIB, PYMOD


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
    print(PYMOD)
