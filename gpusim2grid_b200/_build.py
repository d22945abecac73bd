"""In-tree build of the native library and its Python binding.

Produces, next to this file:
  lib/libgs2g.so                       C-ABI core (include/gs2g.h): C++ host code
                                       + sm_100a CUDA kernels, static cudart
  _gs2g<EXT_SUFFIX>                    pybind11 binding of that C-ABI

Run ``python gpusim2grid_b200/_build.py`` (or ``__graft_entry__.build()``).
nvcc cross-compiles for sm_100a without a GPU.  Rebuilds only what is stale.
"""

from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libgs2g.so"
EXT = PKG / ("_gs2g" + sysconfig.get_config_var("EXT_SUFFIX"))
CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["nr_kernel.cu", "mlp_kernels.cu"]
CPP_SOURCES = ["plan.cpp", "session.cpp"]
HEADERS = ["nr_kernel.cuh", "chord_sweep.cuh", "adjoint.cuh", "plan.hpp", "dense_lu.cuh", "dense_lu_f32.cuh",
           "dense_lu_f64.cuh"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def build(verbose: bool = False) -> None:
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    hdrs = [CSRC / h for h in HEADERS] + [INCLUDE / "gs2g.h"]
    jobs = []
    objs = []
    for src in CU_SOURCES:
        obj = BUILD / (src + ".o")
        objs.append(obj)
        if _stale(obj, [CSRC / src] + hdrs):
            # GS2G_NVCC_DEFINES: build-time tunables, e.g. "-DGS2G_DENSE_KC=32"
            extra = os.environ.get("GS2G_NVCC_DEFINES", "").split()
            jobs.append([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", *extra,
                         "-Xptxas", "-v", "-c", str(CSRC / src), "-o", str(obj)])
    for src in CPP_SOURCES:
        obj = BUILD / (src + ".o")
        objs.append(obj)
        if _stale(obj, [CSRC / src] + hdrs):
            jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-Wall", "-I", str(CUDA_HOME / "include"),
                         "-c", str(CSRC / src), "-o", str(obj)])
    with ThreadPoolExecutor(max_workers=4) as ex:
        for r in ex.map(_run, jobs):
            if verbose:
                sys.stdout.write(r.stdout + r.stderr)
    if _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs),
              "-Xlinker", "--no-undefined", "-lpthread", "-ldl", "-lrt"])
    import pybind11

    binding = CSRC / "pybind_module.cpp"
    if _stale(EXT, [binding, LIB, INCLUDE / "gs2g.h"]):
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I", pybind11.get_include(),
              "-I", sysconfig.get_paths()["include"], str(binding), "-o", str(EXT),
              "-L", str(LIB.parent), "-lgs2g", "-Wl,-rpath,$ORIGIN/lib"])


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print("built", LIB, EXT)
