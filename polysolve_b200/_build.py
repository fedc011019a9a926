"""Builds the native libraries of polysolve_b200 in-tree.

* ``libpolysolve_mas.so``   - the MAS-PCG solver: sm_100a CUDA kernels + C++ host + C-ABI
  (``include/polysolve_mas.h``).
* ``libpolysolve_syn.so``   - the seeded synthetic elasticity generator (host C++, OpenMP).
* ``mas_cpp_test``          - a C++ program that drives the solver through the C++ header
  ``include/polysolve/linear/MASSolver.hpp`` the way polysolve's own tests drive ``Solver``.

The oracle under ``oracle/`` (test infrastructure) has its own recipe: ``oracle.oracle.build()``.
Everything is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
INCLUDE = ROOT / "include"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

MAS_LIB = PKG / "libpolysolve_mas.so"
SYN_LIB = PKG / "libpolysolve_syn.so"
CPP_TEST = PKG / "mas_cpp_test"

CU_SOURCES = [
    "mas_bsr.cu",
    "mas_spmv.cu",
    "mas_build.cu",
    "mas_apply.cu",
    "mas_pcg.cu",
    "mas_noalloc.cu",
    "mas_multi.cu",
    "mas_multi16.cu",
    "mas_warmstart.cu",
    "mas_ws_train.cu",
]
CPP_SOURCES = ["mas_capi.cpp", "mas_trainer.cpp", "mas_ordering.cpp", "mas_json.cpp", "mas_market.cpp"]


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if res.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + res.stdout)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.hpp")) + sorted(
        INCLUDE.rglob("*.h*")
    )


def build_syn(force: bool = False) -> Path:
    src = CSRC / "synthetic.cpp"
    if force or _stale(SYN_LIB, [src]):
        _run(["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-o", str(SYN_LIB), str(src)])
    return SYN_LIB


def build_mas(force: bool = False, verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    objs = []
    hdrs = _headers()
    common_inc = ["-I", str(CSRC), "-I", str(INCLUDE)]
    for name in CU_SOURCES:
        src = CSRC / name
        obj = BUILD / (name + ".o")
        if force or _stale(obj, [src] + hdrs):
            cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++20", "-Xcompiler", "-fPIC,-fopenmp",
                   "--expt-relaxed-constexpr", *common_inc, "-c", str(src), "-o", str(obj)]
            if verbose_ptxas:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
        objs.append(obj)
    for name in CPP_SOURCES:
        src = CSRC / name
        obj = BUILD / (name + ".o")
        if force or _stale(obj, [src] + hdrs):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", *common_inc,
                  "-I", str(CUDA_HOME / "include"), "-c", str(src), "-o", str(obj)])
        objs.append(obj)
    if force or _stale(MAS_LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(MAS_LIB), *map(str, objs),
              "-Xcompiler", "-fopenmp", "-lcudart", "-Xlinker", "--no-undefined"])
    return MAS_LIB


def build_cpp_test(force: bool = False) -> Path:
    src = CSRC / "mas_cpp_test.cpp"
    if force or _stale(CPP_TEST, [src, MAS_LIB] + _headers()):
        _run(["g++", "-O2", "-std=c++17", "-Wall", "-I", str(INCLUDE), "-o", str(CPP_TEST), str(src),
              f"-L{PKG}", "-lpolysolve_mas", f"-Wl,-rpath,{PKG}", "-Wl,-rpath,$ORIGIN"])
    return CPP_TEST


def build_all(force: bool = False) -> None:
    build_syn(force)
    build_mas(force)
    build_cpp_test(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", MAS_LIB, SYN_LIB, CPP_TEST)
