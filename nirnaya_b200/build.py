"""Builds the native libraries in-tree.

  nirnaya_b200/libnir_pdhg.so   CUDA engine + C ABI (nvcc, sm_100a only)
  nirnaya_b200/libnir_lpgen.so  seeded instance generator (g++)
  nirnaya_b200/libnir_mlp.so    warm-start network (nvcc, sm_100a)
  nirnaya_b200/libnir_mps.so    multi-threaded MPS and SOL file I/O, solution check (g++, host only)
  nirnaya_b200/libnir_facade.so presolve and scaling before the path (g++, host only)

Run `python -m nirnaya_b200.build` or call build_all().
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")

NVCC_FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared", "-I" + INC]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources(pattern_dir: str, exts) -> list:
    out = []
    for d in (pattern_dir, INC):
        for f in os.listdir(d):
            if f.endswith(exts):
                out.append(os.path.join(d, f))
    return out


def build_engine(force: bool = False, verbose: bool = False) -> str:
    target = os.path.join(HERE, "libnir_pdhg.so")
    srcs = _sources(CSRC, (".cu", ".cuh", ".h", ".hpp"))
    if force or _stale(target, srcs):
        cmd = [_nvcc(), *NVCC_FLAGS, os.path.join(CSRC, "engine.cu"), "-o", target]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return target


def build_mlp(force: bool = False, verbose: bool = False) -> str:
    target = os.path.join(HERE, "libnir_mlp.so")
    srcs = [os.path.join(CSRC, "mlp.cu"), os.path.join(INC, "nir_mlp.h")]
    if force or _stale(target, srcs):
        cmd = [_nvcc(), *NVCC_FLAGS, srcs[0], "-o", target]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return target


def build_lpgen(force: bool = False, verbose: bool = False) -> str:
    target = os.path.join(HERE, "libnir_lpgen.so")
    srcs = [os.path.join(CSRC, "lpgen.cpp"), os.path.join(INC, "nir_lpgen.h"), os.path.join(INC, "nir_lp.h")]
    if force or _stale(target, srcs):
        cxx = os.environ.get("CXX", "g++")
        cmd = [cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-I" + INC, srcs[0], "-o", target]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return target


def build_mps(force: bool = False, verbose: bool = False) -> str:
    target = os.path.join(HERE, "libnir_mps.so")
    srcs = [os.path.join(CSRC, "mps.cpp"), os.path.join(CSRC, "mps_write.cpp"), os.path.join(CSRC, "sol.cpp"),
            os.path.join(CSRC, "decimal.hpp"), os.path.join(CSRC, "text.hpp"), os.path.join(INC, "nir_mps.h"),
            os.path.join(INC, "nir_sol.h"), os.path.join(INC, "nir_lp.h")]
    if force or _stale(target, srcs):
        cxx = os.environ.get("CXX", "g++")
        # no FMA contraction: the double-double steps of sol.cpp need each rounding
        cmd = [cxx, "-std=c++17", "-O3", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-pthread",
               "-I" + INC, *srcs[:3], "-o", target]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return target


def build_facade(force: bool = False, verbose: bool = False) -> str:
    target = os.path.join(HERE, "libnir_facade.so")
    srcs = [os.path.join(CSRC, "facade.cpp"), os.path.join(CSRC, "text.hpp"), os.path.join(INC, "nir_facade.h"),
            os.path.join(INC, "nir_lp.h")]
    if force or _stale(target, srcs):
        cxx = os.environ.get("CXX", "g++")
        # no FMA contraction: the reference's x86-64 build has none
        cmd = [cxx, "-std=c++17", "-O3", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-pthread",
               "-I" + INC, srcs[0], "-o", target]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return target


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_lpgen(force, verbose)
    build_mps(force, verbose)
    build_facade(force, verbose)
    build_engine(force, verbose)
    build_mlp(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
