"""Builds the native library in-tree: orion_b200/liborion_gpu.so (sm_100a).

    python -m orion_b200.build            # build (skips when up to date)
    python -m orion_b200.build --force

The FP64 translation unit is compiled with --fmad=false so no multiply-add is
contracted: the reference CPU build has no FMA either, and the plain form is
meant to reproduce its arithmetic operation by operation.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "liborion_gpu.so")
OBJDIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")) +
                  glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) +
                  glob.glob(os.path.join(INCLUDE, "*.h")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in _sources())


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False, out: str = None, defines=()) -> str:
    lib = out or LIB
    if not force and out is None and not _stale():
        return LIB
    nvcc = _nvcc()
    os.makedirs(OBJDIR, exist_ok=True)
    common = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC,
              *[f"-D{d}" for d in defines]]
    objdir = OBJDIR if out is None else out + ".objs"
    os.makedirs(objdir, exist_ok=True)
    objs = []
    # device TUs
    strict = ["--fmad=false", "-prec-div=true", "-prec-sqrt=true"]
    units = {
        "orion_gpu.cu": strict,
        "stages_fp64.cu": strict,
        "stages_mixed.cu": ["--fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
        "noalloc.cu": strict,
    }
    for name, extra in units.items():
        obj = os.path.join(objdir, name + ".o")
        log = _run([nvcc, *ARCH, *common, *extra, "-Xptxas", "-v", "-c", os.path.join(CSRC, name), "-o", obj])
        if verbose:
            print(log)
        objs.append(obj)
    # host set-up code: plain C++ without contraction
    for name in ("metrics_host.cpp",):
        obj = os.path.join(objdir, name + ".o")
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-I", INCLUDE, "-c",
              os.path.join(CSRC, name), "-o", obj])
        objs.append(obj)
    tmp = lib + ".tmp"
    _run([nvcc, *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", tmp, "-lcudart"])
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
