"""Build the in-tree native libraries.

* ``alpacc_b200/_lib/libalpacc_b200.so`` - the CUDA path and C ABI, compiled
  for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
* ``alpacc_b200/grammar/_closure.so``  - the generator's endomorphism closure.

The wire-protocol programs are built per grammar by ``wire_program.py``.

Run ``python -m alpacc_b200.build``; rebuilds only when sources are newer.
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libalpacc_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(REPO, "include", "*.h")))


def build_lib(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sources()
    if not force and not _newer(LIB, srcs + headers()):
        return LIB
    objs = []
    for s in srcs:
        o = os.path.join(LIBDIR, os.path.basename(s) + ".o")
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-c", s, "-o", o,
               "-I", os.path.join(REPO, "include")]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.check_call(cmd)
        objs.append(o)
    subprocess.check_call([NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"])
    for o in objs:
        os.remove(o)
    return LIB


def build_all(force: bool = False, verbose: bool = False) -> None:
    from .grammar import lexgen

    lexgen._closure_lib()
    build_lib(force=force, verbose=verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
