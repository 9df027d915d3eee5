"""Build the in-tree native libraries.

* ``_lib/libalpacc_b200.so`` -- the CUDA kernels and the C ABI
  (``include/alpacc_b200.h``), compiled for sm_100a only.
* ``_lib/libalpsynth.so``    -- the seeded workload generators (gcc).

Run ``python -m alpacc_b200.build`` (or ``__graft_entry__.build()``).
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libalpacc_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
                  glob.glob(os.path.join(CSRC, "*.h")) + [os.path.join(HERE, "..", "include", "alpacc_b200.h")])


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in _sources())


def build_cuda(force: bool = False, verbose: bool = False, extra=()) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    if not force and not needs_build():
        return LIB
    tmp = LIB + ".tmp%d" % os.getpid()
    cmd = [NVCC] + NVCC_FLAGS + list(extra) + ["-o", tmp, os.path.join(CSRC, "capi.cu")]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


def build_all(force: bool = False, verbose: bool = False) -> None:
    from . import synth
    synth.build(force=force)
    build_cuda(force=force, verbose=verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
