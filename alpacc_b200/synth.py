"""Seeded synthetic workloads (host side, backed by ``csrc/synth.c``).

The reference ships no benchmark corpus for this path, so every benchmark
input is generated: JSON for ``json.alp``, arithmetic expressions for
``arithmetic.alp`` and s-expressions for ``sexp.alp``, each exactly the
requested size and deterministic in its seed.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "synth.c")
LIB = os.path.join(HERE, "_lib", "libalpsynth.so")

SEED_BASE = 0xA1FACC00


def build(force: bool = False) -> str:
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        tmp = LIB + ".tmp%d" % os.getpid()
        subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", "-o", tmp, SRC])
        os.replace(tmp, LIB)
    return LIB


_lib = None


def _L():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        for name in ("alp_synth_json", "alp_synth_arith", "alp_synth_sexp"):
            f = getattr(L, name)
            f.restype = ctypes.c_int64
            f.argtypes = [ctypes.c_uint64, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p]
        for name in ("alp_synth_json_batch", "alp_synth_sexp_batch"):
            f = getattr(L, name)
            f.restype = ctypes.c_int64
            f.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p,
                          ctypes.c_void_p]
        _lib = L
    return _lib


def _one(fn: str, seed: int, size: int, depth: int) -> np.ndarray:
    out = np.empty(max(size, 2), dtype=np.uint8)
    n = getattr(_L(), fn)(seed, size, depth, out.ctypes.data_as(ctypes.c_void_p))
    return out[:n]


def json_doc(size: int, depth: int = 8, seed: int = SEED_BASE + 2) -> np.ndarray:
    """One JSON document of exactly ``size`` bytes, nesting depth <= ``depth``."""
    return _one("alp_synth_json", seed, size, depth)


def arith_doc(size: int, depth: int = 12, seed: int = SEED_BASE + 1) -> np.ndarray:
    """Arithmetic expressions joined by '+', exactly ``size`` bytes."""
    return _one("alp_synth_arith", seed, size, depth)


def sexp_doc(size: int, depth: int = 20, seed: int = SEED_BASE + 4) -> np.ndarray:
    return _one("alp_synth_sexp", seed, size, depth)


def lognormal_sizes(n_docs: int, median: int = 4096, sigma: float = 1.5, cap: int = 4 << 20,
                    seed: int = SEED_BASE + 4) -> np.ndarray:
    rng = np.random.default_rng(seed)
    s = np.exp(np.log(median) + sigma * rng.standard_normal(n_docs))
    return np.clip(np.rint(s), 2, cap).astype(np.int64)


def batch(grammar: str, sizes: np.ndarray, depth: int, seed: int) -> Tuple[np.ndarray, np.ndarray]:
    """Documents of the given sizes back to back: (bytes, offsets[n+1])."""
    sizes = np.ascontiguousarray(sizes, dtype=np.int64)
    total = int(np.maximum(sizes, 2).sum())
    out = np.empty(max(total, 1), dtype=np.uint8)
    off = np.empty(len(sizes) + 1, dtype=np.int64)
    fn = {"json": _L().alp_synth_json_batch, "sexp": _L().alp_synth_sexp_batch}[grammar]
    fn(seed, sizes.ctypes.data_as(ctypes.c_void_p), len(sizes), depth,
       out.ctypes.data_as(ctypes.c_void_p), off.ctypes.data_as(ctypes.c_void_p))
    return out[:total], off
