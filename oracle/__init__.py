"""ctypes front end of the CPU oracle.

* ``oracle.c`` -- the sequential restatement of the reference's lexer and
  parser (the checker);
* ``par.c``    -- the same results by the templates' data-parallel algorithm,
  one document on all host cores with OpenMP (the timed CPU baseline);
* the seeded workload generators, compiled from ``alpacc_b200/csrc/synth.c``
  into this library as well, so that the CPU baseline generates its inputs
  without loading the product's libraries.

TEST INFRASTRUCTURE ONLY: the tests, ``__graft_entry__.smoke()`` and the CPU
baseline legs of ``bench.py`` use it.  The product package ``alpacc_b200``
never imports it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "oracle.c")
SRCS = [SRC, os.path.join(HERE, "par.c"), os.path.join(HERE, "..", "alpacc_b200", "csrc", "synth.c")]
DEPS = SRCS + [os.path.join(HERE, "oracle.h")]


def build(force: bool = False) -> str:
    """Compile the oracle with gcc (``-O2 -fopenmp``, no GPU needed)."""
    if force or not os.path.exists(LIB) or any(os.path.getmtime(LIB) < os.path.getmtime(x) for x in DEPS):
        tmp = LIB + ".tmp%d" % os.getpid()
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-shared", "-fPIC", "-o", tmp] + SRCS)
        os.replace(tmp, LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        vp, i64, u64p = ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p
        L.orc_load.restype = vp
        L.orc_load.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        L.orc_free.argtypes = [vp]
        for name in ("orc_tokenize",):
            getattr(L, name).argtypes = [vp, vp, i64, vp, vp, vp, i64, vp]
        L.orc_lex_futhark.argtypes = [vp, vp, i64, i64, vp, vp, vp, i64, vp]
        L.orc_pre_productions.argtypes = [vp, vp, i64, vp, i64, vp]
        for name in ("orc_parse_futhark", "orc_parse_glue"):
            getattr(L, name).argtypes = [vp, vp, vp, vp, i64, vp, vp, vp, vp, vp, i64, vp]
        L.orc_max_pair_prods.restype = i64
        L.orc_max_pair_prods.argtypes = [vp]
        L.par_create.restype = vp
        L.par_create.argtypes = [vp, ctypes.c_int]
        L.par_free.argtypes = [vp]
        L.par_threads.argtypes = [vp]
        L.par_lex.argtypes = [vp, vp, i64, vp, vp, vp, vp]
        L.par_parse.argtypes = [vp, vp, vp, vp, i64, vp, vp, vp, vp, vp, vp]
        L.par_lex_parse.argtypes = [vp, vp, i64, vp, vp, vp, vp, vp, vp]
        for name in ("alp_synth_json", "alp_synth_arith", "alp_synth_sexp"):
            f = getattr(L, name)
            f.restype = i64
            f.argtypes = [ctypes.c_uint64, i64, ctypes.c_int, vp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    """Sequential restatement of the reference lexer and parser over one
    grammar's table blob."""

    def __init__(self, blob: bytes):
        self._blob = blob
        self.h = lib().orc_load(blob, len(blob))
        if not self.h:
            raise ValueError("oracle: bad table blob")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_free(self.h)
            self.h = None

    # ---- lexer --------------------------------------------------------------
    def _lex(self, fn, data: bytes, *extra) -> Optional[Tuple[np.ndarray, np.ndarray, np.ndarray]]:
        buf = np.frombuffer(data, dtype=np.uint8) if len(data) else np.zeros(1, np.uint8)
        cap = len(data) + 1
        term = np.zeros(cap, np.uint32)
        start = np.zeros(cap, np.int64)
        end = np.zeros(cap, np.int64)
        n = ctypes.c_int64(0)
        rc = fn(self.h, _p(buf), len(data), *extra, _p(term), _p(start), _p(end), cap, ctypes.byref(n))
        if rc < 0:
            raise RuntimeError("oracle capacity")
        if rc == 0:
            return None
        k = n.value
        return term[:k].copy(), start[:k].copy(), end[:k].copy()

    def tokenize(self, data: bytes):
        """``tokenize``: None when the input is rejected."""
        return self._lex(lib().orc_tokenize, data)

    def lex_futhark(self, data: bytes, chunk: int = 0):
        """The generated ``lex_int`` with its chunk loop (``chunk`` <= 0: one chunk)."""
        return self._lex(lib().orc_lex_futhark, data, ctypes.c_int64(chunk))

    # ---- parser -------------------------------------------------------------
    def max_pair_prods(self) -> int:
        return int(lib().orc_max_pair_prods(self.h))

    def pre_productions(self, terms: np.ndarray):
        terms = np.ascontiguousarray(terms, dtype=np.uint32)
        cap = (len(terms) + 2) * max(1, self.max_pair_prods())
        out = np.zeros(cap, np.uint32)
        n = ctypes.c_int64(0)
        t = terms if len(terms) else np.zeros(1, np.uint32)
        rc = lib().orc_pre_productions(self.h, _p(t), len(terms), _p(out), cap, ctypes.byref(n))
        if rc < 0:
            raise RuntimeError("oracle capacity")
        return None if rc == 0 else out[:n.value].copy()

    def _parse(self, fn, terms, starts, ends):
        terms = np.ascontiguousarray(terms, dtype=np.uint32)
        starts = np.ascontiguousarray(starts, dtype=np.int64)
        ends = np.ascontiguousarray(ends, dtype=np.int64)
        m = len(terms)
        cap = (m + 2) * max(1, self.max_pair_prods())
        parent = np.zeros(cap, np.int64)
        tag = np.zeros(cap, np.uint32)
        kind = np.zeros(cap, np.uint8)
        ns = np.zeros(cap, np.int64)
        ne = np.zeros(cap, np.int64)
        n = ctypes.c_int64(0)
        if m == 0:
            terms, starts, ends = np.zeros(1, np.uint32), np.zeros(1, np.int64), np.zeros(1, np.int64)
        rc = fn(self.h, _p(terms), _p(starts), _p(ends), m, _p(parent), _p(tag), _p(kind), _p(ns),
                _p(ne), cap, ctypes.byref(n))
        if rc < 0:
            raise RuntimeError("oracle capacity")
        if rc == 0:
            return None
        k = n.value
        return parent[:k].copy(), tag[:k].copy(), kind[:k].copy(), ns[:k].copy(), ne[:k].copy()

    def parse_futhark(self, terms, starts, ends):
        """The generated ``parse_int`` over a token array: (parent, tag, kind,
        start, end) per node, or None."""
        return self._parse(lib().orc_parse_futhark, terms, starts, ends)

    def parse_glue(self, terms, starts, ends):
        """Sequential ``llpParse`` + tree flattening (cross-check)."""
        return self._parse(lib().orc_parse_glue, terms, starts, ends)

    def lex_parse(self, data: bytes):
        """The generated lexer+parser ``parse_int``: bytes in, tree out."""
        toks = self.lex_futhark(data)
        if toks is None:
            return None
        return self.parse_futhark(*toks)


def _take(ptr: ctypes.c_void_p, n: int, dtype) -> np.ndarray:
    """Copy n elements out of a context-owned par.c buffer."""
    if n == 0 or not ptr.value:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(np.ctypeslib.as_ctypes_type(dtype))),
                                 shape=(n,)).copy()


class Par:
    """The data-parallel restatement (``par.c``) over one grammar's table
    blob: one document at a time on ``threads`` host threads (0: all).  Its
    buffers live in the context; the methods copy results out."""

    def __init__(self, blob: bytes, threads: int = 0):
        self._o = Oracle(blob)
        self.h = lib().par_create(self._o.h, threads)
        if not self.h:
            raise ValueError("par: key space too large for the direct index")
        self.threads = int(lib().par_threads(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            lib().par_free(self.h)
            self.h = None

    def lex(self, data):
        """Tokens (term, start, end) or None when rejected."""
        buf = np.frombuffer(data, dtype=np.uint8) if len(data) else np.zeros(1, np.uint8)
        p = [ctypes.c_void_p() for _ in range(3)]
        n = ctypes.c_int64(0)
        ok = lib().par_lex(self.h, _p(buf), len(data), *[ctypes.byref(x) for x in p], ctypes.byref(n))
        if ok < 0:
            raise MemoryError("par.c: out of host memory")
        out = (_take(p[0], n.value, np.uint32), _take(p[1], n.value, np.int64), _take(p[2], n.value, np.int64))
        return out if ok else None

    def parse(self, terms, starts, ends):
        """Tree (parent, tag, kind, start, end) over a token array, or None."""
        terms = np.ascontiguousarray(terms, dtype=np.uint32)
        starts = np.ascontiguousarray(starts, dtype=np.int64)
        ends = np.ascontiguousarray(ends, dtype=np.int64)
        m = len(terms)
        if m == 0:
            terms, starts, ends = np.zeros(1, np.uint32), np.zeros(1, np.int64), np.zeros(1, np.int64)
        p = [ctypes.c_void_p() for _ in range(5)]
        n = ctypes.c_int64(0)
        ok = lib().par_parse(self.h, _p(terms), _p(starts), _p(ends), m, *[ctypes.byref(x) for x in p],
                             ctypes.byref(n))
        return self._tree(ok, p, n.value)

    def lex_parse(self, data):
        """Bytes in, tree (parent, tag, kind, start, end) out, or None."""
        buf = np.frombuffer(data, dtype=np.uint8) if len(data) else np.zeros(1, np.uint8)
        p = [ctypes.c_void_p() for _ in range(5)]
        n = ctypes.c_int64(0)
        ok = lib().par_lex_parse(self.h, _p(buf), len(data), *[ctypes.byref(x) for x in p], ctypes.byref(n))
        return self._tree(ok, p, n.value)

    def lex_parse_count(self, data):
        """(valid, nodes) of a lex+parse whose outputs stay in the context:
        the timed form, without the copies into numpy arrays."""
        buf = np.frombuffer(data, dtype=np.uint8) if len(data) else np.zeros(1, np.uint8)
        p = [ctypes.c_void_p() for _ in range(5)]
        n = ctypes.c_int64(0)
        ok = lib().par_lex_parse(self.h, _p(buf), len(data), *[ctypes.byref(x) for x in p], ctypes.byref(n))
        if ok < 0:
            raise MemoryError("par.c: out of host memory")
        return int(ok), n.value

    @staticmethod
    def _tree(ok, p, n):
        if ok < 0:
            raise MemoryError("par.c: out of host memory")
        out = (_take(p[0], n, np.int64), _take(p[1], n, np.uint32), _take(p[2], n, np.uint8),
               _take(p[3], n, np.int64), _take(p[4], n, np.int64))
        return out if ok else None


def synth_json(size: int, depth: int, seed: int) -> np.ndarray:
    """The seeded JSON generator (same source as the product's generator)."""
    out = np.empty(max(size, 2), dtype=np.uint8)
    n = lib().alp_synth_json(seed, size, depth, _p(out))
    return out[:n]
