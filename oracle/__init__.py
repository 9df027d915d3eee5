"""ctypes front end of the CPU oracle (``oracle/oracle.c``).

TEST INFRASTRUCTURE ONLY: the tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use it as the checker.  The product package
``alpacc_b200`` never imports it.
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


def build(force: bool = False) -> str:
    """Compile the oracle with gcc (``-O2``, no GPU needed)."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        tmp = LIB + ".tmp%d" % os.getpid()
        subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", "-o", tmp, SRC])
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
