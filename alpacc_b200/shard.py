"""One document lexed by several GPUs (alp_lex_shard_*).

Rank r holds bytes [pos_r, pos_r + n_r) of the document.  The ranks exchange
two small records:

1. each range's state function (32 bytes), from which every rank composes its
   entry state (the reference's chunk loop carries that state from one chunk
   to the next: futhark/lexer.fut:148-160, cuda/lexer.cu:452-543);
2. each range's token count and last token start, from which every rank gets
   its first token index and the start of the token it continues.

Any all-gather does the exchange: ``torch.distributed.all_gather_object``
between processes (NCCL or gloo), or a plain list in one process.
"""

from __future__ import annotations

import ctypes
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from .api import ALP_OK, AlpError, Grammar, _torch, native

INITIAL_STATE = 1


def _lib():
    L = native()
    vp, i64, i32, P = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.POINTER
    L.alp_lex_shard_begin.argtypes = [vp, vp, i64, i64, i32, vp, P(vp)]
    L.alp_lex_shard_count.argtypes = [vp, ctypes.c_uint32, P(i64), P(i64)]
    L.alp_lex_shard_emit.argtypes = [vp, i64, vp, vp, vp, i64, P(i64), P(i32)]
    L.alp_lex_shard_free.argtypes = [vp]
    L.alp_lex_shard_free.restype = None
    return L


class Shard:
    """One byte range of a document on this process's GPU (one per Grammar at a time)."""

    def __init__(self, g: Grammar, data, pos: int, is_last: bool):
        self.g = g
        self.x = g._as_device_bytes(data)
        self.pos = pos
        self.fn = np.zeros(32, np.uint8)
        g._stream()
        h = ctypes.c_void_p()
        rc = _lib().alp_lex_shard_begin(g.h, ctypes.c_void_p(self.x.data_ptr()), self.x.numel(), pos,
                                        1 if is_last else 0, self.fn.ctypes.data_as(ctypes.c_void_p),
                                        ctypes.byref(h))
        if rc != ALP_OK:
            g._err(rc)
        self.h = h

    def count(self, entry_state: int) -> Tuple[int, int]:
        n, last = ctypes.c_int64(0), ctypes.c_int64(0)
        rc = _lib().alp_lex_shard_count(self.h, entry_state, ctypes.byref(n), ctypes.byref(last))
        if rc != ALP_OK:
            self.g._err(rc)
        self.n_tok = n.value
        return n.value, last.value

    def emit(self, carried_start: int):
        torch = _torch()
        k = max(self.n_tok, 1)
        dev = self.g.device
        term = torch.empty(k, dtype=torch.int32, device=dev)
        start = torch.empty(k, dtype=torch.int64, device=dev)
        end = torch.empty(k, dtype=torch.int64, device=dev)
        n, valid = ctypes.c_int64(0), ctypes.c_int(0)
        rc = _lib().alp_lex_shard_emit(self.h, carried_start, ctypes.c_void_p(term.data_ptr()),
                                       ctypes.c_void_p(start.data_ptr()), ctypes.c_void_p(end.data_ptr()), k,
                                       ctypes.byref(n), ctypes.byref(valid))
        if rc != ALP_OK:
            self.g._err(rc)
        m = n.value
        return (term[:m], start[:m], end[:m]), bool(valid.value)

    def close(self):
        if self.h:
            _lib().alp_lex_shard_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def entry_state(fns: Sequence[np.ndarray], rank: int) -> int:
    s = INITIAL_STATE
    for f in fns[:rank]:
        s = int(f[s])
    return s


def placement(totals: Sequence[Tuple[int, int]], rank: int) -> Tuple[int, int]:
    """(first token index, carried token start) of range `rank`."""
    base = sum(int(c) for c, _ in totals[:rank])
    starts = [int(l) for _, l in totals[:rank] if int(l) >= 0]
    return base, (max(starts) if starts else 0)


def lex_shard(g: Grammar, data, pos: int, is_last: bool, rank: int, all_gather: Callable[[object], List[object]]):
    """This rank's part of the document: ((term, start, end), first token
    index, valid).  `all_gather(x)` returns every rank's x in rank order."""
    s = Shard(g, data, pos, is_last)
    try:
        fns = all_gather(s.fn.copy())
        cnt, last = s.count(entry_state(fns, rank))
        base, carried = placement(all_gather((cnt, last)), rank)
        toks, valid = s.emit(carried)
        return toks, base, valid
    finally:
        s.close()


def lex_split(grammars: Sequence[Grammar], data: bytes, cuts: Sequence[int]):
    """The whole document through len(cuts) + 1 ranges in one process (one
    Grammar per range; the exchanges are plain lists): the tokens of the
    document, or None when it is rejected."""
    torch = _torch()
    cuts = sorted(set(int(c) for c in cuts if 0 < c < len(data)))
    bounds = [0] + cuts + [len(data)]
    if len(grammars) < len(bounds) - 1:
        raise ValueError("one Grammar per range")
    shards = [Shard(g, np.frombuffer(data[a:b], np.uint8), a, i == len(bounds) - 2)
              for i, (g, a, b) in enumerate(zip(grammars, bounds[:-1], bounds[1:]))]
    try:
        fns = [s.fn.copy() for s in shards]
        totals = [s.count(entry_state(fns, r)) for r, s in enumerate(shards)]
        parts, valid = [], True
        for r, s in enumerate(shards):
            toks, v = s.emit(placement(totals, r)[1])
            parts.append(toks)
            valid = v
        if not valid:
            return None
        return tuple(torch.cat([p[i] for p in parts]) for i in range(3))
    finally:
        for s in shards:
            s.close()
