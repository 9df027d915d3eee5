"""One document lexed (alp_lex_shard_*) and parsed (alp_parse_shard_*) by
several GPUs.

Lexing.  Rank r holds bytes [pos_r, pos_r + n_r) of the document.  The ranks
exchange two small records:

1. each range's state function (32 bytes), from which every rank composes its
   entry state (the reference's chunk loop carries that state from one chunk
   to the next: futhark/lexer.fut:148-160, cuda/lexer.cu:452-543);
2. each range's token count and last token start, from which every rank gets
   its first token index and the start of the token it continues.

Parsing.  Rank r holds a contiguous slice of the document's tokens (the
first slice's positions start with ⊢, the last's end with ⊣).  The ranks
exchange three small records:

1. the terminals at each slice's edges, from which every rank builds the key
   windows across its edges (futhark/parser.fut:117-122, 235-240);
2. each slice's position sums, from which every rank gets the sums of the
   slices before it: node, bracket and terminal offsets, depth and
   exscan(arity - 1) (futhark/parser.fut:153-166, 286-290);
3. each slice's staircases (node values and bracket depths strictly below
   everything after them in the slice), which answer the previous
   smaller-or-equal searches that leave a slice: parents and bracket matches
   (futhark/parser.fut:72-108, 174-184, 291-298).

Any all-gather does the exchange: ``torch.distributed.all_gather_object``
between processes (NCCL or gloo), or a plain list in one process.
"""

from __future__ import annotations

import ctypes
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from .api import ALP_OK, AlpError, Grammar, Tree, _torch, native

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


# ---- parsing ------------------------------------------------------------------

HALO = 16  # terminals each slice keeps on either side (lookback + lookahead <= 16)


def _plib():
    L = native()
    vp, i64, i32, P = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.POINTER
    L.alp_parse_shard_begin.argtypes = [vp, vp, vp, vp, i64, i32, i32, vp, P(i64), P(vp)]
    L.alp_parse_shard_sums.argtypes = [vp, vp, vp, vp]
    L.alp_parse_shard_expand.argtypes = [vp, vp, i64, i64, P(i64), P(i64), P(i64)]
    L.alp_parse_shard_stairs.argtypes = [vp, vp, vp, vp, vp]
    L.alp_parse_shard_resolve.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, P(i32)]
    L.alp_parse_shard_tree.argtypes = [vp] + [P(vp)] * 5 + [P(i64), P(i64)]
    L.alp_parse_shard_free.argtypes = [vp]
    L.alp_parse_shard_free.restype = None
    return L


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class ParseShard:
    """One slice of a document's tokens on this process's GPU (one per Grammar at a time)."""

    def __init__(self, g: Grammar, term, start, end, is_first: bool, is_last: bool):
        torch = _torch()
        self.g = g
        self.term = torch.as_tensor(term).to(g.device, torch.int32).contiguous()
        self.start = torch.as_tensor(start).to(g.device, torch.int64).contiguous()
        self.end = torch.as_tensor(end).to(g.device, torch.int64).contiguous()
        self.edge = np.zeros(2 * HALO, np.uint32)
        n_pos = ctypes.c_int64(0)
        g._stream()
        h = ctypes.c_void_p()
        rc = _plib().alp_parse_shard_begin(g.h, ctypes.c_void_p(self.term.data_ptr()),
                                           ctypes.c_void_p(self.start.data_ptr()),
                                           ctypes.c_void_p(self.end.data_ptr()), self.term.numel(),
                                           1 if is_first else 0, 1 if is_last else 0, _ptr(self.edge),
                                           ctypes.byref(n_pos), ctypes.byref(h))
        if rc != ALP_OK:
            g._err(rc)
        self.h = h
        self.n_pos = n_pos.value

    def sums(self, halo_l: np.ndarray, halo_r: np.ndarray) -> np.ndarray:
        out = np.zeros(10, np.int64)
        hl = np.ascontiguousarray(halo_l, np.uint32)
        hr = np.ascontiguousarray(halo_r, np.uint32)
        rc = _plib().alp_parse_shard_sums(self.h, _ptr(hl), _ptr(hr), _ptr(out))
        if rc != ALP_OK:
            self.g._err(rc)
        return out

    def expand(self, pre: Sequence[int], pos_base: int, closed_next: int) -> Tuple[int, int, int]:
        p = np.asarray(pre, np.int64)
        n, sn, sb = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
        rc = _plib().alp_parse_shard_expand(self.h, _ptr(p), pos_base, closed_next, ctypes.byref(n),
                                            ctypes.byref(sn), ctypes.byref(sb))
        if rc != ALP_OK:
            self.g._err(rc)
        self.sizes = (n.value, sn.value, sb.value)
        return self.sizes

    def stairs(self):
        """(node values, node indices, bracket values, bracket symbols) of the slice's staircases."""
        _, sn, sb = self.sizes
        nv, ni = np.zeros(max(sn, 1), np.int32), np.zeros(max(sn, 1), np.int64)
        bv, bs = np.zeros(max(sb, 1), np.int32), np.zeros(max(sb, 1), np.uint32)
        rc = _plib().alp_parse_shard_stairs(self.h, _ptr(nv), _ptr(ni), _ptr(bv), _ptr(bs))
        if rc != ALP_OK:
            self.g._err(rc)
        return nv[:sn], ni[:sn], bv[:sb], bs[:sb]

    def resolve(self, earlier) -> bool:
        """This slice's verdict, with the staircases of the slices before it (rank order)."""
        k = len(earlier)
        n_off = np.zeros(k + 1, np.int64)
        b_off = np.zeros(k + 1, np.int64)
        n_off[1:] = np.cumsum([len(x[0]) for x in earlier]) if k else []
        b_off[1:] = np.cumsum([len(x[2]) for x in earlier]) if k else []
        cat = lambda j, dt: np.ascontiguousarray(np.concatenate([x[j] for x in earlier]) if k else np.zeros(1, dt),
                                                 dt)
        nv, ni, bv, bs = cat(0, np.int32), cat(1, np.int64), cat(2, np.int32), cat(3, np.uint32)
        if len(nv) == 0:
            nv, ni = np.zeros(1, np.int32), np.zeros(1, np.int64)
        if len(bv) == 0:
            bv, bs = np.zeros(1, np.int32), np.zeros(1, np.uint32)
        valid = ctypes.c_int(0)
        rc = _plib().alp_parse_shard_resolve(self.h, k, _ptr(n_off), _ptr(nv), _ptr(ni), _ptr(b_off), _ptr(bv),
                                             _ptr(bs), ctypes.byref(valid))
        if rc != ALP_OK:
            self.g._err(rc)
        return bool(valid.value)

    def tree(self) -> Tuple[Tree, int]:
        """The slice's nodes (copies) and the global index of its first node."""
        from .api import _wrap
        torch = _torch()
        pp = [ctypes.c_void_p() for _ in range(5)]
        n, first = ctypes.c_int64(0), ctypes.c_int64(0)
        rc = _plib().alp_parse_shard_tree(self.h, *[ctypes.byref(x) for x in pp], ctypes.byref(n),
                                          ctypes.byref(first))
        if rc != ALP_OK:
            self.g._err(rc)
        k = n.value
        parts = [_wrap(self.g.h, p.value, k, dt, self.g.device) if k else torch.zeros(0, dtype=dt, device=self.g.device)
                 for p, dt in zip(pp, (torch.int64, torch.int32, torch.uint8, torch.int64, torch.int64))]
        return Tree(*parts), first.value

    def close(self):
        if self.h:
            _plib().alp_parse_shard_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def halos(edges: Sequence[Tuple[np.ndarray, int]], rank: int, empty: int) -> Tuple[np.ndarray, np.ndarray]:
    """The terminals of the HALO positions before and after slice `rank`, from
    every slice's (edge terminals, position count), walking past short slices."""
    left: List[int] = []
    for r in range(rank - 1, -1, -1):
        e, n = edges[r]
        k = min(HALO, int(n))
        left = [int(x) for x in e[2 * HALO - k:]] + left
        if len(left) >= HALO:
            break
    left = [empty] * max(0, HALO - len(left)) + left[-HALO:]
    right: List[int] = []
    for r in range(rank + 1, len(edges)):
        e, n = edges[r]
        k = min(HALO, int(n))
        right += [int(x) for x in e[:k]]
        if len(right) >= HALO:
            break
    right = (right + [empty] * HALO)[:HALO]
    return np.array(left, np.uint32), np.array(right, np.uint32)


def _combine(a, b):
    """Position sums of a slice followed by b (depth, v, terminals and the last
    head restart at a head, futhark's segmented scans)."""
    h = int(b[5]) != 0
    return (a[0] + b[0], a[1] + b[1], b[2] if h else a[2] + b[2], b[3] if h else a[3] + b[3],
            b[4] if h else a[4] + b[4], a[5] + b[5], b[6] if h else a[6], a[7] + b[7])


def prefix(sums: Sequence[np.ndarray], rank: int):
    p = (0, 0, 0, 0, 0, 0, -1, 0)
    for x in sums[:rank]:
        p = _combine(p, tuple(int(v) for v in x[:8]))
    return p


def closed_next(sums: Sequence[np.ndarray], edges: Sequence[Tuple[np.ndarray, int]], rank: int) -> int:
    """Bracket pairs the next slice with positions closes at its first
    position (the slices between, if any, are empty); none for an empty slice."""
    if int(edges[rank][1]) == 0:
        return 0
    for r in range(rank + 1, len(sums)):
        if int(edges[r][1]) > 0:
            return int(sums[r][8])
    return 0


def parse_shard(g: Grammar, toks, is_first: bool, is_last: bool, rank: int,
                all_gather: Callable[[object], List[object]]):
    """This rank's slice of the tree: (Tree, global index of its first node,
    valid for the whole document).  `toks` = (term, start, end) of the
    slice; `all_gather(x)` returns every rank's x in rank order."""
    s = ParseShard(g, *toks, is_first, is_last)
    try:
        empty = int(g.tables.parser.empty)
        edges = all_gather((s.edge.copy(), s.n_pos))
        hl, hr = halos(edges, rank, empty)
        sums = all_gather(s.sums(hl, hr))
        s.expand(prefix(sums, rank), sum(int(n) for _, n in edges[:rank]), closed_next(sums, edges, rank))
        stairs = all_gather(s.stairs())
        valid = s.resolve(stairs[:rank])
        ok = all(all_gather(valid))
        tree, first = s.tree()
        return tree, first, ok
    finally:
        s.close()


def parse_split(grammars: Sequence[Grammar], toks, cuts: Sequence[int]):
    """A document's tokens parsed as len(cuts) + 1 slices in one process (one
    Grammar per slice; the exchanges are plain lists; repeated cuts give empty
    slices): the whole tree as numpy arrays (parent, tag, kind, start, end),
    or None when rejected."""
    term, start, end = (np.asarray(x) for x in toks)
    m = len(term)
    cuts = sorted(int(c) for c in cuts if 0 <= c <= m)
    bounds = [0] + cuts + [m]
    R = len(bounds) - 1
    if len(grammars) < R:
        raise ValueError("one Grammar per slice")
    shards = [ParseShard(g, term[a:b], start[a:b], end[a:b], i == 0, i == R - 1)
              for i, (g, a, b) in enumerate(zip(grammars, bounds[:-1], bounds[1:]))]
    try:
        empty = int(grammars[0].tables.parser.empty)
        edges = [(s.edge.copy(), s.n_pos) for s in shards]
        sums = [s.sums(*halos(edges, r, empty)) for r, s in enumerate(shards)]
        for r, s in enumerate(shards):
            s.expand(prefix(sums, r), sum(int(n) for _, n in edges[:r]), closed_next(sums, edges, r))
        stairs = [s.stairs() for s in shards]
        valid = [s.resolve(stairs[:r]) for r, s in enumerate(shards)]
        parts = [s.tree() for s in shards]
        if not all(valid):
            return None
        return tuple(np.concatenate([getattr(t, f).cpu().numpy() for t, _ in parts])
                     for f in ("parent", "tag", "kind", "start", "end"))
    finally:
        for s in shards:
            s.close()
