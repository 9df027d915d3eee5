"""alpacc's test wire format, read and written on the host.

alpacc's test harness exchanges inputs and expected outputs as
``Data.Binary`` files: big-endian 64-bit integers, 1-byte booleans.

* inputs (lexer, lexer+parser): ``u64 count; repeat { u64 len; len bytes }``
  (src/Alpacc/Test/Lexer.hs:87-105);
* inputs (parser only): ``u64 count; repeat { u64 n; n x u64 terminal }``
  (src/Alpacc/Test/Parser.hs:58-66);
* lexer outputs: ``u64 count; repeat { u8 valid; [u64 n; n x (u64 term,
  u64 start, u64 end)] }`` (src/Alpacc/Test/Lexer.hs:59-85);
* parser-only outputs: ``u64 count; repeat { u8 valid; [u64 n; n x u64
  production] }`` (src/Alpacc/Test/Parser.hs:41-56);
* lexer+parser outputs: ``u64 count; repeat { u8 valid; [u64 n; n x (u8
  kind, u64 parent, u64 id, u64 start, u64 end)] }``, kind 0 = production
  with start = end = 0, 1 = terminal (src/Alpacc/Test/LexerParser.hs:54-99).

``run`` produces an output file for an input file through the batched GPU
entry points (one launch sequence for all inputs), so that results of this
backend can be diffed byte for byte against files alpacc generated, and
``compare`` reports the first difference the way ``alpacc test compare``
checks them.  The files carry no grammar; the caller supplies it.
"""

from __future__ import annotations

import struct
from typing import List, Optional, Sequence, Tuple

import numpy as np

_U64 = struct.Struct(">Q")
_NODE = np.dtype([("kind", "u1"), ("parent", ">u8"), ("id", ">u8"), ("start", ">u8"), ("end", ">u8")])
_TOKEN = np.dtype([("term", ">u8"), ("start", ">u8"), ("end", ">u8")])

Tokens = Tuple[np.ndarray, np.ndarray, np.ndarray]            # term, start, end
Tree = Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray, np.ndarray]  # parent, tag, kind, start, end


class _Reader:
    def __init__(self, buf: bytes):
        self.b = memoryview(buf)
        self.p = 0

    def u64(self) -> int:
        if self.p + 8 > len(self.b):
            raise ValueError("truncated wire file at byte %d" % self.p)
        v = _U64.unpack_from(self.b, self.p)[0]
        self.p += 8
        return v

    def u8(self) -> int:
        if self.p + 1 > len(self.b):
            raise ValueError("truncated wire file at byte %d" % self.p)
        v = self.b[self.p]
        self.p += 1
        return v

    def take(self, n: int) -> bytes:
        if self.p + n > len(self.b):
            raise ValueError("truncated wire file at byte %d" % self.p)
        v = bytes(self.b[self.p:self.p + n])
        self.p += n
        return v

    def array(self, dtype, n: int) -> np.ndarray:
        nb = np.dtype(dtype).itemsize * n
        return np.frombuffer(self.take(nb), dtype=dtype, count=n)

    def done(self):
        if self.p != len(self.b):
            raise ValueError("%d trailing bytes in wire file" % (len(self.b) - self.p))


# ---------------------------------------------------------------- inputs
def write_inputs(docs: Sequence[bytes]) -> bytes:
    out = [_U64.pack(len(docs))]
    for d in docs:
        out.append(_U64.pack(len(d)))
        out.append(bytes(d))
    return b"".join(out)


def read_inputs(buf: bytes) -> List[bytes]:
    r = _Reader(buf)
    docs = [r.take(r.u64()) for _ in range(r.u64())]
    r.done()
    return docs


def write_token_inputs(seqs: Sequence[Sequence[int]]) -> bytes:
    out = [_U64.pack(len(seqs))]
    for s in seqs:
        a = np.asarray(s, dtype=">u8")
        out.append(_U64.pack(len(a)))
        out.append(a.tobytes())
    return b"".join(out)


def read_token_inputs(buf: bytes) -> List[np.ndarray]:
    r = _Reader(buf)
    seqs = []
    for _ in range(r.u64()):
        seqs.append(r.array(">u8", r.u64()).astype(np.uint64))
    r.done()
    return seqs


# ---------------------------------------------------------------- outputs
def write_lexer_outputs(results: Sequence[Optional[Tokens]]) -> bytes:
    out = [_U64.pack(len(results))]
    for t in results:
        if t is None:
            out.append(b"\x00")
            continue
        term, start, end = (np.asarray(x) for x in t)
        rec = np.empty(len(term), dtype=_TOKEN)
        rec["term"], rec["start"], rec["end"] = term, start, end
        out.append(b"\x01" + _U64.pack(len(term)) + rec.tobytes())
    return b"".join(out)


def read_lexer_outputs(buf: bytes) -> List[Optional[Tokens]]:
    r = _Reader(buf)
    res = []
    for _ in range(r.u64()):
        if not _bool(r):
            res.append(None)
            continue
        rec = r.array(_TOKEN, r.u64())
        res.append((rec["term"].astype(np.uint64), rec["start"].astype(np.uint64), rec["end"].astype(np.uint64)))
    r.done()
    return res


def write_parser_outputs(results: Sequence[Optional[Sequence[int]]]) -> bytes:
    out = [_U64.pack(len(results))]
    for p in results:
        if p is None:
            out.append(b"\x00")
            continue
        a = np.asarray(p, dtype=">u8")
        out.append(b"\x01" + _U64.pack(len(a)) + a.tobytes())
    return b"".join(out)


def read_parser_outputs(buf: bytes) -> List[Optional[np.ndarray]]:
    r = _Reader(buf)
    res = []
    for _ in range(r.u64()):
        res.append(r.array(">u8", r.u64()).astype(np.uint64) if _bool(r) else None)
    r.done()
    return res


def write_lexparse_outputs(results: Sequence[Optional[Tree]]) -> bytes:
    out = [_U64.pack(len(results))]
    for t in results:
        if t is None:
            out.append(b"\x00")
            continue
        parent, tag, kind, start, end = (np.asarray(x) for x in t)
        rec = np.zeros(len(parent), dtype=_NODE)
        rec["kind"], rec["parent"], rec["id"] = kind, parent, tag
        term = kind.astype(bool)
        rec["start"] = np.where(term, start, 0)
        rec["end"] = np.where(term, end, 0)
        out.append(b"\x01" + _U64.pack(len(parent)) + rec.tobytes())
    return b"".join(out)


def read_lexparse_outputs(buf: bytes) -> List[Optional[Tree]]:
    r = _Reader(buf)
    res = []
    for _ in range(r.u64()):
        if not _bool(r):
            res.append(None)
            continue
        rec = r.array(_NODE, r.u64())
        if np.any(rec["kind"] > 1):
            raise ValueError("invalid node kind in wire file")
        res.append((rec["parent"].astype(np.int64), rec["id"].astype(np.uint64), rec["kind"].astype(np.uint8),
                    rec["start"].astype(np.int64), rec["end"].astype(np.int64)))
    r.done()
    return res


def _bool(r: _Reader) -> bool:
    v = r.u8()
    if v > 1:
        raise ValueError("invalid boolean byte %d in wire file" % v)
    return v == 1


# ---------------------------------------------------------------- run / compare
def run(grammar, mode: str, inputs: bytes) -> bytes:
    """Outputs for an inputs file through the GPU batch entry points.

    grammar: an ``alpacc_b200.api.Grammar`` built for the matching tables mode;
    mode: "lexer" (lexer outputs), "lexer-parser" (tree outputs) or "parser"
    (parser-only: token-id inputs, production outputs)."""
    if mode == "parser":
        seqs = read_token_inputs(inputs)
        res = []
        for s in seqs:
            p = grammar.pre_productions_int(np.asarray(s, dtype=np.uint32))
            res.append(None if p is None else p.cpu().numpy())
        return write_parser_outputs(res)
    docs = read_inputs(inputs)
    off = np.zeros(len(docs) + 1, np.int64)
    off[1:] = np.cumsum([len(d) for d in docs])
    data = np.frombuffer(b"".join(docs), np.uint8) if off[-1] else np.zeros(0, np.uint8)
    if len(docs) == 0:
        return _U64.pack(0)
    if mode == "lexer":
        term, start, end, tok_off, valid = (x.cpu().numpy() for x in grammar.lex_batch_int(data, off))
        res = [(term[tok_off[i]:tok_off[i + 1]].astype(np.uint32), start[tok_off[i]:tok_off[i + 1]],
                end[tok_off[i]:tok_off[i + 1]]) if valid[i] else None for i in range(len(docs))]
        return write_lexer_outputs(res)
    if mode == "lexer-parser":
        tree, node_off, valid = grammar.parse_batch_int(data, off)
        par, tag, kind, st, en = (x.cpu().numpy() for x in (tree.parent, tree.tag, tree.kind, tree.start, tree.end))
        node_off, valid = node_off.cpu().numpy(), valid.cpu().numpy()
        res = []
        for i in range(len(docs)):
            a, b = node_off[i], node_off[i + 1]
            res.append((par[a:b], tag[a:b].astype(np.uint32), kind[a:b], st[a:b], en[a:b]) if valid[i] else None)
        return write_lexparse_outputs(res)
    raise ValueError("mode must be 'lexer', 'parser' or 'lexer-parser'")


def compare(expected: bytes, got: bytes, mode: str) -> Optional[str]:
    """None if the two output files hold the same results, else a message
    naming the first input whose result differs."""
    reader = {"lexer": read_lexer_outputs, "parser": read_parser_outputs,
              "lexer-parser": read_lexparse_outputs}[mode]
    a, b = reader(expected), reader(got)
    if len(a) != len(b):
        return "%d results expected, %d given" % (len(a), len(b))
    for i, (x, y) in enumerate(zip(a, b)):
        if (x is None) != (y is None):
            return "input %d: expected %s, got %s" % (i, "rejection" if x is None else "a result",
                                                     "rejection" if y is None else "a result")
        if x is None:
            continue
        xs = x if isinstance(x, tuple) else (x,)
        ys = y if isinstance(y, tuple) else (y,)
        for k, (u, v) in enumerate(zip(xs, ys)):
            if len(u) != len(v) or not np.array_equal(np.asarray(u, np.int64), np.asarray(v, np.int64)):
                return "input %d: field %d differs" % (i, k)
    return None
