"""Assemble every table of one grammar and serialise it as the blob that the
C-ABI library (``alp_ctx_create``) and the CPU oracle load.

Modes mirror alpacc's three generators (``src/Alpacc/Generator/Analyzer.hs``):

* ``"lexer"``  -- ``mkLexer`` (lines 106-131): lexer-only terminal ids.
* ``"parser"`` -- ``mkParser`` (lines 149-191): token ids in, productions out.
* ``"both"``   -- ``mkLexerParser`` (lines 193-250): bytes in, tree out; the
  lexer emits the parser's symbol ids.

Blob layout (little endian; every section 4-byte aligned)::

    u32 magic 'ALPB', u32 version, u32 has_lexer, u32 has_parser
    lexer:  u32 S, C, E, ignore_term (0xffffffff = none), dead_term, n_terminals
            u8  byte_class[256]                     (padded to 4)
            u16 delta256[S][256]  next | produce<<15 (oracle form, every byte)
            u16 cls_delta[S][C+1] next | produce<<15 (class C = identity pad) (padded to 4)
            u32 token[S]          terminal id (dead_term when not accepting)
            u8  accept[S]                          (padded to 4)
            u16 endo_step[E][C+1]; u16 endo_comp[E][E]; u16 endo_apply[E][S]  (each padded to 4)
    parser: u32 q, k, n_term_syms, empty, start(⊢), end(⊣), n_prods, n_terminals
            u32 arity[n_prods]; i32 prod_term[n_prods]
            u32 n_pairs; u32 pair[n_pairs][4]  (stack_begin, stack_end, prod_begin, prod_end)
            u32 n_stack; u32 stack[n_stack]    (symbol | is_left<<31)
            u32 n_pseq;  u32 pseq[n_pseq]
            u32 n_keys;  u32 keys[n_keys][q+k]; u32 key_pair[n_keys]
"""

from __future__ import annotations

import hashlib
import os
import struct
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

from . import grammar as G
from .lexgen import LexerTables, build_lexer_dfa, build_lexer_tables
from .llp import CFGInt, LLPTableBuilder

MAGIC = 0x42504C41  # 'ALPB'
VERSION = 1


@dataclass
class ParserTables:
    q: int
    k: int
    n_term_syms: int
    empty: int
    start: int
    end: int
    arity: List[int]
    prod_term: List[int]
    pairs: List[Tuple[int, int, int, int]]
    stack: List[int]
    pseq: List[int]
    keys: List[Tuple[int, ...]]
    key_pair: List[int]
    triples: Dict[Tuple[Tuple[int, ...], Tuple[int, ...]], tuple] = field(default_factory=dict)


@dataclass
class Tables:
    mode: str
    lexer: Optional[LexerTables]
    parser: Optional[ParserTables]
    terminal_names: List[str]
    production_names: List[str]
    ignore_term: Optional[int]
    dead_term: int
    lexer_token_ids: Dict[str, int]

    def blob(self) -> bytes:
        return serialize(self)


def _pad4(b: bytearray):
    while len(b) % 4:
        b.append(0)


def build_tables(alp_text: str, mode: str = "both") -> Tables:
    cfg = G.parse_cfg(alp_text)
    lex = None
    par = None
    term_enc: Dict[tuple, int]
    prod_names: List[str] = []
    if mode == "lexer":
        order, regex = G.lexer_spec(cfg)
        term_enc = G.encode_lexer_terminals(order)
    else:
        pg = G.parsing_grammar(cfg)
        sym_enc = G.encode_symbols(pg)
        term_enc = {s[1]: i for s, i in sym_enc.items() if s[0] == "t" and s[1][0] in ("used", "unused")}
        prod_names = G.production_names(pg)
        par = _build_parser(cfg, pg, sym_enc, term_enc)
    dead_term = term_enc[("unused",)]
    ignore_term = term_enc.get(("used", G.IGNORE))
    if mode in ("lexer", "both"):
        order, regex = G.lexer_spec(cfg)
        dfa = build_lexer_dfa(order, regex)
        lex = build_lexer_tables(dfa)
    names = G.terminal_names(term_enc)
    tok_ids = {}
    for s, i in term_enc.items():
        if s[0] == "used":
            tok_ids[s[1].pretty()] = i
    return Tables(mode, lex, par, names, prod_names, ignore_term, dead_term, tok_ids)


def _build_parser(cfg: G.CFG, pg: G.ParsingGrammar, sym_enc, term_enc) -> ParserTables:
    # integer grammar: terminals first (by symbol id), then nonterminals
    n_t = sum(1 for s in sym_enc if s[0] == "t")
    def sid(sym):
        return sym_enc[sym]
    prods = []
    for lhs, rhs in pg.productions:
        prods.append((sid(("n", lhs)), tuple(sid(x) for x in rhs)))
    g = CFGInt(n_t, len(sym_enc), prods, sid(("n", pg.start)))
    q, k = cfg.lookback, cfg.lookahead
    b = LLPTableBuilder(g, q, k)
    table = b.collection_table()
    starts = b.starts()
    triples = dict(starts)
    triples.update(table)  # table entries win (src/Alpacc/LLP.hs:562)
    empty = term_enc[("unused",)]
    rts = sym_enc[("t", ("rts",))]
    lts = sym_enc[("t", ("lts",))]
    # homomorphisms (src/Alpacc/LLP.hs:568-572) and key padding
    # (src/Alpacc/Encode.hs:259-282)
    items = []
    for (x, y), (alpha, omega, pi) in triples.items():
        if (x, y) in starts and (x, y) not in table:
            br = [(1 << 31) | o for o in reversed(omega)]
        else:
            br = [a for a in alpha] + [(1 << 31) | o for o in reversed(omega)]
        key = tuple([empty] * (q - len(x[:q])) + list(x[:q]) + list(y[:k]) + [empty] * (k - len(y[:k])))
        items.append((key, br, list(pi)))
    items.sort()
    pairs, stack, pseq, keys, key_pair = [], [], [], [], []
    for key, br, pi in items:
        pairs.append((len(stack), len(stack) + len(br), len(pseq), len(pseq) + len(pi)))
        stack.extend(br)
        pseq.extend(pi)
        keys.append(key)
        key_pair.append(len(pairs) - 1)
    arity = [sum(1 for s in rhs if not g.is_t(s)) for _, rhs in prods]
    prod_term = []
    for lhs, _rhs in pg.productions:
        if lhs[0] == "wrap":
            prod_term.append(term_enc[("used", lhs[1])])
        else:
            prod_term.append(-1)
    return ParserTables(q, k, n_t, empty, rts, lts, arity, prod_term, pairs, stack, pseq,
                        keys, key_pair, triples)


def serialize(t: Tables) -> bytes:
    b = bytearray()
    b += struct.pack("<4I", MAGIC, VERSION, 1 if t.lexer else 0, 1 if t.parser else 0)
    n_terms = len(t.terminal_names)
    if t.lexer:
        L = t.lexer
        d = L.dfa
        S, C, E = d.n_states, L.n_classes, len(L.endo)
        b += struct.pack("<6I", S, C, E, 0xFFFFFFFF if t.ignore_term is None else t.ignore_term,
                         t.dead_term, n_terms)
        b += bytes(L.byte_class)
        for s in range(S):
            b += struct.pack("<256H", *[d.delta[s][x] | (d.produce[s][x] << 15) for x in range(256)])
        for s in range(S):
            b += struct.pack("<%dH" % (C + 1), *[L.cls_delta[s][c] | (L.cls_produce[s][c] << 15)
                                                 for c in range(C + 1)])
        _pad4(b)
        tok = []
        for s in range(S):
            tt = d.token[s]
            tok.append(t.dead_term if tt is None else t.lexer_token_ids[tt.pretty()])
        b += struct.pack("<%dI" % S, *tok)
        b += bytes([1 if d.token[s] is not None else 0 for s in range(S)])
        _pad4(b)
        for e in range(E):
            b += struct.pack("<%dH" % (C + 1), *L.endo_step[e])
        _pad4(b)
        for e in range(E):
            b += struct.pack("<%dH" % E, *L.endo_comp[e])
        _pad4(b)
        for e in range(E):
            b += struct.pack("<%dH" % S, *L.endo[e])
        _pad4(b)
    if t.parser:
        P = t.parser
        b += struct.pack("<8I", P.q, P.k, P.n_term_syms, P.empty, P.start, P.end, len(P.arity), n_terms)
        b += struct.pack("<%dI" % len(P.arity), *P.arity)
        b += struct.pack("<%di" % len(P.prod_term), *P.prod_term)
        b += struct.pack("<I", len(P.pairs))
        for p in P.pairs:
            b += struct.pack("<4I", *p)
        b += struct.pack("<I", len(P.stack)) + struct.pack("<%dI" % len(P.stack), *P.stack)
        b += struct.pack("<I", len(P.pseq)) + struct.pack("<%dI" % len(P.pseq), *P.pseq)
        b += struct.pack("<I", len(P.keys))
        for key in P.keys:
            b += struct.pack("<%dI" % (P.q + P.k), *key)
        b += struct.pack("<%dI" % len(P.key_pair), *P.key_pair)
    return bytes(b)


# --------------------------------------------------------------------------
# Grammar files and a cache of built blobs
# --------------------------------------------------------------------------

GRAMMAR_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "grammars")


def grammar_path(name: str) -> str:
    if os.path.exists(name):
        return name
    return os.path.join(GRAMMAR_DIR, name if name.endswith(".alp") else name + ".alp")


_CACHE: Dict[Tuple[str, str], Tables] = {}


def load(name: str, mode: str = "both") -> Tables:
    """Build (once per process) the tables of a grammar file by name or path."""
    path = grammar_path(name)
    with open(path, "r", encoding="utf-8") as f:
        text = f.read()
    key = (hashlib.sha256(text.encode()).hexdigest(), mode)
    if key not in _CACHE:
        _CACHE[key] = build_tables(text, mode)
    return _CACHE[key]
