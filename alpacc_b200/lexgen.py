"""Lexer tables: regexes -> one deterministic lexer automaton with "producing"
transitions -> the integer tables the GPU lexer and the CPU oracle read.

Host-side table generation.  The automaton restates the semantics of alpacc's
lexer DFA (``lexerDFA``, ``src/Alpacc/Lexer/DFA.hs:333-406``):

* the union of every terminal's regex is determinised by subset construction
  (``src/Alpacc/Lexer/DFA.hs:123-151``); a state accepts terminal ``t`` when it
  contains an accepting state of ``t``'s automaton, and ties go to the
  terminal declared first (``src/Alpacc/Lexer/DFA.hs:371-384``);
* a *producing* transition is added from every accepting state ``q`` on every
  byte ``b`` that ``q`` cannot take but the initial state can: it ends the
  current token and continues as if ``b`` were read from the initial state
  (``tokenProducingTransitions``, ``src/Alpacc/Lexer/DFA.hs:272-310``).

The tokens produced depend only on the regex languages, not on how the states
are numbered, so this module builds its own automaton (Thompson NFA, subset
construction, then Moore minimisation over the produce-labelled transitions)
and its own GPU tables:

* byte classes (bytes whose columns are identical) so the per-byte tables are
  ``states x classes`` instead of ``states x 256``;
* the transition monoid ("endomorphisms", ``src/Alpacc/Lexer/ParallelLexing.hs``):
  every distinct state->state function of a byte string, with the step table
  ``f . class``, the composition table ``f . g`` and the apply table ``f(s)``.
  alpacc closes only "connected" endomorphism pairs and maps the rest to dead
  (``src/Alpacc/Lexer/ParallelLexing.hs:222-292,371-397``); a pair that can never
  be adjacent composes to the constant-dead function either way, so the full
  closure used here gives the same states.
"""

from __future__ import annotations

from collections import deque
from dataclasses import dataclass
from typing import Dict, List, Optional, Tuple

from .grammar import GrammarError, T

DEAD = 0
INIT = 1


# --------------------------------------------------------------------------
# Thompson NFA over bytes
# --------------------------------------------------------------------------

class _NFA:
    def __init__(self):
        self.eps: List[List[int]] = []
        self.byte: List[List[Tuple[int, int]]] = []
        self.accept: Dict[int, T] = {}

    def new(self) -> int:
        self.eps.append([])
        self.byte.append([])
        return len(self.eps) - 1

    def chain(self, s: int, bs: bytes, t: int):
        cur = s
        for i, b in enumerate(bs):
            nxt = t if i == len(bs) - 1 else self.new()
            self.byte[cur].append((b, nxt))
            cur = nxt

    def build(self, s: int, t: int, r):
        tag = r[0]
        if tag == "eps":
            self.eps[s].append(t)
        elif tag == "lit":
            self.chain(s, r[1], t)
        elif tag == "range":
            for item in r[1]:
                self.chain(s, item, t)
        elif tag == "star":
            m = self.new()
            self.eps[s].append(m)
            self.eps[m].append(t)
            self.build(m, m, r[1])
        elif tag == "cat":
            m = self.new()
            self.build(s, m, r[1])
            self.build(m, t, r[2])
        elif tag == "alt":
            self.build(s, t, r[1])
            self.build(s, t, r[2])
        else:
            raise ValueError(tag)

    def closure(self, states) -> frozenset:
        seen = set(states)
        stack = list(states)
        while stack:
            s = stack.pop()
            for t in self.eps[s]:
                if t not in seen:
                    seen.add(t)
                    stack.append(t)
        return frozenset(seen)


def regex_dfa(regex) -> Tuple[List[Dict[int, int]], List[bool]]:
    """Plain DFA of one regex (trimmed, no dead state): ``(delta, accepting)``
    with state 0 initial.  Used by the regex known-answer tests
    (``haskell-tests/RegularExpression.hs``)."""
    nfa = _NFA()
    s, t = nfa.new(), nfa.new()
    nfa.build(s, t, regex)
    start = nfa.closure([s])
    ids = {start: 0}
    delta: List[Dict[int, int]] = [{}]
    acc = [t in start]
    q = deque([start])
    while q:
        cur = q.popleft()
        moves: Dict[int, set] = {}
        for st in cur:
            for b, nx in nfa.byte[st]:
                moves.setdefault(b, set()).add(nx)
        for b, tgt in moves.items():
            c = nfa.closure(tgt)
            if c not in ids:
                ids[c] = len(delta)
                delta.append({})
                acc.append(t in c)
                q.append(c)
            delta[ids[cur]][b] = ids[c]
    return delta, acc


def regex_match(regex, data: bytes) -> bool:
    delta, acc = regex_dfa(regex)
    s = 0
    for b in data:
        if b not in delta[s]:
            return False
        s = delta[s][b]
    return acc[s]


# --------------------------------------------------------------------------
# Lexer automaton
# --------------------------------------------------------------------------

@dataclass
class LexerDFA:
    """Minimal lexer automaton.  State 0 is dead, state 1 is initial.

    ``delta[s][b]`` is the next state on byte ``b`` (0 = dead) and
    ``produce[s][b]`` is 1 when that transition ends a token.  ``token[s]`` is
    the terminal a token ending in ``s`` gets (None when ``s`` accepts
    nothing)."""

    delta: List[List[int]]
    produce: List[List[int]]
    token: List[Optional[T]]

    @property
    def n_states(self) -> int:
        return len(self.delta)


def build_lexer_dfa(order: Dict[T, int], regex: Dict[T, tuple]) -> LexerDFA:
    nfa = _NFA()
    root = nfa.new()
    for t, rx in regex.items():
        s, a = nfa.new(), nfa.new()
        nfa.eps[root].append(s)
        nfa.build(s, a, rx)
        nfa.accept[a] = t
    start = nfa.closure([root])
    sets = [None, start]  # index 0 reserved for dead
    ids = {start: 1}
    trans: List[Dict[int, int]] = [{}, {}]
    q = deque([start])
    while q:
        cur = q.popleft()
        moves: Dict[int, set] = {}
        for st in cur:
            for b, nx in nfa.byte[st]:
                moves.setdefault(b, set()).add(nx)
        ci = ids[cur]
        for b, tgt in moves.items():
            c = nfa.closure(tgt)
            if c not in ids:
                ids[c] = len(sets)
                sets.append(c)
                trans.append({})
                q.append(c)
            trans[ci][b] = ids[c]
    n = len(sets)
    token: List[Optional[T]] = [None] * n
    for i in range(1, n):
        best = None
        for st in sets[i]:
            t = nfa.accept.get(st)
            if t is not None and (best is None or order[t] < order[best]):
                best = t
        token[i] = best
    if token[1] is not None:
        raise GrammarError("the lexer accepts the empty string")
    delta = [[DEAD] * 256 for _ in range(n)]
    produce = [[0] * 256 for _ in range(n)]
    for i in range(1, n):
        for b, j in trans[i].items():
            delta[i][b] = j
    # producing transitions (src/Alpacc/Lexer/DFA.hs:272-310)
    for i in range(1, n):
        if token[i] is None:
            continue
        for b in range(256):
            if delta[i][b] == DEAD and trans[1].get(b) is not None:
                delta[i][b] = trans[1][b]
                produce[i][b] = 1
    return _minimize(LexerDFA(delta, produce, token))


def _minimize(d: LexerDFA) -> LexerDFA:
    """Moore refinement: states with the same token and, byte by byte, the
    same produce bit and equivalent targets are merged.  Dead stays 0 and the
    initial state stays 1; the rest are numbered in BFS order."""
    n = d.n_states
    labels = {}
    block = []
    for s in range(n):
        key = ("dead",) if s == DEAD else ("tok", d.token[s].lit if d.token[s] else None,
                                               d.token[s].name if d.token[s] else None)
        block.append(labels.setdefault(key, len(labels)))
    while True:
        sigs = {}
        new_block = []
        for s in range(n):
            sig = (block[s],) + tuple((d.produce[s][b], block[d.delta[s][b]]) for b in range(256))
            new_block.append(sigs.setdefault(sig, len(sigs)))
        if len(sigs) == len(set(block)):
            block = new_block
            break
        block = new_block
    # renumber: dead 0, init 1, BFS
    order = {block[DEAD]: 0, block[INIT]: 1}
    q = deque([INIT])
    seen = {INIT}
    while q:
        s = q.popleft()
        for b in range(256):
            t = d.delta[s][b]
            if t not in seen:
                seen.add(t)
                q.append(t)
                if block[t] not in order:
                    order[block[t]] = len(order)
    rep = {}
    for s in range(n):
        if block[s] in order:
            rep.setdefault(order[block[s]], s)
    m = len(order)
    delta = [[0] * 256 for _ in range(m)]
    produce = [[0] * 256 for _ in range(m)]
    token: List[Optional[T]] = [None] * m
    for ns in range(m):
        s = rep[ns]
        token[ns] = d.token[s] if s != DEAD else None
        for b in range(256):
            delta[ns][b] = order[block[d.delta[s][b]]]
            produce[ns][b] = d.produce[s][b]
    return LexerDFA(delta, produce, token)


# --------------------------------------------------------------------------
# Byte classes and the transition monoid
# --------------------------------------------------------------------------

@dataclass
class LexerTables:
    dfa: LexerDFA
    byte_class: List[int]                 # 256 -> class
    n_classes: int                        # real classes; class n_classes is the identity pad
    cls_delta: List[List[int]]            # [S][C+1] next state
    cls_produce: List[List[int]]          # [S][C+1] produce bit
    endo: List[Tuple[int, ...]]           # E functions; endo[0] is the identity
    endo_step: List[List[int]]            # [E][C+1]
    endo_comp: List[List[int]]            # [E][E]  comp[f][g] = g after f
    class_endo: List[int]                 # [C+1]  endo id of one byte of the class


def build_lexer_tables(dfa: LexerDFA, max_endos: int = 65535) -> LexerTables:
    S = dfa.n_states
    cols = {}
    byte_class = []
    for b in range(256):
        col = tuple((dfa.delta[s][b], dfa.produce[s][b]) for s in range(S))
        byte_class.append(cols.setdefault(col, len(cols)))
    C = len(cols)
    rep = [byte_class.index(c) for c in range(C)]
    cls_delta = [[dfa.delta[s][rep[c]] for c in range(C)] + [s] for s in range(S)]
    cls_produce = [[dfa.produce[s][rep[c]] for c in range(C)] + [0] for s in range(S)]
    ident = tuple(range(S))
    cls_fun = [tuple(cls_delta[s][c] for s in range(S)) for c in range(C)]
    endo = [ident]
    ids = {ident: 0}
    step: List[List[int]] = []
    q = deque([0])
    while q:
        e = q.popleft()
        f = endo[e]
        row = []
        for c in range(C):
            g = cls_fun[c]
            h = tuple(g[f[s]] for s in range(S))
            if h not in ids:
                if len(endo) >= max_endos:
                    raise GrammarError("too many lexer endomorphisms for the GPU tables")
                ids[h] = len(endo)
                endo.append(h)
                q.append(ids[h])
            row.append(ids[h])
        row.append(e)  # identity pad class
        while len(step) <= e:
            step.append(None)
        step[e] = row
    E = len(endo)
    comp = _compose_table(endo, S)
    class_endo = [step[0][c] for c in range(C)] + [0]
    return LexerTables(dfa, byte_class, C, cls_delta, cls_produce, endo, step, comp, class_endo)


def _compose_table(endo: List[Tuple[int, ...]], S: int) -> List[List[int]]:
    """``comp[a][b]`` = id of "apply endo a, then endo b", vectorised: every
    function is hashed to a 64-bit key and looked up by binary search."""
    import numpy as np

    A = np.asarray(endo, dtype=np.int64)              # E x S
    E = A.shape[0]
    rng = np.random.default_rng(0x5EED)
    w = rng.integers(1, 2 ** 62, size=S, dtype=np.int64)
    keys = (A * w).sum(axis=1)                         # wraps mod 2^64: fine for hashing
    order = np.argsort(keys, kind="stable")
    sk = keys[order]
    if np.any(sk[1:] == sk[:-1]):
        raise RuntimeError("endomorphism hash collision")
    out = np.empty((E, E), dtype=np.int64)
    for a in range(E):
        rows = A[:, A[a]]                              # rows[b][s] = endo[b][endo[a][s]]
        hk = (rows * w).sum(axis=1)
        pos = np.searchsorted(sk, hk)
        pos = np.minimum(pos, E - 1)
        if not np.all(sk[pos] == hk):
            raise RuntimeError("composition left the endomorphism closure")
        out[a] = order[pos]
    return out.tolist()
