"""LLP(q,k) parser tables (Vagner & Melichar 2007, Algorithm 8) as alpacc
builds them.

Host-side table generation.  The table decides which inputs are accepted, so
this is a step-by-step restatement of alpacc's construction, not a different
LLP algorithm:

* FIRST_k / FOLLOW_k with truncated products and the End-padded extended
  grammar (``src/Alpacc/LL.hs:188-551``); LAST_q / BEFORE_q are FIRST / FOLLOW
  of the reversed grammar with every string reversed (``src/Alpacc/LL.hs:482-491``).
* the LL(k) table with its conflict check (``llTableM``, ``src/Alpacc/LL.hs:589-612``)
  and the configuration parse of one admissible pair (``parseLlpConfig``,
  ``src/Alpacc/LLP.hs:471-491``, shortest prefix first: ``src/Alpacc/LLP.hs:97-114``).
* the item-set collection: initial set D0 (``src/Alpacc/LLP.hs:83-95``), step
  3(a) (``src/Alpacc/LLP.hs:238-275``), step 3(b) closure
  (``src/Alpacc/LLP.hs:281-335``), grouping by the symbol before the dot
  (``src/Alpacc/LLP.hs:351-373``) and the breadth-first collection with the
  non-LLP conflict check (``src/Alpacc/LLP.hs:377-447``).
* start pairs and the bracket homomorphism (``src/Alpacc/LLP.hs:495-572``).

Symbols are small integers: ``0 .. n_terminals-1`` are terminals, the rest are
nonterminals.  A string is a tuple of symbols.
"""

from __future__ import annotations

from collections import deque
from functools import lru_cache
from typing import Dict, FrozenSet, Iterable, List, Optional, Sequence, Set, Tuple

from .grammar import GrammarError

Str = Tuple[int, ...]


def trunc_product(k: int, a: Iterable[Str], b: Iterable[Str]) -> FrozenSet[Str]:
    """``truncatedProduct`` (``src/Alpacc/LL.hs:188-193``)."""
    b = list(b)
    out = set()
    for x in a:
        if len(x) >= k:
            if b:
                out.add(x[:k])
            continue
        for y in b:
            out.add((x + y)[:k])
    return frozenset(out)


class CFGInt:
    """An integer grammar: ``prods[i] = (lhs, rhs)``."""

    def __init__(self, n_terms: int, n_syms: int, prods: Sequence[Tuple[int, Str]], start: int):
        self.n_terms = n_terms
        self.n_syms = n_syms
        self.prods = [(l, tuple(r)) for l, r in prods]
        self.start = start
        self.by_lhs: Dict[int, List[int]] = {}
        for i, (l, _) in enumerate(self.prods):
            self.by_lhs.setdefault(l, []).append(i)
        self.nonterminals = sorted({l for l, _ in self.prods} | {start})

    def is_t(self, s: int) -> bool:
        return s < self.n_terms

    def reversed(self) -> "CFGInt":
        return CFGInt(self.n_terms, self.n_syms, [(l, tuple(reversed(r))) for l, r in self.prods], self.start)


class FirstFollow:
    """FIRST_k and FOLLOW_k of one grammar (``firstAndFollow'``,
    ``src/Alpacc/LL.hs:502-536``)."""

    def __init__(self, g: CFGInt, k: int):
        self.g = g
        self.k = k
        self.first_map = self._first_map(g, k)
        self._memo: Dict[Str, FrozenSet[Str]] = {}
        self.follow_map = self._follow_map()

    @staticmethod
    def _first_of(g: CFGInt, k: int, fm: Dict[int, FrozenSet[Str]], syms: Str) -> FrozenSet[Str]:
        cur: FrozenSet[Str] = frozenset([()])
        for s in syms:
            if all(len(x) >= k for x in cur):
                break
            if g.is_t(s):
                cur = trunc_product(k, cur, [(s,)])
            else:
                cur = trunc_product(k, cur, fm.get(s, frozenset()))
            if not cur:
                break
        return cur

    @classmethod
    def _first_map(cls, g: CFGInt, k: int) -> Dict[int, FrozenSet[Str]]:
        fm: Dict[int, FrozenSet[Str]] = {nt: frozenset() for nt in g.nonterminals}
        while True:
            new = dict(fm)
            for l, r in g.prods:
                new[l] = new[l] | cls._first_of(g, k, fm, r)
            if new == fm:
                return fm
            fm = new

    def first(self, syms: Str) -> FrozenSet[Str]:
        syms = tuple(syms)
        r = self._memo.get(syms)
        if r is None:
            r = self._first_of(self.g, self.k, self.first_map, syms)
            self._memo[syms] = r
        return r

    def _follow_map(self) -> Dict[int, FrozenSet[Str]]:
        # Extended grammar: ExtendedStart -> S End^k, End a fresh terminal
        # (src/Alpacc/LL.hs:389-409,448-480).  End is encoded as -1.
        g, k = self.g, self.k
        END = -1
        ext_start = g.n_syms  # fresh nonterminal id
        fm = dict(self.first_map)
        fm[ext_start] = frozenset([tuple([END] * k)]) if True else frozenset()

        def first_ext(syms: Str) -> FrozenSet[Str]:
            cur: FrozenSet[Str] = frozenset([()])
            for s in syms:
                if all(len(x) >= k for x in cur):
                    break
                if s == END or g.is_t(s):
                    cur = trunc_product(k, cur, [(s,)])
                else:
                    cur = trunc_product(k, cur, fm[s])
                if not cur:
                    break
            return cur

        prods = [(ext_start, (g.start,) + tuple([END] * k))] + list(g.prods)
        right = []
        for aj, syms in prods:
            for i, s in enumerate(syms):
                if s != END and not g.is_t(s):
                    right.append((aj, s, syms[i + 1:]))
        fol: Dict[int, FrozenSet[Str]] = {nt: frozenset() for nt in g.nonterminals}
        fol[ext_start] = frozenset()
        fol[g.start] = frozenset([tuple([END] * k)])
        firsts = {w: first_ext(w) for _, _, w in right}
        while True:
            new = dict(fol)
            for aj, ai, w in right:
                new[ai] = new[ai] | trunc_product(k, firsts[w], fol[aj])
            if new == fol:
                break
            fol = new
        out = {}
        for nt, ss in fol.items():
            if nt == ext_start:
                continue
            out[nt] = frozenset(tuple(x for x in s if x != END) for s in ss)
        return out

    def follow(self, nt: int) -> FrozenSet[Str]:
        return self.follow_map[nt]


class LLPTableBuilder:
    """Builds the LLP(q,k) admissible-pair table of an augmented grammar whose
    start production is ``Start -> ⊢ S ⊣``."""

    def __init__(self, g: CFGInt, q: int, k: int):
        if q < 0:
            raise GrammarError("Error: Lookback must be non-negative.")
        if k < 1:
            raise GrammarError("Error: Lookahead must be positive.")
        self.g, self.q, self.k = g, q, k
        self.ff = FirstFollow(g, k)
        rg = g.reversed()
        self.ffr = FirstFollow(rg, q)
        self._last_memo: Dict[Str, FrozenSet[Str]] = {}
        self._before = {nt: frozenset(tuple(reversed(s)) for s in ss)
                        for nt, ss in self.ffr.follow_map.items()}
        self.ll_table = self._ll_table()
        self._cfg_memo: Dict[Tuple[Str, Str], Optional[tuple]] = {}

    # -- LAST / BEFORE ----------------------------------------------------
    def last(self, syms: Str) -> FrozenSet[Str]:
        r = self._last_memo.get(syms)
        if r is None:
            r = frozenset(tuple(reversed(s)) for s in self.ffr.first(tuple(reversed(syms))))
            self._last_memo[syms] = r
        return r

    def before(self, nt: int) -> FrozenSet[Str]:
        return self._before[nt]

    # -- LL(k) table --------------------------------------------------------
    def _ll_table(self) -> Dict[Tuple[int, Str], int]:
        table: Dict[Tuple[int, Str], Set[int]] = {}
        for i, (a, rhs) in enumerate(self.g.prods):
            for y in trunc_product(self.k, self.ff.first(rhs), self.ff.follow(a)):
                table.setdefault((a, y), set()).add(i)
        conflicts = {key: v for key, v in table.items() if len(v) > 1}
        if conflicts:
            raise GrammarError("LL(%d) Table Conflicts: %d entries" % (self.k, len(conflicts)))
        return {key: min(v) for key, v in table.items()}

    def parse_config(self, inp: Str, alpha: Str) -> Optional[Tuple[Str, Str, Str]]:
        """``parseLlpConfig`` (``src/Alpacc/LLP.hs:471-491``)."""
        key = (inp, alpha)
        if key in self._cfg_memo:
            return self._cfg_memo[key]
        g, k = self.g, self.k
        stack = list(alpha)
        parsed: List[int] = []
        res = None
        steps = 0
        while True:
            steps += 1
            if steps > 100000:
                raise GrammarError("configuration parse does not terminate")
            if inp and stack and g.is_t(stack[0]):
                if inp[0] == stack[0]:
                    res = (alpha, tuple(stack[1:]), tuple(parsed))
                break
            if stack and not g.is_t(stack[0]):
                idx = self.ll_table.get((stack[0], inp[:k]))
                if idx is None:
                    break
                stack = list(g.prods[idx][1]) + stack[1:]
                parsed.append(idx)
                continue
            if not inp and not stack:
                res = (alpha, (), tuple(parsed))
            break
        self._cfg_memo[key] = res
        return res

    def shortest_prefix(self, v: Str, x_delta: Str) -> Tuple[Str, Str, Str]:
        for n in range(1, len(x_delta) + 1):
            r = self.parse_config(v, x_delta[:n])
            if r is not None:
                return r
        raise GrammarError("no configuration for an LLP item; the grammar is not LLP(%d,%d)"
                           % (self.q, self.k))

    # -- item sets ----------------------------------------------------------
    # An item is (lhs, alpha, beta, suffix, prefix, (cfg_alpha, cfg_omega, cfg_pi)):
    # the dot production lhs -> alpha . beta with the 4-tuple of Algorithm 8.

    def init_d(self) -> FrozenSet[tuple]:
        g = self.g
        ps = g.by_lhs.get(g.start, [])
        if len(ps) != 1:
            return frozenset()
        lhs, rhs = g.prods[ps[0]]
        return frozenset((lhs, rhs, (), l, (), ((), (), ())) for l in self.last(rhs))

    def new_items(self, item) -> Set[tuple]:
        y, alpha_x, beta, _u, v_i, delta = item
        if not alpha_x:
            return set()
        x = alpha_x[-1]
        alpha = alpha_x[:-1]
        uj = set()
        for b in self.before(y):
            uj |= self.last(b + alpha)
        vj = self.ff.first((x,) + v_i)
        x_delta = (x,) + delta[0]
        x_beta = (x,) + beta
        out = set()
        for u in uj:
            for v in vj:
                out.add((y, alpha, x_beta, u, v, self.shortest_prefix(v, x_delta)))
        return out

    def extra_items(self, item) -> Set[tuple]:
        _y, alpha_y, _beta, _u, v, gamma = item
        if not alpha_y or self.g.is_t(alpha_y[-1]):
            return set()
        Y = alpha_y[-1]
        out = set()
        for pi in self.g.by_lhs.get(Y, []):
            delta = self.g.prods[pi][1]
            for b in self.before(Y):
                for u in self.last(b + delta):
                    out.add((Y, delta, (), u, v, gamma))
        return out

    def close(self, items: Set[tuple]) -> FrozenSet[tuple]:
        out = set(items)
        work = list(items)
        while work:
            it = work.pop()
            for e in self.extra_items(it):
                if e not in out:
                    out.add(e)
                    work.append(e)
        return frozenset(out)

    def solve(self, items: FrozenSet[tuple]) -> Set[FrozenSet[tuple]]:
        groups: Dict[int, Set[tuple]] = {}
        for it in items:
            if it[1]:
                groups.setdefault(it[1][-1], set()).add(it)
        out = set()
        for grp in groups.values():
            new = set()
            for it in grp:
                new |= self.new_items(it)
            out.add(self.close(new))
        return out

    def collection_table(self) -> Dict[Tuple[Str, Str], Tuple[Str, Str, Str]]:
        table: Dict[Tuple[Str, Str], Tuple[Str, Str, Str]] = {}
        visited: Set[FrozenSet[tuple]] = set()
        queue = deque([self.init_d()])
        while queue:
            top = queue.popleft()
            if top in visited:
                continue
            for it in top:
                alpha_z = it[1]
                if alpha_z and self.g.is_t(alpha_z[-1]):
                    key = (it[3], it[4])
                    old = table.get(key)
                    if old is not None and old != it[5]:
                        raise GrammarError(
                            "The grammar is not LLP(%d, %d) due to the admissible pair %r" % (self.q, self.k, key))
                    table[key] = it[5]
            visited.add(top)
            queue.extend(self.solve(top))
        return table

    def starts(self) -> Dict[Tuple[Str, Str], Tuple[Str, Str, Str]]:
        g = self.g
        ps = g.by_lhs.get(g.start, [])
        if not ps or not g.prods[ps[0]][1]:
            s, tail = (), ()
        else:
            s = g.prods[ps[0]][1]
            tail = s[1:]
        return {((), y): ((g.start,), tail, ()) for y in self.ff.first(s)}

    def pair_table(self):
        """``llpParserTableWithStartsHomomorphisms``: key (lookback, lookahead)
        -> (brackets, productions); a bracket is (is_left, symbol)."""
        table = self.collection_table()
        out = {}
        for key, (alpha, omega, pi) in self.starts().items():
            out[key] = (tuple((True, o) for o in reversed(omega)), pi)
        for key, (alpha, omega, pi) in table.items():
            out[key] = (tuple((False, a) for a in alpha) + tuple((True, o) for o in reversed(omega)), pi)
        return out


def llp_parse(pairs, q: int, k: int, string: Sequence[int], rts: int, lts: int) -> Optional[List[int]]:
    """Sequential ``llpParse`` with ``pairLookup`` and ``glue``
    (``src/Alpacc/LLP.hs:595-650``) over a table of (alpha, omega, pi) triples.
    Used to check the table on the reference's own known-answer tests."""
    padded = [rts] + list(string) + [lts]
    cur = None
    for i, x in enumerate(padded):
        back = tuple(padded[max(0, i - q):i])
        fwd = tuple(padded[i:i + k])
        v = pairs.get((back, fwd))
        if v is None:
            return None
        a, w, p = list(v[0]), list(v[1]), list(v[2])
        if cur is None:
            cur = (a, w, p)
            continue
        al, wl, pl = cur
        if wl == a:
            cur = (al, w, pl + p)
        elif a[:len(wl)] == wl:
            cur = (al + a[len(wl):], w, pl + p)
        elif wl[:len(a)] == a:
            cur = (al, w + wl[len(a):], pl + p)
        else:
            return None
    return None if cur is None else cur[2]
