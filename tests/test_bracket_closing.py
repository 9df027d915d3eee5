"""The parser closes the bracket pairs between adjacent positions (a
position's first rights against the previous position's top lefts) before
its bracket search, and searches only the brackets left.  These CPU tests pin
that step on its own: over the LLP pair sequence of generated and corrupted
documents, checking the closed pairs' symbols and matching the rest gives the
verdict of matching every bracket (futhark/parser.fut:153-184), and the
brackets left are the count the kernels place them by."""

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables

_CACHE = {}


def _ctx(name):
    if name not in _CACHE:
        tb = tables.load(name, "both")
        _CACHE[name] = (tb, oracle.Oracle(tb.blob()))
    return _CACHE[name]


def _pair_brackets(tb, o, data):
    """Per position of ⊢ tokens ⊣: (rights, lefts) as symbol lists in stack
    order, or None when some position has no admissible pair."""
    p = tb.parser
    lexed = o.lex_futhark(data)
    if lexed is None:
        return None
    arr = [p.start] + [int(t) for t in lexed[0]] + [p.end]
    kmap = dict(zip(p.keys, p.key_pair))
    n = len(arr)
    out = []
    for i in range(n):
        pid = kmap.get(tuple(arr[j] if 0 <= j < n else p.empty for j in range(i - p.q, i + p.k)))
        if pid is None:
            return None
        s0, s1, _, _ = p.pairs[pid]
        br = p.stack[s0:s1]
        rights = [b & 0x7fffffff for b in br if not b >> 31]
        lefts = [b & 0x7fffffff for b in br if b >> 31]
        assert [b for b in br if not b >> 31] + [b for b in br if b >> 31] == list(br), "rights before lefts"
        out.append((rights, lefts))
    return out


def _match_all(seq):
    """Stack matching of a (kind, symbol) sequence: depth never below zero,
    zero at the end, every right against the last open left of its symbol."""
    st = []
    for kind, sym in seq:
        if kind == "L":
            st.append(sym)
        elif not st or st.pop() != sym:
            return False
    return not st


def _flat(pos):
    return [x for r, l in pos for x in [("R", s) for s in r] + [("L", s) for s in l]]


def _close_adjacent(pos):
    """(verdict of the closed pairs' symbols, the brackets left in order)."""
    ok = True
    kept = []
    closed = [0] * (len(pos) + 1)
    for i in range(1, len(pos)):
        m = min(len(pos[i - 1][1]), len(pos[i][0]))
        for t in range(m):
            ok &= pos[i - 1][1][-1 - t] == pos[i][0][t]
        closed[i] = m
    for i, (r, l) in enumerate(pos):
        kept += [("R", s) for s in r[closed[i]:]]
        kept += [("L", s) for s in l[:len(l) - closed[i + 1]]]
    return ok, kept, sum(closed)


def _docs(name):
    closers = {"json": b"]}", "arithmetic": b")", "sexp": b")"}[name]
    gen = {"json": lambda n, s: synth.json_doc(n, 16, s), "arithmetic": lambda n, s: synth.arith_doc(n, 12, s),
           "sexp": lambda n, s: synth.sexp_doc(n, 20, s)}[name]
    rng = np.random.default_rng(31)
    for i, size in enumerate([40, 300, 5000, 30000]):
        d = bytes(gen(size, 1200 + i))
        yield d
        pos = [j for j, c in enumerate(d) if c in closers]
        for k in range(6):
            if not pos:
                break
            b = bytearray(d)
            j = pos[int(rng.integers(0, len(pos)))]
            if k % 3 == 0:
                del b[j]
            elif k % 3 == 1:
                b.insert(j, b[j])
            else:
                b[j] = closers[(closers.index(b[j]) + 1) % len(closers)]
            yield bytes(b)


@pytest.mark.parametrize("name", ["json", "arithmetic", "sexp"])
def test_closing_adjacent_pairs_keeps_the_verdict(name):
    tb, o = _ctx(name)
    seen = 0
    for d in _docs(name):
        pos = _pair_brackets(tb, o, d)
        if pos is None:
            continue
        seen += 1
        full = _match_all(_flat(pos))
        ok, kept, n_closed = _close_adjacent(pos)
        assert (ok and _match_all(kept)) == full
        assert len(kept) == len(_flat(pos)) - 2 * n_closed
        if full:
            assert o.lex_parse(d) is not None, "brackets match but the oracle rejects"
    assert seen > 10
