"""json.alp checked without the repository's table generator.

The oracle reads the tables that alpacc_b200/{lexgen,llp,tables}.py build, so
a mistake in those builders would show in the oracle and the kernels alike.
For the benchmark grammar this test restates json.alp a second way, sharing
no code with them:

* tokens: greedy longest match without backtracking (a token ends only when
  the next byte cannot extend any terminal; src/Alpacc/Lexer/DFA.hs:415-447)
  over the grammar's regular expressions, run by the third-party `regex`
  engine's partial matching;
* tree: a recursive-descent parser written from the productions of
  alpacc_b200/grammars/json.alp, giving the leftmost derivation in preorder
  with parents, terminals as leaves with their spans (the shape of the
  README's tree, README.md:84-106);
* ids: terminal and production ids assigned by hand from alpacc's published
  numbering rules (src/Alpacc/CFG.hs:131,219-224; src/Alpacc/Grammar.hs:90;
  src/Alpacc/Encode.hs:122-162): ordinary terminals with names first in file
  order, then literals sorted by their text, then ignore; productions in file
  and alternative order; lexer-only ids sorted with names before literals.

Both are compared with the oracle on generated documents and edge cases.
"""

import numpy as np
import pytest
import regex

import oracle
from alpacc_b200 import synth, tables

# The grammar's regular expressions in alpacc's syntax (`.` is a literal dot,
# `\s` a space), written for the `regex` engine.
STRING = regex.compile(rb'"(?:[\x00-\x21\x23-\xff]|\\")*"')
NUMBER = regex.compile(rb"-?[0-9]+(?:\.[0-9]+)?")
IGNORE = regex.compile(rb"[ \n\t\r]")
LITERALS = [b",", b":", b"[", b"]", b"false", b"null", b"true", b"{", b"}"]  # sorted by text

# lexer+parser ids: names in file order, literals by text, then ignore
TERM_BOTH = {"string": 0, "number": 1, **{lit: 2 + i for i, lit in enumerate(LITERALS)}, "ignore": 11}
# lexer-only ids: every terminal sorted, names before literals, then ignore
TERM_LEX = {"number": 0, "string": 1, **{lit: 2 + i for i, lit in enumerate(LITERALS)}, "ignore": 11}
# productions in file and alternative order
P = dict(J_obj=0, J_arr=1, J_str=2, J_num=3, J_null=4, J_true=5, J_false=6, O=7, FS0_e=8, FS0=9, FS1_e=10,
         FS1=11, F=12, A=13, EL0_e=14, EL0=15, EL1_e=16, EL1=17)

# terminals in priority order (implicit literal rules before the named ones,
# src/Alpacc/CFG.hs:162); for json no two of them match the same text
TERMINALS = [(lit, regex.compile(regex.escape(lit))) for lit in LITERALS] + \
    [("string", STRING), ("number", NUMBER), ("ignore", IGNORE)]


def tokenize(s: bytes):
    """[(name, start, end)] without ignore tokens, or None when rejected."""
    out, i, n = [], 0, len(s)
    if n == 0:
        return None  # the initial state does not accept
    while i < n:
        j = i
        while j < n and any(p.fullmatch(s, i, j + 1, partial=True) for _, p in TERMINALS):
            j += 1
        name = next((nm for nm, p in TERMINALS if j > i and p.fullmatch(s, i, j)), None)
        if name is None:
            return None
        if name != "ignore":
            out.append((name, i, j))
        i = j
    return out


class _Reject(Exception):
    pass


def parse(toks):
    """(parent, tag, kind, start, end) lists of the preorder tree, or None."""
    nodes = []
    pos = [0]

    def peek():
        return toks[pos[0]][0] if pos[0] < len(toks) else None

    def node(parent, prod):
        nodes.append((parent, prod, 0, 0, 0))
        return len(nodes) - 1

    def leaf(parent, name):
        if peek() != name:
            raise _Reject()
        _, a, b = toks[pos[0]]
        pos[0] += 1
        nodes.append((parent, TERM_BOTH[name], 1, a, b))

    def J(parent):
        t = peek()
        if t == b"{":
            O(node(parent, P["J_obj"]))
        elif t == b"[":
            A(node(parent, P["J_arr"]))
        elif t in ("string", "number", b"null", b"true", b"false"):
            me = node(parent, {"string": P["J_str"], "number": P["J_num"], b"null": P["J_null"],
                               b"true": P["J_true"], b"false": P["J_false"]}[t])
            leaf(me, t)
        else:
            raise _Reject()

    def O(parent):
        me = node(parent, P["O"])
        leaf(me, b"{")
        if peek() == "string":
            f = node(me, P["FS0"])
            F(f)
            FS1(f)
        else:
            node(me, P["FS0_e"])
        leaf(me, b"}")

    def FS1(parent):
        if peek() == b",":
            me = node(parent, P["FS1"])
            leaf(me, b",")
            F(me)
            FS1(me)
        else:
            node(parent, P["FS1_e"])

    def F(parent):
        me = node(parent, P["F"])
        leaf(me, "string")
        leaf(me, b":")
        J(me)

    def A(parent):
        me = node(parent, P["A"])
        leaf(me, b"[")
        if peek() in (b"{", b"[", "string", "number", b"null", b"true", b"false"):
            e = node(me, P["EL0"])
            J(e)
            EL1(e)
        else:
            node(me, P["EL0_e"])
        leaf(me, b"]")

    def EL1(parent):
        if peek() == b",":
            me = node(parent, P["EL1"])
            leaf(me, b",")
            J(me)
            EL1(me)
        else:
            node(parent, P["EL1_e"])

    try:
        J(0)
    except _Reject:
        return None
    if pos[0] != len(toks):
        return None
    return [np.array([x[k] for x in nodes], dt) for k, dt in
            enumerate((np.int64, np.uint32, np.uint8, np.int64, np.int64))]


def _docs():
    out = [synth.json_doc(size, depth, seed).tobytes()
           for size, depth, seed in ((120_000, 16, 0xA1FACC00 + 71), (90_000, 8, 0xA1FACC00 + 72),
                                     (60_000, 16, 0xA1FACC00 + 73))]
    out += [b'{"a": 1}', b"[]", b"{}", b' [1.5, -2, "x\\"y", null, true, false, {"k": [[]]}] ', b'"s"', b"7",
            b'{"a": 1,}', b"[1 2]", b"1.", b"-", b'"open', b"[", b"nul", b'{"a"}', b"", b" ", b'"a\\", "b"']
    return out


@pytest.fixture(scope="module")
def oracles():
    both, lex = tables.load("json", "both"), tables.load("json", "lexer")
    return oracle.Oracle(both.blob()), oracle.Oracle(lex.blob())


def test_tokens_match_independent_tokenizer(oracles):
    ob, ol = oracles
    for d in _docs():
        want = tokenize(d)
        for o, ids in ((ob, TERM_BOTH), (ol, TERM_LEX)):
            got = o.tokenize(d)
            assert (got is None) == (want is None), d[:60]
            if want is None:
                continue
            np.testing.assert_array_equal(got[0], np.array([ids[t] for t, _, _ in want], np.uint32))
            np.testing.assert_array_equal(got[1], np.array([a for _, a, _ in want], np.int64))
            np.testing.assert_array_equal(got[2], np.array([b for _, _, b in want], np.int64))


def test_tree_matches_recursive_descent(oracles):
    ob, _ = oracles
    n_valid = 0
    for d in _docs():
        toks = tokenize(d)
        want = parse(toks) if toks is not None else None
        got = ob.lex_parse(d)
        assert (got is None) == (want is None), d[:60]
        if want is None:
            continue
        n_valid += 1
        for g, w in zip(got, want):
            np.testing.assert_array_equal(g, w)
    assert n_valid >= 9
