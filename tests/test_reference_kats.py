"""Known-answer tests transcribed from the reference's own test suite and
README, run against this project's restatement of the table generator and
the CPU oracle (no GPU)."""

import itertools
import json
import os
from collections import deque

import numpy as np
import pytest

import oracle
from alpacc_b200 import grammar as G
from alpacc_b200 import lexgen, tables
from alpacc_b200.llp import CFGInt, FirstFollow, LLPTableBuilder, llp_parse

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


# ---------------------------------------------------------------- README ----
def test_readme_tree_oracle():
    """README.md:84-106: the tree of 12+(3*4) with parents and spans."""
    with open(os.path.join(GOLDEN, "readme_arith_tree.json")) as f:
        gold = json.load(f)
    tb = tables.load("arithmetic", "both")
    o = oracle.Oracle(tb.blob())
    res = o.lex_parse(gold["input"].encode())
    assert res is not None
    par, tag, kind, s, e = res
    got = []
    for i in range(len(par)):
        if kind[i]:
            got.append((int(par[i]), ["terminal", tb.terminal_names[tag[i]], [int(s[i]), int(e[i])]]))
        else:
            got.append((int(par[i]), ["production", tb.production_names[tag[i]]]))
    assert got == [(p, n) for p, n in gold["tree"]]
    glue = o.parse_glue(*o.tokenize(gold["input"].encode()))
    for a, b in zip(res, glue):
        np.testing.assert_array_equal(a, b)


# ------------------------------------------------------ haskell-tests/LLP.hs -
# Grammar of haskell-tests/LLP.hs:18-31: E -> T E'; E' -> + T E' | eps;
# T -> a | [ E ].  Terminals [ ] + a = 0..3, ⊢ 4, ⊣ 5; E 6, E' 7, T 8, Start 9.
LLP_PRODS = [(6, (8, 7)), (7, (2, 8, 7)), (7, ()), (8, (3,)), (8, (0, 6, 1)), (9, (4, 6, 5))]


def _llp_parser(q, k):
    g = CFGInt(6, 10, LLP_PRODS, 9)
    b = LLPTableBuilder(g, q, k)
    pairs = dict(b.collection_table())
    for key, v in b.starts().items():
        pairs.setdefault(key, v)  # llpParserTableWithStarts: starts win on ties
    return lambda s: llp_parse(pairs, q, k, s, 4, 5)


def _derivable(max_len):
    """Every terminal string of length <= max_len derivable from E."""
    prods = {}
    for l, r in LLP_PRODS[:-1]:
        prods.setdefault(l, []).append(r)
    out, seen = set(), set()
    q = deque([(6,)])
    while q:
        form = q.popleft()
        if form in seen:
            continue
        seen.add(form)
        nts = [i for i, x in enumerate(form) if x >= 6]
        if sum(1 for x in form if x < 6) > max_len:
            continue
        if not nts:
            out.add(form)
            continue
        i = nts[0]
        for r in prods[form[i]]:
            q.append(form[:i] + r + form[i + 1:])
    return out


@pytest.mark.parametrize("q,k", [(q, k) for q in range(1, 4) for k in range(1, 4)])
def test_llp_parse_kat(q, k):
    """haskell-tests/LLP.hs:495-499: a+[a+a] -> [0,3,1,4,0,3,1,3,2,2]."""
    parse = _llp_parser(q, k)
    assert parse([3, 2, 0, 3, 2, 3, 1]) == [0, 3, 1, 4, 0, 3, 1, 3, 2, 2]


@pytest.mark.parametrize("q,k", [(1, 1), (2, 2), (3, 3)])
def test_llp_derivable_and_not(q, k):
    """haskell-tests/LLP.hs:517-534: derivable strings parse, nonderivable
    strings of length 3 do not."""
    parse = _llp_parser(q, k)
    der = _derivable(9)
    for s in der:
        assert parse(list(s)) is not None, s
    for s in itertools.product(range(4), repeat=3):
        if s not in der:
            assert parse(list(s)) is None, s


def test_llp_table_keys_contain_psls_fixture():
    """haskell-tests/LLP.hs:82-97: every admissible pair of the PSLS fixture
    is a key of the LLP(1,1) table."""
    g = CFGInt(6, 10, LLP_PRODS, 9)
    keys = set(LLPTableBuilder(g, 1, 1).collection_table().keys())
    T = {"[": 0, "]": 1, "+": 2, "a": 3, "⊢": 4, "⊣": 5}
    fixture = [("+", "["), ("+", "a"), ("[", "["), ("[", "a"), ("]", "+"), ("]", "]"), ("]", "⊣"),
               ("a", "+"), ("a", "]"), ("a", "⊣"), ("⊢", "["), ("⊢", "a")]
    for x, y in fixture:
        assert ((T[x],), (T[y],)) in keys


# ------------------------------------------------------- haskell-tests/LL.hs -
def test_first_small():
    """haskell-tests/LL.hs:15-25,75-84: T -> R | a T c; R -> eps | b R."""
    # a b c = 0 1 2; R 3, T 4
    prods = [(4, (3,)), (4, (0, 4, 2)), (3, ()), (3, (1, 3))]
    ff = FirstFollow(CFGInt(3, 5, prods, 4), 1)
    got = [ff.first(r) for _, r in prods]
    assert got == [{(), (1,)}, {(0,)}, {()}, {(1,)}]


def test_follow_small():
    """haskell-tests/LL.hs:27-38,100-108 on followExtendedGrammar."""
    # $ a b c = 0..3; T' 4, R 5, T 6
    prods = [(4, (6, 0)), (6, (5,)), (6, (1, 6, 3)), (5, ()), (5, (5, 2, 5))]
    ff = FirstFollow(CFGInt(4, 7, prods, 4), 1)
    assert [ff.follow(n) for n in (4, 5, 6)] == [{()}, {(0,), (3,), (2,)}, {(0,), (3,)}]


BOOK = [(3, (4, 0)), (4, (5, 6)), (4, (6, 5)), (5, (1,)), (5, (7, 5, 7)), (6, (2,)), (6, (7, 6, 7)),
        (7, (1,)), (7, (2,))]  # $ a b = 0..2; N' 3, N 4, A 5, B 6, C 7


def test_follow_large():
    """haskell-tests/LL.hs:56-71,110-121 on bookGrammar."""
    ff = FirstFollow(CFGInt(3, 8, BOOK, 3), 1)
    ab = {(1,), (2,), (0,)}
    assert [ff.follow(n) for n in (3, 4, 5, 6, 7)] == [{()}, {(0,)}, ab, ab, ab]


def test_first_book():
    """haskell-tests/LL.hs:86-98: FIRST_1 of every right-hand side of bookGrammar."""
    ff = FirstFollow(CFGInt(3, 8, BOOK, 3), 1)
    a, b, ab = {(1,)}, {(2,)}, {(1,), (2,)}
    assert [ff.first(r) for _, r in BOOK] == [ab, ab, ab, a, ab, b, ab, a, b]


@pytest.mark.parametrize("k", range(1, 6))
def test_ll_parse(k):
    """haskell-tests/LL.hs:123-135: LL(k) parse of aabbbcc$ on extendedGrammar."""
    prods = [(4, (6, 0)), (6, (5,)), (6, (1, 6, 3)), (5, ()), (5, (2, 5))]
    g = CFGInt(4, 7, prods, 4)
    b = LLPTableBuilder.__new__(LLPTableBuilder)
    b.g, b.k, b.q = g, k, 0
    b.ff = FirstFollow(g, k)
    table = b._ll_table()
    stack, inp, out = [4], [1, 1, 2, 2, 2, 3, 3, 0], []
    while stack:
        top = stack.pop(0)
        if top < 4:
            assert inp and inp[0] == top
            inp.pop(0)
        else:
            i = table[(top, tuple(inp[:k]))]
            out.append(i)
            stack = list(prods[i][1]) + stack
    assert out == [0, 2, 2, 1, 4, 4, 4, 3] and not inp


# ----------------------------------------- haskell-tests/RegularExpression.hs
REGEX_CASES = [  # haskell-tests/RegularExpression.hs:38-120
    ("a*|b*", ["", "a", "aa", "aaa", "b", "bb", "bbb"], ["ab", "ba", "c", "aba", "bba", "xy"]),
    ("a*b*", ["", "ab", "aab", "b", "bb", "aaa", "abb", "aabbb"], ["aba", "bab", "xy", "abab", "bbaaa"]),
    ("a|b|c", ["a", "b", "c"], ["ab", "abc", "cba", "ac", "bb", "cc", "abcab", "xy", ""]),
    ("a+b+c+", ["abc", "aabbcc", "aaabbbccc", "aaaaaabbbbbbcccccc", "abbc"],
     ["ab", "acb", "bca", "aabccx", "aabcbccc", "abcabc", "xy", ""]),
    ("[a-z]+", ["abc", "aabbcc", "aaabbbccc", "aaaaaabbbbbbcccccc", "abbc", "ab", "acb", "bca", "aabccx",
                "aabcbccc", "abcabc", "xy"], ["", "4234", "324", "1", "<", "#", "\\"]),
    ("(a*b|c)d+(e|)", ["bd", "bde", "abd", "cd", "abdde", "cdde", "abde"],
     ["a", "b", "aa", "bb", "cc", "ade", "de", "xbdde", "abbddee"]),
    ("(xy*|z)ab+(c|)", ["xab", "xyab", "xyyab", "zab", "xabc", "xyabc", "xyyyabc"],
     ["x", "xy", "xz", "ab", "abb", "xyyy", "abc4", "zatbc"]),
    ("a*b+c*(d|)e+f", ["aabcdeef", "aabbcdeef", "abbcdef", "abbcccdeef", "abdeef"],
     ["aaaeef", "abcdf", "aabbcczdeef", "aabccddeef", "abccddef", "xy", ""]),
    ("(cat|dog|fish)+([0-9]|)", ["catfish", "catcatfish", "dogdogdog4", "fish3", "catdogfish0", "cat3"],
     ["catdoga", "0fishfish", "4cat4", " dogdogdogdog", "ddogfish3", "xy", ""]),
    ("()", [""], ["catdoga", "0fishfish", "4cat4", " dogdogdogdog", "ddogfish3", "xy"]),
    ("", [""], ["catdoga", "0fishfish", "4cat4", " dogdogdogdog", "ddogfish3", "xy"]),
]


@pytest.mark.parametrize("rx,good,bad", REGEX_CASES)
def test_regex(rx, good, bad):
    r = G.parse_regex(rx)
    for s in good:
        assert lexgen.regex_match(r, s.encode()), (rx, s)
    for s in bad:
        assert not lexgen.regex_match(r, s.encode()), (rx, s)
