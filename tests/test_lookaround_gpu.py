"""The parser at other lookback / lookahead settings: the arithmetic and sexp
grammars rebuilt with params (q, k) in {(1,2), (2,1), (2,2), (3,1), (1,3)}
(an LLP(1,1) grammar is LLP(q,k) for larger q, k) and parsed on the GPU
against the oracle.  These reach every instantiation of the pair kernel,
the generic one included, and key windows wider than the bundled grammars'."""

import itertools

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu

SETTINGS = [(1, 2), (2, 1), (2, 2), (3, 1), (1, 3)]
_CACHE = {}


def _ctx(name, q, k):
    from alpacc_b200.api import Grammar
    key = (name, q, k)
    if key not in _CACHE:
        with open(tables.grammar_path(name)) as f:
            src = f.read()
        src = src.replace("lookback = 1.", "lookback = %d." % q).replace("lookahead = 1.", "lookahead = %d." % k)
        tb = tables.build_tables(src, "both")
        assert (tb.parser.q, tb.parser.k) == (q, k)
        _CACHE[key] = (Grammar(tb), oracle.Oracle(tb.blob()))
    return _CACHE[key]


def _same(g, o, data: bytes):
    want = o.lex_parse(data)
    got = g.parse_int(data)
    assert (got is None) == (want is None), data[:60]
    if want is None:
        return
    for a, b in zip((got.parent, got.tag, got.kind, got.start, got.end), want):
        np.testing.assert_array_equal(a.cpu().numpy().astype(np.int64), np.asarray(b).astype(np.int64))


@pytest.mark.parametrize("name", ["arithmetic", "sexp"])
@pytest.mark.parametrize("qk", SETTINGS)
def test_parse_at_other_lookaround(has_gpu, name, qk):
    g, o = _ctx(name, *qk)
    gen = synth.arith_doc if name == "arithmetic" else synth.sexp_doc
    for i, size in enumerate([1, 2, 5, 100, 4097, 70000, 1 << 20]):
        _same(g, o, gen(size, 12 if name == "arithmetic" else 20, 900 + i).tobytes())
    alpha = b"1+*()a " if name == "arithmetic" else b"()a "
    for n in range(0, 4):
        for t in itertools.product(alpha, repeat=n):
            _same(g, o, bytes(t))
    # batches: key windows that would cross a document boundary
    docs = [gen(s, 8, 950 + j).tobytes() for j, s in enumerate([3, 40, 1, 900, 7])] + [b"", b"(", b")"]
    off = np.zeros(len(docs) + 1, np.int64)
    off[1:] = np.cumsum([len(d) for d in docs])
    data = np.frombuffer(b"".join(docs), np.uint8)
    tree, node_off, valid = g.parse_batch_int(data, off)
    node_off, valid = node_off.cpu().numpy(), valid.cpu().numpy()
    for j, d in enumerate(docs):
        want = o.lex_parse(d)
        assert bool(valid[j]) == (want is not None), (j, d)
        if want is None:
            continue
        a, b = node_off[j], node_off[j + 1]
        for col, w in zip((tree.parent, tree.tag, tree.kind, tree.start, tree.end), want):
            np.testing.assert_array_equal(col[a:b].cpu().numpy().astype(np.int64), np.asarray(w).astype(np.int64))
