"""Bit-exact parity at the benchmark configurations' full sizes.

The other GPU tests stop at a few MiB; a tiling, 32-bit-overflow or
look-back bug that only shows at hundreds of MiB (positions, bracket counts,
exscan values, tile and document counts) would pass them.  Here every
configuration of the benchmark runs at its stated size through the C ABI and
is compared with the sequential oracle, element for element:

* arithmetic.alp lex+parse, 1 MiB of random derivations;
* json.alp lexer only (lexer-mode ids), one 512 MiB document, depth <= 8;
* json.alp lex+parse, one 256 MiB document, depth <= 16;
* the batch: 100,000 json documents (depth <= 8) and 50,000 sexp documents with
  log-normal sizes (median 4 KiB, sigma 1.5, capped at 4 MiB), each set in
  one segmented call, every document against the oracle run on it alone.

The reference checks its own generated pipeline the same way on one long
generated input (tests/testjson.sh:81-94).
"""

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu

SEED = 0xA1FACC00


def _threads():
    try:
        return max(1, min(len(os.sched_getaffinity(0)), 64))
    except AttributeError:
        return os.cpu_count() or 1


def _tree_equal(got, want):
    assert want is not None, "the oracle rejected a generated document"
    assert got is not None, "the GPU rejected a document the oracle accepts"
    arrs = [x.cpu().numpy() for x in (got.parent, got.tag, got.kind, got.start, got.end)]
    assert len(arrs[0]) == len(want[0])
    for a, w in zip(arrs, want):
        np.testing.assert_array_equal(a.astype(w.dtype), w)


def test_arithmetic_1mib_parse(has_gpu):
    from alpacc_b200.api import Grammar
    tb = tables.load("arithmetic", "both")
    doc = synth.arith_doc(1 << 20, 12, SEED + 0).tobytes()
    _tree_equal(Grammar(tb).parse_int(doc), oracle.Oracle(tb.blob()).lex_parse(doc))


def test_json_512mib_lex(has_gpu):
    from alpacc_b200.api import Grammar
    tb = tables.load("json", "lexer")
    doc = synth.json_doc(512 << 20, 8, SEED + 1)
    g = Grammar(tb)
    got = g.lex_int(doc)
    want = oracle.Oracle(tb.blob()).tokenize(doc.tobytes())
    assert got is not None and want is not None
    for a, w in zip(got, want):
        a = a.cpu().numpy()
        assert len(a) == len(w)
        np.testing.assert_array_equal(a.astype(w.dtype), w)


def test_json_256mib_parse(has_gpu):
    from alpacc_b200.api import Grammar
    tb = tables.load("json", "both")
    doc = synth.json_doc(256 << 20, 16, SEED + 2)
    g = Grammar(tb)
    got = g.parse_int(doc)
    del g
    _tree_equal(got, oracle.Oracle(tb.blob()).lex_parse(doc.tobytes()))


@pytest.mark.parametrize("name,n_docs,seed", [("json", 100_000, SEED + 3), ("sexp", 50_000, SEED + 4)])
def test_batch_full(has_gpu, name, n_docs, seed):
    from alpacc_b200.api import Grammar
    tb = tables.load(name, "both")
    sizes = synth.lognormal_sizes(n_docs, median=4096, sigma=1.5, cap=4 << 20, seed=seed)
    data, off = synth.batch(name, sizes, 8 if name == "json" else 20, seed)
    g = Grammar(tb)
    tree, node_off, valid = g.parse_batch_int(data, off)
    par, tag, kind, st, en = (x.cpu().numpy() for x in (tree.parent, tree.tag, tree.kind, tree.start, tree.end))
    node_off, valid = node_off.cpu().numpy(), valid.cpu().numpy()
    assert valid.all(), "the GPU rejected generated documents"
    o = oracle.Oracle(tb.blob())

    def one(i):
        return o.lex_parse(data[off[i]:off[i + 1]].tobytes())

    with ThreadPoolExecutor(_threads()) as ex:
        want = list(ex.map(one, range(n_docs), chunksize=64))
    assert all(w is not None for w in want), "the oracle rejected generated documents"
    counts = np.array([len(w[0]) for w in want], np.int64)
    np.testing.assert_array_equal(np.diff(node_off), counts)
    for j, got in enumerate((par, tag, kind, st, en)):
        w = np.concatenate([x[j] for x in want])
        np.testing.assert_array_equal(got.astype(w.dtype), w)
