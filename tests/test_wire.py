"""alpacc's test wire format (big-endian Data.Binary): byte layout on small
known cases, round trips of oracle results, and malformed files."""

import json
import os
import struct

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables, wire

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def u64(x):
    return struct.pack(">Q", x)


def test_input_layout():
    b = wire.write_inputs([b"ab", b""])
    assert b == u64(2) + u64(2) + b"ab" + u64(0)
    assert wire.read_inputs(b) == [b"ab", b""]
    t = wire.write_token_inputs([[1, 2], []])
    assert t == u64(2) + u64(2) + u64(1) + u64(2) + u64(0)
    assert [list(x) for x in wire.read_token_inputs(t)] == [[1, 2], []]


def test_output_layouts():
    lx = wire.write_lexer_outputs([None, (np.array([3]), np.array([0]), np.array([2]))])
    assert lx == u64(2) + b"\x00" + b"\x01" + u64(1) + u64(3) + u64(0) + u64(2)
    pr = wire.write_parser_outputs([[4, 5], None])
    assert pr == u64(2) + b"\x01" + u64(2) + u64(4) + u64(5) + b"\x00"
    tree = (np.array([0, 0]), np.array([7, 1]), np.array([0, 1], np.uint8), np.array([0, 3]), np.array([0, 4]))
    lp = wire.write_lexparse_outputs([tree])
    node0 = b"\x00" + u64(0) + u64(7) + u64(0) + u64(0)
    node1 = b"\x01" + u64(0) + u64(1) + u64(3) + u64(4)
    assert lp == u64(1) + b"\x01" + u64(2) + node0 + node1


def test_readme_tree_round_trip():
    with open(os.path.join(GOLDEN, "readme_arith_tree.json")) as f:
        g = json.load(f)
    tb = tables.load("arithmetic", "both")
    o = oracle.Oracle(tb.blob())
    got = o.lex_parse(g["input"].encode())
    b = wire.write_lexparse_outputs([got])
    assert len(b) == 8 + 1 + 8 + 33 * len(got[0])
    back = wire.read_lexparse_outputs(b)[0]
    for x, y in zip(back, got):
        np.testing.assert_array_equal(np.asarray(x, np.int64), np.asarray(y, np.int64))
    assert wire.compare(b, b, "lexer-parser") is None


@pytest.mark.parametrize("name", ["json", "sexp", "arithmetic"])
def test_oracle_results_round_trip(name):
    tb = tables.load(name, "both")
    o = oracle.Oracle(tb.blob())
    gen = {"json": lambda s, i: synth.json_doc(s, 8, i), "sexp": lambda s, i: synth.sexp_doc(s, 20, i),
           "arithmetic": lambda s, i: synth.arith_doc(s, 12, i)}[name]
    docs = [gen(3000 + 100 * i, 40 + i).tobytes() for i in range(6)] + [b"", b"#"]
    lex = [o.lex_futhark(d) for d in docs]
    lp = [o.lex_parse(d) for d in docs]
    pp = [None if t is None else o.pre_productions(t[0]) for t in lex]
    for write, read, res, mode in ((wire.write_lexer_outputs, wire.read_lexer_outputs, lex, "lexer"),
                                   (wire.write_lexparse_outputs, wire.read_lexparse_outputs, lp, "lexer-parser"),
                                   (wire.write_parser_outputs, wire.read_parser_outputs, pp, "parser")):
        b = write(res)
        back = read(b)
        assert len(back) == len(res)
        for x, y in zip(back, res):
            assert (x is None) == (y is None)
            if x is None:
                continue
            xs = x if isinstance(x, tuple) else (x,)
            ys = y if isinstance(y, tuple) else (y,)
            for u, v in zip(xs, ys):
                np.testing.assert_array_equal(np.asarray(u, np.int64), np.asarray(v, np.int64))
        assert wire.compare(b, b, mode) is None
        if any(r is not None for r in res):
            i = next(k for k, r in enumerate(res) if r is not None)
            other = list(res)
            other[i] = None
            assert "input %d" % i in wire.compare(b, write(other), mode)


def test_malformed_files_are_rejected():
    with pytest.raises(ValueError):
        wire.read_inputs(u64(1) + u64(5) + b"ab")
    with pytest.raises(ValueError):
        wire.read_lexer_outputs(u64(1) + b"\x02")
    with pytest.raises(ValueError):
        wire.read_lexparse_outputs(u64(1) + b"\x01" + u64(1) + b"\x05" + u64(0) * 4)
    with pytest.raises(ValueError):
        wire.read_inputs(wire.write_inputs([b"x"]) + b"\x00")
