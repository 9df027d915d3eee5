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


def _c_writer():
    import ctypes
    from alpacc_b200 import build
    lib = ctypes.CDLL(build.build_cuda())
    f = lib.alp_write_reference_format
    vp = ctypes.c_void_p
    f.argtypes = [ctypes.c_int, ctypes.c_int64, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_size_t,
                  ctypes.POINTER(ctypes.c_size_t)]
    return f


def _ptr(a):
    return None if a is None else a.ctypes.data


def _c_write(f, mode, valid, off, id_=None, parent=None, kind=None, start=None, end=None, cap=None):
    import ctypes
    n = ctypes.c_size_t(0)
    rc = f(mode, len(valid), _ptr(valid), _ptr(off), _ptr(id_), _ptr(parent), _ptr(kind), _ptr(start), _ptr(end),
           None, 0, ctypes.byref(n))
    assert rc == 0
    buf = np.zeros(max(n.value if cap is None else cap, 1), np.uint8)
    rc = f(mode, len(valid), _ptr(valid), _ptr(off), _ptr(id_), _ptr(parent), _ptr(kind), _ptr(start), _ptr(end),
           _ptr(buf), len(buf) if cap is None else cap, ctypes.byref(n))
    return rc, bytes(buf[:n.value]), n.value


def test_c_abi_writer_matches_wire_module():
    """alp_write_reference_format (host code in the C library, no GPU) writes the
    same bytes as this module for every output kind, rejected inputs and empty
    ones included."""
    f = _c_writer()
    rng = np.random.default_rng(3)
    counts = [0, 5, 1, 0, 17, 3]
    valid = np.array([1, 1, 0, 1, 1, 0], np.uint8)
    off = np.zeros(len(counts) + 1, np.int64)
    off[1:] = np.cumsum(counts)
    m = int(off[-1])
    term = rng.integers(0, 40, m).astype(np.uint32)
    start = rng.integers(0, 1 << 40, m).astype(np.int64)
    end = start + rng.integers(1, 9, m)
    parent = rng.integers(0, 1 << 33, m).astype(np.int64)
    kind = rng.integers(0, 2, m).astype(np.uint8)
    sl = [slice(off[i], off[i + 1]) for i in range(len(counts))]

    rc, got, _ = _c_write(f, 0, valid, off, id_=term, start=start, end=end)
    assert rc == 0
    assert got == wire.write_lexer_outputs([(term[s], start[s], end[s]) if v else None for s, v in zip(sl, valid)])

    rc, got, _ = _c_write(f, 1, valid, off, id_=term, parent=parent, kind=kind, start=start, end=end)
    assert rc == 0
    want = wire.write_lexparse_outputs([(parent[s], term[s], kind[s], start[s], end[s]) if v else None
                                        for s, v in zip(sl, valid)])
    assert got == want

    rc, got, _ = _c_write(f, 2, valid, off, id_=term)
    assert rc == 0
    assert got == wire.write_parser_outputs([term[s] if v else None for s, v in zip(sl, valid)])

    empty = np.zeros(0, np.uint8)
    rc, got, _ = _c_write(f, 2, empty, np.zeros(1, np.int64), id_=term)
    assert rc == 0 and got == u64(0)


def test_c_abi_writer_errors():
    import ctypes
    f = _c_writer()
    valid = np.array([1], np.uint8)
    off = np.array([0, 2], np.int64)
    ids = np.array([3, 4], np.uint32)
    kind = np.array([1, 2], np.uint8)
    z = np.zeros(2, np.int64)
    rc, _, need = _c_write(f, 2, valid, off, id_=ids, cap=4)
    assert rc == 5 and need == 8 + 1 + 8 + 16  # ALP_ERR_CAPACITY, with the size needed
    rc, _, _ = _c_write(f, 1, valid, off, id_=ids, parent=z, kind=kind, start=z, end=z)
    assert rc == 1  # kind 2
    n = ctypes.c_size_t(0)
    assert f(7, 1, _ptr(valid), _ptr(off), _ptr(ids), None, None, None, None, None, 0, ctypes.byref(n)) == 1
    assert f(0, 1, _ptr(valid), _ptr(off), _ptr(ids), None, None, None, None, None, 0, ctypes.byref(n)) == 1
    bad = np.array([2, 1], np.int64)
    assert f(2, 1, _ptr(valid), _ptr(bad), _ptr(ids), None, None, None, None, None, 0, ctypes.byref(n)) == 1


def _c_compare():
    import ctypes
    from alpacc_b200 import build
    lib = ctypes.CDLL(build.build_cuda())
    f = lib.alp_compare_reference_format
    f.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t,
                  ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int)]

    def cmp(mode, a: bytes, b: bytes):
        d, k = ctypes.c_int64(7), ctypes.c_int(7)
        rc = f(mode, a, len(a), b, len(b), ctypes.byref(d), ctypes.byref(k))
        return rc, d.value, k.value
    return cmp


def test_c_abi_comparator():
    """alp_compare_reference_format (host code in the C library, no GPU) agrees with
    this module's compare on equal files and on each kind of difference, names the
    first differing input and field, and refuses malformed files."""
    cmp = _c_compare()
    rng = np.random.default_rng(5)

    def tree(n):
        kind = rng.integers(0, 2, n).astype(np.uint8)
        start = rng.integers(0, 1000, n).astype(np.int64)
        return (rng.integers(0, 50, n).astype(np.int64), rng.integers(0, 30, n).astype(np.uint32), kind,
                np.where(kind == 1, start, 0), np.where(kind == 1, start + 3, 0))

    res = [tree(5), None, tree(0), tree(9), tree(2)]
    res[3][2][4] = 1  # a terminal: its start and end are written
    a = wire.write_lexparse_outputs(res)
    assert cmp(1, a, a) == (0, -1, -1) and wire.compare(a, a, "lexer-parser") is None
    # each field of element 4 of input 3, in record order (kind, parent, id, start, end)
    for k, f in ((0, 2), (1, 0), (2, 1), (3, 3), (4, 4)):
        r2 = [None if t is None else tuple(x.copy() for x in t) for t in res]
        if f == 2:  # a kind flip makes start/end 0 on the production side too
            r2[3][2][4] ^= 1
        else:
            r2[3][f][4] += 1
        b = wire.write_lexparse_outputs(r2)
        got = cmp(1, a, b)
        assert got[0] == 0 and got[1] == 3 and got[2] == k, (k, got)
        assert wire.compare(a, b, "lexer-parser") is not None
    # acceptance differs; element counts differ; result counts differ
    assert cmp(1, a, wire.write_lexparse_outputs([res[0], tree(1)] + res[2:]))[:2] == (0, 1)
    assert cmp(1, a, wire.write_lexparse_outputs(res[:3] + [tree(8), res[4]]))[:3] == (0, 3, -1)
    assert cmp(1, a, wire.write_lexparse_outputs(res[:4]))[:3] == (0, 4, -1)
    # lexer and parser-only files
    toks = [(np.array([1, 2], np.uint64), np.array([0, 3], np.uint64), np.array([3, 5], np.uint64)), None]
    la = wire.write_lexer_outputs(toks)
    lb = wire.write_lexer_outputs([(toks[0][0], toks[0][1], np.array([3, 6], np.uint64)), None])
    assert cmp(0, la, la)[1] == -1 and cmp(0, la, lb) == (0, 0, 2)
    pa = wire.write_parser_outputs([np.array([4, 5, 6]), None, np.array([], np.int64)])
    pb = wire.write_parser_outputs([np.array([4, 5, 6]), None, np.array([1])])
    assert cmp(2, pa, pa)[1] == -1 and cmp(2, pa, pb) == (0, 2, -1)
    assert cmp(2, pa, wire.write_parser_outputs([np.array([4, 7, 6]), None, np.array([], np.int64)])) == (0, 0, 0)
    # malformed: truncated, trailing bytes, a boolean or kind byte out of range, unknown mode
    assert cmp(1, a, a[:-1])[0] == 1 and cmp(1, a + b"\x00", a)[0] == 1
    bad_bool = bytearray(a)
    bad_bool[8] = 2
    assert cmp(1, bytes(bad_bool), a)[0] == 1
    bad_kind = bytearray(a)
    bad_kind[8 + 1 + 8] = 3
    assert cmp(1, bytes(bad_kind), a)[0] == 1
    assert cmp(9, a, a)[0] == 1


@pytest.mark.parametrize("mode,name", [(0, "lexer"), (1, "lexer-parser"), (2, "parser")])
def test_c_abi_comparator_fuzz(mode, name):
    """Single-byte changes to a file of each kind: the C comparator and this module's
    compare agree on equal / different, and on what is malformed (ValueError here,
    ALP_ERR_ARG there)."""
    cmp = _c_compare()
    rng = np.random.default_rng(11 + mode)
    res = []
    for i in range(6):
        if i == 2:
            res.append(None)
            continue
        n = int(rng.integers(0, 5))
        if mode == 0:
            s = rng.integers(0, 100, n).astype(np.uint64)
            res.append((rng.integers(0, 9, n).astype(np.uint64), s, s + 2))
        elif mode == 1:
            kind = rng.integers(0, 2, n).astype(np.uint8)
            s = rng.integers(0, 100, n).astype(np.int64)
            res.append((rng.integers(0, 9, n).astype(np.int64), rng.integers(0, 9, n).astype(np.uint32), kind,
                        np.where(kind == 1, s, 0), np.where(kind == 1, s + 2, 0)))
        else:
            res.append(rng.integers(0, 9, n).astype(np.uint64))
    writer = {0: wire.write_lexer_outputs, 1: wire.write_lexparse_outputs, 2: wire.write_parser_outputs}[mode]
    a = writer(res)
    for _ in range(300):
        b = bytearray(a)
        j = int(rng.integers(0, len(b)))
        b[j] = int(rng.integers(0, 256))
        b = bytes(b)
        rc, diff, _ = cmp(mode, a, b)
        try:
            py = wire.compare(a, b, name)
        except ValueError:
            assert rc == 1, (j, b[j])
            continue
        assert rc == 0, (j, b[j])
        assert (diff == -1) == (py is None), (j, b[j], diff, py)
