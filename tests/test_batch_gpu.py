"""Batched (segmented) lex and parse: every document of a batch against the
oracle run on that document alone (the reference API lexes/parses one
document per call), bit-exact, including empty, one-byte, rejected and
tile-aligned documents."""

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu

_CACHE = {}


def _ctx(name, mode):
    from alpacc_b200.api import Grammar
    key = (name, mode)
    if key not in _CACHE:
        tb = tables.load(name, mode)
        _CACHE[key] = (Grammar(tb), oracle.Oracle(tb.blob()))
    return _CACHE[key]


def _docs(name, n_docs, seed, median=600, cap=20000):
    sizes = synth.lognormal_sizes(n_docs, median=median, sigma=1.5, cap=cap, seed=seed)
    data, off = synth.batch(name, sizes, 8 if name == "json" else 20, seed)
    return [data[off[i]:off[i + 1]].tobytes() for i in range(n_docs)]


def _special(name):
    good = {"json": [b"[1]", b"{}", b"  [ 1 , 2 ] ", b"\"x\"", b"7"],
            "sexp": [b"a", b"()", b"(a (b c))", b" (x) "]}[name]
    bad = {"json": [b"[1", b"\"open", b"#", b"]"], "sexp": [b"(a", b")", b"(("]}[name]
    return good, bad


def _layout(name, docs):
    """Insert empty documents at the front, middle and end, and a padding
    document so that the next one starts exactly on a 4096-byte tile boundary."""
    out = [b"", b""] + docs[:3] + [b""] + docs[3:] + [b"", b""]
    pos = sum(len(d) for d in out[:5])
    pad = (-pos) % 4096
    o, c, one = (b"[", b"]", b"1") if name == "json" else (b"(", b")", b"a")
    if pad == 1:
        out.insert(5, one)
    elif pad >= 2:
        out.insert(5, o + b" " * (pad - 2) + c)
    return out


def _pack(docs):
    off = np.zeros(len(docs) + 1, np.int64)
    off[1:] = np.cumsum([len(d) for d in docs])
    data = np.frombuffer(b"".join(docs), np.uint8) if off[-1] else np.zeros(0, np.uint8)
    return data, off


@pytest.mark.parametrize("name", ["json", "sexp"])
@pytest.mark.parametrize("mode", ["lexer", "both"])
def test_lex_batch(has_gpu, name, mode):
    g, o = _ctx(name, mode)
    rng = np.random.default_rng(3)
    good, bad = _special(name)
    docs = _layout(name, _docs(name, 300, 77) + good + bad)
    data, off = _pack(docs)
    term, start, end, tok_off, valid = (x.cpu().numpy() for x in g.lex_batch_int(data, off))
    assert tok_off[0] == 0 and tok_off[-1] == len(term)
    for i, d in enumerate(docs):
        want = o.lex_futhark(d)
        assert bool(valid[i]) == (want is not None), (i, d[:40])
        if want is None:
            continue
        a, b = tok_off[i], tok_off[i + 1]
        np.testing.assert_array_equal(term[a:b].astype(np.uint32), want[0])
        np.testing.assert_array_equal(start[a:b], want[1])
        np.testing.assert_array_equal(end[a:b], want[2])


@pytest.mark.parametrize("name", ["json", "sexp"])
def test_parse_batch(has_gpu, name):
    g, o = _ctx(name, "both")
    rng = np.random.default_rng(5)
    good, bad = _special(name)
    docs = _docs(name, 400, 91)
    # structurally broken documents (a closer removed) among valid ones
    for i in range(0, 40, 4):
        d = bytearray(docs[i])
        j = max((k for k, c in enumerate(d) if c in b")]}"), default=None)
        if j is not None:
            del d[j]
            docs[i] = bytes(d)
    docs = _layout(name, docs + good + bad)
    data, off = _pack(docs)
    tree, node_off, valid = g.parse_batch_int(data, off)
    par, tag, kind, st, en = (x.cpu().numpy() for x in (tree.parent, tree.tag, tree.kind, tree.start, tree.end))
    node_off, valid = node_off.cpu().numpy(), valid.cpu().numpy()
    n_valid = 0
    for i, d in enumerate(docs):
        want = o.lex_parse(d)
        assert bool(valid[i]) == (want is not None), (i, d[:60])
        if want is None:
            continue
        n_valid += 1
        a, b = node_off[i], node_off[i + 1]
        for got, w in zip((par[a:b], tag[a:b].astype(np.uint32), kind[a:b], st[a:b], en[a:b]), want):
            np.testing.assert_array_equal(got, w)
    assert n_valid > 300


@pytest.mark.parametrize("name", ["json", "sexp"])
def test_parse_batch_host(has_gpu, name):
    """alp_parse_batch_host (host offsets in, parents and spans back as 32-bit values
    widened on the host): the same arrays as alp_parse_batch on the device, for a batch
    with empty, rejected and broken documents and one large enough for several copy
    chunks; every accepted document against the oracle; a short capacity reports the
    node total; offsets that decrease are refused."""
    import ctypes
    from alpacc_b200 import api
    g, o = _ctx(name, "both")
    good, bad = _special(name)
    docs = _docs(name, 300, 93)
    for i in range(0, 30, 3):
        d = bytearray(docs[i])
        j = max((k for k, c in enumerate(d) if c in b")]}"), default=None)
        if j is not None:
            del d[j]
            docs[i] = bytes(d)
    big = synth.json_doc(12 << 20, 16, 95) if name == "json" else synth.sexp_doc(12 << 20, 20, 95)
    docs = _layout(name, docs + good + bad + [big.tobytes()])
    data, off = _pack(docs)
    tree, node_off, valid = g.parse_batch_int(data, off)
    want = [x.cpu().numpy() for x in (tree.parent, tree.tag, tree.kind, tree.start, tree.end)]
    want_off, want_valid = node_off.cpu().numpy(), valid.cpu().numpy()
    got = g.parse_batch_host(data, off)
    assert len(got[0]) == len(want[0]) > (1 << 21)
    for a, b in zip(got[:5], want):
        np.testing.assert_array_equal(a, b.astype(a.dtype))
    np.testing.assert_array_equal(got[5], want_off)
    np.testing.assert_array_equal(got[6], want_valid)
    for i in list(range(0, 60)) + [len(docs) - 3]:
        w = o.lex_parse(docs[i])
        assert bool(got[6][i]) == (w is not None)
        if w is not None:
            a, b = got[5][i], got[5][i + 1]
            for x, y in zip(got[:5], w):
                np.testing.assert_array_equal(x[a:b], y)
    L = api.native()
    total = ctypes.c_int64(0)
    bufs = [np.empty(16, dt) for dt in (np.int64, np.uint32, np.uint8, np.int64, np.int64)]
    no, nv = np.empty(len(docs) + 1, np.int64), np.empty(len(docs), np.uint8)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = L.alp_parse_batch_host(g.h, vp(data), vp(off), len(docs), *[vp(b) for b in bufs], vp(no), vp(nv), 16,
                                ctypes.byref(total))
    assert rc == 5 and total.value == len(want[0])
    off2 = off.copy()
    off2[3], off2[4] = off2[4], off2[3] - 1
    rc = L.alp_parse_batch_host(g.h, vp(data), vp(off2), len(docs), *[vp(b) for b in bufs], vp(no), vp(nv), 16,
                                ctypes.byref(total))
    assert rc == 1


def test_single_doc_batch_equals_parse(has_gpu):
    g, o = _ctx("json", "both")
    d = synth.json_doc(300000, 16, 12345)
    data, off = _pack([d.tobytes()])
    tree, node_off, valid = g.parse_batch_int(data, off)
    one = g.parse_int(d)
    assert valid.cpu().numpy()[0] == 1
    np.testing.assert_array_equal(tree.parent.cpu().numpy(), one.parent.cpu().numpy())
    np.testing.assert_array_equal(tree.start.cpu().numpy(), one.start.cpu().numpy())


def _stress_layout(name):
    """Documents that start exactly on 8 KiB and 16 KiB tile boundaries, runs
    of hundreds of one- and two-byte documents (tiles holding more documents
    than the shared offset list), empty documents between them, and documents
    dense in tokens and nodes (a token every other byte)."""
    o, c, one = (b"[", b"]", b"1") if name == "json" else (b"(", b")", b"a")
    sep = b"," if name == "json" else b" "
    dense = o + sep.join([one] * 6000) + c
    docs, pos = [], 0

    def add(d):
        nonlocal pos
        docs.append(d)
        pos += len(d)

    for boundary in (8192, 16384, 3 * 8192, 4 * 16384):
        add(dense)
        pad = (-pos) % boundary
        if pad >= 2:
            add(o + b" " * (pad - 2) + c)
        elif pad == 1:
            add(one)
        add(b"")
        add(o + one + c)
    for i in range(700):
        add(one if i % 3 else b"")
        if i % 50 == 0:
            add(o + c)
    add(dense)
    return docs


@pytest.mark.parametrize("name", ["json", "sexp"])
def test_parse_batch_tile_boundaries_and_dense(has_gpu, name):
    g, o = _ctx(name, "both")
    docs = _stress_layout(name)
    data, off = _pack(docs)
    tree, node_off, valid = g.parse_batch_int(data, off)
    par, tag, kind, st, en = (x.cpu().numpy() for x in (tree.parent, tree.tag, tree.kind, tree.start, tree.end))
    node_off, valid = node_off.cpu().numpy(), valid.cpu().numpy()
    for i, d in enumerate(docs):
        want = o.lex_parse(d)
        assert bool(valid[i]) == (want is not None), (i, d[:40])
        if want is None:
            continue
        a, b = node_off[i], node_off[i + 1]
        for got, w in zip((par[a:b], tag[a:b].astype(np.uint32), kind[a:b], st[a:b], en[a:b]), want):
            np.testing.assert_array_equal(got, w)
    term, start, end, tok_off, lvalid = (x.cpu().numpy() for x in g.lex_batch_int(data, off))
    for i, d in enumerate(docs):
        want = o.lex_futhark(d)
        assert bool(lvalid[i]) == (want is not None)
        if want is not None:
            a, b = tok_off[i], tok_off[i + 1]
            np.testing.assert_array_equal(term[a:b].astype(np.uint32), want[0])
            np.testing.assert_array_equal(start[a:b], want[1])
            np.testing.assert_array_equal(end[a:b], want[2])


@pytest.mark.parametrize("name", ["json", "sexp"])
def test_parse_batch_bracket_mismatches(has_gpu, name):
    """Brackets are matched inside threads and warps, and only the rest crosses
    tiles: documents whose one flaw is a closer of the wrong kind (depth
    intact) at the start, the middle or the end, documents that end open
    followed by documents that start with closers, and many small documents
    per warp, each document's validity against the oracle."""
    g, o = _ctx(name, "both")
    rng = np.random.default_rng(23)
    docs = _docs(name, 600, 47, median=120, cap=60000)
    closers = b"]}" if name == "json" else b")"
    for i in range(0, len(docs), 3):
        d = bytearray(docs[i])
        pos = [k for k, c in enumerate(d) if c in closers]
        if not pos:
            continue
        j = pos[[0, len(pos) // 2, len(pos) - 1, int(rng.integers(0, len(pos)))][i % 4]]
        if name == "json":
            d[j] = closers[(closers.index(d[j]) + 1) % 2]
        else:
            del d[j]
        docs[i] = bytes(d)
    opener, closer = (b"[", b"]") if name == "json" else (b"(", b")")
    extra = []
    for k in range(1, 40):
        extra += [opener * k + (b"1" if name == "json" else b"a"), closer * k, opener * k + closer * k]
    docs = docs[:300] + extra + docs[300:]
    data, off = _pack(docs)
    tree, node_off, valid = g.parse_batch_int(data, off)
    par = tree.parent.cpu().numpy()
    node_off, valid = node_off.cpu().numpy(), valid.cpu().numpy()
    n_bad = 0
    for i, d in enumerate(docs):
        want = o.lex_parse(d)
        assert bool(valid[i]) == (want is not None), (i, d[:60])
        if want is None:
            n_bad += 1
            continue
        np.testing.assert_array_equal(par[node_off[i]:node_off[i + 1]], want[0])
    assert n_bad > 100
