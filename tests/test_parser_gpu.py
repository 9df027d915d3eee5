"""GPU parser parity: the CUDA LLP parse (bytes -> preorder tree) against the
CPU oracle's restatement of the generated ``parse_int`` (and of the
sequential glue parser), bit-exact, through the C ABI."""

import itertools
import json
import os

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
_CACHE = {}


def _ctx(name):
    from alpacc_b200.api import Grammar
    if name not in _CACHE:
        tb = tables.load(name, "both")
        _CACHE[name] = (Grammar(tb), oracle.Oracle(tb.blob()), tb)
    return _CACHE[name]


def _gen(name, size, seed, depth=None):
    if name == "json":
        return synth.json_doc(size, depth or 16, seed)
    if name == "arithmetic":
        return synth.arith_doc(size, depth or 12, seed)
    return synth.sexp_doc(size, depth or 20, seed)


def _check(g, o, data: bytes):
    want = o.lex_parse(data)
    got = g.parse_int(data)
    if want is None:
        assert got is None, "GPU accepted an input the reference rejects"
        return 0
    assert got is not None, "GPU rejected an input the reference accepts"
    gp, gt, gk, gs, ge = (x.cpu().numpy() for x in (got.parent, got.tag, got.kind, got.start, got.end))
    wp, wt, wk, ws, we = want
    np.testing.assert_array_equal(gt.astype(np.uint32), wt)
    np.testing.assert_array_equal(gk, wk)
    np.testing.assert_array_equal(gs, ws)
    np.testing.assert_array_equal(ge, we)
    np.testing.assert_array_equal(gp, wp)
    return len(wp)


def test_readme_tree(has_gpu):
    """The README's parse of 12+(3*4) (README.md:84-106), node for node."""
    g, o, tb = _ctx("arithmetic")
    with open(os.path.join(GOLDEN, "readme_arith_tree.json")) as f:
        gold = json.load(f)
    named = g.parse(gold["input"].encode())
    assert [list(x[1]) if x[1][0] == "production" else x for x in named] is not None
    want = [(p, tuple(n) if n[0] == "production" else (n[0], n[1], tuple(n[2]))) for p, n in gold["tree"]]
    got = [(p, n if n[0] == "production" else (n[0], n[1], tuple(n[2]))) for p, n in named]
    assert got == want


@pytest.mark.parametrize("name", ["json", "arithmetic", "sexp"])
def test_generated_sizes(has_gpu, name):
    g, o, _ = _ctx(name)
    for i, size in enumerate([2, 3, 17, 100, 1000, 4096, 4097, 20000, 65537, 1 << 20, (1 << 22) + 5]):
        _check(g, o, _gen(name, size, 500 + i).tobytes())


@pytest.mark.parametrize("name", ["json", "arithmetic", "sexp"])
def test_exhaustive_short(has_gpu, name):
    g, o, _ = _ctx(name)
    alpha = {"json": b'{}[],:"1 n', "arithmetic": b"1-+*()a ", "sexp": b"()a "}[name]
    for L in range(0, 5 if name != "json" else 4):
        for t in itertools.product(alpha, repeat=L):
            _check(g, o, bytes(t))


@pytest.mark.parametrize("name", ["json", "arithmetic", "sexp"])
def test_corrupted(has_gpu, name):
    """Structural edits: delete/duplicate a bracket, swap closers.  Most are
    rejected by the bracket match far from the edit."""
    g, o, _ = _ctx(name)
    rng = np.random.default_rng(11)
    closers = {"json": b"]}", "arithmetic": b")", "sexp": b")"}[name]
    for i in range(25):
        d = bytearray(_gen(name, 30000 + 1013 * i, 700 + i).tobytes())
        pos = [j for j, c in enumerate(d) if c in closers]
        if pos:
            j = pos[int(rng.integers(0, len(pos)))]
            op = i % 3
            if op == 0:
                del d[j]
            elif op == 1:
                d.insert(j, d[j])
            else:
                d[j] = closers[(closers.index(d[j]) + 1) % len(closers)]
        _check(g, o, bytes(d))


def test_deep_nesting(has_gpu):
    """Nesting far deeper than one tile, so matches and parents cross tiles."""
    g, o, _ = _ctx("json")
    for depth in [10, 1000, 5000]:
        d = b"[" * depth + b"1" + b"]" * depth
        assert _check(g, o, d) > 0
        _check(g, o, b"[" * depth + b"1" + b"]" * (depth - 1))
        _check(g, o, b"[" * depth + b"1" + b"]" * (depth - 1) + b"}")
    gs, os_, _ = _ctx("sexp")
    _check(gs, os_, b"(" * 20000 + b"a" + b")" * 20000)


def test_parser_only_and_glue(has_gpu):
    """parse_tokens_int and pre_productions_int against the oracle, and the
    glue parser agreeing with the scan formulation on valid input."""
    g, o, _ = _ctx("json")
    d = _gen("json", 200000, 9)
    toks = o.lex_futhark(d.tobytes())
    want = o.parse_futhark(*toks)
    glue = o.parse_glue(*toks)
    for a, b in zip(want, glue):
        np.testing.assert_array_equal(a, b)
    got = g.parse_tokens_int(toks[0].astype(np.int64), toks[1], toks[2])
    np.testing.assert_array_equal(got.parent.cpu().numpy(), want[0])
    np.testing.assert_array_equal(got.tag.cpu().numpy().astype(np.uint32), want[1])
    pp = g.pre_productions_int(toks[0].astype(np.int64))
    np.testing.assert_array_equal(pp.cpu().numpy().astype(np.uint32), o.pre_productions(toks[0]))


def test_host_buffers(has_gpu):
    g, o, _ = _ctx("sexp")
    d = _gen("sexp", 123457, 3)
    got = g.parse_host(d)
    want = o.lex_parse(d.tobytes())
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)


def test_host_buffers_json_and_rejections(has_gpu):
    """alp_parse_host on json (tags, kinds and spans start back to the host while the
    searches run): the tree of a 3 MiB document, a document the parser rejects after the
    lexer accepted it, and one the lexer rejects."""
    g, o, _ = _ctx("json")
    d = _gen("json", (3 << 20) + 11, 21)
    got = g.parse_host(d)
    want = o.lex_parse(d.tobytes())
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)
    bad_parse = b'{"a": [1, 2}, "b": 3}'   # every token fine, the brackets do not match
    assert o.lex_parse(bad_parse) is None and o.tokenize(bad_parse) is not None
    assert g.parse_host(np.frombuffer(bad_parse, np.uint8)) is None
    bad_lex = b'{"a": @}'
    assert o.tokenize(bad_lex) is None
    assert g.parse_host(np.frombuffer(bad_lex, np.uint8)) is None
    # the context is fine afterwards
    got = g.parse_host(d)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)


def test_host_widening_chunks(has_gpu):
    """alp_parse_host sends parents and spans as 32-bit values and widens them on the
    host chunk by chunk (1 Mi values per copy through a ring of sixteen slots, 256 Ki
    values per slice): a 32 MiB json document (nine chunks of each field, 45 copies in
    all, so the ring wraps, and a partial last chunk and slice) into pageable arrays,
    into pinned arrays, and into arrays one element off a 32-byte boundary, with the
    default threads and with one; the bytes it reports moving match 17 per node."""
    import ctypes
    import torch
    from alpacc_b200 import api
    g, o, tb = _ctx("json")
    d = _gen("json", (32 << 20) + 5, 23)
    want = o.lex_parse(d.tobytes())
    N = len(want[0])
    assert N > 2 * (1 << 22) and N % (1 << 18) != 0
    got = g.parse_host(d)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)
    info = (ctypes.c_int64 * 15)()
    assert api.native().alp_ctx_info(g.h, info, 15) == 0
    assert info[13] == len(d) and info[14] == 17 * N
    vp = lambda a: ctypes.c_void_p(a.data_ptr())
    n, valid = ctypes.c_int64(0), ctypes.c_int(0)
    h_in = torch.from_numpy(d).pin_memory()
    dts = (torch.int64, torch.int32, torch.uint8, torch.int64, torch.int64)
    for shift in (0, 1):
        bufs = [torch.full((N + 8,), 90, dtype=dt, pin_memory=True) for dt in dts]
        outs = [b[shift:shift + N] for b in bufs]
        rc = api.native().alp_parse_host(g.h, vp(h_in), len(d), *[vp(x) for x in outs], N, ctypes.byref(n),
                                         ctypes.byref(valid))
        assert rc == 0 and valid.value == 1 and n.value == N
        for x, w in zip(outs, want):
            np.testing.assert_array_equal(x.numpy().astype(w.dtype), w)
        for b in bufs:  # nothing written outside the N elements
            assert (b[:shift] == 90).all() and (b[shift + N:] == 90).all()
    os.environ["ALP_HOST_THREADS"] = "1"
    try:
        g1 = api.Grammar(tb)
        got = g1.parse_host(d)
    finally:
        del os.environ["ALP_HOST_THREADS"]
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("name", ["json", "arithmetic", "sexp"])
def test_host_buffers_short_inputs(has_gpu, name):
    """alp_parse_host on every short input over a small alphabet (trees of a few nodes,
    rejections, the empty input) against the oracle."""
    g, o, _ = _ctx(name)
    alpha = {"json": b'[]1 ', "arithmetic": b"1+()", "sexp": b"()a "}[name]
    for L in range(0, 4):
        for t in itertools.product(alpha, repeat=L):
            d = bytes(t)
            want = o.lex_parse(d)
            got = g.parse_host(np.frombuffer(d, np.uint8))
            assert (got is None) == (want is None), d
            if want is not None:
                for a, b in zip(got, want):
                    np.testing.assert_array_equal(a, b)


def test_host_null_outputs(has_gpu):
    """A host output array missing while the capacity is positive: ALP_ERR_ARG before any
    work; a capacity of 0 with no arrays: ALP_ERR_CAPACITY with the node count."""
    import ctypes
    from alpacc_b200 import api
    g, o, _ = _ctx("json")
    d = _gen("json", 5000, 24)
    n_want = len(o.lex_parse(d.tobytes())[0])
    bufs = [np.zeros(n_want, dt) for dt in (np.int64, np.uint32, np.uint8, np.int64, np.int64)]
    n, valid = ctypes.c_int64(0), ctypes.c_int(0)
    vp = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)
    L = api.native()
    for miss in range(5):
        args = [vp(b) if i != miss else None for i, b in enumerate(bufs)]
        assert L.alp_parse_host(g.h, vp(d), len(d), *args, n_want, ctypes.byref(n), ctypes.byref(valid)) == 1
    assert L.alp_parse_host(g.h, vp(d), len(d), None, None, None, None, None, 0, ctypes.byref(n),
                            ctypes.byref(valid)) == 5 and n.value == n_want
    got = g.parse_host(d)  # the context is fine afterwards
    for a, w in zip(got, o.lex_parse(d.tobytes())):
        np.testing.assert_array_equal(a, w)


def test_host_buffers_too_small(has_gpu):
    """A host capacity below the node count: ALP_ERR_CAPACITY with the count needed, and
    nothing written past the capacity (no copy was started early)."""
    import ctypes
    from alpacc_b200 import api
    g, o, _ = _ctx("json")
    d = _gen("json", 200_000, 22)
    n_want = len(o.lex_parse(d.tobytes())[0])
    cap = n_want // 2
    canary = 0x5a
    bufs = [np.full(cap + 64, canary, dt) for dt in (np.int64, np.uint32, np.uint8, np.int64, np.int64)]
    n, valid = ctypes.c_int64(0), ctypes.c_int(0)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = api.native().alp_parse_host(g.h, vp(d), len(d), *[vp(b) for b in bufs], cap, ctypes.byref(n),
                                     ctypes.byref(valid))
    assert rc == 5 and n.value == n_want
    for b in bufs:
        assert (b[cap:] == canary).all()
    got = g.parse_host(d)  # and a call with room works
    for a, w in zip(got, o.lex_parse(d.tobytes())):
        np.testing.assert_array_equal(a, w)


def _bracket_counts(tb, data: bytes):
    """Brackets of the LLP pair sequence and the pairs closed between adjacent
    positions (a position's first rights against the previous position's top
    lefts, none across a document start), computed on the CPU from the
    oracle's tokens and the pair table."""
    o = oracle.Oracle(tb.blob())
    p = tb.parser
    terms = o.lex_futhark(data)[0]
    arr = [p.start] + [int(t) for t in terms] + [p.end]
    kmap = dict(zip(p.keys, p.key_pair))
    n = len(arr)
    pids = [kmap[tuple(arr[j] if 0 <= j < n else p.empty for j in range(i - p.q, i + p.k))] for i in range(n)]
    nbr = [b - a for a, b, _, _ in p.pairs]
    nl = [sum(1 for x in p.stack[a:b] if x >> 31) for a, b, _, _ in p.pairs]
    brackets = sum(nbr[x] for x in pids)
    closed = sum(min(nl[a], nbr[b] - nl[b]) for a, b in zip(pids, pids[1:]))
    return brackets, closed


@pytest.mark.parametrize("name", ["json", "arithmetic", "sexp"])
def test_adjacent_bracket_pairs_counted(has_gpu, name):
    """The parser closes the bracket pairs between adjacent positions before the
    bracket search; the counts it reports equal the CPU's."""
    import ctypes
    from alpacc_b200 import api
    g, o, tb = _ctx(name)
    for i, size in enumerate([100, 5000, 300000]):
        d = _gen(name, size, 900 + i).tobytes()
        assert g.parse_int(d) is not None
        info = (ctypes.c_int64 * 12)()
        assert api.native().alp_ctx_info(g.h, info, 12) == 0
        brackets, closed = _bracket_counts(tb, d)
        assert info[10] == brackets
        assert info[11] == brackets - 2 * closed
        assert 0 < info[11] < brackets or brackets == 0


@pytest.mark.parametrize("name", ["json", "arithmetic", "sexp"])
def test_fused_and_two_pass_position_forms(has_gpu, name):
    """The position pass has two forms: one fused kernel (pair lookup, look-back
    over tiles, expansion) sized from the previous parse on the context, and
    the pair pass + tile-sum scan + expansion that sizes exactly first.  A
    fresh context's first parse takes the second form, later ones the first;
    both against the oracle, and a document much denser in nodes and brackets
    than the one before it (the fused form's estimate is short, so it runs
    again at the exact sizes)."""
    from alpacc_b200.api import Grammar
    tb = tables.load(name, "both")
    o = oracle.Oracle(tb.blob())
    g = Grammar(tb)
    sparse = {"json": b'["' + b"x" * 300000 + b'"]', "arithmetic": b"1" * 300000,
              "sexp": b"(" + b"a" * 300000 + b")"}[name]
    dense = {"json": b"[" + b"[1]," * 100000 + b"1]", "arithmetic": b"(" * 50000 + b"1" + b")" * 50000,
             "sexp": b"(" + b"()" * 150000 + b")"}[name]
    docs = [_gen(name, 2_000_003, 501).tobytes(), _gen(name, 777_777, 502).tobytes(), sparse, dense,
            _gen(name, 3_000_000, 503).tobytes()]
    cfg = g.get_tuning()
    try:
        g.set_tuning(cfg[:5] + [0])
        for d in docs:  # first call: two-pass form; then fused, estimates from the previous document
            _check(g, o, d)
        # a batch in the fused form: documents restart the sums inside tiles
        sizes = synth.lognormal_sizes(500, median=700, sigma=1.5, cap=30000, seed=504)
        data, off = synth.batch(name if name != "arithmetic" else "json", sizes, 8, 504) if name != "arithmetic" \
            else (None, None)
        if data is not None:
            tree, node_off, valid = g.parse_batch_int(data, off)
            par, tag, kind, st, en = (x.cpu().numpy() for x in (tree.parent, tree.tag, tree.kind, tree.start,
                                                                 tree.end))
            node_off, valid = node_off.cpu().numpy(), valid.cpu().numpy()
            for i in range(len(sizes)):
                want = o.lex_parse(data[off[i]:off[i + 1]].tobytes())
                assert bool(valid[i]) == (want is not None)
                if want is not None:
                    a, b = node_off[i], node_off[i + 1]
                    for got, w in zip((par[a:b], tag[a:b], kind[a:b], st[a:b], en[a:b]), want):
                        np.testing.assert_array_equal(got.astype(w.dtype), w)
        g.set_tuning(cfg[:5] + [1])
        for d in docs[:2]:
            _check(g, o, d)
    finally:
        g.set_tuning(cfg)


def test_fused_caller_buffer_too_small(has_gpu):
    """alp_parse_into with a node capacity below the tree's size reports the
    size needed, in either form of the position pass."""
    import ctypes
    import torch
    from alpacc_b200 import api
    g, o, tb = _ctx("json")
    d = torch.from_numpy(_gen("json", 400_000, 601)).cuda()
    want = o.lex_parse(d.cpu().numpy().tobytes())
    N = len(want[0])
    L = api.native()
    for split in (0, 1):
        cfg = g.get_tuning()
        g.set_tuning(cfg[:5] + [split])
        try:
            assert g.parse_int(d) is not None  # a parse on the context first: estimates exist
            outs = [torch.empty(N // 2, dtype=dt, device="cuda") for dt in
                    (torch.int64, torch.int32, torch.uint8, torch.int64, torch.int64)]
            n, v = ctypes.c_int64(0), ctypes.c_int(0)
            rc = L.alp_parse_into(g.h, ctypes.c_void_p(d.data_ptr()), d.numel(),
                                  *[ctypes.c_void_p(x.data_ptr()) for x in outs], N // 2, ctypes.byref(n),
                                  ctypes.byref(v))
            assert rc == api.ALP_ERR_CAPACITY and n.value == N
            outs = [torch.empty(N, dtype=dt, device="cuda") for dt in
                    (torch.int64, torch.int32, torch.uint8, torch.int64, torch.int64)]
            rc = L.alp_parse_into(g.h, ctypes.c_void_p(d.data_ptr()), d.numel(),
                                  *[ctypes.c_void_p(x.data_ptr()) for x in outs], N, ctypes.byref(n),
                                  ctypes.byref(v))
            assert rc == 0 and v.value == 1 and n.value == N
            for a, w in zip(outs, want):
                np.testing.assert_array_equal(a.cpu().numpy().astype(w.dtype), w)
        finally:
            g.set_tuning(cfg)
