"""GPU lexer parity: the CUDA single-pass lexer against the CPU oracle's
restatement of the generated ``lex_int`` (single chunk) and of ``tokenize``,
bit-exact, through the C ABI."""

import itertools

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu

GRAMMARS = ["json", "arithmetic", "sexp"]
_CACHE = {}


def _ctx(name, mode):
    from alpacc_b200.api import Grammar
    key = (name, mode)
    if key not in _CACHE:
        tb = tables.load(name, mode)
        _CACHE[key] = (Grammar(tb), oracle.Oracle(tb.blob()))
    return _CACHE[key]


def _gen(name, size, seed):
    if name == "json":
        return synth.json_doc(size, 8, seed)
    if name == "arithmetic":
        return synth.arith_doc(size, 12, seed)
    return synth.sexp_doc(size, 20, seed)


def _check(g, o, data: bytes):
    want = o.lex_futhark(data)
    want2 = o.tokenize(data)
    got = g.lex_int(data)
    if want is None:
        assert want2 is None
        assert got is None, "GPU accepted an input the reference rejects"
        return
    assert got is not None, "GPU rejected an input the reference accepts"
    gt, gs, ge = (x.cpu().numpy() for x in got)
    for a, b in zip(want, want2):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(gt.astype(np.uint32), want[0])
    np.testing.assert_array_equal(gs, want[1])
    np.testing.assert_array_equal(ge, want[2])


@pytest.mark.parametrize("name", GRAMMARS)
@pytest.mark.parametrize("mode", ["lexer", "both"])
@pytest.mark.parametrize("split", [1, 0])
def test_generated_sizes(has_gpu, name, mode, split):
    """split: the token pass as count pass + tile scan + token pass (1) or as
    one fused pass with a look-back over tiles (0)."""
    g, o = _ctx(name, mode)
    sizes = [1, 2, 3, 15, 16, 17, 255, 4095, 4096, 4097, 8191, 65536 + 7, 131072 * 8 + 3, 1 << 22]
    saved = g.get_tuning()
    try:
        g.set_tuning(saved[:4] + [split])
        for i, size in enumerate(sizes):
            _check(g, o, _gen(name, size, 100 + i).tobytes())
    finally:
        g.set_tuning(saved)


@pytest.mark.parametrize("name", GRAMMARS)
def test_readme_and_edge_inputs(has_gpu, name):
    g, o = _ctx(name, "both")
    cases = [b"", b" ", b"\n\n", b"12+(3*4)", b"{\"a\": [1, 2.5, null]}", b"(a (b c) d)", b"\"unterminated",
             b"#", bytes(range(256)), b"a" * 5000, b" " * 9000, b"(" * 4097 + b")" * 4097]
    for c in cases:
        _check(g, o, c)


@pytest.mark.parametrize("name", GRAMMARS)
def test_exhaustive_short(has_gpu, name):
    """Every string of length <= 3 over the grammar's alphabet plus one
    foreign byte (the reference's exhaustive test mode)."""
    g, o = _ctx(name, "both")
    alpha = {"json": b'{}[],:"\\ 1-.tn', "arithmetic": b"1-+*/()a ", "sexp": b"()a1 "}[name]
    for L in range(0, 4):
        for t in itertools.product(alpha, repeat=L):
            _check(g, o, bytes(t))


@pytest.mark.parametrize("name", GRAMMARS)
def test_random_corruptions(has_gpu, name):
    """Valid documents with random byte edits (mostly rejected somewhere in
    the middle, so the dead state must propagate across tiles)."""
    g, o = _ctx(name, "both")
    rng = np.random.default_rng(7)
    for i in range(20):
        d = bytearray(_gen(name, 20000 + 997 * i, 300 + i).tobytes())
        for _ in range(int(rng.integers(1, 4))):
            d[int(rng.integers(0, len(d)))] = int(rng.integers(0, 256))
        _check(g, o, bytes(d))


def test_host_buffers(has_gpu):
    g, o = _ctx("json", "lexer")
    d = _gen("json", 300000, 5)
    got = g.lex_host(d)
    want = o.lex_futhark(d.tobytes())
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)


def test_dense_tokens_and_unaligned_input(has_gpu):
    """Tiles with more tokens than the shared-memory staging holds (every
    other byte a token) next to sparse tiles, and inputs that start off a
    16-byte boundary (byte loads instead of vector loads)."""
    import torch
    g, o = _ctx("json", "both")
    dense = b"[" + b"1," * 300000 + b"1]"
    _check(g, o, dense)
    mixed = b"[" + b"1," * 20000 + b'"' + b"x" * 50000 + b'",' + b"1," * 20000 + b"1]"
    _check(g, o, mixed)
    doc = _gen("json", 200003, 11).tobytes()
    buf = torch.frombuffer(bytearray(b"   " + doc), dtype=torch.uint8).to("cuda")
    for off in (1, 3):
        view = buf[off:]
        assert view.data_ptr() % 16 != 0
        got = g.lex_int(view)
        want = o.lex_futhark(bytes(b"   "[off:]) + doc)
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a.cpu().numpy().astype(b.dtype), b)


@pytest.mark.parametrize("mode", ["lexer", "both"])
def test_token_pass_fallbacks(has_gpu, mode):
    """The fused token pass keeps up to 16 token records per 32-byte chunk and
    stages up to 2048 tokens per 8 KiB tile: chunks with more tokens re-run
    the DFA, tiles with more take their prefix first and write directly.
    Both against the oracle, and the split passes (count pass, tile scan,
    token pass) against the fused one."""
    g, o = _ctx("json", mode)
    ga, oa = _ctx("arithmetic", mode)
    unit = b"[" * 20 + b"]" * 20 + b',"' + b"x" * 200 + b'",'   # dense chunks in staged tiles
    doc = b"[" + unit * 3000 + b"1]"
    saved = [x.get_tuning() for x in (g, ga)]
    try:
        for x, c in zip((g, ga), saved):
            x.set_tuning(c[:4] + [0])
        _check(ga, oa, b"1+" * 100000 + b"1")                     # every byte a token
        _check(ga, oa, b"(" * 70000 + b"1" + b")" * 70000)
        _check(g, o, doc)
        _check(g, o, b"[" + b"1," * 8 + b"1" * 9 + b"," + (b"[1]," * 10000) + b"1]")
    finally:
        for x, c in zip((g, ga), saved):
            x.set_tuning(c)
    d = _gen("json", 3_000_000, 41).tobytes()
    cfg = g.get_tuning()
    try:
        g.set_tuning(cfg[:4] + [0])
        fused = [x.cpu().numpy() for x in g.lex_int(d)]
        _check(g, o, doc)
        g.set_tuning(cfg[:4] + [1])
        split = [x.cpu().numpy() for x in g.lex_int(d)]
        _check(g, o, doc)
    finally:
        g.set_tuning(cfg)
    for a, b in zip(fused, split):
        np.testing.assert_array_equal(a, b)
