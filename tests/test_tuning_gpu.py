"""Autotuned launch shapes: every tile shape of the previous-smaller-or-equal
kernel and every persistent grid size must give the oracle's trees (only the
speed may differ), and alp_tune_parse must leave a valid, equally exact
setting in the context."""

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu

_CACHE = {}


def _ctx(name):
    from alpacc_b200.api import Grammar
    if name not in _CACHE:
        tb = tables.load(name, "both")
        _CACHE[name] = (Grammar(tb), oracle.Oracle(tb.blob()))
    return _CACHE[name]


def _gen(name, size, seed, depth):
    if name == "json":
        return synth.json_doc(size, depth, seed).tobytes()
    if name == "arithmetic":
        return synth.arith_doc(size, depth, seed).tobytes()
    return synth.sexp_doc(size, depth, seed).tobytes()


def _tree(g, data):
    t = g.parse_int(data)
    return None if t is None else tuple(x.cpu().numpy() for x in (t.parent, t.tag, t.kind, t.start, t.end))


def _oracle(o, data):
    w = o.lex_parse(data)
    return None if w is None else tuple(np.asarray(x) for x in w)


def _same(got, want):
    assert (got is None) == (want is None)
    if want is None:
        return
    for a, b in zip(got, want):
        np.testing.assert_array_equal(np.asarray(a).astype(np.int64), np.asarray(b).astype(np.int64))


@pytest.mark.parametrize("name", ["json", "arithmetic", "sexp"])
def test_every_tile_shape_matches_oracle(has_gpu, name):
    from alpacc_b200.api import Grammar
    g, o = _ctx(name)
    docs = [_gen(name, s, 40 + i, d) for i, (s, d) in
            enumerate([(3, 4), (100, 4), (5000, 8), (70000, 16), (300000, 3000)])]
    # nesting far deeper than a tile: parents and bracket matches across tiles
    o_, c_ = ("[", "]") if name == "json" else ("(", ")")
    if name != "json":
        docs.append((o_ * 9000 + "a" + c_ * 9000).encode() if name == "sexp" else (o_ * 9000 + "1" + c_ * 9000).encode())
    else:
        docs.append(("[" * 9000 + "1" + "]" * 9000).encode())
    docs.append(docs[2][:-1])  # rejected
    wants = [_oracle(o, d) for d in docs]
    saved = g.get_tuning()
    try:
        for shape in range(len(Grammar.tile_shapes())):
            for ctas in (0, 1):
                g.set_tuning([shape, ctas, ctas])
                for d, w in zip(docs, wants):
                    _same(_tree(g, d), w)
    finally:
        g.set_tuning(saved)


def test_tuner_keeps_a_valid_exact_setting(has_gpu):
    from alpacc_b200.api import AlpError, Grammar
    g, o = _ctx("json")
    sample = _gen("json", 4 << 20, 77, 16)
    want = _tree(g, sample)
    saved = g.get_tuning()
    try:
        res = g.tune(sample, reps=2)
        cfg = res["config"]
        assert 0 <= cfg[0] < len(Grammar.tile_shapes()) and cfg[2] >= 1
        assert cfg[4] in (0, 1) and cfg[5] in (0, 1) and cfg[6] in (8, 16, 32)
        names = {k for k, _, _ in res["timings"]}
        assert {"expand_ctas_per_sm", "best_ms", "lex_token_pass_split", "lex_scan_chunks_per_lane",
                "parse_position_pass_split"} <= names
        assert ("pairs_ctas_per_sm" in names) == (cfg[5] == 1)
        assert sum(1 for k, _, _ in res["timings"] if k.startswith("ple_shape_")) == len(Grammar.tile_shapes())
        _same(_tree(g, sample), want)
        small = _gen("json", 20000, 3, 8)
        _same(_tree(g, small), _oracle(o, small))
        with pytest.raises(AlpError):
            g.set_tuning([len(Grammar.tile_shapes()), 0, 0])
    finally:
        g.set_tuning(saved)


@pytest.mark.parametrize("name", ["json", "sexp"])
def test_every_lexer_knob_against_oracle(has_gpu, name):
    """Every lexer setting the tuner may pick (state-scan chunks per lane 8,
    16, 32; fused or split token pass) and both forms of the parser's position
    pass give the oracle's tree."""
    g, o = _ctx(name)
    docs = [_gen(name, 3_000_001, 88, 16 if name == "json" else 20), b"", b"x"]
    docs.append(_gen(name, 200_000, 89, 16 if name == "json" else 20))
    wants = [_oracle(o, d) for d in docs]
    saved = g.get_tuning()
    try:
        for gs in (8, 16, 32):
            for lex_split in (0, 1):
                for parse_split in (0, 1):
                    g.set_tuning(saved[:4] + [lex_split, parse_split, gs])
                    for d, w in zip(docs, wants):
                        _same(_tree(g, d), w)
    finally:
        g.set_tuning(saved)
