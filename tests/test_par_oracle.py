"""The data-parallel CPU restatement (oracle/par.c, the timed CPU baseline)
against the sequential oracle: the same tokens and trees, and the same
rejections, for every grammar, at sizes that cut documents into many blocks."""

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables

GENS = {
    "json": lambda size, seed: synth.json_doc(size, 16, seed),
    "arithmetic": lambda size, seed: synth.arith_doc(size, 12, seed),
    "sexp": lambda size, seed: synth.sexp_doc(size, 20, seed),
}


def _same(a, b):
    assert (a is None) == (b is None)
    if a is not None:
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("name", sorted(GENS))
def test_par_matches_oracle(name):
    for mode in ("both", "lexer"):
        blob = tables.load(name, mode).blob()
        o, P = oracle.Oracle(blob), oracle.Par(blob, 4)
        for i, size in enumerate((0, 1, 2, 3, 17, 4096, 65537, 1 << 20, (3 << 20) + 5)):
            d = GENS[name](size, 900 + i).tobytes() if size else b""
            _same(o.lex_futhark(d), P.lex(d))
            if mode == "both":
                _same(o.lex_parse(d), P.lex_parse(d))


@pytest.mark.parametrize("name", sorted(GENS))
def test_par_rejections_match_oracle(name):
    blob = tables.load(name, "both").blob()
    o, P = oracle.Oracle(blob), oracle.Par(blob, 4)
    rng = np.random.default_rng(5)
    base = GENS[name](1 << 20, 77)
    cases = [rng.integers(0, 256, 300000, dtype=np.uint8).tobytes()]
    for _ in range(12):  # one byte changed, one byte dropped, a truncation
        j = int(rng.integers(0, base.size))
        x = base.copy()
        x[j] = rng.integers(0, 256)
        cases.append(x.tobytes())
        cases.append(np.delete(base, j).tobytes())
        cases.append(base[:j].tobytes())
    for d in cases:
        _same(o.lex_parse(d), P.lex_parse(d))
