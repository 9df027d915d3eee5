"""Output files of this backend for alpacc test inputs, byte for byte equal
to the files written from the oracle's results (the form alpacc's own test
harness compares), through the batched GPU entry points."""

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables, wire

pytestmark = pytest.mark.gpu


def _docs(name):
    gen = {"json": lambda s, i: synth.json_doc(s, 8, i), "sexp": lambda s, i: synth.sexp_doc(s, 20, i)}[name]
    sizes = synth.lognormal_sizes(60, median=800, sigma=1.5, cap=50000, seed=5)
    docs = [gen(int(s), 70 + i).tobytes() for i, s in enumerate(sizes)]
    bad = {"json": [b"[1,", b"#"], "sexp": [b"(a", b")"]}[name]
    return [b""] + docs[:30] + bad + [b""] + docs[30:]


@pytest.mark.parametrize("name", ["json", "sexp"])
def test_lexer_and_parser_outputs_match_oracle_files(has_gpu, name):
    from alpacc_b200.api import Grammar
    tb = tables.load(name, "both")
    g, o = Grammar(tb), oracle.Oracle(tb.blob())
    docs = _docs(name)
    inputs = wire.write_inputs(docs)
    want_lex = wire.write_lexer_outputs([o.lex_futhark(d) for d in docs])
    got_lex = wire.run(g, "lexer", inputs)
    assert wire.compare(want_lex, got_lex, "lexer") is None
    assert got_lex == want_lex
    want_lp = wire.write_lexparse_outputs([o.lex_parse(d) for d in docs])
    got_lp = wire.run(g, "lexer-parser", inputs)
    assert wire.compare(want_lp, got_lp, "lexer-parser") is None
    assert got_lp == want_lp
    toks = [o.lex_futhark(d) for d in docs]
    seqs = [t[0] for t in toks if t is not None]
    want_p = wire.write_parser_outputs([o.pre_productions(s) for s in seqs])
    got_p = wire.run(g, "parser", wire.write_token_inputs(seqs))
    assert wire.compare(want_p, got_p, "parser") is None
    assert got_p == want_p
