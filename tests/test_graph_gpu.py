"""The batched parse as a CUDA graph (alp_parse_graph_*): one capture, many
replays.  Every replay must give exactly what alp_parse_batch gives for the
same documents (which the batch tests pin to the oracle document by document),
also after the input buffers are refilled with other documents of the same
shape; too-small capacities must be reported, not overrun."""

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


def _batch(name, sizes, seed, bad_every=0):
    data, off = synth.batch(name, sizes, 8 if name == "json" else 20, seed)
    data = data.copy()
    if bad_every:
        # corrupt some documents in place (same sizes): a stray closer at their middle
        closer = ord("]") if name == "json" else ord(")")
        for i in range(0, len(sizes), bad_every):
            if sizes[i] > 2:
                data[off[i] + sizes[i] // 2] = closer
    return data, off


def _same(got, want):
    (gt, gno, gv), (wt, wno, wv) = got, want
    np.testing.assert_array_equal(gv.cpu().numpy(), wv.cpu().numpy())
    np.testing.assert_array_equal(gno.cpu().numpy(), wno.cpu().numpy())
    assert len(gt) == len(wt)
    for f in ("parent", "tag", "kind", "start", "end"):
        np.testing.assert_array_equal(getattr(gt, f).cpu().numpy(), getattr(wt, f).cpu().numpy(), err_msg=f)


@pytest.mark.parametrize("name", ["json", "sexp"])
def test_graph_replays_equal_batch(has_gpu, name):
    g, o = _ctx(name)
    sizes = synth.lognormal_sizes(300, median=700, sigma=1.5, cap=30000, seed=21)
    data, off = _batch(name, sizes, 21, bad_every=37)
    want = g.parse_batch_int(data, off)
    assert 0 < int(want[2].sum()) < len(sizes)  # accepted and rejected documents both present
    pg = g.parse_batch_graph(data, off)
    try:
        for _ in range(3):
            pg.launch()
            _same(pg.result(), want)
        # other documents of the same shape, loaded into the captured buffers
        data2, off2 = _batch(name, sizes, 99, bad_every=11)
        assert np.array_equal(off2, off)
        want2 = g.parse_batch_int(data2, off2)
        pg.load(data2, off2)
        pg.launch()
        _same(pg.result(), want2)
        # the parent context keeps working while the graph lives
        t = g.lex_int(data[off[1]:off[2]].tobytes())
        assert (t is None) == (o.lex_futhark(data[off[1]:off[2]].tobytes()) is None)
        pg.load(data, off)
        pg.launch()
        _same(pg.result(), want)
    finally:
        pg.close()


def test_graph_capacity_reported(has_gpu):
    from alpacc_b200.api import AlpError
    g, _ = _ctx("json")
    sizes = synth.lognormal_sizes(40, median=2000, sigma=1.0, cap=20000, seed=5)
    data, off = _batch("json", sizes, 5)
    tree, _, _ = g.parse_batch_int(data, off)
    for caps in ((len(tree) // 2, 1 << 20), (len(tree) + 100, 10)):
        pg = g.parse_batch_graph(data, off, cap_nodes=caps[0], cap_brackets=caps[1])
        try:
            pg.launch()
            with pytest.raises(AlpError) as e:
                pg.result()
            assert e.value.code == 5  # ALP_ERR_CAPACITY
        finally:
            pg.close()
    # exact capacities are enough
    import ctypes
    from alpacc_b200.api import native
    info = (ctypes.c_int64 * 11)()
    g.parse_batch_int(data, off)
    native().alp_ctx_info(g.h, info, 11)
    pg = g.parse_batch_graph(data, off, cap_nodes=len(tree), cap_brackets=int(info[10]))
    try:
        pg.launch()
        got = pg.result()
        assert len(got[0]) == len(tree)
    finally:
        pg.close()
