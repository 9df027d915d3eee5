"""Token streams (alp_lex_stream_*, alp_lex_host_stream): input pushed in
pieces gives the tokens of the concatenation, bit-exact against the CPU oracle
(the generated ``lex_int`` restated) on small inputs and against the whole-input
GPU lexer on large ones.  Cut points fall inside tokens, inside ignored runs,
at tile and chunk edges, and include empty and one-byte pieces."""

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu

GRAMMARS = ["json", "arithmetic", "sexp"]
_CACHE = {}


def _ctx(name):
    from alpacc_b200.api import Grammar
    if name not in _CACHE:
        tb = tables.load(name, "lexer")
        _CACHE[name] = (Grammar(tb), oracle.Oracle(tb.blob()))
    return _CACHE[name]


def _gen(name, size, seed):
    if name == "json":
        return synth.json_doc(size, 8, seed)
    if name == "arithmetic":
        return synth.arith_doc(size, 12, seed)
    return synth.sexp_doc(size, 20, seed)


def _pieces(data: bytes, cuts):
    cuts = sorted(set(int(c) for c in cuts if 0 <= c <= len(data)))
    bounds = [0] + cuts + [len(data)]
    return [data[a:b] for a, b in zip(bounds[:-1], bounds[1:])]


def _stream(g, pieces, cap=None):
    total = sum(len(p) for p in pieces)
    s = g.lex_stream(total + 1 if cap is None else cap)
    try:
        for p in pieces:
            s.push(p)
        r = s.end()
        return None if r is None else tuple(x.cpu().numpy() for x in r)
    finally:
        s.close()


def _same(got, want):
    if want is None:
        assert got is None, "stream accepted an input the reference rejects"
        return
    assert got is not None, "stream rejected an input the reference accepts"
    np.testing.assert_array_equal(got[0].astype(np.uint32), np.asarray(want[0], np.uint32))
    np.testing.assert_array_equal(got[1], want[1])
    np.testing.assert_array_equal(got[2], want[2])


@pytest.mark.parametrize("name", GRAMMARS)
def test_stream_random_cuts_vs_oracle(has_gpu, name):
    g, o = _ctx(name)
    rng = np.random.default_rng(7)
    for i, size in enumerate([1, 2, 31, 32, 33, 1000, 8191, 8192, 8193, 40000]):
        data = _gen(name, size, 300 + i).tobytes()
        want = o.lex_futhark(data)
        for trial in range(4):
            k = int(rng.integers(1, 12))
            cuts = rng.integers(0, size + 1, k)
            if trial == 1:
                cuts = np.concatenate([cuts, cuts])  # empty pieces
            _same(_stream(g, _pieces(data, cuts)), want)


@pytest.mark.parametrize("name", GRAMMARS)
def test_stream_byte_at_a_time(has_gpu, name):
    g, o = _ctx(name)
    data = _gen(name, 300, 41).tobytes()
    _same(_stream(g, [data[i:i + 1] for i in range(len(data))]), o.lex_futhark(data))
    # every single cut point of a small document
    small = _gen(name, 64, 43).tobytes()
    want = o.lex_futhark(small)
    for c in range(len(small) + 1):
        _same(_stream(g, _pieces(small, [c])), want)


def test_stream_long_token_across_pieces_and_tiles(has_gpu):
    # a JSON string of 50 000 bytes: the token in progress is carried through
    # pieces and 8 KiB tiles that hold no token start
    g, o = _ctx("json")
    body = b'{"k": "' + b"x" * 50000 + b'", "n": [1, 2, 3]}'
    want = o.lex_futhark(body)
    assert want is not None
    for cuts in ([10], [7, 9000, 30000, 50006], list(range(5, len(body), 8192)), [50007, 50008]):
        _same(_stream(g, _pieces(body, cuts)), want)


@pytest.mark.parametrize("name", GRAMMARS)
def test_stream_rejected_and_empty(has_gpu, name):
    g, o = _ctx(name)
    rng = np.random.default_rng(11)
    for i in range(6):
        data = rng.integers(0, 256, 500 + 97 * i, dtype=np.uint8).tobytes()
        want = o.lex_futhark(data)
        _same(_stream(g, _pieces(data, rng.integers(0, len(data), 5))), want)
    # a valid prefix followed by a bad byte
    data = _gen(name, 4000, 5).tobytes() + b"\x01" + _gen(name, 100, 6).tobytes()
    _same(_stream(g, _pieces(data, [1000, 3999, 4000, 4001])), o.lex_futhark(data))
    _same(_stream(g, []), o.lex_futhark(b""))
    _same(_stream(g, [b"", b""]), o.lex_futhark(b""))
    _same(g.lex_host_stream(np.zeros(0, np.uint8)), o.lex_futhark(b""))


@pytest.mark.parametrize("name", ["json", "sexp"])
def test_stream_large_vs_whole_input(has_gpu, name):
    g, _ = _ctx(name)
    data = _gen(name, (24 << 20) + 12345, 77).tobytes()
    want = tuple(x.cpu().numpy() for x in g.lex_int(data))
    rng = np.random.default_rng(3)
    cuts = np.sort(rng.integers(0, len(data), 9))
    _same(_stream(g, _pieces(data, cuts)), want)


def test_stream_capacity_and_count(has_gpu):
    from alpacc_b200.api import AlpError
    g, o = _ctx("json")
    data = _gen("json", 5000, 9).tobytes()
    want = o.lex_futhark(data)
    s = g.lex_stream(len(data) + 1)
    s.push(data[:2500])
    k = s.tokens()
    # tokens final after the first half: those ending before the token in progress
    assert k == int(np.sum(np.asarray(want[2]) < 2500))
    s.push(data[2500:])
    r = s.end()
    s.close()
    _same(tuple(x.cpu().numpy() for x in r), want)
    with pytest.raises(AlpError) as e:
        _stream(g, _pieces(data, [100, 3000]), cap=5)
    assert e.value.code == 5  # ALP_ERR_CAPACITY


@pytest.mark.parametrize("name", GRAMMARS)
def test_host_stream_vs_oracle(has_gpu, name):
    g, o = _ctx(name)
    for i, (size, piece) in enumerate([(1, 0), (1000, 256), (70000, 256), (70000, 4096), (300000, 1 << 16)]):
        data = _gen(name, size, 500 + i)
        _same(g.lex_host_stream(data, piece), o.lex_futhark(data.tobytes()))


def test_host_stream_large_pinned(has_gpu):
    """40 MiB through 8 MiB pieces into pinned buffers, against alp_lex_host and against
    the device tokens of alp_lex (both host calls send the spans as 32-bit values and
    widen them on the host; alp_lex's are the 64-bit device arrays)."""
    import torch
    g, _ = _ctx("json")
    data = _gen("json", (40 << 20) + 999, 91)
    want = g.lex_host(data)
    dev = tuple(x.cpu().numpy() for x in g.lex_int(data))
    assert len(want[0]) > 4 * (1 << 20)  # several 1 Mi-value chunks of each field
    _same(want, dev)
    cap = len(data) + 1
    out = (torch.empty(cap, dtype=torch.int32).pin_memory(), torch.empty(cap, dtype=torch.int64).pin_memory(),
           torch.empty(cap, dtype=torch.int64).pin_memory())
    pin = torch.from_numpy(data).pin_memory()
    got = g.lex_host_stream(pin, 8 << 20, out)
    assert got is not None
    got = tuple(x.numpy() for x in got)
    _same(got, want)
    # rejected input
    bad = np.frombuffer(data[:100000].tobytes() + b"\x01", np.uint8)
    assert g.lex_host_stream(bad, 4096) is None
    assert g.lex_host(bad) is None


def test_lexstream_tool(has_gpu):
    import io
    from alpacc_b200 import lexstream
    _, o = _ctx("json")
    data = _gen("json", 20000, 13).tobytes()
    want = o.lex_futhark(data)
    out = io.BytesIO()
    assert lexstream.run("json", io.BytesIO(data), out, piece=777) == 0
    assert out.getvalue().decode().splitlines() == ["%d %d %d" % (a, b, t) for t, a, b in zip(*want)]
    names = tables.load("json", "lexer").terminal_names
    out = io.BytesIO()
    assert lexstream.run("json", io.BytesIO(data), out, piece=4096, names=True) == 0
    assert out.getvalue().decode().splitlines() == ["%d %d %s" % (a, b, names[t]) for t, a, b in zip(*want)]
    # rejected: the tokens before the bad byte are printed, exit status 255
    bad = data[:5000] + b"\x01"
    out = io.BytesIO()
    assert lexstream.run("json", io.BytesIO(bad), out, piece=1000) == 255
    assert len(out.getvalue().decode().splitlines()) >= int(np.sum(np.asarray(want[2]) < 4000))
