"""One document lexed in ranges (alp_lex_shard_*): the union of the ranges'
tokens must equal the whole document's, bit-exact against the CPU oracle on
small documents and against the whole-document GPU lexer on large ones.
Ranges are cut inside tokens, inside long string tokens that span several
ranges, and down to one byte; rejected documents too.  The last test runs two
processes that exchange the ranges' records through torch.distributed (gloo),
as separate GPUs would."""

import os
import socket

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu

_CACHE = {}


def _ctxs(name, k=4):
    from alpacc_b200.api import Grammar
    if name not in _CACHE:
        tb = tables.load(name, "lexer")
        _CACHE[name] = ([Grammar(tb) for _ in range(k)], oracle.Oracle(tb.blob()))
    return _CACHE[name]


def _gen(name, size, seed):
    if name == "json":
        return synth.json_doc(size, 8, seed).tobytes()
    if name == "arithmetic":
        return synth.arith_doc(size, 12, seed).tobytes()
    return synth.sexp_doc(size, 20, seed).tobytes()


def _np(t):
    return None if t is None else tuple(x.cpu().numpy() for x in t)


def _same(got, want):
    assert (got is None) == (want is None)
    if want is None:
        return
    np.testing.assert_array_equal(np.asarray(got[0]).astype(np.uint32), np.asarray(want[0], np.uint32))
    np.testing.assert_array_equal(got[1], want[1])
    np.testing.assert_array_equal(got[2], want[2])


@pytest.mark.parametrize("name", ["json", "arithmetic", "sexp"])
def test_ranges_vs_oracle(has_gpu, name):
    from alpacc_b200 import shard
    gs, o = _ctxs(name)
    rng = np.random.default_rng(13)
    for i, size in enumerate([2, 40, 1000, 9000, 70000]):
        data = _gen(name, size, 600 + i)
        want = o.lex_futhark(data)
        for k in (1, 2, 3):
            cuts = rng.integers(1, size, k) if size > 1 else []
            _same(_np(shard.lex_split(gs, data, cuts)), want)
        if size <= 40:
            for c in range(1, size):  # every single cut
                _same(_np(shard.lex_split(gs, data, [c])), want)


def test_long_token_over_ranges(has_gpu):
    from alpacc_b200 import shard
    gs, o = _ctxs("json")
    body = b'{"k": "' + b"y" * 60000 + b'", "n": [1, 22, 333]}'
    want = o.lex_futhark(body)
    for cuts in ([8], [10, 20000, 40000], [7, 60006], [60007, 60010, 60012]):
        _same(_np(shard.lex_split(gs, body, cuts)), want)


@pytest.mark.parametrize("name", ["json", "sexp"])
def test_rejected_documents(has_gpu, name):
    from alpacc_b200 import shard
    gs, o = _ctxs(name)
    rng = np.random.default_rng(2)
    for i in range(4):
        data = rng.integers(0, 256, 3000 + 101 * i, dtype=np.uint8).tobytes()
        _same(_np(shard.lex_split(gs, data, rng.integers(1, len(data), 2))), o.lex_futhark(data))
    data = _gen(name, 5000, 8) + b"\x01" + _gen(name, 300, 9)
    _same(_np(shard.lex_split(gs, data, [2500, 5000, 5001])), o.lex_futhark(data))


@pytest.mark.parametrize("name", ["json", "sexp"])
def test_large_document_in_four_ranges(has_gpu, name):
    from alpacc_b200 import shard
    gs, _ = _ctxs(name)
    data = _gen(name, (16 << 20) + 777, 31)
    want = _np(gs[0].lex_int(data))
    n = len(data)
    _same(_np(shard.lex_split(gs, data, [n // 4 + 3, n // 2 - 5, 3 * n // 4 + 1])), want)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    from alpacc_b200 import shard
    from alpacc_b200.api import Grammar
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = Grammar(tables.load("json", "lexer"))
        data = _gen("json", (4 << 20) + 123, 55)
        n = len(data)
        bounds = [0, n // 3 + 1, 2 * n // 3 - 2, n][: world + 1] if world == 3 else [0, n // 2 + 7, n]
        a, b = bounds[rank], bounds[rank + 1]

        def gather(x):
            out = [None] * world
            dist.all_gather_object(out, x)
            return out

        toks, base, valid = shard.lex_shard(g, np.frombuffer(data[a:b], np.uint8), a, rank == world - 1, rank, gather)
        parts = gather((base, [t.cpu().numpy() for t in toks], valid))
        if rank == 0:
            parts.sort(key=lambda p: p[0])
            got = tuple(np.concatenate([p[1][i] for p in parts]) for i in range(3))
            assert parts[-1][2]
            want = _np(g.lex_int(data))
            _same(got, want)
            for (b0, t0, _), (b1, _, _) in zip(parts, parts[1:]):
                assert b0 + len(t0[0]) == b1
        q.put((rank, "ok"))
    except BaseException as e:  # report, do not hang the other rank's test
        q.put((rank, repr(e)))
        raise
    finally:
        dist.destroy_process_group()


def test_two_processes_exchange_through_torch_distributed(has_gpu):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=120)
    assert res == [(0, "ok"), (1, "ok")], res
    assert all(p.exitcode == 0 for p in procs)
