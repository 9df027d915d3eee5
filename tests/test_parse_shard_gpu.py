"""One document parsed as slices of its tokens (alp_parse_shard_*), one
context per slice standing in for one GPU each, against the whole-document
oracle: the key windows across slice edges, the pairs closed between the last
position of one slice and the first of the next, depth / exscan(arity - 1) /
terminal offsets carried across slices, and the previous-smaller-or-equal
searches (parents, bracket matches) answered by earlier slices' staircases.
The last test runs two processes that exchange through torch.distributed
(gloo), lexing their byte ranges (alp_lex_shard_*) and parsing the tokens."""

import os
import socket

import numpy as np
import pytest

import oracle
from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu

GRAMMARS = ["json", "arithmetic", "sexp"]
_CACHE = {}


def _ctx(name, k=6):
    from alpacc_b200.api import Grammar
    if name not in _CACHE:
        tb = tables.load(name, "both")
        _CACHE[name] = ([Grammar(tb) for _ in range(k)], oracle.Oracle(tb.blob()))
    return _CACHE[name]


def _gen(name, size, seed):
    if name == "json":
        return synth.json_doc(size, 16, seed).tobytes()
    if name == "arithmetic":
        return synth.arith_doc(size, 12, seed).tobytes()
    return synth.sexp_doc(size, 20, seed).tobytes()


def _toks(g, data):
    t = g.lex_int(data)
    return None if t is None else tuple(x.cpu().numpy() for x in t)


def _check(gs, o, data, cuts):
    from alpacc_b200 import shard
    toks = _toks(gs[0], data)
    want = o.lex_parse(data)
    if toks is None:
        assert want is None
        return
    got = shard.parse_split(gs, toks, cuts)
    assert (got is None) == (want is None), (cuts, data[:60])
    if want is None:
        return
    for a, w in zip(got, want):
        np.testing.assert_array_equal(a.astype(w.dtype), w)


@pytest.mark.parametrize("name", GRAMMARS)
def test_slices_match_whole_document(has_gpu, name):
    gs, o = _ctx(name)
    rng = np.random.default_rng(11)
    for i, size in enumerate((300, 20_000, 400_000, 3_000_000)):
        data = _gen(name, size, 700 + i)
        m = len(_toks(gs[0], data)[0])
        cut_sets = [[m // 2], [1], [m - 1], [0], [m], [1, 2, 3], [m // 3, m // 3, 2 * m // 3],
                    sorted(rng.integers(0, m + 1, 4).tolist())]
        for cuts in cut_sets:
            _check(gs, o, data, cuts)


@pytest.mark.parametrize("name", ["json", "sexp"])
def test_deep_nesting_across_slices(has_gpu, name):
    """Brackets opened in one slice and closed two slices later; parents in
    earlier slices far beyond any tile."""
    gs, o = _ctx(name)
    op, cl, leaf = (b"[", b"]", b"1") if name == "json" else (b"(", b")", b"a")
    data = op * 30000 + leaf + cl * 30000
    m = len(_toks(gs[0], data)[0])
    for cuts in ([m // 2], [m // 4, m // 2, 3 * m // 4], [5000, 30001, 30002, 55000]):
        _check(gs, o, data, cuts)
    inner = op + (op + leaf + cl + b" ") * 20000 + cl
    m = len(_toks(gs[0], inner)[0])
    _check(gs, o, inner, [m // 3, 2 * m // 3])


@pytest.mark.parametrize("name", ["json", "sexp"])
def test_rejections_across_slices(has_gpu, name):
    """A closer of the wrong kind, or one too many or too few, on one side of a
    cut and its opener on the other: every slice's verdict combined."""
    gs, o = _ctx(name)
    base = _gen(name, 200_000, 801)
    variants = []
    if name == "json":
        j = base.index(b"[", 1000)
        variants += [base[:j] + b"{" + base[j + 1:], base[:-1], base + b"]", b"[" + base]
        k = base.rindex(b"]")
        variants.append(base[:k] + b"}" + base[k + 1:])
    else:
        j = base.index(b"(", 1000)
        variants += [base[:j] + base[j + 1:], base[:-1] + b"))", b"(" + base]
    for d in variants:
        toks = _toks(gs[0], d)
        if toks is None:
            continue
        m = len(toks[0])
        for cuts in ([m // 2], [7, m - 7], [m // 3, 2 * m // 3]):
            _check(gs, o, d, cuts)


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
        g = Grammar(tables.load("json", "both"))
        data = _gen("json", (3 << 20) + 77, 56)
        n = len(data)
        bounds = [0, n // 2 + 13, n]
        a, b = bounds[rank], bounds[rank + 1]

        def gather(x):
            out = [None] * world
            dist.all_gather_object(out, x)
            return out

        toks, base, lex_ok = shard.lex_shard(g, np.frombuffer(data[a:b], np.uint8), a, rank == world - 1, rank,
                                             gather)
        assert all(gather(lex_ok)[-1:])
        tree, first, ok = shard.parse_shard(g, toks, rank == 0, rank == world - 1, rank, gather)
        parts = gather((first, [getattr(tree, f).cpu().numpy() for f in ("parent", "tag", "kind", "start", "end")],
                        ok))
        if rank == 0:
            parts.sort(key=lambda p: p[0])
            assert all(p[2] for p in parts)
            got = tuple(np.concatenate([p[1][i] for p in parts]) for i in range(5))
            want = oracle.Oracle(tables.load("json", "both").blob()).lex_parse(data)
            for x, w in zip(got, want):
                np.testing.assert_array_equal(x.astype(w.dtype), w)
            assert parts[0][0] == 0 and parts[1][0] == len(parts[0][1][0])
        q.put((rank, "ok"))
    except BaseException as e:  # report, do not hang the other rank's test
        q.put((rank, repr(e)))
        raise
    finally:
        dist.destroy_process_group()


def test_two_processes_lex_and_parse(has_gpu):
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
