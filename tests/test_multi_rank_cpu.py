"""The N > 1 path of bench.py on CPU: two gloo ranks, one process each, go
through the same process-group set-up, max-over-ranks step time and
whole-job throughput that the torchrun launch uses on GPUs (there each rank
parses its own document: replicas, no data-path collective)."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench
    dist = bench._dist_init(world, backend="gloo")
    ms = bench._max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")  # rank 1 is the slower one
    dist.barrier()
    out.put((rank, ms, bench._gbs(world, 256 << 20, ms)))
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_step():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, _, _ in res] == [0, 1]
    for _, ms, gbs in res:
        assert ms == pytest.approx(15.0)
        assert gbs == pytest.approx(2 * (256 << 20) / 15e-3 / 1e9)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench._dist_init(1) is None
    assert bench._max_over_ranks(3.5, None, "cpu") == 3.5
