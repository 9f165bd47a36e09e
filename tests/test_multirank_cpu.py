"""bench.py with several ranks (one replica per GPU, "replicas only": the path has no
exchange step): the host logic that combines the ranks -- the slowest rank's time and
end-to-end rate, and the whole-job throughput -- checked with two gloo ranks on CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r timed 1 + r seconds and saw an end-to-end rate of 10 - r GB/s
        total, e2e = bench.reduce_over_ranks(dist, 1.0 + rank, 10.0 - rank, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()
    out.put((rank, total, e2e))


def test_two_ranks_take_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(out.get(timeout=10) for _ in range(world))
    assert got == [(0, 2.0, 9.0), (1, 2.0, 9.0)]


def test_aggregate_is_all_ranks_bytes_over_the_slowest_time():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate_gbs(4, 512 * 2 ** 20, 10, 2.0) == pytest.approx(4 * 512 * 2 ** 20 * 10 / 2.0 / 1e9)
