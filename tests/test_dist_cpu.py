"""The N > 1 path of bench.py on the CPU: two gloo ranks run its process
group set-up, barrier and max-over-ranks timing, and the whole-job value
is every rank's work over the slowest rank's time."""
import os
import pathlib
import socket
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    r, w, _ = bench.dist_setup(world, backend="gloo")
    bench.barrier(w)
    ms = 100.0 + 50.0 * r                    # rank 1 is the slow one
    slowest = bench.max_over_ranks(ms, w)
    out.put((r, w, slowest, bench.job_value(1_000_000, slowest, w)))
    import torch.distributed as dist
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1]
    for _, w, slowest, value in got:
        assert w == 2 and slowest == pytest.approx(150.0)
        assert value == pytest.approx(2 * 1_000_000 / 0.150)
