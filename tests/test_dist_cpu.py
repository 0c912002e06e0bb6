"""The N > 1 path of bench.py on the CPU: two gloo ranks run its process
group set-up, barrier, max-over-ranks timing and sum-over-ranks counts; the
whole-job value is every rank's work over the slowest rank's time; the
batched workload's maps are dealt whole to the ranks (disjoint shares that
cover the batch, largest first), and each rank's stage map is its own."""
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
    total = bench.sum_over_ranks(1000.0 + r, w)
    from hl2sdk_tools_sharp_b200 import roomgrid as rg
    cfgs = [rg.config_batch(i, seed=bench.CONFIG_SEED) for i in range(32)]
    share = bench.deal_maps([c.side ** 2 for c in cfgs], w)[r]
    seed_map = bench.world_for(3, bench.CONFIG_SEED + r).light_origin.tolist()
    out.put((r, w, slowest, bench.job_value(1_000_000, slowest, w), total, share, seed_map))
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
    for _, w, slowest, value, total, _, _ in got:
        assert w == 2 and slowest == pytest.approx(150.0)
        assert value == pytest.approx(2 * 1_000_000 / 0.150)
        assert total == 2001.0
    a, b = got[0][5], got[1][5]
    assert not set(a) & set(b) and sorted(a + b) == list(range(32))
    assert got[0][6] != got[1][6]                  # each rank lights a map of its own


def test_deal_maps_is_largest_first_and_balanced():
    sys.path.insert(0, str(ROOT))
    import bench
    w = [100, 4, 81, 9, 64, 36, 49, 25]
    shares = bench.deal_maps(w, 3)
    assert sorted(i for s in shares for i in s) == list(range(8))
    loads = [sum(w[i] for i in s) for s in shares]
    assert max(loads) - min(loads) <= max(w[i] for s in shares for i in s[-1:])
    assert shares[0][0] == 0 and shares[1][0] == 2 and shares[2][0] == 4   # the three largest, one each
    assert bench.deal_maps(w, 1) == [sorted(range(8), key=lambda k: -w[k])]
