"""The N > 1 path of bench.py on the CPU: two gloo ranks shard each workload (no collective on
the data path) and combine their timings with the max / sum reductions the GPU runs use. Every
simulation must land on exactly one rank, and the reductions must see both ranks."""
import datetime
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


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    uneven = [s["seed"] for s in bench.uneven_sims(96)[rank::world]]
    sweep = [int(t) for t in bench.sweep_descs(49, 2, (2, 3), rank, world)["tag"]]
    serve = [float(t) for t, _ in bench.serve_requests(9, 200.0)[rank::world]]
    mx = bench.max_over_ranks(dist, None, float(rank + 1))
    sm = bench.sum_over_ranks(dist, None, float(len(uneven)))
    out.put((rank, uneven, sweep, serve, mx, sm))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_ranks_shard_without_overlap():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=150) for _ in range(world))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    import sys

    sys.path.insert(0, ROOT)
    import bench

    all_uneven = [s["seed"] for s in bench.uneven_sims(96)]
    assert sorted(res[0][1] + res[1][1]) == sorted(all_uneven)
    assert not set(res[0][1]) & set(res[1][1])
    all_sweep = [int(t) for t in bench.sweep_descs(49, 2, (2, 3))["tag"]]
    assert sorted(res[0][2] + res[1][2]) == sorted(all_sweep)
    assert len(res[0][3]) + len(res[1][3]) == 9
    for r in res:
        assert r[4] == 2.0                      # max over ranks
        assert r[5] == len(all_uneven)          # sum over ranks
