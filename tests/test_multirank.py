"""The N > 1 path of bench.py on the CPU: two and three gloo ranks shard each workload (no collective on
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
@pytest.mark.parametrize("world", [2, 3])
def test_ranks_shard_without_overlap(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
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
    got_uneven = [v for r in res for v in r[1]]
    assert sorted(got_uneven) == sorted(all_uneven) and len(set(got_uneven)) == len(got_uneven)
    all_sweep = [int(t) for t in bench.sweep_descs(49, 2, (2, 3))["tag"]]
    got_sweep = [v for r in res for v in r[2]]
    assert sorted(got_sweep) == sorted(all_sweep) and len(set(got_sweep)) == len(got_sweep)
    assert sum(len(r[3]) for r in res) == 9
    for r in res:
        assert r[4] == float(world)             # max over ranks
        assert r[5] == len(all_uneven)          # sum over ranks
