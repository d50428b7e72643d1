#!/usr/bin/env python
"""bench.py -- throughput of the B200 CA stepping path on the reference's headline workloads.

Default workload (one GPU): a 512^3 grid, Moore-26 neighbourhood, C = 16 states (maxCellState
15), survive {4,5}, birth {5}, 40% of the whole volume seeded alive by the reference's cell
hash (seed 0), 1000 ticks with statistics every tick. One "step" is one full 1000-tick run
through the C ABI (cave_run: nibble layout in HBM -> bit-plane layout -> 1000 tick launches ->
back). `value` is cell-updates/s with the grid already resident in HBM; `e2e` is the same
through cave_run_host with the grid read from and written back to pinned host memory.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl reference]

Under torchrun (N > 1) every rank runs an independent replica (a single grid does not shard
without a halo exchange the reference does not do in search mode); value = all ranks' cell
updates / max over ranks of the device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (edge, ticks)
    "large512": (512, 1000),
    "large256": (256, 1000),
    "large1024": (1024, 200),
    "sweep49": (49, 20),
    "uneven2048": (0, 0),
    "serve": (0, 0),
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="large512")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ticks", type=int, default=0, help="override the workload's tick count (profiling runs)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: mean request arrivals per second")
    ap.add_argument("--requests", type=int, default=64, help="serve: requests in the timed window")
    ap.add_argument("--sims", type=int, default=2048, help="uneven2048: simulations in the batch")
    ap.add_argument("--stride", type=int, default=1,
                    help="sweep49: run every n-th simulation of the sweep (small profiling runs)")
    ap.add_argument("--no-autotune", action="store_true")
    return ap.parse_args()


# ----------------------------------------------------------------------------- helpers
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for i, n in enumerate(names):
                    if r[5 + i].strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        os.unlink(self.f.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_profile_value(kernel_key, name):
    """A `name: value` line of the committed ncu summary profiles/<kernel_key>.md (or None)."""
    p = os.path.join(ROOT, "profiles", f"{kernel_key}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(name + ":"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def committed_traffic(kernel_key):
    """DRAM bytes per launch from the committed ncu summary (profiles/<kernel_key>.md)."""
    return committed_profile_value(kernel_key, "traffic_bytes_per_launch")


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def barrier(pg, local):
    import torch

    torch.cuda.synchronize(local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(local)


def _reduce(pg, local, v, op):
    """All-reduce of one float over the ranks (no-op without a process group). local = None
    reduces on the CPU (gloo), else on cuda:local (nccl)."""
    if not pg:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device="cpu" if local is None else f"cuda:{local}")
    pg.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(pg, local, v):
    return _reduce(pg, local, v, pg.ReduceOp.MAX if pg else None)


def sum_over_ranks(pg, local, v):
    return _reduce(pg, local, v, pg.ReduceOp.SUM if pg else None)


# ----------------------------------------------------------------------------- CPU baseline
def cpu_baseline_large(G, init, params, budget_s=12.0):
    """The oracle's OpenMP step (bit-identical to the literal restatement) on the same grid."""
    import oracle as O

    cores = os.cpu_count() or 1
    cells = init
    t0 = time.perf_counter()
    ticks = 0
    while True:
        cells, _ = O.step_fast(G, G, G, params, cells, nthreads=cores)
        ticks += 1
        el = time.perf_counter() - t0
        if el > budget_s or ticks >= 50:
            break
    return {"value": G ** 3 * ticks / el, "unit": "cell-updates/s", "cores": cores, "kind": "port",
            "sample": f"{ticks} ticks of the {G}^3 grid (of {WORKLOADS.get(f'large{G}', (G, 0))[1]}), oracle "
                      f"OpenMP z-slab step, {el:.1f} s"}


# ----------------------------------------------------------------------------- workloads
def large_workload(args, world, rank, local, pg):
    import numpy as np
    import torch

    import cave_b200 as cb

    G, T = WORKLOADS[args.workload]
    T = args.ticks or T
    cells_per_step = G ** 3 * T
    thr = cb.threshold_from_fill(0.40)
    params = cb.make_params(15, 0x7, 0x10, 0x18)
    ctx = cb.Context(local)
    ctx.set_timing(True)
    g = cb.Grid(ctx, G, G, G)
    g.seed_threshold((G, G, G), thr, 0, 15)
    init_host = g.download()
    words = init_host.size
    pin_in = torch.from_numpy(init_host.view(np.int32)).pin_memory()
    pin_out = torch.empty(words, dtype=torch.int32).pin_memory()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device=f"cuda:{local}")  # 256 MiB > L2

    def reset():
        g.upload(init_host)
        flush.zero_()
        torch.cuda.synchronize(local)

    # the tick kernel compiled for this rule (NVRTC, cached), unless CAVE_JIT=off
    t_prep = time.perf_counter()
    ctx.prepare_rule(params)
    prep_s = time.perf_counter() - t_prep
    for _ in range(args.warmup):
        reset()
        g.run(params, T, T, stats=True)
    barrier(pg, local)
    dev_ms, tick_ms, conv_ms, launches = [], [], [], 0
    _, jit0 = cb.jit_stats()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            reset()
            g.run(params, T, T, stats=True)
            t = ctx.last_timing()
            dev_ms.append(t.total_ms)
            tick_ms.append(t.tick_ms)
            conv_ms.append(t.convert_ms)
            launches += t.launches
        barrier(pg, local)
    clocks = clk.summary()
    _, jit1 = cb.jit_stats()
    specialised = jit1 - jit0 == T * args.steps
    # end-to-end through the C ABI with host buffers
    e2e_ms = []
    for i in range(0 if args.no_e2e else args.steps + 1):
        flush.zero_()
        torch.cuda.synchronize(local)
        g.run_host(pin_in.data_ptr(), pin_out.data_ptr(), params, T, T, stats=True)
        if i > 0:
            e2e_ms.append(ctx.last_timing().total_ms)
    barrier(pg, local)

    tot_dev = max_over_ranks(pg, local, sum(dev_ms))
    tot_e2e = max_over_ranks(pg, local, sum(e2e_ms)) if e2e_ms else float("nan")
    tot_tick = max_over_ranks(pg, local, sum(tick_ms))
    value = world * cells_per_step * args.steps / (tot_dev / 1e3)
    e2e_value = world * cells_per_step * args.steps / (tot_e2e / 1e3)
    per_launch_s = (tot_tick / 1e3) / (T * args.steps)
    alg_bytes = G ** 3  # 1 byte per cell update: 0.5 B read + 0.5 B written
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / per_launch_s / 1e9
    traffic = committed_traffic(f"stream_tick_{G}")
    line = {
        "metric": "cell-updates/s",
        "value": value,
        "unit": "cell-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": tot_dev / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u4 (packed nibble states, bit-sliced integer logic)",
        "data": "synthetic: reference cell hash (searchSystem.cpp:244-262), seed 0, 40% fill of the whole volume",
        "config": {"workload": f"{G}^3 Moore-26, C=16 (maxCellState 15), survive {{4,5}} birth {{5}}, "
                               f"{T} ticks, stats every tick", "grid": [G, G, G], "ticks": T,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "256 MiB buffer written between timed steps (a step is one whole run; within a run each "
                         "tick reads the previous tick's output)",
                   "tick_kernel": ("compiled for the rule at run time (NVRTC, cached; cave_prepare_rule took "
                                   f"{prep_s:.2f} s before the warm-up)") if specialised else
                                  "generic (rule read at run time)"},
        "tick_kernel_us": per_launch_s * 1e6,
        "convert_ms_per_step": sum(conv_ms) / len(conv_ms),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": traffic,
                     "note": "algorithmic bytes = 1 B per cell update (packed 4-bit state read once, written once)"},
        "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": int(words * 4),
                "d2h_bytes_per_step": int(words * 4 + T * 48)},
        "gpu_launches": int(sum_over_ranks(pg, local, launches)),
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        params_np = np.array([params.birthAndMaxCellStateRules, params.survivalAndNeighborhoodRules, 0],
                             dtype=np.uint64)
        line["cpu_baseline"] = cpu_baseline_large(G, init_host, params_np)
    g.close()
    ctx.close()
    return line


def sweep_descs(G, seeds, cs_values, rank=0, world=1, stride=1):
    """The config-3 sweep: FE neighbourhood, every survive/birth set with <= 2 bits (171 each),
    C in cs_values (maxCellState = C - 1), `seeds` seeds; sims of this rank's shard."""
    import numpy as np

    import cave_b200 as cb

    n_masks = 171
    per = n_masks * n_masks
    idx = np.arange(per, dtype=np.int64)
    si, bi = idx // n_masks, idx % n_masks
    parts = []
    init_ix = 0
    for c in cs_values:
        mcs = c - 1
        for s in range(seeds):
            d = np.zeros(per, dtype=cb.SIM_DESC_DTYPE)
            d["birth"] = (np.uint64((mcs - 1) & 0xF) << np.uint64(60)) | (bi + 1).astype(np.uint64)
            d["survival"] = (np.uint64(3) << np.uint64(60)) | (si + 1).astype(np.uint64)
            d["init"] = init_ix
            d["maxTicks"] = 20
            parts.append(d)
            init_ix += 1
    allv = np.concatenate(parts)
    allv["tag"] = np.arange(allv.size, dtype=np.uint32)
    mine = allv[rank::world]
    return np.ascontiguousarray(mine[::stride])


def sweep_workload(args, world, rank, local, pg):
    import numpy as np

    import cave_b200 as cb

    G, T = WORKLOADS["sweep49"]
    seeds, cs_values = 32, (2, 3, 4, 5)
    thr = cb.threshold_from_fill(0.30)
    ctx = cb.Context(local)
    ctx.set_timing(True)
    vb = cb.valid_bitmasks(18, 2)

    def make_batch():
        b = cb.Batch(ctx)
        for c in cs_values:
            for s in range(seeds):
                b.add_init_seeded(G, G, G, (16, 16, 16), thr, s, c - 1)
        b.add_table(vb)
        return b

    full = sweep_descs(G, seeds, cs_values, rank, world)
    if args.stride > 1:
        full = np.ascontiguousarray(full[::args.stride])
    warm = np.ascontiguousarray(full[::32])
    for _ in range(args.warmup):
        with make_batch() as b:
            b.add_sims_array(warm, max_rule_bits=2)
            b.launch()
            b.results_array()
    barrier(pg, local)
    kern_ms, tot_ms, wall, cats, ticks, launches = [], [], [], None, 0, 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            with make_batch() as b:
                t0 = time.perf_counter()
                b.add_sims_array(full, max_rule_bits=2)
                b.launch()
                res = b.results_array()
                wall.append(time.perf_counter() - t0)
                t = ctx.last_timing()
                kern_ms.append(t.tick_ms)
                tot_ms.append(t.total_ms)
                launches += t.launches
            cats = np.bincount(res["category"], minlength=3)
            ticks = int(res["info"][:, 2].sum())
        barrier(pg, local)
    clocks = clk.summary()
    n_all = sum_over_ranks(pg, local, float(full.size))
    kern = max_over_ranks(pg, local, sum(kern_ms) / len(kern_ms))
    tot = max_over_ranks(pg, local, sum(tot_ms) / len(tot_ms))
    sims_s = n_all / (kern / 1e3)
    # plain per-simulation path on a stride sample of the same sweep (rank 0)
    plain = {}
    if rank == 0:
        sample = sweep_descs(G, seeds, cs_values, stride=997)
        best = None
        for slots in (6, 64, 256):
            with make_batch() as b:
                b.add_sims_array(sample, max_rule_bits=2)
                dev_s = b.run_plain(slots)
                r = b.results_array()
            v = sample.size / dev_s
            plain[f"slots{slots}_sims_per_s"] = v
            best = v if best is None else max(best, v)
        plain["best_sims_per_s"] = best
        plain["sample"] = f"{sample.size} simulations (every 997th of the sweep)"
    line = {
        "metric": "search sims/s", "value": sims_s, "unit": "sims/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": kern, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "u4 (packed nibble states, bit-sliced integer logic)",
        "data": "synthetic: reference cell hash, 30% fill of a centred 16^3 box, seeds 0..31",
        "config": {"workload": f"49^3 FE sweep: 171 x 171 rules (<= 2 bits) x C in {{2,3,4,5}} x 32 seeds, "
                               f"{T} ticks with early stop"
                               + (f", every {args.stride}th simulation" if args.stride > 1 else ""),
                   "simulations": int(n_all),
                   "parallelism": f"shards x{world}" if world > 1 else "single GPU",
                   "l2": "grids resident in shared memory; initial grids read once per simulation"},
        "cell_updates_per_s": ticks * G ** 3 * world / (kern / 1e3),
        "categories": {"viable": int(cats[0]), "possible": int(cats[1]), "unviable": int(cats[2])},
        "plain_path": plain,
        "batched_over_plain": (sims_s / plain["best_sims_per_s"]) if plain else None,
        "e2e": {"value": n_all / (tot / 1e3), "unit": "sims/s", "h2d_bytes_per_step": int(full.size * 16),
                "d2h_bytes_per_step": int(full.size * cb.SIM_RESULT_DTYPE.itemsize)},
        "gpu_launches": int(sum_over_ranks(pg, local, launches)),
        "clocks": clocks,
        # grids stay in shared memory, so the bound is integer issue: utilisation from the
        # committed ncu capture of this workload (not measured live)
        "int_issue": {"issue_active_frac": committed_profile_value("resident_sweep49", "issue_active_frac"),
                      "alu_pipe_frac": committed_profile_value("resident_sweep49", "alu_pipe_frac"),
                      "source": "ncu --set full, profiles/resident_sweep49.md"},
    }
    ctx.close()
    return line



# ----------------------------------------------------------------------------- config 4 / 5 inputs
NB_COUNT = {0x1: 6, 0x3: 18, 0x7: 26}


def _rule_bits(g, n):
    """1..4 distinct neighbour counts among 1..n as a reference rule mask (bit c-1 = count c)."""
    k = int(g.integers(1, 5))
    return sum(1 << int(c) for c in g.choice(n, size=k, replace=False))


def uneven_sims(n, seed=20261203):
    """The uneven-size batch: per simulation, in this draw order, edge from {33,49,65,97,129,193},
    neighbourhood from {F, FE, Moore}, C from 2..16 (maxCellState C-1), survival and birth sets
    of 1-4 counts, ticks from 10..500 and fill from [0.20, 0.50); spawn = the whole grid, seed =
    the simulation index. numpy Generator over MT19937(seed)."""
    g = np.random.Generator(np.random.MT19937(seed))
    edges, flags = (33, 49, 65, 97, 129, 193), (0x1, 0x3, 0x7)
    out = []
    for i in range(n):
        e = edges[int(g.integers(6))]
        fl = flags[int(g.integers(3))]
        C = int(g.integers(2, 17))
        S = _rule_bits(g, NB_COUNT[fl])
        B = _rule_bits(g, NB_COUNT[fl])
        T = int(g.integers(10, 501))
        p = float(g.uniform(0.20, 0.50))
        out.append(dict(edge=e, flags=fl, maxcs=C - 1, birth=B, survival=S, ticks=T, fill=p, seed=i))
    return out


def uneven_workload(args, world, rank, local, pg):
    import cave_b200 as cb

    sims = uneven_sims(args.sims)
    mine = sims[rank::world]
    ctx = cb.Context(local)
    ctx.set_timing(True)

    def make_batch(subset, autotune):
        b = cb.Batch(ctx)
        b.set_options(autotune=autotune)
        descs = []
        for j, s in enumerate(subset):
            ix = b.add_init_seeded(s["edge"], s["edge"], s["edge"], (s["edge"],) * 3, cb.threshold_from_fill(s["fill"]),
                                   s["seed"], s["maxcs"])
            descs.append(cb.SimDesc(cb.make_params(s["maxcs"], s["flags"], s["birth"], s["survival"]), ix, s["ticks"], 0,
                                    j))
        b.add_sims(descs)
        return b

    autotune = not args.no_autotune
    tune_ms = 0.0
    t0 = time.perf_counter()
    for _ in range(args.warmup):
        with make_batch(mine, autotune) as b:
            b.launch()
            b.results_array()
            plan = b.plan()
    tune_wall = time.perf_counter() - t0
    barrier(pg, local)
    kern_ms, tot_ms, wall = [], [], []
    updates, launches = 0, 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            with make_batch(mine, autotune) as b:
                w0 = time.perf_counter()
                b.launch()
                res = b.results_array()
                wall.append(time.perf_counter() - w0)
                t = ctx.last_timing()
                kern_ms.append(t.tick_ms)
                tot_ms.append(t.total_ms)
                launches += t.launches
                plan = b.plan()
            vol = np.array([s["edge"] ** 3 for s in mine], dtype=np.int64)
            updates = int((res["info"][:, 2].astype(np.int64) * vol).sum())
            assert int(res["error"].max(initial=0)) == 0
        barrier(pg, local)
    clocks = clk.summary()
    kern = max_over_ranks(pg, local, sum(kern_ms) / len(kern_ms))
    tot = max_over_ranks(pg, local, sum(tot_ms) / len(tot_ms))
    n_all = sum_over_ranks(pg, local, float(len(mine)))
    upd_all = sum_over_ranks(pg, local, float(updates))
    # the plain per-simulation path (one launch per slot per tick, a host fence per tick) and
    # the batched path on the same sample (every 64th simulation)
    plain = {}
    if rank == 0:
        sample = sims[::64]
        vol_s = np.array([s["edge"] ** 3 for s in sample], dtype=np.int64)
        with make_batch(sample, autotune) as b:
            dev_s = b.run_plain(len(sample))
            r = b.results_array()
        upd_s = int((r["info"][:, 2].astype(np.int64) * vol_s).sum())
        with make_batch(sample, autotune) as b:
            b.launch()
            rb = b.results_array()
            tb = ctx.last_timing().tick_ms / 1e3
        assert np.array_equal(rb["info"], r["info"]), "plain and batched paths disagree"
        plain = {"sample": f"{len(sample)} simulations (every 64th)", "plain_sims_per_s": len(sample) / dev_s,
                 "plain_cell_updates_per_s": upd_s / dev_s, "batched_sims_per_s_same_sample": len(sample) / tb,
                 "batched_cell_updates_per_s_same_sample": upd_s / tb, "batched_over_plain_same_sample": dev_s / tb}
    line = {
        "metric": "search sims/s", "value": n_all / (kern / 1e3), "unit": "sims/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": kern, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "u4 (packed nibble states, bit-sliced integer logic)",
        "data": "synthetic: reference cell hash, 20-50% fill of the whole grid, seeds 0..2047",
        "config": {"workload": f"uneven batch: {len(sims)} simulations, edges {{33,49,65,97,129,193}}, F/FE/Moore, "
                               f"C 2..16, 1-4 counts per set, 10-500 ticks with early stop",
                   "simulations": int(n_all), "autotune": autotune,
                   "parallelism": f"shards x{world}" if world > 1 else "single GPU",
                   "l2": "grids up to 65^3 resident in shared memory; larger grids in HBM (two copies each)"},
        "cell_updates_per_s": upd_all / (kern / 1e3),
        "plan": plan,
        "autotune_and_warmup_wall_s": tune_wall,
        "plain_path": plain,
        "e2e": {"value": n_all / (tot / 1e3), "unit": "sims/s", "h2d_bytes_per_step": int(len(mine) * 40),
                "d2h_bytes_per_step": int(len(mine) * cb.SIM_RESULT_DTYPE.itemsize)},
        "host_wall_s_per_step": sum(wall) / len(wall),
        "gpu_launches": int(sum_over_ranks(pg, local, launches)),
        "clocks": clocks,
    }
    ctx.close()
    return line


def serve_requests(n, rate, seed=20261204):
    """Request stream: Poisson arrivals (mean `rate`/s); each request 1-256 simulations with
    edge 32..256, ticks 10..500 and rules / fills as the uneven batch; spawn = whole grid."""
    import cave_b200 as cb

    g = np.random.Generator(np.random.MT19937(seed))
    t, out = 0.0, []
    flags = (0x1, 0x3, 0x7)
    sid = 0
    for _ in range(n):
        t += float(g.exponential(1.0 / rate))
        k = int(g.integers(1, 257))
        r = cb.request_sims(k)
        for i in range(k):
            e = int(g.integers(32, 257))
            fl = flags[int(g.integers(3))]
            C = int(g.integers(2, 17))
            S = _rule_bits(g, NB_COUNT[fl])
            B = _rule_bits(g, NB_COUNT[fl])
            p = cb.make_params(C - 1, fl, B, S)
            r[i]["X"] = r[i]["Y"] = r[i]["Z"] = e
            r[i]["maxTicks"] = int(g.integers(10, 501))
            r[i]["birth"], r[i]["survival"] = p.birthAndMaxCellStateRules, p.survivalAndNeighborhoodRules
            r[i]["spawnX"] = r[i]["spawnY"] = r[i]["spawnZ"] = e
            r[i]["runSeedIndex"] = sid
            r[i]["threshold"] = cb.threshold_from_fill(float(g.uniform(0.20, 0.50)))
            r[i]["tag"] = i
            sid += 1
        out.append((t, r))
    return out


def serve_workload(args, world, rank, local, pg):
    import cave_b200 as cb

    reqs = serve_requests(args.requests, args.rate)[rank::world]
    ctx = cb.Context(local)
    budget = 120 * 10 ** 9
    total_sims = sum(r.size for _, r in reqs)

    def run(srv, timed_arrivals):
        ids, lat = {}, []
        t0 = time.perf_counter()
        for t_arr, r in reqs:
            if timed_arrivals:
                d = t_arr - (time.perf_counter() - t0)
                if d > 0:
                    time.sleep(d)
            ids[srv.submit(r)] = r.size
        done = 0
        upd = 0
        while done < len(ids):
            for rid in srv.poll():
                res, l = srv.fetch(rid)
                assert int(res["error"].max(initial=0)) == 0
                lat.append(l)
                done += 1
            time.sleep(0.0005)
        span = time.perf_counter() - t0
        st = srv.stats()
        return span, sorted(lat), st

    with cb.Server(ctx, hbm_budget=budget, autotune=False) as srv:
        warm = serve_requests(2, args.rate, seed=7)
        for _, r in warm:
            srv.wait(srv.submit(r), 600.0)
        for rid in srv.poll():
            pass
    with cb.Server(ctx, hbm_budget=budget) as srv, ClockSampler(local) as clk:
        span_served, lat, st_served = run(srv, True)
    clocks = clk.summary()
    with cb.Server(ctx, hbm_budget=budget) as srv:
        span_off, _, st_off = run(srv, False)

    def pct(p):
        return lat[min(len(lat) - 1, int(p * (len(lat) - 1) + 0.5))] if lat else None

    served_ups = st_served.cellUpdates / span_served
    off_ups = st_off.cellUpdates / span_off
    arrival_span = reqs[-1][0] if reqs else 0.0
    line = {
        "metric": "served cell-updates/s", "value": served_ups, "unit": "cell-updates/s", "n_gpus": world,
        "steps": 1, "warmup": 1, "ms_per_step": span_served * 1e3, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "u4 (packed nibble states, bit-sliced integer logic)",
        "data": "synthetic: Poisson request stream, reference cell hash seeding",
        "config": {"workload": f"served: {len(reqs)} requests, Poisson {args.rate}/s, 1-256 sims each, edge 32..256, "
                               f"ticks 10..500, F/FE/Moore, C 2..16", "requests": len(reqs), "simulations": total_sims,
                   "hbm_budget_bytes": budget, "arrival_window_s": arrival_span},
        "latency_p50_s": pct(0.50), "latency_p99_s": pct(0.99),
        "server_p50_s": st_served.p50LatencySeconds, "server_p99_s": st_served.p99LatencySeconds,
        "offline_cell_updates_per_s": off_ups, "throughput_loss_vs_offline": 1.0 - served_ups / off_ups,
        "served_span_s": span_served, "offline_span_s": span_off, "peak_hbm_bytes": st_served.peakBytes,
        "tick_launches": st_served.tickLaunches, "resident_launches": st_served.residentLaunches,
        "rounds": st_served.rounds,
        "gpu_launches": int(st_served.tickLaunches + st_served.residentLaunches + st_served.rounds),
        "clocks": clocks,
        "e2e": {"value": served_ups, "unit": "cell-updates/s", "h2d_bytes_per_step": int(total_sims * 72),
                "d2h_bytes_per_step": int(total_sims * cb.SIM_RESULT_DTYPE.itemsize)},
    }
    ctx.close()
    return line


def reference_arm(args, world, rank, local, pg):
    """The oracle port of the reference's CPU-free arithmetic on the host cores (no CPU stepping
    exists in the reference; its GPU path needs Vulkan, which this box does not have)."""
    import oracle as O

    if rank != 0:
        return None
    G, T = WORKLOADS[args.workload]
    params = O.make_params(15, 0x7, 0x10, 0x18)
    init = O.seed(G, G, G, random=True, threshold=O.threshold_from_float(0.40), run_seed=0, max_cell_state=15)
    cores = os.cpu_count() or 1
    ticks_per_step = 1
    cells = init
    for _ in range(args.warmup):
        cells, _ = O.step_fast(G, G, G, params, cells, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps * ticks_per_step):
        cells, _ = O.step_fast(G, G, G, params, cells, nthreads=cores)
    el = time.perf_counter() - t0
    v = G ** 3 * args.steps * ticks_per_step / el
    return {
        "impl": "reference", "metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u4", "data": "synthetic (same seed and fill)",
        "config": {"workload": f"{G}^3 Moore-26, C=16, survive {{4,5}} birth {{5}}; one tick per step "
                               f"(bounded sample of the {T}-tick run)", "grid": [G, G, G]},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": "port",
                         "sample": f"{args.steps} ticks of {G}^3 after {args.warmup} warm-up ticks"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse_args()
    if args.impl == "reference":
        # rank 0 alone runs the CPU arm; other ranks exit without work (no process group).
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        line = reference_arm(args, world, rank, 0, None)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
        return
    world, rank, local, pg = dist_setup(args)
    if args.workload == "sweep49":
        line = sweep_workload(args, world, rank, local, pg)
    elif args.workload == "uneven2048":
        line = uneven_workload(args, world, rank, local, pg)
    elif args.workload == "serve":
        line = serve_workload(args, world, rank, local, pg)
    else:
        line = large_workload(args, world, rank, local, pg)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
