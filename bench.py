#!/usr/bin/env python
"""bench.py -- throughput of the B200 CA stepping path on the reference's headline workloads.

Default line (one GPU): a 512^3 grid, Moore-26 neighbourhood, C = 16 states (maxCellState 15),
survive {4,5}, birth {5}, 40% of the whole volume seeded alive by the reference's cell hash
(seed 0), 1000 ticks with statistics every tick. One "step" is one full 1000-tick run through
the C ABI (cave_run: nibble layout in HBM -> bit-plane layout -> tick launches -> back).
`value` is cell-updates/s with the grid already resident in HBM; `e2e` is the same through
cave_run_host with the grid read from and written back to pinned host memory. The last timed
run and the last end-to-end run are checked against the oracle fixture
(tests/golden/large_fixtures.json): every cell, every tick's statistics and the GridInfo.

The default line also carries `extra`: the other workloads, each timed on the device, checked
against its oracle fixture where one exists, with its CPU baseline and clocks:
  plain49     the plain single simulation (49^3 FE, C=4, 20 ticks): plain, streaming and
              resident paths
  large256    256^3, same rule as the default, 1000 ticks (L2-resident ping-pong)
  large1024   1024^3, 200 ticks (out of L2)
  sweep49     the batched search sweep (3,742,848 simulations of 49^3) vs the plain path
  uneven2048  the uneven-size batch with the autotuner vs the plain path
  serve       the served request stream at 200 requests/s (overload) and 16 requests/s

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl reference]

Under torchrun (N > 1) every rank runs an independent replica of the large grids (a single
grid does not shard without a halo exchange the reference does not do in search mode) and a
shard of the simulation workloads; value = all ranks' work / max over ranks of the device time.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import platform
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")

WORKLOADS = {
    # name: (edge, ticks)
    "large512": (512, 1000),
    "large256": (256, 1000),
    "large1024": (1024, 200),
    "plain49": (49, 20),
    "sweep49": (49, 20),
    "uneven2048": (0, 0),
    "serve": (0, 0),
}
LARGE_RULE = (15, 0x7, 1 << 4, (1 << 3) | (1 << 4))  # maxCellState, flags, birth, survival
PLAIN_RULE = (3, 0x3, 0x60, 0x70)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="large512")
    ap.add_argument("--no-extra", action="store_true", help="default line only (no other workloads)")
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


def fixture(name):
    p = os.path.join(GOLDEN, name)
    return json.load(open(p)) if os.path.exists(p) else {}


def sha256_u32(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).astype("<u4").tobytes()).hexdigest()


class ParityError(AssertionError):
    pass


def require(ok, what):
    if not ok:
        raise ParityError(f"parity check failed: {what}")


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


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


# ----------------------------------------------------------------------------- CPU baselines
# The oracle (oracle/, test infrastructure) is the CPU restatement of the reference's shader
# arithmetic; the reference itself has no CPU stepping. Only these functions load it.
def _oracle_params(rule):
    import oracle as O

    return O.make_params(*rule)


def cpu_baseline_grid(G, init, rule, ticks_full, budget_s=10.0, single=True, spawn=None):
    """The oracle's OpenMP z-slab step on the same grid, all host cores, then one thread."""
    import oracle as O

    params = _oracle_params(rule)
    cores = os.cpu_count() or 1

    def rate(nthreads, budget, most):
        cells, ticks, t0 = init, 0, time.perf_counter()
        while True:
            cells, _ = O.step_fast(G, G, G, params, cells, nthreads=nthreads)
            ticks += 1
            el = time.perf_counter() - t0
            if el > budget or ticks >= most:
                return G ** 3 * ticks / el, ticks, el

    v, n, el = rate(cores, budget_s, 50)
    out = {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": "port", "cpu_model": cpu_model(),
           "sample": f"{n} ticks of the {G}^3 grid (of {ticks_full}), oracle OpenMP z-slab step on {cores} threads, "
                     f"{el:.1f} s"}
    if single:
        v1, n1, el1 = rate(1, budget_s / 3, 20)
        out["single_thread"] = {"value": v1, "unit": "cell-updates/s",
                                "sample": f"{n1} ticks, 1 thread, {el1:.1f} s"}
    return out


def _pool_init():
    os.environ["OMP_NUM_THREADS"] = "1"


def _cpu_sweep_sim(a):
    """One sweep simulation on one host thread (oracle): (ticks run, cells per tick)."""
    import oracle as O

    mcs, s, si, bi = a
    init = O.seed(49, 49, 49, spawn=(16, 16, 16), random=True, threshold=O.threshold_from_float(0.30), run_seed=s,
                  max_cell_state=mcs)
    info, _, _ = O.run_sim(49, 49, 49, O.make_params(mcs, 0x3, bi + 1, si + 1), init, 20,
                           valid=O.valid_bitmasks(18, 2), max_rule_bits=2, fast=True)
    return info.ticks, 49 ** 3


def _cpu_uneven_sim(s):
    import oracle as O

    e = s["edge"]
    init = O.seed(e, e, e, random=True, threshold=O.threshold_from_float(s["fill"]), run_seed=s["seed"],
                  max_cell_state=s["maxcs"])
    info, _, _ = O.run_sim(e, e, e, O.make_params(s["maxcs"], s["flags"], s["birth"], s["survival"]), init,
                           s["ticks"], fast=True)
    return info.ticks, e ** 3


def cpu_baseline_sims(fn, items, what):
    """A sample of simulations run by the oracle, one per host thread over all cores (a spawn
    process pool: safe after CUDA is initialised), then the first few on one thread."""
    from multiprocessing import get_context

    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    with get_context("spawn").Pool(cores, initializer=_pool_init) as pool:
        t1 = time.perf_counter()
        res = pool.map(fn, items, chunksize=1)
        el = time.perf_counter() - t1
    updates = sum(t * v for t, v in res)
    one = items[:max(1, len(items) // (4 * cores))]
    _pool_init()
    t2 = time.perf_counter()
    r1 = [fn(x) for x in one]
    el1 = time.perf_counter() - t2
    return {"value": len(items) / el, "unit": "sims/s", "cell_updates_per_s": updates / el, "cores": cores,
            "kind": "port", "cpu_model": cpu_model(),
            "sample": f"{len(items)} simulations ({what}), oracle, one simulation per thread on {cores} threads, "
                      f"{el:.1f} s (pool start {t1 - t0:.1f} s not counted)",
            "single_thread": {"value": len(one) / el1, "unit": "sims/s",
                              "cell_updates_per_s": sum(t * v for t, v in r1) / el1,
                              "sample": f"first {len(one)} of them on 1 thread, {el1:.1f} s"}}


# ----------------------------------------------------------------------------- large grids
def large_workload(args, world, rank, local, pg, G, T, steps, warmup, e2e=True, cpu=True):
    import torch

    import cave_b200 as cb

    cells_per_step = G ** 3 * T
    thr = cb.threshold_from_fill(0.40)
    params = cb.make_params(*LARGE_RULE)
    ctx = cb.Context(local)
    ctx.set_timing(True)
    g = cb.Grid(ctx, G, G, G)
    g.seed_threshold((G, G, G), thr, 0, 15)
    init_host = g.download()
    words = init_host.size
    fx = fixture("large_fixtures.json").get(str(G), {})
    want = fx.get("checkpoints", {}).get(str(T))
    if fx:
        require(sha256_u32(init_host) == fx["seed_sha256"], f"{G}^3 seeded cells")
    pin_in = torch.from_numpy(init_host.view(np.int32)).pin_memory()
    pin_out = torch.empty(words, dtype=torch.int32).pin_memory()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device=f"cuda:{local}")  # 256 MiB > L2

    def reset():
        g.upload(init_host)
        flush.zero_()
        torch.cuda.synchronize(local)

    def check(cells, ticks, info, what):
        if not want:
            return
        rec = cb.tick_records(ticks)
        require(hashlib.sha256(rec.tobytes()).hexdigest() == want["ticks_sha256"], f"{what}: per-tick statistics")
        require(list(info.as_tuple()) == want["gridinfo"], f"{what}: GridInfo")
        require(sha256_u32(cells) == want["cells_sha256"], f"{what}: cells")

    # the tick kernel compiled for this rule (NVRTC, cached), unless CAVE_JIT=off
    t_prep = time.perf_counter()
    ctx.prepare_rule(params)
    prep_s = time.perf_counter() - t_prep
    for _ in range(warmup):
        reset()
        g.run(params, T, T, stats=True)
    barrier(pg, local)
    dev_ms, tick_ms, conv_ms, launches = [], [], [], 0
    _, jit0 = cb.jit_stats()
    with ClockSampler(local) as clk:
        for _ in range(steps):
            reset()
            ticks, info = g.run(params, T, T, stats=True)
            t = ctx.last_timing()
            dev_ms.append(t.total_ms)
            tick_ms.append(t.tick_ms)
            conv_ms.append(t.convert_ms)
            launches += t.launches
        barrier(pg, local)
    clocks = clk.summary()
    _, jit1 = cb.jit_stats()
    specialised = jit1 - jit0 > 0
    pairs = specialised and launches <= steps * (T // 2 + 1 + 4)  # two ticks per launch (+ conversion/fold kernels)
    check(g.download(), ticks, info, f"{G}^3 x {T} ticks, device-resident run")
    # end-to-end through the C ABI with host buffers
    e2e_ms = []
    for i in range(steps + 1 if e2e else 0):
        flush.zero_()
        torch.cuda.synchronize(local)
        ticks, info = g.run_host(pin_in.data_ptr(), pin_out.data_ptr(), params, T, T, stats=True)
        if i > 0:
            e2e_ms.append(ctx.last_timing().total_ms)
    if e2e:
        check(pin_out.numpy().view(np.uint32), ticks, info, f"{G}^3 x {T} ticks, host-buffer run")
    barrier(pg, local)

    tot_dev = max_over_ranks(pg, local, sum(dev_ms))
    tot_e2e = max_over_ranks(pg, local, sum(e2e_ms)) if e2e_ms else float("nan")
    tot_tick = max_over_ranks(pg, local, sum(tick_ms))
    value = world * cells_per_step * steps / (tot_dev / 1e3)
    per_launch_s = (tot_tick / 1e3) / (T * steps)
    alg_bytes = G ** 3  # 1 byte per cell update: 0.5 B read + 0.5 B written
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / per_launch_s / 1e9
    line = {
        "metric": "cell-updates/s",
        "value": value,
        "unit": "cell-updates/s",
        "n_gpus": world,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": tot_dev / steps,
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
                                   f"{prep_s:.2f} s before the warm-up), "
                                   + ("two ticks per launch" if pairs else "one tick per launch"))
                                  if specialised else "generic (rule read at run time), one tick per launch"},
        "tick_kernel_us": per_launch_s * 1e6,
        "ticks_per_launch": 2 if pairs else 1,
        "convert_ms_per_step": sum(conv_ms) / len(conv_ms),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind,
                     # DRAM bytes per tick from the committed ncu summary of the kernel that ran
                     "traffic": (lambda t: t / 2 if (t is not None and pairs) else t)(
                         committed_traffic(f"stream_tick2_{G}" if pairs else f"stream_tick_{G}")),
                     "note": "algorithmic bytes = 1 B per cell update (packed 4-bit state read once, written once "
                             "per tick); achieved = G^3 B x ticks / tick-loop time (CUDA events on the library's "
                             "stream); traffic = ncu DRAM bytes (read + write) per tick of the same kernel"
                             + ("; two ticks per launch: the grid crosses HBM once per two ticks, so traffic is "
                                "about half the algorithmic bytes and the achieved rate may exceed the copy "
                                "bandwidth" if pairs else "")},
        "parity": ({"ok": True, "checked": f"last timed run{' and last end-to-end run' if e2e else ''}: every cell, "
                                          f"every tick's statistics and the GridInfo equal "
                                          f"tests/golden/large_fixtures.json ({G}^3, {T} ticks)"}
                   if want else {"ok": None, "checked": f"no oracle fixture for {G}^3 x {T} ticks"}),
        "gpu_launches": int(sum_over_ranks(pg, local, launches)),
        "clocks": clocks,
    }
    if e2e:
        line["e2e"] = {"value": world * cells_per_step * steps / (tot_e2e / 1e3), "unit": "cell-updates/s",
                       "h2d_bytes_per_step": int(words * 4), "d2h_bytes_per_step": int(words * 4 + T * 48)}
    if rank == 0 and world == 1 and cpu and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_grid(G, init_host, LARGE_RULE, T, single=G <= 512,
                                                 budget_s=10.0 if G <= 512 else 12.0)
    g.close()
    ctx.close()
    return line


# ----------------------------------------------------------------------------- config 1
def plain49_workload(args, world, rank, local, pg, steps, warmup):
    """The plain single simulation: 49^3, FE, C = 4, survive {5,6,7} birth {6,7}, 30% fill of
    the centred 16^3 box, seed 0, 20 ticks, statistics every tick -- through the plain path
    (cave_step: one launch per tick, the reference's per-tick dispatch), the streaming path
    (cave_run) and the resident kernel (a batch of this one simulation, all ticks on chip)."""
    import cave_b200 as cb

    G, T = WORKLOADS["plain49"]
    thr = cb.threshold_from_fill(0.30)
    params = cb.make_params(*PLAIN_RULE)
    ctx = cb.Context(local)
    ctx.set_timing(True)
    want = fixture("large_fixtures.json").get("49", {}).get("checkpoints", {}).get(str(T))
    out = {"workload": "49^3 FE, C=4 (maxCellState 3), survive {5,6,7} birth {6,7}, 30% fill of a centred 16^3 box, "
                       "seed 0, 20 ticks, statistics every tick", "unit": "sims/s"}
    launches = 0
    with cb.Grid(ctx, G, G, G) as g, ClockSampler(local) as clk:
        g.seed_threshold((16, 16, 16), thr, 0, 3)
        init = g.download()
        for path in ("plain", "streaming"):
            ms = []
            for i in range(warmup + steps):
                g.upload(init)
                if path == "plain":
                    ticks = g.step(params, T)
                    info = None
                else:
                    ticks, info = g.run(params, T, T)
                t = ctx.last_timing()
                if i >= warmup:
                    ms.append(t.tick_ms)
                    launches += t.launches
            if want:
                rec = cb.tick_records(ticks)
                require(hashlib.sha256(rec.tobytes()).hexdigest() == want["ticks_sha256"],
                        f"plain 49^3 ({path}): per-tick statistics")
                require(sha256_u32(g.download()) == want["cells_sha256"], f"plain 49^3 ({path}): cells")
                if info is not None:
                    require(list(info.as_tuple()) == want["gridinfo"], f"plain 49^3 ({path}): GridInfo")
            dev = max_over_ranks(pg, local, statistics.median(ms))
            out[path] = {"sims_per_s": 1e3 / dev, "cell_updates_per_s": G ** 3 * T / (dev / 1e3),
                         "us_per_tick": dev * 1e3 / T, "ms_per_sim": dev,
                         "how": "cave_step: one launch per tick" if path == "plain" else
                                "cave_run: layout conversion, one tick launch per tick, deferred fold"}
        # resident: one simulation in one CTA's shared memory for all its ticks
        ms = []
        for i in range(warmup + steps):
            with cb.Batch(ctx) as b:
                ix = b.add_init(G, G, G, init)
                b.add_sims([cb.SimDesc(params, ix, T, 0, 0)])
                b.launch()
                r = b.results_array()
                t = ctx.last_timing()
            if i >= warmup:
                ms.append(t.tick_ms)
                launches += t.launches
        if want:
            require(list(r[0]["info"]) == want["gridinfo"], "plain 49^3 (resident): GridInfo")
        dev = max_over_ranks(pg, local, statistics.median(ms))
        out["resident"] = {"sims_per_s": 1e3 / dev, "cell_updates_per_s": G ** 3 * T / (dev / 1e3),
                           "us_per_tick": dev * 1e3 / T, "ms_per_sim": dev,
                           "how": "a batch of this one simulation: one persistent launch, grid in shared memory"}
    out["clocks"] = clk.summary()
    out["gpu_launches"] = launches
    out["parity"] = ({"ok": True, "checked": "plain and streaming: every cell after tick 20, every tick's statistics; "
                                             "streaming and resident: GridInfo; vs tests/golden/large_fixtures.json"}
                     if want else {"ok": None, "checked": "no oracle fixture"})
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_grid(G, init, PLAIN_RULE, T, budget_s=3.0)
        # per simulation of 20 ticks
        cpu["sims_per_s"] = cpu["value"] / (G ** 3 * T)
        cpu["single_thread"]["sims_per_s"] = cpu["single_thread"]["value"] / (G ** 3 * T)
        out["cpu_baseline"] = cpu
    ctx.close()
    return out


# ----------------------------------------------------------------------------- config 3
def sweep_descs(G, seeds, cs_values, rank=0, world=1, stride=1):
    """The config-3 sweep: FE neighbourhood, every survive/birth set with <= 2 bits (171 each),
    C in cs_values (maxCellState = C - 1), `seeds` seeds; sims of this rank's shard."""
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


def sweep_workload(args, world, rank, local, pg, steps, warmup):
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
    for _ in range(warmup):
        with make_batch() as b:
            b.add_sims_array(warm, max_rule_bits=2)
            b.launch()
            b.results_array()
    barrier(pg, local)
    kern_ms, tot_ms, cats, ticks, launches, res = [], [], None, 0, 0, None
    # the step's results land in pinned host memory (the end-to-end read-back)
    import torch

    pinned = torch.empty(full.size * cb.SIM_RESULT_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
    out = pinned.numpy().view(cb.SIM_RESULT_DTYPE)
    with ClockSampler(local) as clk:
        for _ in range(steps):
            with make_batch() as b:
                b.add_sims_array(full, max_rule_bits=2)
                b.launch()
                res = b.results_array(out)
                t = ctx.last_timing()
                kern_ms.append(t.tick_ms)
                tot_ms.append(t.total_ms)
                launches += t.launches
            cats = np.bincount(res["category"], minlength=3)
            ticks = int(res["info"][:, 2].sum())
        barrier(pg, local)
    clocks = clk.summary()
    # parity: every 64th simulation of the sweep against the oracle fixture
    fx = fixture("sweep49_fixture.json")
    parity = {"ok": None, "checked": "not checked (sharded or strided run, or no fixture)"}
    if fx and world == 1 and args.stride == 1:
        sample = res[::fx["stride"]]
        rec = cb.result_records(sample, np.asarray(full["tag"][::fx["stride"]], dtype=np.uint64))
        blocks = [hashlib.sha256(rec[i:i + fx["block"]].tobytes()).hexdigest()
                  for i in range(0, rec.shape[0], fx["block"])]
        bad = [i for i, (a, b) in enumerate(zip(blocks, fx["block_sha256"])) if a != b]
        require(len(blocks) == len(fx["block_sha256"]) and not bad,
                f"sweep49: result blocks {bad[:8]} of every-64th-simulation sample differ from the oracle fixture")
        parity = {"ok": True, "checked": f"every {fx['stride']}th simulation ({rec.shape[0]}): GridInfo, category, "
                                         f"population, active ticks, changed cells, bounding box equal "
                                         f"tests/golden/sweep49_fixture.json"}
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
            v = sample.size / dev_s
            plain[f"slots{slots}_sims_per_s"] = v
            best = v if best is None else max(best, v)
        plain["best_sims_per_s"] = best
        plain["sample"] = f"{sample.size} simulations (every 997th of the sweep)"
    line = {
        "metric": "search sims/s", "value": sims_s, "unit": "sims/s", "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": kern, "higher_is_better": True, "scaling": "strong",
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
        "parity": parity,
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
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        sample = sweep_descs(G, seeds, cs_values, stride=997)[:16 * cores]
        items = [(int((int(d["birth"]) >> 60) & 0xF) + 1, int(d["init"]) % seeds,
                  int((int(d["survival"]) & 0xFFFFFFFF) - 1), int((int(d["birth"]) & 0xFFFFFFFF) - 1))
                 for d in sample]
        line["cpu_baseline"] = cpu_baseline_sims(_cpu_sweep_sim, items, "every 997th simulation of the sweep")
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


def uneven_spec_digest(sims):
    keys = ("edge", "flags", "maxcs", "birth", "survival", "ticks", "fill", "seed")
    return hashlib.sha256(json.dumps([[s[k] for k in keys] for s in sims]).encode()).hexdigest()


def uneven_workload(args, world, rank, local, pg, steps, warmup):
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
    t0 = time.perf_counter()
    plan = None
    for _ in range(warmup):
        with make_batch(mine, autotune) as b:
            b.launch()
            b.results_array()
            plan = b.plan()
    tune_wall = time.perf_counter() - t0
    barrier(pg, local)
    kern_ms, tot_ms, wall = [], [], []
    updates, launches, res = 0, 0, None
    vol = np.array([s["edge"] ** 3 for s in mine], dtype=np.int64)
    with ClockSampler(local) as clk:
        for _ in range(steps):
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
            updates = int((res["info"][:, 2].astype(np.int64) * vol).sum())
            require(int(res["error"].max(initial=0)) == 0, "uneven: a simulation raised an error flag")
        barrier(pg, local)
    clocks = clk.summary()
    fx = fixture("engine_fixture.json").get("uneven", {})
    parity = {"ok": None, "checked": "not checked (sharded run, another batch size, or no fixture)"}
    if fx and world == 1 and len(sims) == fx["sims"] and uneven_spec_digest(sims) == fx["spec_sha256"]:
        rec = cb.result_records(res, np.arange(len(sims)))
        blocks = [hashlib.sha256(rec[i:i + fx["block"]].tobytes()).hexdigest()
                  for i in range(0, rec.shape[0], fx["block"])]
        bad = [i for i, (a, b) in enumerate(zip(blocks, fx["block_sha256"])) if a != b]
        require(not bad, f"uneven2048: result blocks {bad[:8]} differ from the oracle fixture")
        parity = {"ok": True, "checked": f"all {len(sims)} simulations: GridInfo, category, population, active ticks, "
                                         f"changed cells, bounding box equal tests/golden/engine_fixture.json"}
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
        require(np.array_equal(rb["info"], r["info"]), "uneven: plain and batched paths disagree")
        plain = {"sample": f"{len(sample)} simulations (every 64th)", "plain_sims_per_s": len(sample) / dev_s,
                 "plain_cell_updates_per_s": upd_s / dev_s, "batched_sims_per_s_same_sample": len(sample) / tb,
                 "batched_cell_updates_per_s_same_sample": upd_s / tb, "batched_over_plain_same_sample": dev_s / tb}
    line = {
        "metric": "search sims/s", "value": n_all / (kern / 1e3), "unit": "sims/s", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": kern, "higher_is_better": True,
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
        # the whole batch against the plain path's rate on its every-64th sample (a 32-simulation
        # batch cannot fill the GPU, so the same-sample ratio understates batching)
        "batched_over_plain": ((n_all / (kern / 1e3)) / plain["plain_sims_per_s"]) if plain else None,
        "batched_over_plain_cell_updates": ((upd_all / (kern / 1e3)) / plain["plain_cell_updates_per_s"])
        if plain else None,
        "parity": parity,
        "e2e": {"value": n_all / (tot / 1e3), "unit": "sims/s", "h2d_bytes_per_step": int(len(mine) * 40),
                "d2h_bytes_per_step": int(len(mine) * cb.SIM_RESULT_DTYPE.itemsize)},
        "host_wall_s_per_step": sum(wall) / len(wall),
        "gpu_launches": int(sum_over_ranks(pg, local, launches)),
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sims(_cpu_uneven_sim, sims[::64], "every 64th simulation of the batch")
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


def serve_workload(args, world, rank, local, pg, rate=None, nreq=None):
    import cave_b200 as cb

    rate = rate or args.rate
    nreq = nreq or args.requests
    reqs = serve_requests(nreq, rate)[rank::world]
    ctx = cb.Context(local)
    budget = 120 * 10 ** 9
    total_sims = sum(r.size for _, r in reqs)

    def run(srv, timed_arrivals):
        ids, lat, by_id = {}, [], {}
        t0 = time.perf_counter()
        for t_arr, r in reqs:
            if timed_arrivals:
                d = t_arr - (time.perf_counter() - t0)
                if d > 0:
                    time.sleep(d)
            ids[srv.submit(r)] = r.size
        done = 0
        while done < len(ids):
            for rid in srv.poll():
                res, lt = srv.fetch(rid)
                require(int(res["error"].max(initial=0)) == 0, "serve: a simulation raised an error flag")
                lat.append(lt)
                by_id[rid] = res
                done += 1
            time.sleep(0.0005)
        span = time.perf_counter() - t0
        return span, sorted(lat), srv.stats(), [by_id[i] for i in sorted(by_id)]

    with cb.Server(ctx, hbm_budget=budget, autotune=False) as srv:
        warm = serve_requests(2, rate, seed=7)
        for _, r in warm:
            srv.wait(srv.submit(r), 600.0)
        for _ in srv.poll():
            pass
    with cb.Server(ctx, hbm_budget=budget) as srv, ClockSampler(local) as clk:
        span_served, lat, st_served, res_served = run(srv, True)
    clocks = clk.summary()
    with cb.Server(ctx, hbm_budget=budget) as srv:
        span_off, _, st_off, res_off = run(srv, False)
    # every simulation's result is the same in the served mix as in the offline run
    same = all(np.array_equal(cb.result_records(a, np.zeros(a.size)), cb.result_records(b, np.zeros(b.size)))
               for a, b in zip(res_served, res_off))
    require(same, "serve: a result differs between the served stream and the offline run")

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
        "config": {"workload": f"served: {len(reqs)} requests, Poisson {rate}/s, 1-256 sims each, edge 32..256, "
                               f"ticks 10..500, F/FE/Moore, C 2..16", "requests": len(reqs), "simulations": total_sims,
                   "hbm_budget_bytes": budget, "arrival_window_s": arrival_span},
        "latency_p50_s": pct(0.50), "latency_p99_s": pct(0.99),
        "server_p50_s": st_served.p50LatencySeconds, "server_p99_s": st_served.p99LatencySeconds,
        "offline_cell_updates_per_s": off_ups, "throughput_loss_vs_offline": 1.0 - served_ups / off_ups,
        "served_span_s": span_served, "offline_span_s": span_off, "peak_hbm_bytes": st_served.peakBytes,
        "tick_launches": st_served.tickLaunches, "resident_launches": st_served.residentLaunches,
        "rounds": st_served.rounds,
        "parity": {"ok": True, "checked": "every simulation's result in the served stream equals the offline run's "
                                          "(all requests submitted at once)"},
        "gpu_launches": int(st_served.tickLaunches + st_served.residentLaunches + st_served.rounds),
        "clocks": clocks,
        "e2e": {"value": served_ups, "unit": "cell-updates/s", "h2d_bytes_per_step": int(total_sims * 72),
                "d2h_bytes_per_step": int(total_sims * cb.SIM_RESULT_DTYPE.itemsize)},
    }
    ctx.close()
    return line


# ----------------------------------------------------------------------------- reference arm
def reference_arm(args, world, rank, local, pg):
    """The oracle port of the reference's shader arithmetic on the host cores (no CPU stepping
    exists in the reference; its GPU path needs Vulkan, which this box does not have)."""
    import oracle as O

    if rank != 0:
        return None
    G, T = WORKLOADS["large512"]
    params = O.make_params(*LARGE_RULE)
    init = O.seed(G, G, G, random=True, threshold=O.threshold_from_float(0.40), run_seed=0, max_cell_state=15)
    cores = os.cpu_count() or 1
    per_step = 5  # ticks per step: a bounded sample (about half a second on 16 cores)
    cells = init
    for _ in range(args.warmup * per_step):
        cells, _ = O.step_fast(G, G, G, params, cells, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps * per_step):
        cells, _ = O.step_fast(G, G, G, params, cells, nthreads=cores)
    el = time.perf_counter() - t0
    v = G ** 3 * args.steps * per_step / el
    return {
        "impl": "reference", "metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u4", "data": "synthetic (same seed and fill)",
        "config": {"workload": f"{G}^3 Moore-26, C=16, survive {{4,5}} birth {{5}}; {per_step} ticks per step "
                               f"(bounded sample of the {T}-tick run)", "grid": [G, G, G]},
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": "port", "cpu_model": cpu_model(),
                         "sample": f"{args.steps * per_step} ticks of {G}^3 after {args.warmup * per_step} "
                                   f"warm-up ticks"},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_extras(args, world, rank, local, pg):
    """The other workloads, each as a compact object of the default line."""
    steps, warmup = max(2, min(args.steps, 3)), 3
    extra = {}

    def keep(line, drop=("n_gpus", "higher_is_better", "vs_baseline", "dtype")):
        return {k: v for k, v in line.items() if k not in drop}

    extra["plain49"] = plain49_workload(args, world, rank, local, pg, steps, warmup)
    for G in (256, 1024):
        extra[f"large{G}"] = keep(large_workload(args, world, rank, local, pg, G, WORKLOADS[f"large{G}"][1],
                                                 steps, warmup, e2e=False))
    extra["sweep49"] = keep(sweep_workload(args, world, rank, local, pg, steps, warmup))
    extra["uneven2048"] = keep(uneven_workload(args, world, rank, local, pg, 2, warmup))
    extra["serve200"] = keep(serve_workload(args, world, rank, local, pg, rate=200.0, nreq=64))
    extra["serve16"] = keep(serve_workload(args, world, rank, local, pg, rate=16.0, nreq=48))
    return extra


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
        line = sweep_workload(args, world, rank, local, pg, args.steps, args.warmup)
    elif args.workload == "uneven2048":
        line = uneven_workload(args, world, rank, local, pg, args.steps, args.warmup)
    elif args.workload == "serve":
        line = serve_workload(args, world, rank, local, pg)
    elif args.workload == "plain49":
        line = plain49_workload(args, world, rank, local, pg, args.steps, args.warmup)
    else:
        G, T = WORKLOADS[args.workload]
        line = large_workload(args, world, rank, local, pg, G, args.ticks or T, args.steps, args.warmup,
                              e2e=not args.no_e2e)
        if args.workload == "large512" and not args.no_extra and not args.ticks:
            line["extra"] = run_extras(args, world, rank, local, pg)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
