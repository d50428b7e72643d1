"""Generates tests/golden/engine_fixture.json with the CPU oracle (test infrastructure).

Two parts, both run by the oracle's per-rule lifecycle (searchSystem.cpp:496-526 plus
searchManager.slang:98-149: step until the manager reports status > 0):

* "uneven": the uneven-size batch of the benchmark (bench.py uneven_sims: 2048 simulations,
  edges {33, 49, 65, 97, 129, 193}, F / FE / Moore, C = 2..16, 1-4 counts per rule set,
  10..500 ticks, 20-50% fill of the whole grid, seed = the simulation's index). Each result is
  packed as 18 little-endian uint32 (index, GridInfo (6), category, population after the last
  tick, ticks in which a cell changed, cells changed over all ticks (low, high word), bbox_min
  (3), bbox_max (3)); the fixture stores the SHA-256 of every block of 64 records, the
  category counts, the ticks run, and the SHA-256 of the simulation list itself (so a change
  of the draw is caught).
* "long": hand-picked long-lived simulations for the tiled and served paths at the large end
  of their size ranges (193^3 and 256^3 with the Moore rule S{4,5} B{5}, C = 16, 300 ticks),
  with their records in the clear.

Usage: python tests/golden/make_engine_fixture.py [--procs N] [--parts uneven,long]
"""
import argparse
import hashlib
import json
import os
import sys
import time
from multiprocessing import get_context

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
os.environ.setdefault("OMP_NUM_THREADS", "1")

BLOCK = 64
LONG = [
    # name, edge, maxCellState, flags, birth, survival, ticks, fill, seed
    ("tiled193", 193, 15, 0x7, 1 << 4, (1 << 3) | (1 << 4), 300, 0.40, 3),
    ("served256", 256, 15, 0x7, 1 << 4, (1 << 3) | (1 << 4), 300, 0.35, 11),
]


def spec_digest(sims):
    keys = ("edge", "flags", "maxcs", "birth", "survival", "ticks", "fill", "seed")
    return hashlib.sha256(json.dumps([[s[k] for k in keys] for s in sims]).encode()).hexdigest()


def record(index, e, maxcs, flags, birth, survival, ticks, fill, seed):
    import oracle as O

    init = O.seed(e, e, e, random=True, threshold=O.threshold_from_float(fill), run_seed=seed,
                  max_cell_state=maxcs)
    p = O.make_params(maxcs, flags, birth, survival)
    info, per, _ = O.run_sim(e, e, e, p, init, ticks, fast=True, per_tick=True)
    last = per[-1]
    chg = sum(t.changed for t in per)
    return [index, *info.as_tuple(), O.classify(info, maxcs), last.population, sum(1 for t in per if t.changed),
            chg & 0xFFFFFFFF, chg >> 32, *last.bbox_min, *last.bbox_max]


def work(a):
    i, s = a
    return record(i, s["edge"], s["maxcs"], s["flags"], s["birth"], s["survival"], s["ticks"], s["fill"], s["seed"])


def work_long(a):
    name, e, maxcs, flags, birth, survival, ticks, fill, seed = a
    return record(0, e, maxcs, flags, birth, survival, ticks, fill, seed)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--parts", default="uneven,long")
    a = ap.parse_args()
    import numpy as np

    import bench
    import oracle as O

    O.build()
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "engine_fixture.json")
    fixture = json.load(open(path)) if os.path.exists(path) else {}
    parts = a.parts.split(",")
    if "uneven" in parts:
        sims = bench.uneven_sims(2048)
        order = sorted(range(len(sims)), key=lambda i: -sims[i]["edge"] ** 3 * sims[i]["ticks"])
        t0 = time.time()
        with get_context("spawn").Pool(a.procs) as pool:
            got = pool.map(work, [(i, sims[i]) for i in order], chunksize=1)
        rows = np.zeros((len(sims), 18), dtype="<u4")
        for r in got:
            rows[r[0]] = r
        cats = np.bincount(rows[:, 7], minlength=3)
        vol = np.array([s["edge"] ** 3 for s in sims], dtype=np.int64)
        fixture["uneven"] = {
            "sims": len(sims), "block": BLOCK, "spec_sha256": spec_digest(sims),
            "viable": int(cats[0]), "possible": int(cats[1]), "unviable": int(cats[2]),
            "ticks": int(rows[:, 3].astype(np.int64).sum()),
            "cell_updates": int((rows[:, 3].astype(np.int64) * vol).sum()),
            "block_sha256": [hashlib.sha256(rows[i:i + BLOCK].tobytes()).hexdigest()
                             for i in range(0, len(sims), BLOCK)],
            "seconds": round(time.time() - t0, 1),
        }
        print(json.dumps({k: v for k, v in fixture["uneven"].items() if k != "block_sha256"}), flush=True)
    if "long" in parts:
        with get_context("spawn").Pool(min(a.procs, len(LONG))) as pool:
            got = pool.map(work_long, LONG, chunksize=1)
        fixture["long"] = {
            L[0]: {"edge": L[1], "maxCellState": L[2], "flags": L[3], "birth": L[4], "survival": L[5],
                   "maxTicks": L[6], "fill": L[7], "seed": L[8], "record": r}
            for L, r in zip(LONG, got)}
        print(json.dumps(fixture["long"]), flush=True)
    fixture["record"] = ("index, GridInfo[6], category, population, activeTicks, totalChanged lo, hi, bbox_min[3], "
                         "bbox_max[3] as little-endian uint32")
    with open(path + ".tmp", "w") as f:
        json.dump(fixture, f, indent=1, sort_keys=True)
    os.replace(path + ".tmp", path)


if __name__ == "__main__":
    main()
