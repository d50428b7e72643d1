"""Generates tests/golden/sweep49_fixture.json with the CPU oracle (test infrastructure).

The batched search sweep on 49^3 cubes: FE neighbourhood (flags 0x3), every survival and
birth set with 1 or 2 of the 18 counts (171 K-indexed masks each, permutationMath.h:101-128
order), maxCellState 1..4 (C = 2..5 states), seeds 0..31, each initial grid a centred 16^3 box
filled to 30% by the reference's cell hash (searchSystem.cpp:244-262; threshold
(uint32)((double)0.3f * 2^32)), 20 ticks with the manager's early stop
(searchManager.slang:98-139). Simulations are numbered in the order (C, seed, survival index,
birth index) -- 3,742,848 in all -- and the fixture covers every 64th one (index % 64 == 0).

Per sampled simulation the result is packed as 18 little-endian uint32:
  index, GridInfo (6, structs.h:79-87), category (searchSystem.cpp:697-711), population after
  the last tick, ticks in which a cell changed, cells changed over all ticks (low, high word),
  bbox_min (3), bbox_max (3) of the non-zero cells after the last tick
and the fixture stores the SHA-256 of each block of 1024 consecutive records, the category
counts and the number of ticks run.

Usage: python tests/golden/make_sweep49_fixture.py [--procs N]
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

G = 49
SPAWN = 16
FILL = 0.30
TICKS = 20
CS = (2, 3, 4, 5)
SEEDS = 32
NMASKS = 171
STRIDE = 64
BLOCK = 1024
PER_INIT = NMASKS * NMASKS


def work(args):
    import numpy as np

    import oracle as O

    ci, s = args
    mcs = CS[ci] - 1
    vb = O.valid_bitmasks(18, 2)
    init = O.seed(G, G, G, spawn=(SPAWN, SPAWN, SPAWN), random=True, threshold=O.threshold_from_float(FILL),
                  run_seed=s, max_cell_state=mcs)
    base = (ci * SEEDS + s) * PER_INIT
    first = (-base) % STRIDE
    rows = []
    for k in range(first, PER_INIT, STRIDE):
        si, bi = divmod(k, NMASKS)
        p = O.make_params(mcs, 0x3, bi + 1, si + 1)
        info, ticks, _ = O.run_sim(G, G, G, p, init, TICKS, valid=vb, max_rule_bits=2, fast=True, per_tick=True)
        last = ticks[-1]
        chg = sum(t.changed for t in ticks)
        rows.append([base + k, *info.as_tuple(), O.classify(info, mcs), last.population,
                     sum(1 for t in ticks if t.changed), chg & 0xFFFFFFFF, chg >> 32, *last.bbox_min,
                     *last.bbox_max])
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    a = ap.parse_args()
    import numpy as np

    import oracle as O

    O.build()
    tasks = [(ci, s) for ci in range(len(CS)) for s in range(SEEDS)]
    t0 = time.time()
    with get_context("spawn").Pool(a.procs) as pool:
        parts = pool.map(work, tasks, chunksize=1)
    rows = np.array([r for p in parts for r in p], dtype="<u4")
    assert np.all(np.diff(rows[:, 0].astype(np.int64)) == STRIDE)
    cats = np.bincount(rows[:, 7], minlength=3)
    out = {
        "workload": "49^3 FE sweep: 171 x 171 K<=2 rules x C in {2,3,4,5} x seeds 0..31, 30% fill of a centred "
                    "16^3 box, 20 ticks with early stop; simulations in (C, seed, survival index, birth index) order",
        "stride": STRIDE, "block": BLOCK, "sims_total": len(CS) * SEEDS * PER_INIT, "sims": int(rows.shape[0]),
        "record": "index, GridInfo[6], category, population, activeTicks, totalChanged lo, hi, bbox_min[3], "
                  "bbox_max[3] as little-endian uint32",
        "viable": int(cats[0]), "possible": int(cats[1]), "unviable": int(cats[2]),
        "ticks": int(rows[:, 3].astype(np.int64).sum()),
        "block_sha256": [hashlib.sha256(rows[i:i + BLOCK].tobytes()).hexdigest()
                         for i in range(0, rows.shape[0], BLOCK)],
        "seconds": round(time.time() - t0, 1),
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sweep49_fixture.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(json.dumps({k: v for k, v in out.items() if k != "block_sha256"}))


if __name__ == "__main__":
    main()
