"""Generates tests/golden/large_fixtures.json with the CPU oracle (test infrastructure).

The large-grid workload of the bandwidth benchmark (grids 256 and 512, also 1024): a cube of
G^3 cells, Moore neighbourhood (flags 0x7, 26 neighbours), maxCellState 15 (C = 16 states),
survival {4,5}, birth {5}, the reference's cell hash (searchSystem.cpp:244-262) with seed 0
filling 40% of the whole volume (threshold (uint32)((double)0.4f * 2^32)), stepped `ticks`
times with statistics every tick (raw stepping: the run never stops on the manager's status).
Grid 49 is the plain single-simulation workload instead: 49^3, FE (flags 0x3), maxCellState 3
(C = 4), survival {5,6,7}, birth {6,7}, 30% fill of a centred 16^3 box, seed 0, 20 ticks.
The benchmark rule settles into a still life within about 100 ticks, so three more entries keep
every tick busy at the same geometries ("active..."): Moore, maxCellState 3, birth {5,6,7},
survival {5,6,7,8} at 256^3 (300 ticks) and 512^3 (200 ticks), and FE, maxCellState 5, birth
{4,5}, survival {3,4,5,6} at 256^3 (200 ticks), each with a 30% fill of the whole volume, seed 1.

For each grid the fixture stores, at every checkpoint tick T:
  * the SHA-256 of the cells after tick T in the reference's padded nibble layout
    (little-endian uint32 words, x/8 + y*W + z*W*Y);
  * the SHA-256 of the per-tick statistics of ticks 0..T-1, each tick packed as 12
    little-endian uint32 (dead, dying, born, surviving -- the GridSnapshot of structs.h:130-136
    -- then population, changed, bbox_min[3], bbox_max[3]);
  * the GridInfo after T ticks with MAX_NUMBER_OF_TICKS_TO_SURVIVE = T (searchManager.slang:
    98-139 applied once per tick);
and, in the clear, the statistics of a few ticks (for diagnosing a mismatch).

Usage: python tests/golden/make_large_fixtures.py [--grids 49,256,512,...] [--threads N]
"""
import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

def _mask(counts):
    return sum(1 << (c - 1) for c in counts)


LARGE = dict(max_cell_state=15, flags=0x7, birth=_mask([5]), survival=_mask([4, 5]), fill=0.40, spawn=None, seed=0)
ACTIVE = dict(max_cell_state=3, flags=0x7, birth=_mask([5, 6, 7]), survival=_mask([5, 6, 7, 8]), fill=0.30,
              spawn=None, seed=1)
ACTIVE_FE = dict(max_cell_state=5, flags=0x3, birth=_mask([4, 5]), survival=_mask([3, 4, 5, 6]), fill=0.30,
                 spawn=None, seed=1)
# name: (edge, workload, checkpoint ticks)
ENTRIES = {
    "49": (49, dict(max_cell_state=3, flags=0x3, birth=0x60, survival=0x70, fill=0.30, spawn=16, seed=0), (20,)),
    "256": (256, LARGE, (100, 1000)),
    "512": (512, LARGE, (100, 1000)),
    "1024": (1024, LARGE, (20, 200)),
    "active256": (256, ACTIVE, (6, 100, 300)),
    "active512": (512, ACTIVE, (6, 200)),
    "activeFE256": (256, ACTIVE_FE, (6, 200)),
}
SAMPLE_TICKS = (0, 1, 2, 49, 99, 199, 499, 999)


def stats_row(st):
    return [st.dead, st.dying, st.born, st.surviving, st.population, st.changed, *st.bbox_min, *st.bbox_max]


def grid_info(rows, max_ticks):
    """GridInfo after len(rows) manager updates (searchManager.slang:115-139), no early stop."""
    died = born = ticks = maxs = final = status = 0
    for r in rows:
        ticks += 1
        died += r[0]
        born += r[2]
        final = r[3]
        maxs = max(maxs, r[3])
        status = 1 if (r[3] == 0 and r[2] == 0) else (2 if ticks >= max_ticks else 0)
    m = 0xFFFFFFFF
    return [died & m, born & m, ticks, status, maxs, final]


def make(name, threads):
    import oracle as O

    G, w, checkpoints = ENTRIES[name]
    p = O.make_params(w["max_cell_state"], w["flags"], w["birth"], w["survival"])
    sp = w["spawn"] or G
    cells = O.seed(G, G, G, spawn=(sp, sp, sp), random=True, threshold=O.threshold_from_float(w["fill"]),
                   run_seed=w["seed"], max_cell_state=w["max_cell_state"])
    out = {"grid": G, "seed_sha256": hashlib.sha256(cells.tobytes()).hexdigest(), "checkpoints": {}, "sample": {},
           "rule": {k: w[k] for k in ("max_cell_state", "flags", "birth", "survival", "fill", "spawn", "seed")}}
    rows = []
    t0 = time.time()
    last = max(checkpoints)
    for t in range(last):
        cells, st = O.step_stats_fast(G, G, G, p, cells, nthreads=threads)
        rows.append(stats_row(st))
        if t in SAMPLE_TICKS:
            out["sample"][str(t)] = rows[-1]
        if t + 1 in checkpoints:
            T = t + 1
            out["checkpoints"][str(T)] = {
                "cells_sha256": hashlib.sha256(cells.astype("<u4").tobytes()).hexdigest(),
                "ticks_sha256": hashlib.sha256(np.array(rows, dtype="<u4").tobytes()).hexdigest(),
                "gridinfo": grid_info(rows, T),
            }
            print(f"{name}: tick {T} after {time.time() - t0:.0f} s", flush=True)
    out["seconds"] = round(time.time() - t0, 1)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grids", default="49,256,512,active256,active512,activeFE256")
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    a = ap.parse_args()
    import oracle as O

    O.build()
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "large_fixtures.json")
    fixture = json.load(open(path)) if os.path.exists(path) else {}
    fixture["workload"] = ("cube G^3, Moore (flags 0x7), maxCellState 15, survival {4,5}, birth {5}, cell hash seed 0, "
                           "40% fill of the whole volume, raw stepping with statistics every tick; G = 49: FE, "
                           "maxCellState 3, survival {5,6,7}, birth {6,7}, 30% fill of a centred 16^3 box, 20 ticks")
    for name in a.grids.split(","):
        fixture[name] = make(name, a.threads)
        with open(path + ".tmp", "w") as f:
            json.dump(fixture, f, indent=1, sort_keys=True)
        os.replace(path + ".tmp", path)


if __name__ == "__main__":
    main()
