"""Generates tests/golden/sweep_fixture.json with the CPU oracle (test infrastructure).

The sweep is the reference's published benchmark workload (benchmarks/scripts/debug/
bench_chunks.ps1:21-32): cube, neighbourhood selection FE (subsets F, E, FE), K <= 2 rule bits,
maxCellState 2..3, 20 ticks, default 11^3 filled spawn (src/main.cpp:34-35), grids 25^3 and
49^3 -- 71,532 rules per grid. For each grid the fixture stores the viable / possible /
unviable counts and a SHA-256 over every rule's final GridInfo in canonical order
(maxCS, flags, survival index, birth index), packed as little-endian uint32 x 6.

Usage: python tests/golden/make_sweep_fixture.py [--grids 25,49] [--procs 8]
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

NEIGHBOURS = {1: 6, 2: 12, 3: 18}
MAXCS = (2, 3)
TICKS = 20
SPAWN = 11


def rules():
    """Canonical order of the sweep's (maxCS, flags, survival index, birth index)."""
    import oracle as O

    out = []
    for mcs in MAXCS:
        for flags in (1, 2, 3):
            n = len(O.valid_bitmasks(NEIGHBOURS[flags], 2))
            for si in range(n):
                for bi in range(n):
                    out.append((mcs, flags, si, bi))
    return out


def work(args):
    import numpy as np

    import oracle as O

    G, mcs, flags, si = args
    vb = O.valid_bitmasks(NEIGHBOURS[flags], 2)
    init = O.seed(G, G, G, spawn=(SPAWN, SPAWN, SPAWN), random=False, max_cell_state=mcs)
    rows = []
    for bi in range(len(vb)):
        p = O.make_params(mcs, flags, bi + 1, si + 1)
        info, _, _ = O.run_sim(G, G, G, p, init, TICKS, valid=vb, max_rule_bits=2, fast=True)
        rows.append(list(info.as_tuple()) + [O.classify(info, mcs)])
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grids", default="25,49")
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    a = ap.parse_args()
    import numpy as np

    import oracle as O

    O.build()
    out_path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sweep_fixture.json")
    fixture = json.load(open(out_path)) if os.path.exists(out_path) else {}
    for G in [int(g) for g in a.grids.split(",")]:
        tasks = []
        for mcs in MAXCS:
            for flags in (1, 2, 3):
                for si in range(len(O.valid_bitmasks(NEIGHBOURS[flags], 2))):
                    tasks.append((G, mcs, flags, si))
        t0 = time.time()
        with get_context("spawn").Pool(a.procs) as pool:
            res = pool.map(work, tasks, chunksize=2)
        rows = [r for chunk in res for r in chunk]
        arr = np.array([r[:6] for r in rows], dtype="<u4")
        cats = np.array([r[6] for r in rows])
        fixture[str(G)] = {
            "rules": len(rows),
            "viable": int((cats == 0).sum()),
            "possible": int((cats == 1).sum()),
            "unviable": int((cats == 2).sum()),
            "gridinfo_sha256": hashlib.sha256(arr.tobytes()).hexdigest(),
            "seconds": round(time.time() - t0, 1),
        }
        print(G, fixture[str(G)], flush=True)
    fixture["workload"] = ("cube, FE subsets (F, E, FE), K<=2, maxCellState 2..3, 20 ticks, 11^3 filled spawn; "
                           "rules in (maxCS, flags, survival index, birth index) order; GridInfo as 6 x uint32 LE")
    with open(out_path, "w") as f:
        json.dump(fixture, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
