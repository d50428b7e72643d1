"""Tiled batch execution (the engine: multi-CTA tick launches over many simulations, rounds,
completion ring, admission in waves, autotuning) against the oracle's per-rule lifecycle
(searchSystem.cpp:496-526 + searchManager.slang:98-149). Integer work: every compared field
is exact."""
import numpy as np
import pytest

import cave_b200 as cb
import oracle as O

pytestmark = pytest.mark.gpu


def expected(X, Y, Z, params_np, init, max_ticks):
    info, ticks, _ = O.run_sim(X, Y, Z, params_np, init, max_ticks, fast=True, per_tick=True)
    maxcs = int((int(params_np[0]) >> 60) & 0xF) + 1
    last = ticks[-1]
    return {
        "info": info.as_tuple(),
        "category": O.classify(info, maxcs),
        "population": last.population,
        "totalChanged": sum(t.changed for t in ticks),
        "activeTicks": sum(1 for t in ticks if t.changed),
        "bbox": (tuple(last.bbox_min), tuple(last.bbox_max)),
    }


def got(r):
    return {
        "info": tuple(int(v) for v in r["info"]),
        "category": int(r["category"]),
        "population": int(r["population"]),
        "totalChanged": int(r["totalChanged"]),
        "activeTicks": int(r["activeTicks"]),
        "bbox": (tuple(int(v) for v in r["bbox_min"]), tuple(int(v) for v in r["bbox_max"])),
    }


def random_case(rng, dims, i):
    X, Y, Z = dims
    flags = int(rng.choice([1, 2, 3, 4, 5, 6, 7]))
    maxcs = int(rng.choice([1, 2, 3, 5, 9, 15]))
    nb = (6 if flags & 1 else 0) + (12 if flags & 2 else 0) + (8 if flags & 4 else 0)
    if i % 3 == 0:  # dense rule: table evaluation
        B, S = int(rng.integers(1, 1 << nb)), int(rng.integers(1, 1 << nb))
    else:           # 1..4 counts each: term evaluation
        B = sum(1 << int(v) for v in rng.choice(nb, size=int(rng.integers(1, 5)), replace=False))
        S = sum(1 << int(v) for v in rng.choice(nb, size=int(rng.integers(1, 5)), replace=False))
    s = np.zeros((Z, Y, X), dtype=np.uint8)
    s[rng.random((Z, Y, X)) < float(rng.uniform(0.2, 0.5))] = maxcs & 0xF
    init = O.pack(s)
    T = int(rng.integers(1, 25))
    return O.make_params(maxcs, flags, B, S), init, T


def run_batch(ctx, cases, dims_of, **opts):
    with cb.Batch(ctx) as b:
        b.set_options(**opts)
        for i, (params_np, init, T) in enumerate(cases):
            X, Y, Z = dims_of(i)
            ix = b.add_init(X, Y, Z, init)
            b.add_sims([cb.SimDesc(cb.SimParams(*[int(v) for v in params_np]), ix, T, 0, i)])
        b.launch()
        res = b.results_array()
        plan = b.plan()
    return res, plan


@pytest.mark.parametrize("dims", [(33, 33, 33), (40, 17, 29), (130, 70, 40), (97, 40, 33)])
def test_tiled_only_matches_oracle(ctx, dims):
    """Every simulation through the tiled path (grids that would fit shared memory included)."""
    rng = np.random.default_rng(sum(dims) + 7)
    cases = [random_case(rng, dims, i) for i in range(12)]
    res, plan = run_batch(ctx, cases, lambda i: dims, tiled_only=True)
    assert all(p["path"] == "tiled" for p in plan)
    for i, (params_np, init, T) in enumerate(cases):
        assert int(res[i]["tag"]) == i and int(res[i]["error"]) == 0
        assert got(res[i]) == expected(*dims, params_np, init, T), f"sim {i}"


def test_mixed_shapes_resident_and_tiled(ctx):
    """One batch mixing grids that run resident and grids too large for shared memory."""
    rng = np.random.default_rng(11)
    shapes = [(33, 33, 33), (130, 70, 40), (49, 49, 49), (97, 97, 24), (8, 8, 8)]
    cases, dims = [], []
    for i in range(20):
        d = shapes[i % len(shapes)]
        dims.append(d)
        cases.append(random_case(rng, d, i))
    res, plan = run_batch(ctx, cases, lambda i: dims[i])
    paths = {tuple(p["grid"]): p["path"] for p in plan}
    assert paths[(130, 70, 40)] == "tiled" and paths[(33, 33, 33)] == "resident"
    for i, (params_np, init, T) in enumerate(cases):
        assert int(res[i]["error"]) == 0
        assert got(res[i]) == expected(*dims[i], params_np, init, T), f"sim {i} {dims[i]}"


def test_waves_under_small_budget(ctx):
    """A memory budget of about three simulations: the rest wait for earlier ones to finish."""
    rng = np.random.default_rng(5)
    dims = (130, 70, 40)
    per_sim = 2 * 5 * 70 * 40 * 16
    cases = [random_case(rng, dims, i) for i in range(10)]
    res, _ = run_batch(ctx, cases, lambda i: dims, memory_budget=3 * per_sim + 4096, ticks_per_round=3)
    for i, (params_np, init, T) in enumerate(cases):
        assert got(res[i]) == expected(*dims, params_np, init, T), f"sim {i}"


def test_autotune_does_not_change_results(ctx):
    rng = np.random.default_rng(9)
    dims = (97, 40, 33)
    cases = [random_case(rng, dims, i) for i in range(8)]
    a, _ = run_batch(ctx, cases, lambda i: dims)
    b, plan = run_batch(ctx, cases, lambda i: dims, autotune=True)
    assert plan and plan[0]["path"] in ("resident", "tiled")
    for i in range(len(cases)):
        assert got(a[i]) == got(b[i])


def test_ticks_per_round_does_not_change_results(ctx):
    rng = np.random.default_rng(21)
    dims = (130, 70, 40)
    cases = [random_case(rng, dims, i) for i in range(6)]
    a, _ = run_batch(ctx, cases, lambda i: dims, ticks_per_round=1)
    b, _ = run_batch(ctx, cases, lambda i: dims, ticks_per_round=16)
    for i in range(len(cases)):
        assert got(a[i]) == got(b[i])
