"""Large grids at the benchmark's own geometry against oracle fixtures.

The benchmark workload: 256^3 and 512^3 cubes, Moore neighbourhood, maxCellState 15, survival
{4,5}, birth {5}, 40% fill by the reference's cell hash with seed 0, stepped 100 and 1000 ticks
by cave_run with statistics every tick (1024^3: 20 and 200 ticks, out of L2). That rule settles into a still life within about 100
ticks, so "active" entries keep every tick busy at the same geometries (Moore C=4 B{5,6,7}
S{5,6,7,8} at 256^3 and 512^3, FE C=6 B{4,5} S{3,4,5,6} at 256^3). Each runs on the
rule-specialised tick kernels (CAVE_JIT=sync; runs of 100 or more ticks also take the tile-timing
pass) and on the generic one (CAVE_JIT=off), on device-resident cells and through cave_run_host
with pinned host buffers (the end-to-end form). Compared with tests/golden/large_fixtures.json
(made by tests/golden/make_large_fixtures.py from the oracle): the SHA-256 of every cell after
the last tick and of every tick's statistics, and the GridInfo. Integer work: exact.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import cave_b200 as cb

pytestmark = pytest.mark.gpu

FIXTURE = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "large_fixtures.json")))
CASES = [(name, int(T)) for name in ("256", "512", "1024", "active256", "active512", "activeFE256") if name in FIXTURE
         for T in FIXTURE[name]["checkpoints"]]


def _setup(ctx, name):
    fx = FIXTURE[name]
    G, r = fx["grid"], fx["rule"]
    g = cb.Grid(ctx, G, G, G)
    sp = r["spawn"] or G
    g.seed_threshold((sp, sp, sp), cb.threshold_from_fill(r["fill"]), r["seed"], r["max_cell_state"])
    assert hashlib.sha256(g.download().astype("<u4").tobytes()).hexdigest() == fx["seed_sha256"], "seeded cells"
    return g, cb.make_params(r["max_cell_state"], r["flags"], r["birth"], r["survival"])


def _check(name, T, cells, ticks, info):
    fx = FIXTURE[name]
    cp = fx["checkpoints"][str(T)]
    rec = cb.tick_records(ticks)
    for t, want in fx["sample"].items():
        if int(t) < T:
            assert rec[int(t)].tolist() == want, f"{name} tick {t} statistics"
    assert hashlib.sha256(rec.tobytes()).hexdigest() == cp["ticks_sha256"], f"{name} per-tick statistics, {T} ticks"
    assert list(info.as_tuple()) == cp["gridinfo"], f"{name} GridInfo after {T} ticks"
    assert hashlib.sha256(cells.astype("<u4").tobytes()).hexdigest() == cp["cells_sha256"], f"{name} cells, {T} ticks"


@pytest.mark.parametrize("jit", ["sync", "off"])
@pytest.mark.parametrize("name,T", CASES)
def test_large_grid_run(ctx, monkeypatch, jit, name, T):
    monkeypatch.setenv("CAVE_JIT", jit)
    g, params = _setup(ctx, name)
    with g:
        launches0 = cb.jit_stats()[1]
        ticks, info = g.run(params, T, T)
        assert (cb.jit_stats()[1] - launches0 > 0) == (jit == "sync")
        _check(name, T, g.download(), ticks, info)


@pytest.mark.parametrize("name", ["512", "active512"])
def test_large_grid_run_host_buffers(ctx, monkeypatch, name):
    """The end-to-end form the benchmark times: pinned host buffers in and out."""
    torch = pytest.importorskip("torch")
    monkeypatch.setenv("CAVE_JIT", "sync")
    T = max(int(t) for t in FIXTURE[name]["checkpoints"])
    g, params = _setup(ctx, name)
    with g:
        init = g.download()
        pin_in = torch.from_numpy(init.view(np.int32)).pin_memory()
        pin_out = torch.zeros_like(pin_in).pin_memory()
        g.upload(np.zeros_like(init))  # the run must take its input from the host buffer
        ticks, info = g.run_host(pin_in.data_ptr(), pin_out.data_ptr(), params, T, T)
        _check(name, T, pin_out.numpy().view(np.uint32), ticks, info)


@pytest.mark.parametrize("pairs", ["1", "0"])
def test_tick_loop_replayed_from_a_graph(ctx, monkeypatch, pairs):
    """CAVE_RUN_GRAPH=1 (a measurement mode): the tick launches captured into a CUDA graph and
    replayed give the same cells, statistics and GridInfo."""
    monkeypatch.setenv("CAVE_JIT", "sync")
    monkeypatch.setenv("CAVE_RUN_GRAPH", "1")
    monkeypatch.setenv("CAVE_TICK2", pairs)
    name, T = "active256", 100
    g, params = _setup(ctx, name)
    with g:
        ticks, info = g.run(params, T, T)
        _check(name, T, g.download(), ticks, info)
