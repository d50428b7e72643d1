"""GPU parity of the rule-specialised tick kernels (NVRTC): with CAVE_JIT=sync every cave_run and
cave_render_step below runs the kernels compiled for its rule, checked bit-exact against the
oracle (every cell, every per-tick statistic, GridInfo), and the launch counter proves that the
specialised kernels, not the generic one, did the ticks. Every cave_run case runs twice: with
two ticks per launch (the default; an odd tick count starts with one single-tick launch) and with
CAVE_TICK2=0 (one tick per launch)."""
import os

import numpy as np
import pytest

import cave_b200 as cb
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["pairs", "single"], autouse=True)
def tick2(request, monkeypatch):
    monkeypatch.setenv("CAVE_TICK2", "1" if request.param == "pairs" else "0")
    return request.param == "pairs"


def expected_launches(nticks, pairs):
    return (nticks & 1) + nticks // 2 if pairs and nticks >= 2 else nticks


@pytest.fixture(scope="module", autouse=True)
def jit_sync(tmp_path_factory):
    saved = {k: os.environ.get(k) for k in ("CAVE_JIT", "CAVE_JIT_CACHE")}
    os.environ["CAVE_JIT"] = "sync"
    os.environ["CAVE_JIT_CACHE"] = str(tmp_path_factory.mktemp("jit_cache"))
    yield
    for k, v in saved.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v


def random_states(rng, X, Y, Z, maxcs, p_alive=0.35, p_other=0.15):
    s = np.zeros((Z, Y, X), dtype=np.uint8)
    r = rng.random((Z, Y, X))
    s[r < p_alive] = maxcs & 0xF
    other = (r >= p_alive) & (r < p_alive + p_other)
    s[other] = rng.integers(1, 16, size=int(other.sum()), dtype=np.uint8)
    return O.pack(s)


def run_and_check(ctx, X, Y, Z, params_np, init, nticks, max_ticks=10 ** 6):
    p = cb.SimParams(*[int(v) for v in params_np])
    cells, expect = init, []
    for _ in range(nticks):
        cells, st = O.step_stats_fast(X, Y, Z, params_np, cells)
        expect.append(st.as_tuple())
    _, launches0 = cb.jit_stats()
    with cb.Grid(ctx, X, Y, Z) as g:
        g.upload(init)
        sts, info = g.run(p, nticks, max_ticks)
        got_cells = g.download()
    _, launches1 = cb.jit_stats()
    pairs = os.environ.get("CAVE_TICK2") != "0"
    assert launches1 - launches0 == expected_launches(nticks, pairs), "the ticks did not run on the specialised kernels"
    assert np.array_equal(got_cells, cells), "cells differ"
    for t in range(nticks):
        assert sts[t].as_tuple() == expect[t], f"statistics differ at tick {t + 1}"
    return info


def test_config2_rule(ctx):
    """Moore-26, C=16, survive {4,5}, birth {5}, 40% fill: the large-grid benchmark rule."""
    G = 128
    init = O.seed(G, G, G, random=True, threshold=O.threshold_from_float(0.40), run_seed=0, max_cell_state=15)
    params = O.make_params(15, 0x7, 0x10, 0x18)
    info = run_and_check(ctx, G, G, G, params, init, 6, max_ticks=6)
    want = O.run_sim(G, G, G, params, init, 6, fast=True)[0]
    assert info.as_tuple() == want.as_tuple()


@pytest.mark.parametrize("flags", [0, 1, 2, 3, 4, 5, 6, 7, 0xB])
def test_every_neighbourhood(ctx, flags):
    rng = np.random.default_rng(1000 + flags)
    X, Y, Z = 70, 33, 21
    nb = (6 if flags & 1 else 0) + (12 if flags & 2 else 0) + (8 if flags & 4 else 0)
    maxcs = int(rng.integers(1, 16))
    B = sum(1 << int(v) for v in rng.choice(nb, size=min(3, nb), replace=False)) if nb else 1
    S = sum(1 << int(v) for v in rng.choice(nb, size=min(4, nb), replace=False)) if nb else 1
    run_and_check(ctx, X, Y, Z, O.make_params(maxcs, flags, B, S), random_states(rng, X, Y, Z, maxcs), 3)


@pytest.mark.parametrize("maxcs,birth,survival", [(1, 0x1F0, 0x3F), (16, 0x10, 0x18), (2, 0x0, 0x0),
                                                   (9, (1 << 26) - 1, (1 << 26) - 1), (5, 0x2AAAAAA, 0x1555555)])
def test_state_counts_and_table_shapes(ctx, maxcs, birth, survival):
    rng = np.random.default_rng(maxcs * 7 + birth % 97)
    X, Y, Z = 97, 29, 18
    run_and_check(ctx, X, Y, Z, O.make_params(maxcs, 0x7, birth, survival), random_states(rng, X, Y, Z, maxcs), 3)


@pytest.mark.parametrize("dims", [(1024, 40, 4), (480, 95, 7), (33, 1, 1)])
def test_tilings(ctx, dims):
    X, Y, Z = dims
    rng = np.random.default_rng(X + Y + Z)
    run_and_check(ctx, X, Y, Z, O.make_params(15, 0x7, 0x10, 0x18), random_states(rng, X, Y, Z, 15), 4)


@pytest.mark.parametrize("nticks", [1, 2, 3, 4, 5, 7, 8])
def test_tick_counts(ctx, nticks):
    """Odd counts start with a single-tick launch, then two ticks per launch."""
    rng = np.random.default_rng(300 + nticks)
    X, Y, Z = 96, 61, 40
    params = O.make_params(3, 0x7, 0x70, 0xF0)  # Moore C=4 B{5,6,7} S{5,6,7,8}: busy every tick
    info = run_and_check(ctx, X, Y, Z, params, random_states(rng, X, Y, Z, 3), nticks, max_ticks=nticks)
    want = O.run_sim(X, Y, Z, params, random_states(np.random.default_rng(300 + nticks), X, Y, Z, 3), nticks,
                     fast=True)[0]
    assert info.as_tuple() == want.as_tuple()


@pytest.mark.parametrize("dims", [(32, 1, 1), (33, 2, 3), (64, 3, 5), (100, 5, 2), (257, 130, 9), (512, 200, 33),
                                  (96, 300, 7), (31, 64, 64)])
def test_pair_tilings(ctx, dims):
    """Grids with fewer rows than a tile, a single plane, one row, partial strips, many y-tiles."""
    X, Y, Z = dims
    rng = np.random.default_rng(X * 7 + Y * 3 + Z)
    run_and_check(ctx, X, Y, Z, O.make_params(5, 0x3, 0x18, 0x3C), random_states(rng, X, Y, Z, 5), 6)


@pytest.mark.parametrize("dims,nticks", [((512, 200, 33), 9), ((512, 90, 150), 10), ((480, 150, 300), 8),
                                         ((64, 40, 1200), 12), ((256, 256, 256), 7)])
def test_long_slab_tilings(ctx, dims, nticks):
    """Slabs of two planes or more with a last slab of one plane, partial strips (480 cells per
    row), one y-tile with 600 small CTAs, many y-tiles; Moore neighbourhood, several launches:
    every tick equals the oracle's."""
    X, Y, Z = dims
    rng = np.random.default_rng(X + 5 * Y + 11 * Z)
    run_and_check(ctx, X, Y, Z, O.make_params(15, 0x7, 0x10, 0x18), random_states(rng, X, Y, Z, 15), nticks)


def test_prepare_then_async(ctx):
    """cave_prepare_rule compiles ahead; an async-mode run of a large grid then uses the kernel."""
    os.environ["CAVE_JIT"] = "async"
    try:
        G = 128  # 2^21 cells: the async threshold
        params = O.make_params(6, 0x3, 0x60, 0x1C0)
        ctx.prepare_rule(cb.SimParams(*[int(v) for v in params]))
        rng = np.random.default_rng(5)
        run_and_check(ctx, G, G, G, params, random_states(rng, G, G, G, 6), 2)
    finally:
        os.environ["CAVE_JIT"] = "sync"


@pytest.mark.parametrize("wrap", [False, True])
def test_render_step(ctx, wrap):
    import torch
    X, Y, Z = 65, 40, 33
    rng = np.random.default_rng(77 + wrap)
    s = np.zeros((Z, Y, X), dtype=np.uint8)
    r = rng.random((Z, Y, X))
    s[r < 0.3] = 5
    mid = (r >= 0.3) & (r < 0.4)
    s[mid] = rng.integers(1, 6, size=int(mid.sum()), dtype=np.uint8)
    params_np = O.make_params(5, 0x3 | (0x8 if wrap else 0), 0x1C, 0x70)
    buf = O.render_pack(s)
    want, want_skip = O.render_step(X, Y, Z, params_np, buf, wrap=wrap, nticks=3, skip=True)
    d_in = torch.from_numpy(buf.view(np.int32)).to("cuda:0")
    d_out = torch.full_like(d_in, -1)
    d_skip = torch.full((cb.render_skip_elements(X, Y, Z),), -1, dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()
    _, l0 = cb.jit_stats()
    cb.render_step(ctx, d_in.data_ptr(), d_out.data_ptr(), X, Y, Z, cb.SimParams(*[int(v) for v in params_np]), 3,
                   d_skip.data_ptr())
    _, l1 = cb.jit_stats()
    assert l1 - l0 == 3
    assert np.array_equal(d_out.cpu().numpy().view(np.uint32), want)
    assert np.array_equal(d_skip.cpu().numpy().view(np.uint32), want_skip)
