"""GPU parity: the CUDA paths against the CPU oracle, bit-exact (integer work).

Every check compares every cell and every statistic after every checked tick.
"""
import numpy as np
import pytest

import cave_b200 as cb
import oracle as O

pytestmark = pytest.mark.gpu

FULL26 = (1 << 26) - 1


def random_states(rng, X, Y, Z, maxcs, p_alive=0.35, p_other=0.15):
    s = np.zeros((Z, Y, X), dtype=np.uint8)
    r = rng.random((Z, Y, X))
    s[r < p_alive] = maxcs & 0xF
    other = (r >= p_alive) & (r < p_alive + p_other)
    s[other] = rng.integers(1, 16, size=int(other.sum()), dtype=np.uint8)
    return O.pack(s)


def stats_tuple(ts):
    return ts.as_tuple()


def oracle_ticks(X, Y, Z, params, init, nticks, valid=None, K=0, fast=False):
    cells, out = init, []
    for _ in range(nticks):
        if fast:
            nxt, snap = O.step_fast(X, Y, Z, params, cells, valid, K)
            out.append((nxt, tuple(int(v) for v in snap)))
        else:
            nxt, st = O.step(X, Y, Z, params, cells, valid, K)
            out.append((nxt, st.as_tuple()))
        cells = nxt
    return out


def check_path(ctx, X, Y, Z, params_np, init, nticks, path, valid=None, K=0, every_tick=True, fast=False):
    p = cb.SimParams(*[int(v) for v in params_np])
    expect = oracle_ticks(X, Y, Z, params_np, init, nticks, valid, K, fast)
    with cb.Grid(ctx, X, Y, Z) as g:
        g.upload(init)
        if every_tick:
            for t in range(nticks):
                st = (g.step(p, 1, valid, K) if path == "step" else g.run(p, 1, 10 ** 6, valid, K)[0])[0]
                cells = g.download()
                assert np.array_equal(cells, expect[t][0]), f"{path}: cells differ at tick {t + 1}"
                got = stats_tuple(st)
                assert got[:len(expect[t][1])] == expect[t][1], f"{path}: stats differ at tick {t + 1}"
        else:
            sts = g.step(p, nticks, valid, K) if path == "step" else g.run(p, nticks, 10 ** 6, valid, K)[0]
            cells = g.download()
            assert np.array_equal(cells, expect[-1][0]), f"{path}: cells differ after {nticks} ticks"
            for t in range(nticks):
                got = stats_tuple(sts[t])
                assert got[:len(expect[t][1])] == expect[t][1], f"{path}: stats differ at tick {t + 1}"


# ---------------------------------------------------------------- config 1 (49^3 FE C=4)
def test_config1_seed_and_20_ticks(ctx):
    G = 49
    thr = O.threshold_from_float(0.30)
    init = O.seed(G, G, G, spawn=(16, 16, 16), random=True, threshold=thr, run_seed=0, max_cell_state=3)
    with cb.Grid(ctx, G, G, G) as g:
        g.seed_threshold((16, 16, 16), thr, 0, 3)
        assert np.array_equal(g.download(), init)
    params = O.make_params(3, 0x3, 0x60, 0x70)
    for path in ("step", "run"):
        check_path(ctx, G, G, G, params, init, 20, path)


# ---------------------------------------------------------------- shapes x neighbourhoods x rules
SHAPES = [(1, 1, 1), (8, 8, 8), (9, 9, 9), (17, 17, 17), (33, 33, 33), (31, 2, 5), (64, 3, 7), (65, 9, 4),
          (100, 37, 20)]


@pytest.mark.parametrize("dims", SHAPES)
@pytest.mark.parametrize("flags", [0, 1, 2, 3, 4, 5, 6, 7, 0xB, 0xF])
def test_shapes_flags_random_rules(ctx, dims, flags):
    X, Y, Z = dims
    rng = np.random.default_rng((X * 131 + Y * 17 + Z) * 16 + flags)
    for maxcs, dense in ((1, False), (3, True), (15, False), (16, True), (7, False)):
        init = random_states(rng, X, Y, Z, maxcs)
        if dense:
            B, S = int(rng.integers(0, FULL26)), int(rng.integers(0, FULL26))
        else:
            B = sum(1 << int(b) for b in rng.choice(26, size=int(rng.integers(1, 4)), replace=False))
            S = sum(1 << int(b) for b in rng.choice(26, size=int(rng.integers(1, 4)), replace=False))
        params = O.make_params(maxcs, flags, B, S)
        for path in ("step", "run"):
            check_path(ctx, X, Y, Z, params, init, 3, path)


def test_k_index_rules(ctx):
    X = Y = Z = 25
    rng = np.random.default_rng(11)
    for flags, n in ((1, 6), (2, 12), (3, 18), (7, 26)):
        vb = O.valid_bitmasks(n, 2)
        init = random_states(rng, X, Y, Z, 3)
        for _ in range(3):
            bi, si = int(rng.integers(0, len(vb))), int(rng.integers(0, len(vb)))
            params = O.make_params(3, flags, bi + 1, si + 1)
            for path in ("step", "run"):
                check_path(ctx, X, Y, Z, params, init, 2, path, valid=vb, K=2)


def test_bad_k_index_rejected(ctx):
    vb = O.valid_bitmasks(6, 2)
    with cb.Grid(ctx, 9, 9, 9) as g:
        for fn in (lambda p: g.step(p, 1, vb, 2), lambda p: g.run(p, 1, 10, vb, 2)):
            with pytest.raises(cb.CaveError) as e:
                fn(cb.make_params(3, 1, 22, 1))  # index 22 > 21 masks
            assert e.value.code == cb.ERR_INVALID_ARG


# ---------------------------------------------------------------- larger grids (streaming tiles)
@pytest.mark.parametrize("G", [96, 128, 200])
def test_config2_shape_reduced(ctx, G):
    """Moore-26, C=16 (maxCS 15), survive {4,5}, birth {5}, 40% fill over the whole volume."""
    thr = O.threshold_from_float(0.40)
    init = O.seed(G, G, G, random=True, threshold=thr, run_seed=0, max_cell_state=15)
    params = O.make_params(15, 0x7, 0x10, 0x18)
    check_path(ctx, G, G, G, params, init, 6, "run", every_tick=False, fast=True)


def test_wide_rows_1024(ctx):
    X, Y, Z = 1024, 6, 5
    rng = np.random.default_rng(3)
    init = random_states(rng, X, Y, Z, 4)
    params = O.make_params(4, 7, 0b11100, 0b1111000)
    for path in ("step", "run"):
        check_path(ctx, X, Y, Z, params, init, 3, path)


@pytest.mark.parametrize("dims", [(512, 70, 5), (1024, 40, 4), (480, 95, 7)])
def test_wide_rows_many_tiles(ctx, dims):
    """Wide rows split into several y-tiles: halo rows are real rows of the neighbouring tile
    and must be neither double-counted nor read past the exchange buffer."""
    X, Y, Z = dims
    rng = np.random.default_rng(X + Y)
    init = random_states(rng, X, Y, Z, 15)
    params = O.make_params(15, 7, 0x10, 0x18)
    check_path(ctx, X, Y, Z, params, init, 4, "run", every_tick=False)


# ---------------------------------------------------------------- seeding
@pytest.mark.parametrize("dims", [(49, 49, 49), (25, 25, 25), (33, 40, 17)])
@pytest.mark.parametrize("random_fill,density_index,seed,size_index", [(0, 15, 0, 0), (1, 7, 3, 0), (1, 2, 9, 5),
                                                                        (1, 15, 0, 0)])
def test_device_seeding_matches_reference_hash(ctx, dims, random_fill, density_index, seed, size_index):
    X, Y, Z = dims
    spawn = (min(16, X), min(11, Y), min(20, Z))
    c = cb.ChunkConfig(0, X, Y, Z, spawn[0], spawn[1], spawn[2], 0, 0 if random_fill else 1, size_index,
                       density_index, seed, 0, 1)
    thr = O.threshold_from_index(density_index) if random_fill else 1 << 32
    expect = O.seed(X, Y, Z, spawn=spawn, spawn_size_index=size_index, random=bool(random_fill), threshold=thr,
                    run_seed=seed, max_cell_state=5)
    with cb.Grid(ctx, X, Y, Z) as g:
        g.seed(c, 5)
        assert np.array_equal(g.download(), expect)


# ---------------------------------------------------------------- tile shapes
def test_tile_timing_pass_and_shapes(ctx, monkeypatch):
    """A long run of a large grid goes through cave_run's tile timing pass (the trial ticks must
    leave the input and the statistics untouched), and every tile shape gives the same cells and
    statistics."""
    G, T = 128, 100  # 2^21 cells and 100 ticks: the smallest run that is tuned
    thr = O.threshold_from_float(0.40)
    init = O.seed(G, G, G, random=True, threshold=thr, run_seed=3, max_cell_state=15)
    params_np = O.make_params(15, 0x7, 0x10, 0x18)
    cells, expect = init, []
    for _ in range(T):
        cells, snap = O.step_fast(G, G, G, params_np, cells)
        expect.append(tuple(int(v) for v in snap))
    p = cb.SimParams(*[int(v) for v in params_np])
    for rows in (None, 8, 12, 20):
        if rows is None:
            monkeypatch.delenv("CAVE_STREAM_ROWS", raising=False)
        else:
            monkeypatch.setenv("CAVE_STREAM_ROWS", str(rows))
        with cb.Grid(ctx, G, G, G) as g:
            g.upload(init)
            sts, _ = g.run(p, T, 10 ** 6)
            assert np.array_equal(g.download(), cells), f"rows {rows}: cells differ after {T} ticks"
        for t in range(T):
            got = sts[t].as_tuple()
            assert got[:len(expect[t])] == expect[t], f"rows {rows}: statistics differ at tick {t + 1}"
