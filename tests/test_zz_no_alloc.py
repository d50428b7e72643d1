"""cave_run_noalloc (static scratch, caller-owned device buffers) against cave_run.

Integer work, so the tolerance is exact: every cell, every per-tick statistic and the
GridInfo must equal cave_run's on the same inputs. The calls run back to back so that each
one starts from the scratch contents the previous call left behind.
"""
import ctypes

import numpy as np
import pytest

import cave_b200 as cb
import oracle as O

pytestmark = pytest.mark.gpu

TICK_BYTES = ctypes.sizeof(cb.TickStats)


def _torch():
    import torch
    return torch


def random_cells(rng, X, Y, Z, maxcs):
    s = np.zeros((Z, Y, X), dtype=np.uint8)
    r = rng.random((Z, Y, X))
    s[r < 0.35] = maxcs & 0xF
    other = (r >= 0.35) & (r < 0.5)
    s[other] = rng.integers(1, 16, size=int(other.sum()), dtype=np.uint8)
    return O.pack(s)


def reference_run(ctx, X, Y, Z, init, params, nticks, max_ticks, valid=None, K=0):
    with cb.Grid(ctx, X, Y, Z) as g:
        g.upload(init)
        ticks, info = g.run(params, nticks, max_ticks, valid, K)
        return g.download(), [bytes(t) for t in ticks], bytes(info)


def noalloc_run(ctx, X, Y, Z, init, params, nticks, max_ticks, valid=None, K=0, in_place=False):
    torch = _torch()
    d_in = torch.from_numpy(init.view(np.int32)).to("cuda:0")
    d_out = d_in if in_place else torch.full_like(d_in, -1)
    d_ticks = torch.full((max(nticks, 1) * TICK_BYTES,), 0xAB, dtype=torch.uint8, device="cuda:0")
    torch.cuda.synchronize()
    info = cb.run_noalloc(ctx, d_in.data_ptr(), d_out.data_ptr(), X, Y, Z, params, nticks, max_ticks, valid, K,
                          d_ticks.data_ptr())
    cells = d_out.cpu().numpy().view(np.uint32)
    raw = d_ticks.cpu().numpy().tobytes()
    return cells, [raw[i * TICK_BYTES:(i + 1) * TICK_BYTES] for i in range(nticks)], bytes(info)


def _case_seeded49():
    G = 49
    init = O.seed(G, G, G, spawn=(16, 16, 16), random=True, threshold=O.threshold_from_float(0.30), run_seed=0,
                  max_cell_state=3)
    return (G, G, G, init, cb.make_params(3, 0x3, 0x60, 0x70), 20, 20, None, 0)


def _case_moore_dense():
    rng = np.random.default_rng(11)
    X, Y, Z = 100, 37, 20
    init = random_cells(rng, X, Y, Z, 16)
    # birth/survive sets with many counts (mux-tree rule evaluation)
    return (X, Y, Z, init, cb.make_params(16, 0x7, 0x2AAAAA8, 0x1555554), 7, 5, None, 0)


def _case_kindex():
    rng = np.random.default_rng(5)
    X, Y, Z = 70, 40, 33
    init = random_cells(rng, X, Y, Z, 6)
    valid = cb.valid_bitmasks(18, 3)
    return (X, Y, Z, init, cb.make_params(6, 0x3, 17, 3), 9, 9, valid, 3)


def _check(ctx, case, in_place=False):
    X, Y, Z, init, params, nticks, max_ticks, valid, K = case
    want = reference_run(ctx, X, Y, Z, init, params, nticks, max_ticks, valid, K)
    got = noalloc_run(ctx, X, Y, Z, init, params, nticks, max_ticks, valid, K, in_place)
    assert np.array_equal(got[0], want[0]), "cells differ from cave_run"
    assert got[1] == want[1], "per-tick statistics differ from cave_run"
    assert got[2] == want[2], "GridInfo differs from cave_run"


def test_two_calls_in_a_row(ctx):
    a = _case_seeded49()
    _check(ctx, a)
    _check(ctx, a)


def test_calls_over_different_shapes_and_rules(ctx):
    for case in (_case_moore_dense(), _case_kindex(), _case_seeded49(), _case_moore_dense()):
        _check(ctx, case)


def test_in_place(ctx):
    _check(ctx, _case_kindex(), in_place=True)
    _check(ctx, _case_kindex(), in_place=True)


def test_256_cubed_fits(ctx):
    G = 256
    rng = np.random.default_rng(2)
    init = random_cells(rng, G, G, G, 16)
    case = (G, G, G, init, cb.make_params(16, 0x7, 1 << 4, (1 << 3) | (1 << 4)), 3, 3, None, 0)
    _check(ctx, case)
    _check(ctx, case)


def test_no_stats_outputs(ctx):
    torch = _torch()
    X, Y, Z, init, params, nticks, max_ticks, _, _ = _case_seeded49()
    want = reference_run(ctx, X, Y, Z, init, params, nticks, max_ticks)
    d_in = torch.from_numpy(init.view(np.int32)).to("cuda:0")
    d_out = torch.zeros_like(d_in)
    torch.cuda.synchronize()
    rc = cb.lib().cave_run_noalloc(ctx.h, ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(d_out.data_ptr()), X, Y,
                                   Z, ctypes.byref(params), None, 0, 0, nticks, max_ticks, None, None)
    assert rc == cb.OK
    assert np.array_equal(d_out.cpu().numpy().view(np.uint32), want[0])


def test_rejects_grid_above_scratch_limit(ctx):
    torch = _torch()
    buf = torch.zeros(64, dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()
    with pytest.raises(cb.CaveError) as e:
        cb.run_noalloc(ctx, buf.data_ptr(), buf.data_ptr(), 1024, 1024, 40, cb.make_params(16, 0x7, 16, 24), 1)
    assert e.value.code == 1  # CAVE_ERR_INVALID_ARG
    assert "maximum" in str(e.value)


def test_rejects_host_buffers(ctx):
    X = Y = Z = 8
    host = np.zeros(cb.grid_words(X, Y, Z), dtype=np.uint32)
    with pytest.raises(cb.CaveError) as e:
        cb.run_noalloc(ctx, host.ctypes.data, host.ctypes.data, X, Y, Z, cb.make_params(16, 0x7, 16, 24), 1)
    assert "device memory" in str(e.value)


def test_call_allocates_no_device_memory(ctx):
    """A call after the first one on the device leaves the device's free memory unchanged:
    nothing is allocated or freed on the device. The first call (which loads the scratch array's
    module and the kernels it uses) has the same rule, so the measured call of another grid shape
    needs no kernel that is not loaded yet."""
    torch = _torch()
    X, Y, Z, init, params, nticks, max_ticks, valid, K = _case_kindex()
    noalloc_run(ctx, X, Y, Z, init, params, nticks, max_ticks, valid, K)
    X2, Y2, Z2 = 50, 30, 41
    init2 = random_cells(np.random.default_rng(9), X2, Y2, Z2, 6)
    d_in = torch.from_numpy(init2.view(np.int32)).to("cuda:0")
    d_out = torch.zeros_like(d_in)
    d_ticks = torch.zeros(nticks * TICK_BYTES, dtype=torch.uint8, device="cuda:0")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    cb.run_noalloc(ctx, d_in.data_ptr(), d_out.data_ptr(), X2, Y2, Z2, params, nticks, max_ticks, valid, K,
                   d_ticks.data_ptr())
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
    want = reference_run(ctx, X2, Y2, Z2, init2, params, nticks, max_ticks, valid, K)
    assert np.array_equal(d_out.cpu().numpy().view(np.uint32), want[0]), "cells differ from cave_run"


def test_rejects_memory_of_another_gpu(ctx):
    """A buffer on another GPU is refused before anything is launched."""
    torch = _torch()
    if torch.cuda.device_count() < 2:
        pytest.skip("needs a second GPU")
    X = Y = Z = 8
    other = torch.zeros(cb.grid_words(X, Y, Z), dtype=torch.int32, device="cuda:1")
    mine = torch.zeros_like(other, device="cuda:0")
    torch.cuda.synchronize(0)
    torch.cuda.synchronize(1)
    for a, b in ((other, mine), (mine, other)):
        with pytest.raises(cb.CaveError) as e:
            cb.run_noalloc(ctx, a.data_ptr(), b.data_ptr(), X, Y, Z, cb.make_params(16, 0x7, 16, 24), 1)
        assert e.value.code == 1  # CAVE_ERR_INVALID_ARG
        assert "context's device" in str(e.value)
