"""cave_render_step (the render mode's tick on its Morton-tiled buffer, with and without
wrap-around) against the oracle's restatement of rayMarchCompute.slang: every buffer element
(block padding included) and every skip-grid element, bit-exact."""
import numpy as np
import pytest

import cave_b200 as cb
import oracle as O

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def random_states(rng, X, Y, Z, maxcs):
    s = np.zeros((Z, Y, X), dtype=np.uint8)
    r = rng.random((Z, Y, X))
    s[r < 0.3] = maxcs & 0xF
    mid = (r >= 0.3) & (r < 0.4)
    s[mid] = rng.integers(1, 16, size=int(mid.sum()), dtype=np.uint8)
    return s


def device_step(ctx, buf, X, Y, Z, params, nticks, with_skip=True, in_place=False):
    torch = _torch()
    d_in = torch.from_numpy(buf.view(np.int32)).to("cuda:0")
    d_out = d_in if in_place else torch.full_like(d_in, -1)
    d_skip = torch.full((cb.render_skip_elements(X, Y, Z),), -1, dtype=torch.int32, device="cuda:0") if with_skip \
        else None
    torch.cuda.synchronize()
    cb.render_step(ctx, d_in.data_ptr(), d_out.data_ptr(), X, Y, Z, params, nticks,
                   d_skip.data_ptr() if with_skip else None)
    out = d_out.cpu().numpy().view(np.uint32)
    skip = d_skip.cpu().numpy().view(np.uint32) if with_skip else None
    return out, skip


CASES = [
    ((9, 5, 3), 0x7, 1, 3), ((31, 17, 12), 0x3, 3, 4), ((32, 32, 8), 0x1, 2, 2), ((33, 9, 20), 0x7, 15, 3),
    ((63, 12, 10), 0x2, 4, 2), ((64, 8, 16), 0x5, 7, 3), ((100, 30, 7), 0x6, 1, 2), ((2, 2, 2), 0x7, 2, 2),
    ((1, 1, 1), 0x7, 1, 2), ((65, 64, 65), 0x3, 3, 1),
]


@pytest.mark.parametrize("wrap", [False, True])
@pytest.mark.parametrize("dims,flags,maxcs,nticks", CASES)
def test_render_step_matches_oracle(ctx, dims, flags, maxcs, nticks, wrap):
    X, Y, Z = dims
    rng = np.random.default_rng(X * 131 + Y * 7 + Z + flags + (100 if wrap else 0))
    nb = (6 if flags & 1 else 0) + (12 if flags & 2 else 0) + (8 if flags & 4 else 0)
    B = sum(1 << int(v) for v in rng.choice(nb, size=min(3, nb), replace=False))
    S = sum(1 << int(v) for v in rng.choice(nb, size=min(3, nb), replace=False))
    params_np = O.make_params(maxcs, flags | (0x8 if wrap else 0), B, S)
    buf = O.render_pack(random_states(rng, X, Y, Z, maxcs))
    want, want_skip = O.render_step(X, Y, Z, params_np, buf, wrap=wrap, nticks=nticks, skip=True)
    got, got_skip = device_step(ctx, buf, X, Y, Z, cb.SimParams(*[int(v) for v in params_np]), nticks)
    assert np.array_equal(got, want)
    assert np.array_equal(got_skip, want_skip)


def test_in_place_and_zero_ticks(ctx):
    X, Y, Z = 40, 21, 13
    rng = np.random.default_rng(5)
    params_np = O.make_params(4, 0xF, 0b1100100, 0b111000)
    buf = O.render_pack(random_states(rng, X, Y, Z, 4))
    want, _ = O.render_step(X, Y, Z, params_np, buf, wrap=True, nticks=2)
    got, _ = device_step(ctx, buf, X, Y, Z, cb.SimParams(*[int(v) for v in params_np]), 2, in_place=True)
    assert np.array_equal(got, want)
    same, _ = device_step(ctx, buf, X, Y, Z, cb.SimParams(*[int(v) for v in params_np]), 0)
    assert np.array_equal(same, buf)


def test_widest_wrapped_grid_and_rejection(ctx):
    torch = _torch()
    rng = np.random.default_rng(9)
    X, Y, Z = 1022, 3, 2
    params_np = O.make_params(2, 0x1 | 0x8, 0b11, 0b1)
    buf = O.render_pack(random_states(rng, X, Y, Z, 2))
    want, _ = O.render_step(X, Y, Z, params_np, buf, wrap=True, nticks=1)
    got, _ = device_step(ctx, buf, X, Y, Z, cb.SimParams(*[int(v) for v in params_np]), 1, with_skip=False)
    assert np.array_equal(got, want)
    n = cb.render_buffer_elements(1023, 3, 2)
    d = torch.zeros(n, dtype=torch.int32, device="cuda:0")
    with pytest.raises(cb.CaveError):
        cb.render_step(ctx, d.data_ptr(), d.data_ptr(), 1023, 3, 2, cb.SimParams(*[int(v) for v in params_np]), 1)
