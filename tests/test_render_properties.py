"""The render-mode oracle against an independent vectorised restatement (numpy, written here from
the shaders, not from the oracle), on hypothesis-drawn grids, rules and neighbourhoods, with
wrap-around on and off:

* layout: cellStateUtils.slang:18-54 -- 2 cells per texel along x (low nibble even x), 8^3-texel
  blocks in x, y, z order, Morton order inside a block (x bit 0, y bit 1, z bit 2 of each bit
  triplet), block padding 0;
* tick: rayMarchCompute.slang:80-113 (neighbour alive test; with WRAP_AT_BOUNDARY every axis
  wraps, else out-of-grid is not alive) and :121-179 (count over the selected face, edge and
  corner deltas; survive, birth and decay exactly as the search tick);
* skip grid: :182-205 -- every cell non-zero after the tick marks the 8-cell chunks from
  floor((c - 1) / 8) to floor((c + 1) / 8) per axis, clamped to the skip grid (never wrapped),
  in the same tiled layout over the skip grid's own dimensions.
Every element of the output buffer and of the skip grid must be equal. Integer work: exact."""
import numpy as np
from hypothesis import given, settings
from hypothesis import strategies as st

import oracle as O

PERM = (1 << 60) - 1


def _morton(x, y, z):
    m = np.zeros_like(x)
    for b in range(3):
        m |= ((x >> b) & 1) << (3 * b)
        m |= ((y >> b) & 1) << (3 * b + 1)
        m |= ((z >> b) & 1) << (3 * b + 2)
    return m


def _tiled(tx, ty, tz, dims):
    """Element index of texel (tx, ty, tz) of a texel grid with dimensions dims = (W, H, D)."""
    nbx, nby = -(-dims[0] // 8), -(-dims[1] // 8)
    block = (tz // 8) * nbx * nby + (ty // 8) * nbx + (tx // 8)
    return block * 512 + _morton(tx % 8, ty % 8, tz % 8)


def _elements(dims):
    return (-(-dims[0] // 8)) * (-(-dims[1] // 8)) * (-(-dims[2] // 8)) * 512


def _pack(s):
    Z, Y, X = s.shape
    W = (X + 1) // 2
    full = np.zeros((Z, Y, 2 * W), dtype=np.int64)
    full[:, :, :X] = s
    texel = full[:, :, 0::2] | (full[:, :, 1::2] << 4)
    tz, ty, tx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(W), indexing="ij")
    buf = np.zeros(_elements((W, Y, Z)), dtype=np.uint32)
    buf[_tiled(tx, ty, tz, (W, Y, Z)).ravel()] = texel.ravel()
    return buf


def _deltas(flags):
    out = []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                k = (dx != 0) + (dy != 0) + (dz != 0)
                if k and (flags >> (k - 1)) & 1:  # k = 1 face, 2 edge, 3 corner
                    out.append((dx, dy, dz))
    return out


def _tick(s, maxcs, flags, birth, survival, wrap):
    Z, Y, X = s.shape
    alive = (s == maxcs).astype(np.int64)
    n = np.zeros_like(alive)
    for dx, dy, dz in _deltas(flags):
        if wrap:
            n += np.roll(alive, shift=(-dz, -dy, -dx), axis=(0, 1, 2))  # alive at (c + d) mod dims
        else:
            p = np.pad(alive, 1)
            n += p[1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X]
    hit = lambda mask: (n > 0) & ((mask >> np.maximum(n - 1, 0)) & 1).astype(bool)
    return np.where(s == maxcs, np.where(hit(survival), maxcs, maxcs - 1),
                    np.where(s == 0, np.where(hit(birth), maxcs, 0), s - 1)).astype(np.int64)


def _skip(new):
    Z, Y, X = new.shape
    dims = (-(-X // 8), -(-Y // 8), -(-Z // 8))
    marked = np.zeros((dims[2], dims[1], dims[0]), dtype=bool)
    for z, y, x in np.argwhere(new != 0):
        lo = [max((c - 1) // 8, 0) for c in (x, y, z)]
        hi = [min((c + 1) // 8, d - 1) for c, d in zip((x, y, z), dims)]
        marked[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = True
    buf = np.zeros(_elements(dims), dtype=np.uint32)
    k, j, i = np.nonzero(marked)
    buf[_tiled(i, j, k, dims)] = 1
    return buf


@settings(max_examples=300, deadline=None)
@given(X=st.integers(1, 21), Y=st.integers(1, 19), Z=st.integers(1, 17), flags=st.integers(1, 7),
       maxcs=st.integers(1, 15), birth=st.integers(0, (1 << 26) - 1), survival=st.integers(0, (1 << 26) - 1),
       wrap=st.booleans(), p_alive=st.floats(0.0, 0.6), seed=st.integers(0, 2**31 - 1))
def test_render_oracle_equals_restatement(X, Y, Z, flags, maxcs, birth, survival, wrap, p_alive, seed):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, maxcs + 1, size=(Z, Y, X)).astype(np.int64)
    s[rng.random((Z, Y, X)) < p_alive] = maxcs
    params = O.make_params(maxcs, flags, birth, survival)
    assert int(params[0]) & PERM == birth and int(params[1]) & PERM == survival
    buf = _pack(s)
    assert np.array_equal(buf, O.render_pack(s.astype(np.uint8)))  # layouts agree
    out, skip = O.render_step(X, Y, Z, params, buf, wrap=wrap, skip=True)
    new = _tick(s, maxcs, flags, birth, survival, wrap)
    assert np.array_equal(out, _pack(new))
    assert np.array_equal(skip, _skip(new))
