"""The render-mode oracle (rayMarchCompute.slang computeMain + cellStateUtils.slang layout):
layout round trips, agreement with the search step when nothing wraps, and hand-derived known
answers for wrap-around and the skip grid."""
import numpy as np
import pytest

import oracle as O


@pytest.mark.parametrize("dims", [(1, 1, 1), (9, 5, 3), (17, 8, 8), (33, 20, 11), (16, 16, 16)])
def test_layout_round_trip(dims):
    X, Y, Z = dims
    s = np.random.default_rng(sum(dims)).integers(0, 16, size=(Z, Y, X)).astype(np.uint8)
    buf = O.render_pack(s)
    assert buf.size == O.render_elements(X, Y, Z)
    assert np.array_equal(O.render_unpack(buf, X, Y, Z), s)
    idx = O.render_indices(X, Y, Z)
    used = np.zeros(buf.size, dtype=bool)
    used[idx.reshape(-1)] = True
    assert np.all(buf[~used] == 0)  # block padding
    assert len(np.unique(idx)) == idx.size


def test_morton_order_inside_a_block():
    # x bit 0, y bit 1, z bit 2 of each coordinate triplet (cellStateUtils.slang:28-34)
    assert O.lib().oracle_render_index(1, 0, 0, 16, 8, 8) == 1
    assert O.lib().oracle_render_index(0, 1, 0, 16, 8, 8) == 2
    assert O.lib().oracle_render_index(0, 0, 1, 16, 8, 8) == 4
    assert O.lib().oracle_render_index(2, 0, 0, 16, 8, 8) == 8
    assert O.lib().oracle_render_index(7, 7, 7, 16, 8, 8) == 511
    assert O.lib().oracle_render_index(0, 0, 0, 32, 8, 8) == 0
    assert O.lib().oracle_render_index(8, 0, 0, 32, 8, 8) == 512  # second block along x


@pytest.mark.parametrize("flags", [1, 2, 3, 4, 7])
def test_no_wrap_equals_search_step(flags):
    X, Y, Z = 19, 10, 9
    rng = np.random.default_rng(flags)
    s = np.zeros((Z, Y, X), dtype=np.uint8)
    s[rng.random((Z, Y, X)) < 0.35] = 5
    s[rng.random((Z, Y, X)) < 0.1] = 2
    p = O.make_params(5, flags, 0b1011010, 0b110101)
    out, _ = O.render_step(X, Y, Z, p, O.render_pack(s), wrap=False)
    ref, _ = O.step(X, Y, Z, p, O.pack(s))
    assert np.array_equal(O.render_unpack(out, X, Y, Z), O.unpack(ref, X, Y, Z))


def test_wrap_births_across_the_boundary():
    # one alive cell at the origin, faces neighbourhood, birth on exactly one neighbour:
    # with wrap the cells at x = X-1, y = Y-1, z = Z-1 are born too
    X, Y, Z = 6, 5, 4
    s = np.zeros((Z, Y, X), dtype=np.uint8)
    s[0, 0, 0] = 1
    p = O.make_params(1, 0x1 | 0x8, 0b1, 0)
    wrapped, _ = O.render_step(X, Y, Z, p, O.render_pack(s), wrap=True)
    w = O.render_unpack(wrapped, X, Y, Z)
    expect = {(0, 0, 1), (0, 1, 0), (1, 0, 0), (0, 0, X - 1), (0, Y - 1, 0), (Z - 1, 0, 0)}
    assert {tuple(int(v) for v in c) for c in np.argwhere(w == 1)} == expect
    flat, _ = O.render_step(X, Y, Z, p, O.render_pack(s), wrap=False)
    assert {tuple(int(v) for v in c) for c in np.argwhere(O.render_unpack(flat, X, Y, Z) == 1)} == {
        (0, 0, 1), (0, 1, 0), (1, 0, 0)}


def test_skip_grid_marks_chunks_within_one_cell():
    X, Y, Z = 24, 16, 16
    s = np.zeros((Z, Y, X), dtype=np.uint8)
    s[4, 4, 8] = 2  # decays to 1: still non-zero after the tick, at x = 8 (chunk 1, next to chunk 0)
    p = O.make_params(3, 0x1, 0, 0)
    out, skip = O.render_step(X, Y, Z, p, O.render_pack(s), wrap=False, skip=True)
    marked = set()
    sx, sy, sz = 3, 2, 2
    for k in range(sz):
        for j in range(sy):
            for i in range(sx):
                # the skip grid is tiled like a texel grid of width sx (X = 2 * sx)
                e = O.lib().oracle_render_index(i, j, k, sx * 2, sy, sz)
                if skip[e]:
                    marked.add((i, j, k))
    assert marked == {(0, 0, 0), (1, 0, 0)}
