"""The C oracle against an independent vectorised restatement of the same tick
(shaders/slang/search/searchSimulationCube.slang:117-247, cube.slang:7-21) over random grids,
neighbourhoods, state counts and rule masks drawn by hypothesis: every cell of the next grid and
every counter must agree, and the counters must satisfy their identities (they partition the
volume; changed = born + dying; population and bounding box are those of the new grid)."""
import numpy as np
from hypothesis import given, settings
from hypothesis import strategies as st

import oracle as O

FACES = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
EDGES = [(dx, dy, 0) for dx in (-1, 1) for dy in (-1, 1)] + [(dx, 0, dz) for dx in (-1, 1) for dz in (-1, 1)] + \
        [(0, dy, dz) for dy in (-1, 1) for dz in (-1, 1)]
CORNERS = [(dx, dy, dz) for dx in (-1, 1) for dy in (-1, 1) for dz in (-1, 1)]


def numpy_tick(s, maxcs, flags, birth, survival):
    """One tick on a (Z, Y, X) array of states: neighbours alive iff their state equals maxcs,
    outside the grid dead; an alive cell survives (stays maxcs) iff n > 0 and survival bit n - 1
    is set, else becomes maxcs - 1; a 0 cell is born (maxcs) iff n > 0 and birth bit n - 1 is
    set; any other state decreases by one; states are stored in 4 bits."""
    Z, Y, X = s.shape
    alive = np.pad((s == maxcs).astype(np.int32), 1)
    deltas = (FACES if flags & 1 else []) + (EDGES if flags & 2 else []) + (CORNERS if flags & 4 else [])
    n = np.zeros((Z, Y, X), dtype=np.int32)
    for dx, dy, dz in deltas:
        n += alive[1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X]
    bit = lambda mask: (n > 0) & ((np.right_shift(np.uint64(mask), np.maximum(n - 1, 0).astype(np.uint64)) & np.uint64(1)) == 1)
    is_alive, is_zero = s == maxcs, s == 0
    surv, born = is_alive & bit(survival), is_zero & bit(birth)
    new = np.where(is_alive, np.where(surv, maxcs, maxcs - 1),
                   np.where(is_zero, np.where(born, maxcs, 0), s.astype(np.int32) - 1))
    new = (new & 0xF).astype(np.uint8)
    counts = (int((is_zero & ~born).sum()), int((~is_zero & ~surv).sum()), int(born.sum()), int(surv.sum()))
    return new, counts


@settings(max_examples=200, deadline=None)
@given(X=st.integers(1, 19), Y=st.integers(1, 9), Z=st.integers(1, 9), flags=st.integers(0, 15),
       maxcs=st.integers(1, 16), birth=st.integers(0, (1 << 27) - 1), survival=st.integers(0, (1 << 27) - 1),
       p_alive=st.floats(0.0, 0.8), seed=st.integers(0, 2 ** 31 - 1))
def test_oracle_equals_vectorised_restatement(X, Y, Z, flags, maxcs, birth, survival, p_alive, seed):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, 16, size=(Z, Y, X), dtype=np.uint8)
    s[rng.random((Z, Y, X)) < p_alive] = maxcs & 0xF
    params = O.make_params(maxcs, flags, birth, survival)
    got, stats = O.step(X, Y, Z, params, O.pack(s))
    want, counts = numpy_tick(s, maxcs, flags & 7, birth, survival)  # the W flag (8) is ignored
    assert np.array_equal(O.unpack(got, X, Y, Z), want)
    assert (stats.dead, stats.dying, stats.born, stats.surviving) == counts
    assert sum(counts) == X * Y * Z and stats.changed == stats.born + stats.dying
    nz = np.argwhere(want != 0)
    assert stats.population == len(nz)
    if len(nz):
        assert tuple(stats.bbox_min) == tuple(int(v) for v in nz.min(axis=0)[::-1])
        assert tuple(stats.bbox_max) == tuple(int(v) for v in nz.max(axis=0)[::-1])
    else:
        assert tuple(stats.bbox_min) == (0xFFFFFFFF,) * 3 and tuple(stats.bbox_max) == (0, 0, 0)


def numpy_run(s, maxcs, flags, birth, survival, max_ticks):
    """searchManager.slang:115-139 over numpy_tick until the status is non-zero; GridInfo as
    (totalDied, totalBorn, ticks, status, maxAlive, finalAlive) and the category of
    searchSystem.cpp:697-711 (0 viable, 1 possible, 2 unviable)."""
    died = born = ticks = max_alive = final = status = 0
    while status == 0:
        s, (dead, _, b, surv) = numpy_tick(s, maxcs, flags, birth, survival)
        ticks += 1
        died += dead
        born += b
        final = surv
        max_alive = max(max_alive, surv)
        status = 1 if surv == 0 and b == 0 else 2 if ticks >= max_ticks else 0
    category = 0 if status == 2 else 1 if ticks > maxcs + 1 else 2
    return (died, born, ticks, status, max_alive, final), category


@settings(max_examples=100, deadline=None)
@given(E=st.integers(2, 9), flags=st.integers(1, 7), maxcs=st.integers(1, 6), birth=st.integers(1, (1 << 26) - 1),
       survival=st.integers(0, (1 << 26) - 1), max_ticks=st.integers(1, 12), seed=st.integers(0, 2 ** 31 - 1))
def test_oracle_lifecycle_equals_restatement(E, flags, maxcs, birth, survival, max_ticks, seed):
    """A rule's whole lifecycle (step until the manager stops it): GridInfo and category."""
    rng = np.random.default_rng(seed)
    s = np.where(rng.random((E, E, E)) < 0.35, maxcs, 0).astype(np.uint8)
    params = O.make_params(maxcs, flags, birth, survival)
    info, _, _ = O.run_sim(E, E, E, params, O.pack(s), max_ticks)
    want_info, want_cat = numpy_run(s, maxcs, flags, birth, survival, max_ticks)
    assert info.as_tuple() == want_info
    assert O.classify(info, maxcs) == want_cat
