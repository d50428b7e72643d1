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


@settings(max_examples=1000, deadline=None)
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


@settings(max_examples=500, deadline=None)
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


def numpy_seed(X, Y, Z, spawn, size_index, random, density_index, run_seed, maxcs):
    """The initial cells of searchSystem.cpp:219-306 (cube layout), vectorised: the spawn box
    centred in the grid (scaled by the size index), cells inside it alive when the cell hash is
    below the density threshold (or always when the spawn is filled), packed 8 per word."""
    def dim(axis, d):
        if size_index == 0:
            return axis
        return max(1, min(axis, (axis * (size_index + 1) + 15) // 16))

    ex, ey, ez = (dim(min(s, d), d) for s, d in zip(spawn, (X, Y, Z)))
    density = np.float32(density_index + 1) / np.float32(16)
    threshold = 0xFFFFFFFF if density >= 1 else int(np.float64(density) * 4294967296.0)

    def wang(v):
        v = (v ^ np.uint32(61)) ^ (v >> np.uint32(16))
        v = v * np.uint32(9)
        v = v ^ (v >> np.uint32(4))
        v = v * np.uint32(0x27D4EB2D)
        return v ^ (v >> np.uint32(15))

    z, y, x = np.meshgrid(np.arange(Z, dtype=np.uint32), np.arange(Y, dtype=np.uint32),
                          np.arange(X, dtype=np.uint32), indexing="ij")
    with np.errstate(over="ignore"):
        h = wang(x * np.uint32(73856093) + np.uint32(run_seed))
        h = wang(h ^ (y * np.uint32(19349663)))
        h = wang(h ^ (z * np.uint32(83492791)))
    inside = ((x >= (X - ex) // 2) & (x < (X + ex) // 2) & (y >= (Y - ey) // 2) & (y < (Y + ey) // 2) &
              (z >= (Z - ez) // 2) & (z < (Z + ez) // 2))
    alive = inside & ((density >= 1) | (h < np.uint32(threshold)) if random else inside)
    return O.pack(np.where(alive, maxcs & 0xF, 0).astype(np.uint8))


@settings(max_examples=500, deadline=None)
@given(X=st.integers(1, 21), Y=st.integers(1, 11), Z=st.integers(1, 11), spawn=st.tuples(*[st.integers(1, 21)] * 3),
       size_index=st.integers(0, 15), random=st.booleans(), density_index=st.integers(0, 15),
       run_seed=st.integers(0, 2 ** 32 - 1), maxcs=st.integers(1, 16))
def test_oracle_seed_equals_restatement(X, Y, Z, spawn, size_index, random, density_index, run_seed, maxcs):
    got = O.seed(X, Y, Z, spawn=spawn, spawn_size_index=size_index, random=random,
                 threshold=O.threshold_from_index(density_index), run_seed=run_seed, max_cell_state=maxcs)
    want = numpy_seed(X, Y, Z, spawn, size_index, random, density_index, run_seed, maxcs)
    assert np.array_equal(got, want)


@settings(max_examples=300, deadline=None)
@given(G=st.integers(3, 8), flags=st.integers(1, 7), maxcs=st.integers(1, 4), kindex=st.booleans(),
       b0=st.integers(1, 6), s0=st.integers(1, 4), maxp=st.integers(1, 6), s_extra=st.integers(0, 2),
       max_ticks=st.integers(1, 8), seed=st.integers(0, 1000))
def test_slot_pipeline_walks_next_permutation_in_order(G, flags, maxcs, kindex, b0, s0, maxp, s_extra, max_ticks,
                                                       seed):
    """The literal SearchSystem slot (oracle_run_slot: reset, tick, manager and host read-back of
    searchSystem.cpp:480-713 with NextPermutation, searchManager.slang:56-96) reports exactly the
    rules of the permutation walk -- birth index from its start to maxPermutation, then the next
    survival index with birth 1, up to survivalEnd -- in that order, once each, and each with the
    result of running that rule alone from the initial cells."""
    b0 = min(b0, maxp)
    s_end = s0 + s_extra
    valid = O.valid_bitmasks(6, 2) if kindex else None
    init = O.seed(G, G, G, spawn=(G // 2 + 1,) * 3, random=True, threshold=1 << 31, run_seed=seed,
                  max_cell_state=maxcs)
    res = O.run_slot(G, G, G, ((maxcs - 1) << 60) | b0, (flags << 60) | s0, maxp, s_end, init, max_ticks,
                     valid=valid, max_rule_bits=2 if kindex else 0)
    walk = [(s0, b) for b in range(b0, maxp + 1)] + [(s, b) for s in range(s0 + 1, s_end + 1)
                                                      for b in range(1, maxp + 1)]
    assert len(res) == len(walk)
    for r, (s, b) in zip(res, walk):
        bm = int(valid[b - 1]) if kindex else b
        sm = int(valid[s - 1]) if kindex else s
        assert r.birthAndMaxCellStateRules == ((maxcs - 1) << 60) | bm
        assert r.survivalAndNeighborhoodRules == (flags << 60) | sm
        p = O.make_params(maxcs, flags, bm, sm)
        info, _, _ = O.run_sim(G, G, G, p, init, max_ticks)
        assert r.info.as_tuple() == info.as_tuple()
        assert r.category == O.classify(info, maxcs)
