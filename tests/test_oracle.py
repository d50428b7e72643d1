"""Known-answer and property tests of the CPU oracle (the parity reference).

Hand-derived expectations follow the reference shader rules
(shaders/slang/search/searchSimulationCube.slang:78-247, searchManager.slang:56-149,
permutationMath.h:101-128, searchSystem.cpp:219-306).
"""
import numpy as np
import pytest

import oracle as O


def states(cells, X, Y, Z):
    return O.unpack(cells, X, Y, Z)


def grid_with(X, Y, Z, cells_and_states):
    s = np.zeros((Z, Y, X), dtype=np.uint8)
    for (x, y, z), v in cells_and_states:
        s[z, y, x] = v
    return O.pack(s)


# ---- permutationMath.h:94-98 documents these sizes
@pytest.mark.parametrize("n,k,count", [(6, 2, 21), (12, 2, 78), (18, 2, 171), (14, 2, 105), (26, 2, 351),
                                       (26, 4, 17901)])
def test_valid_bitmask_counts(n, k, count):
    v = O.valid_bitmasks(n, k)
    assert len(v) == count
    assert np.all(np.diff(v.astype(np.int64)) > 0)  # sorted ascending, unique
    assert 0 not in v
    assert all(1 <= bin(int(m)).count("1") <= k for m in v)
    assert int(v.max()) < (1 << n)


def test_valid_bitmask_order_small():
    # N=3, K=2: {1,2,4} U {3,5,6} sorted
    assert O.valid_bitmasks(3, 2).tolist() == [1, 2, 3, 4, 5, 6]
    assert O.valid_bitmasks(3, 0).tolist() == []


# ---- single cells
def test_single_cell_faces_birth():
    X = Y = Z = 5
    g = grid_with(X, Y, Z, [((2, 2, 2), 1)])
    p = O.make_params(1, 1, birth=0b1, survival=0)  # birth on exactly 1 neighbour
    out, st = O.step(X, Y, Z, p, g)
    s = states(out, X, Y, Z)
    born = {(2 + dx, 2 + dy, 2 + dz) for dx, dy, dz in [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1),
                                                       (0, 0, -1)]}
    for z in range(Z):
        for y in range(Y):
            for x in range(X):
                assert s[z, y, x] == (1 if (x, y, z) in born else 0)
    assert (st.born, st.surviving, st.dying) == (6, 0, 1)
    assert st.dead == X * Y * Z - 7
    assert st.population == 6 and st.changed == 7
    assert tuple(st.bbox_min) == (1, 1, 1) and tuple(st.bbox_max) == (3, 3, 3)


def test_corner_cell_moore_zero_boundary():
    X = Y = Z = 4
    g = grid_with(X, Y, Z, [((0, 0, 0), 2)])
    p = O.make_params(2, 7, birth=0b1, survival=0)
    out, st = O.step(X, Y, Z, p, g)
    s = states(out, X, Y, Z)
    assert st.born == 7  # only the in-grid Moore neighbours of a corner
    assert s[0, 0, 0] == 1  # alive -> maxCS-1
    assert s[1, 1, 1] == 2 and s[0, 0, 1] == 2


def test_row_end_padding_x_mod_8_eq_1():
    X, Y, Z = 9, 3, 3  # the last word of each row holds one cell and 7 padding nibbles
    g = grid_with(X, Y, Z, [((8, 1, 1), 1)])
    p = O.make_params(1, 1, birth=0b1, survival=0)
    out, st = O.step(X, Y, Z, p, g)
    assert st.born == 5  # x=9 does not exist
    w = out.reshape(Z, Y, 2)
    assert np.all((w[:, :, 1] & np.uint32(0xFFFFFFF0)) == 0)  # padding nibbles stay 0


def test_max_cell_state_16_seeds_zero_and_dies():
    X = Y = Z = 12
    init = O.seed(X, Y, Z, spawn=(4, 4, 4), random=False, max_cell_state=16)
    assert not init.any()  # 16 & 0xF == 0 (searchSystem.cpp:302)
    p = O.make_params(16, 7, birth=(1 << 26) - 1, survival=(1 << 26) - 1)
    info, ticks, _ = O.run_sim(X, Y, Z, p, init, 20, per_tick=True)
    assert info.ticks == 1 and info.status == 1
    assert ticks[0].dead == X * Y * Z


def test_count_zero_never_births():
    X = Y = Z = 6
    p = O.make_params(3, 7, birth=(1 << 26) - 1, survival=(1 << 26) - 1)
    out, st = O.step(X, Y, Z, p, np.zeros(O.grid_words(X, Y, Z), np.uint32))
    assert not out.any() and st.dead == X * Y * Z and st.born == 0


def test_decay_chain():
    X = Y = Z = 3
    g = grid_with(X, Y, Z, [((1, 1, 1), 4)])  # maxCS 5: state 4 is decaying
    p = O.make_params(5, 7, birth=0, survival=0)
    for expect in (3, 2, 1, 0):
        g, st = O.step(X, Y, Z, p, g)
        assert states(g, X, Y, Z)[1, 1, 1] == expect
        assert st.dying == 1


def test_state_above_max_decays():
    X = Y = Z = 3
    g = grid_with(X, Y, Z, [((1, 1, 1), 9)])
    p = O.make_params(3, 7, birth=0b1, survival=0)
    g, st = O.step(X, Y, Z, p, g)
    assert states(g, X, Y, Z)[1, 1, 1] == 8 and st.dying == 1 and st.born == 0


def test_wrap_flag_is_ignored():
    X = Y = Z = 5
    g = grid_with(X, Y, Z, [((0, 2, 2), 1)])
    a, sa = O.step(X, Y, Z, O.make_params(1, 0x1, 1, 0), g)
    b, sb = O.step(X, Y, Z, O.make_params(1, 0x9, 1, 0), g)  # W bit set (cube shader ignores it)
    assert np.array_equal(a, b) and sa.as_tuple() == sb.as_tuple()


# ---- properties over random grids
@pytest.mark.parametrize("dims", [(1, 1, 1), (8, 8, 8), (9, 9, 9), (17, 5, 11), (33, 7, 4)])
@pytest.mark.parametrize("flags", range(8))
def test_fast_matches_literal(dims, flags):
    rng = np.random.default_rng(hash((dims, flags)) & 0xFFFF)
    X, Y, Z = dims
    for maxcs in (1, 3, 16):
        st = rng.integers(0, 16, size=(Z, Y, X), dtype=np.uint8)
        st[rng.random((Z, Y, X)) < 0.4] = maxcs & 0xF
        g = O.pack(st)
        B, S = int(rng.integers(0, 1 << 26)), int(rng.integers(0, 1 << 26))
        p = O.make_params(maxcs, flags, B, S)
        a, sa = O.step(X, Y, Z, p, g)
        b, sb = O.step_fast(X, Y, Z, p, g)
        assert np.array_equal(a, b)
        assert tuple(sb) == sa.as_tuple()[:4]
        assert sum(sa.as_tuple()[:4]) == X * Y * Z
        assert sa.changed == sa.born + sa.dying
        assert sa.population == int(np.count_nonzero(states(a, X, Y, Z)))


def test_empty_grid_stays_empty():
    X, Y, Z = 10, 9, 8
    p = O.make_params(4, 7, birth=0xFFF, survival=0xFFF)
    g = np.zeros(O.grid_words(X, Y, Z), np.uint32)
    for _ in range(3):
        g, st = O.step(X, Y, Z, p, g)
        assert not g.any() and st.population == 0 and tuple(st.bbox_min) == (0xFFFFFFFF,) * 3


def test_k_index_params():
    X = Y = Z = 9
    vb = O.valid_bitmasks(18, 2)
    rng = np.random.default_rng(5)
    g = O.pack(np.where(rng.random((Z, Y, X)) < 0.3, 3, 0).astype(np.uint8))
    bi, si = 40, 100
    a, sa = O.step(X, Y, Z, O.make_params(3, 3, bi + 1, si + 1), g, valid=vb, max_rule_bits=2)
    b, sb = O.step(X, Y, Z, O.make_params(3, 3, int(vb[bi]), int(vb[si])), g)
    assert np.array_equal(a, b) and sa.as_tuple() == sb.as_tuple()
    with pytest.raises(ValueError):
        O.step(X, Y, Z, O.make_params(3, 3, 172, 1), g, valid=vb, max_rule_bits=2)


# ---- seeding (searchSystem.cpp:224-306)
def test_seed_box_and_fill():
    G = 49
    thr = O.threshold_from_float(0.30)
    assert thr == 1288490240
    init = O.seed(G, G, G, spawn=(16, 16, 16), random=True, threshold=thr, run_seed=0, max_cell_state=3)
    s = states(init, G, G, G)
    nz = np.argwhere(s)
    assert nz.min(axis=0).tolist() == [16, 16, 16] and nz.max(axis=0).tolist() == [31, 31, 31]
    assert set(np.unique(s).tolist()) == {0, 3}
    assert abs(len(nz) / 16 ** 3 - 0.30) < 0.03
    # the same cells by the literal hash
    expect = sum(1 for x in range(16, 32) for y in range(16, 32) for z in range(16, 32)
                 if O.cell_hash(x, y, z, 0) < thr)
    assert expect == len(nz)


def test_seed_filled_and_density_index():
    init = O.seed(25, 25, 25, spawn=(11, 11, 11), random=False, max_cell_state=2)
    s = states(init, 25, 25, 25)
    assert np.count_nonzero(s) == 11 ** 3 and s[7, 7, 7] == 2 and s[17, 17, 17] == 2 and s[6, 7, 7] == 0
    assert O.threshold_from_index(15) == 1 << 32
    assert O.threshold_from_index(3) == 1 << 30  # density 0.25
    assert O.threshold_from_float(0.4) == 1717986944


def test_wang_hash_known_values():
    # wangHash(x*73856093 + seed) chain for (0,0,0,0): computed by the restated formula
    def wang(s):
        s = ((s ^ 61) ^ (s >> 16)) & 0xFFFFFFFF
        s = (s * 9) & 0xFFFFFFFF
        s = s ^ (s >> 4)
        s = (s * 0x27d4eb2d) & 0xFFFFFFFF
        return s ^ (s >> 15)

    for x, y, z, sd in [(0, 0, 0, 0), (16, 31, 20, 7), (48, 1, 33, 31)]:
        h = wang((x * 73856093 + sd) & 0xFFFFFFFF)
        h = wang(h ^ ((y * 19349663) & 0xFFFFFFFF))
        h = wang(h ^ ((z * 83492791) & 0xFFFFFFFF))
        assert O.cell_hash(x, y, z, sd) == h


# ---- manager (searchManager.slang:98-149)
def test_manager_status_and_next_permutation():
    info, perms = O.GridInfo(), O.Perms((2 << 60) | 5, (3 << 60) | 7)
    ic, pc = O.manager([100, 2, 3, 4], info, perms, max_permutation=10, survival_end=9, max_ticks=2)
    assert ic.as_tuple() == (100, 3, 1, 0, 4, 4) and perms.birthAndMaxCellStateRules == (2 << 60) | 5
    ic, pc = O.manager([50, 1, 0, 0], info, perms, 10, 9, 2)  # surviving == 0 and born == 0
    assert ic.status == 1 and ic.ticks == 2
    assert (perms.birthAndMaxCellStateRules, perms.survivalAndNeighborhoodRules) == ((2 << 60) | 6, (3 << 60) | 7)
    assert info.as_tuple() == (0, 0, 0, 0, 0, 0)  # fresh GridInfo after the advance
    # birth index at its maximum -> survival advances, birth restarts at 1 keeping the maxCS bits
    perms = O.Perms((2 << 60) | 10, (3 << 60) | 7)
    info = O.GridInfo()
    O.manager([0, 0, 0, 0], info, perms, 10, 9, 5)
    assert (perms.birthAndMaxCellStateRules, perms.survivalAndNeighborhoodRules) == ((2 << 60) | 1, (3 << 60) | 8)
    # exhausted -> NULL; a NULL slot only copies
    perms = O.Perms((2 << 60) | 10, (3 << 60) | 9)
    info = O.GridInfo()
    O.manager([0, 0, 0, 0], info, perms, 10, 9, 5)
    assert (perms.birthAndMaxCellStateRules, perms.survivalAndNeighborhoodRules) == (0, 0)
    ic, pc = O.manager([1, 1, 1, 1], info, perms, 10, 9, 5)
    assert ic.as_tuple() == info.as_tuple() and (pc.birthAndMaxCellStateRules, pc.survivalAndNeighborhoodRules) == (0, 0)


def test_manager_viable_at_tick_limit():
    info, perms = O.GridInfo(), O.Perms((1 << 60) | 1, (1 << 60) | 1)
    for t in range(3):
        ic, _ = O.manager([0, 0, 0, 5], info, perms, 1, 1, 3)
    assert ic.status == 2 and ic.ticks == 3 and ic.maxAlive == 5


def test_slot_pipeline_equals_independent_rules():
    """A whole SearchSystem slot (reset + tick pipeline of searchSystem.cpp:480-713) gives each
    rule exactly the result of running it alone from the initial cells."""
    G = 11
    vb = O.valid_bitmasks(6, 2)
    init = O.seed(G, G, G, spawn=(5, 5, 5), random=False, max_cell_state=2)
    res = O.run_slot(G, G, G, ((2 - 1) << 60) | 1, (1 << 60) | 1, len(vb), 3, init, 10, valid=vb, max_rule_bits=2)
    assert len(res) == len(vb) * 3
    for r in res:
        p = np.array([r.birthAndMaxCellStateRules, r.survivalAndNeighborhoodRules, 0], dtype=np.uint64)
        info, _, _ = O.run_sim(G, G, G, p, init, 10)
        assert info.as_tuple() == r.info.as_tuple()
        assert O.classify(info, 2) == r.category


def test_aggregate_lines_known_answer():
    """RuleAggregator (ruleAggregator.h:69-90, :105-135): rule identity, per-category runs, min /
    max ticks, float32 averages printed with six significant digits in the reference's key
    order."""
    runs = [((2 << 60) | 5, (3 << 60) | 9, 20, 0), ((2 << 60) | 5, (3 << 60) | 9, 7, 2),
            ((2 << 60) | 5, (3 << 60) | 9, 20, 0), ((0 << 60) | 5, (3 << 60) | 9, 4, 1)]
    got = O.aggregate_lines(runs)
    assert got[(5, 9, 3, 3, 0)] == ('{"birth":5,"survival":9,"maxCellState":3,"neighborhoodFlags":3,"shapeId":0,'
                                    '"totalRuns":3,"viableRuns":2,"possibleRuns":0,"unviableRuns":1,'
                                    '"viabilityRate":0.666667,"minTicksSurvived":7,"maxTicksSurvived":20,'
                                    '"avgTicksSurvived":15.6667}')
    assert got[(5, 9, 1, 3, 0)] == ('{"birth":5,"survival":9,"maxCellState":1,"neighborhoodFlags":3,"shapeId":0,'
                                    '"totalRuns":1,"viableRuns":0,"possibleRuns":1,"unviableRuns":0,'
                                    '"viabilityRate":0,"minTicksSurvived":4,"maxTicksSurvived":4,'
                                    '"avgTicksSurvived":4}')
