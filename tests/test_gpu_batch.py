"""Batched resident kernel vs the oracle's per-rule lifecycle (searchSystem.cpp:496-526 +
searchManager.slang:98-149): final GridInfo, category and derived statistics, bit-exact."""
import numpy as np
import pytest

import cave_b200 as cb
import oracle as O

pytestmark = pytest.mark.gpu


def expected(X, Y, Z, params_np, init, max_ticks, valid=None, K=0):
    info, ticks, _ = O.run_sim(X, Y, Z, params_np, init, max_ticks, valid=valid, max_rule_bits=K, fast=True,
                               per_tick=True)
    maxcs = int((int(params_np[0]) >> 60) & 0xF) + 1
    last = ticks[-1]
    return {
        "info": info.as_tuple(),
        "category": O.classify(info, maxcs),
        "population": last.population,
        "totalChanged": sum(t.changed for t in ticks),
        "activeTicks": sum(1 for t in ticks if t.changed),
        "bbox": (tuple(last.bbox_min), tuple(last.bbox_max)),
    }


def got(r):
    return {
        "info": r.info.as_tuple(),
        "category": r.category,
        "population": r.population,
        "totalChanged": r.totalChanged,
        "activeTicks": r.activeTicks,
        "bbox": (tuple(r.bbox_min), tuple(r.bbox_max)),
    }


def rand_init(rng, X, Y, Z, maxcs, p=0.3, box=None):
    s = np.zeros((Z, Y, X), dtype=np.uint8)
    if box is None:
        sl = (slice(None),) * 3
    else:
        b = [(d - box) // 2 for d in (Z, Y, X)]
        sl = tuple(slice(b[i], b[i] + box) for i in range(3))
    sub = s[sl]
    sub[rng.random(sub.shape) < p] = maxcs & 0xF
    return O.pack(s)


@pytest.mark.parametrize("dims", [(8, 8, 8), (17, 9, 13), (33, 33, 33), (49, 49, 49), (65, 65, 65), (40, 33, 25)])
def test_batch_mixed_rules(ctx, dims):
    X, Y, Z = dims
    rng = np.random.default_rng(sum(dims))
    cases = []
    with cb.Batch(ctx) as b:
        for i in range(24):
            flags = int(rng.integers(0, 8))
            maxcs = int(rng.choice([1, 2, 3, 4, 7, 15, 16]))
            nb = (6 if flags & 1 else 0) + (12 if flags & 2 else 0) + (8 if flags & 4 else 0)
            if i % 3 == 0:  # dense rule -> mux tree
                B, S = int(rng.integers(0, 1 << 26)), int(rng.integers(0, 1 << 26))
            else:           # sparse rule -> term list
                k = max(nb, 1)
                B = sum(1 << int(v) for v in rng.choice(k, size=min(2, k), replace=False))
                S = sum(1 << int(v) for v in rng.choice(k, size=min(int(rng.integers(1, 3)), k), replace=False))
            init = rand_init(rng, X, Y, Z, maxcs, p=float(rng.uniform(0.15, 0.5)), box=min(X, Y, Z) // 2 + 1)
            T = int(rng.integers(1, 30))
            params_np = O.make_params(maxcs, flags, B, S)
            ix = b.add_init(X, Y, Z, init)
            cases.append((params_np, init, T))
            b.add_sims([cb.SimDesc(cb.SimParams(*[int(v) for v in params_np]), ix, T, 0, i)])
        b.launch()
        res = b.results()
    for i, (params_np, init, T) in enumerate(cases):
        assert res[i].tag == i and res[i].error == 0
        assert got(res[i]) == expected(X, Y, Z, params_np, init, T), f"sim {i}"


def test_batch_k_index_sweep_slice(ctx):
    """A slice of the reference benchmark sweep: FE, K=2, 25^3, 11^3 filled spawn, 20 ticks."""
    G = 25
    rng = np.random.default_rng(7)
    with cb.Batch(ctx) as b:
        descs, cases = [], []
        for mcs in (2, 3):
            init = O.seed(G, G, G, spawn=(11, 11, 11), random=False, max_cell_state=mcs)
            ix = b.add_init(G, G, G, init)
            for flags, n in ((1, 6), (2, 12), (3, 18)):
                vb = O.valid_bitmasks(n, 2)
                tab = b.add_table(vb)
                for _ in range(40):
                    bi, si = int(rng.integers(0, len(vb))), int(rng.integers(0, len(vb)))
                    p = O.make_params(mcs, flags, bi + 1, si + 1)
                    descs.append(cb.SimDesc(cb.SimParams(*[int(v) for v in p]), ix, 20, tab, len(descs)))
                    cases.append((p, init, vb, int(vb[bi]), int(vb[si])))
        b.add_sims(descs, max_rule_bits=2)
        b.launch()
        res = b.results()
    for i, (p, init, vb, bm, sm) in enumerate(cases):
        assert got(res[i]) == expected(G, G, G, p, init, 20, valid=vb, K=2), f"sim {i}"
        # K-indices translated to bitmasks, upper bits kept (searchSystem.cpp:676-684)
        assert res[i].params.birthAndMaxCellStateRules == ((int(p[0]) >> 60) << 60) | bm
        assert res[i].params.survivalAndNeighborhoodRules == ((int(p[1]) >> 60) << 60) | sm


def test_batch_device_seeded_inits(ctx):
    G = 49
    thr = O.threshold_from_float(0.30)
    with cb.Batch(ctx) as b:
        ix = [b.add_init_seeded(G, G, G, (16, 16, 16), thr, s, 3) for s in range(3)]
        descs = [cb.SimDesc(cb.make_params(3, 3, 0x60, 0x70), ix[s], 20, 0, s) for s in range(3)]
        b.add_sims(descs)
        b.launch()
        res = b.results()
    for s in range(3):
        init = O.seed(G, G, G, spawn=(16, 16, 16), random=True, threshold=thr, run_seed=s, max_cell_state=3)
        assert got(res[s]) == expected(G, G, G, O.make_params(3, 3, 0x60, 0x70), init, 20)



def test_results_into_caller_memory(ctx):
    """results_array(out): the same records written into a caller's array (here pinned host memory,
    as the benchmark reads them); an array that is too small or of another dtype is refused before
    the library writes anything."""
    import torch

    G = 49
    thr = O.threshold_from_float(0.30)
    with cb.Batch(ctx) as b:
        ix = [b.add_init_seeded(G, G, G, (16, 16, 16), thr, s, 3) for s in range(5)]
        b.add_sims([cb.SimDesc(cb.make_params(3, 3, 0x60, 0x70), ix[s], 20, 0, s) for s in range(5)])
        b.launch()
        ref = b.results_array().copy()
        pinned = torch.empty(8 * cb.SIM_RESULT_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
        out = pinned.numpy().view(cb.SIM_RESULT_DTYPE)
        got_ = b.results_array(out)
        assert got_.shape == (5,) and np.shares_memory(got_, out)
        assert got_.tobytes() == ref.tobytes()
        for bad in (np.zeros(4, dtype=cb.SIM_RESULT_DTYPE), np.zeros(8, dtype=np.uint64),
                    np.zeros(16, dtype=cb.SIM_RESULT_DTYPE)[::2]):
            with pytest.raises(ValueError):
                b.results_array(bad)

def test_withheld_initial_copy_times_out_without_a_fault(ctx, monkeypatch):
    """Failure path of the bounded device waits: with the failure test switch the resident
    kernel never issues a one-simulation batch's initial-grid copy, gives up its wait after 1 ms
    and raises the timeout flag; the batch reports CAVE_ERR_TIMEOUT and the context stays usable
    (a normal batch right after gives the oracle's result)."""
    G = 21
    init = O.seed(G, G, G, spawn=(9, 9, 9), random=True, threshold=O.threshold_from_float(0.35), run_seed=1,
                  max_cell_state=3)
    params = cb.make_params(3, 0x3, 0x60, 0x70)
    monkeypatch.setenv("CAVE_TEST_WITHHOLD_INIT_COPY", "1")
    with cb.Batch(ctx) as b:
        ix = b.add_init(G, G, G, init)
        b.add_sims([cb.SimDesc(params, ix, 10, 0, 0)])
        b.launch()
        with pytest.raises(cb.CaveError) as e:
            b.results_array()
        assert e.value.code == cb.ERR_TIMEOUT
    monkeypatch.delenv("CAVE_TEST_WITHHOLD_INIT_COPY")
    with cb.Batch(ctx) as b:
        ix = b.add_init(G, G, G, init)
        b.add_sims([cb.SimDesc(params, ix, 10, 0, 0)])
        b.launch()
        r = b.results_array()
    want = O.run_sim(G, G, G, O.make_params(3, 0x3, 0x60, 0x70), init, 10, fast=True)[0]
    assert tuple(int(v) for v in r[0]["info"]) == want.as_tuple()
