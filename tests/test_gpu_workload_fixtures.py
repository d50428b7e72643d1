"""The benchmark's simulation workloads at their own sizes against oracle fixtures.

* The 49^3 search sweep (171 x 171 K<=2 FE rules x C 2..5 x 32 seeds, 20 ticks with early stop):
  every 64th of its 3,742,848 simulations, batched, against tests/golden/sweep49_fixture.json.
* The uneven-size batch (2048 simulations, edges 33..193, F/FE/Moore, C 2..16, 10..500 ticks):
  every simulation, with the autotuner, and with every grid forced onto the tiled (multi-CTA)
  path, against tests/golden/engine_fixture.json ("uneven").
* Long-lived simulations at the large end of the tiled and served size ranges (193^3 and 256^3,
  300 ticks): tiled in a batch, and served alone and in a mix of other requests
  (engine_fixture.json "long").
Each result is compared field by field (GridInfo, category, population, active ticks, changed
cells, bounding box), packed as cave_b200.result_records. Integer work: exact.
"""
import hashlib
import json
import os
import time

import numpy as np
import pytest

import bench
import cave_b200 as cb

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    p = os.path.join(GOLDEN, name)
    if not os.path.exists(p):
        pytest.skip(f"{name} not generated")
    return json.load(open(p))


def _blocks(rec, block):
    return [hashlib.sha256(rec[i:i + block].tobytes()).hexdigest() for i in range(0, rec.shape[0], block)]


def test_sweep49_every_64th_simulation(ctx):
    fx = _load("sweep49_fixture.json")
    full = bench.sweep_descs(49, 32, (2, 3, 4, 5))
    sample = np.ascontiguousarray(full[::fx["stride"]])
    with cb.Batch(ctx) as b:
        for c in (2, 3, 4, 5):
            for s in range(32):
                b.add_init_seeded(49, 49, 49, (16, 16, 16), cb.threshold_from_fill(0.30), s, c - 1)
        b.add_table(cb.valid_bitmasks(18, 2))
        b.add_sims_array(sample, max_rule_bits=2)
        b.launch()
        res = b.results_array()
    rec = cb.result_records(res, sample["tag"])
    cats = np.bincount(rec[:, 7], minlength=3)
    assert [int(c) for c in cats] == [fx["viable"], fx["possible"], fx["unviable"]]
    got = _blocks(rec, fx["block"])
    bad = [i for i, (a, b) in enumerate(zip(got, fx["block_sha256"])) if a != b]
    assert len(got) == len(fx["block_sha256"]) and not bad, f"blocks {bad[:10]} differ"


def _uneven(ctx, **opts):
    fx = _load("engine_fixture.json")["uneven"]
    sims = bench.uneven_sims(fx["sims"])
    assert bench.uneven_spec_digest(sims) == fx["spec_sha256"], "the batch's draw changed"
    with cb.Batch(ctx) as b:
        b.set_options(**opts)
        descs = []
        for j, s in enumerate(sims):
            e = s["edge"]
            ix = b.add_init_seeded(e, e, e, (e, e, e), cb.threshold_from_fill(s["fill"]), s["seed"], s["maxcs"])
            descs.append(cb.SimDesc(cb.make_params(s["maxcs"], s["flags"], s["birth"], s["survival"]), ix,
                                    s["ticks"], 0, j))
        b.add_sims(descs)
        b.launch()
        res = b.results_array()
    assert int(res["error"].max()) == 0
    rec = cb.result_records(res, np.arange(len(sims)))
    got = _blocks(rec, fx["block"])
    bad = [i for i, (a, b) in enumerate(zip(got, fx["block_sha256"])) if a != b]
    assert not bad, f"blocks {bad[:10]} differ"
    assert int(rec[:, 3].astype(np.int64).sum()) == fx["ticks"]


def test_uneven_batch_autotuned(ctx):
    _uneven(ctx, autotune=True)


def test_uneven_batch_all_tiled(ctx):
    _uneven(ctx, tiled_only=True)


def _long(name):
    L = _load("engine_fixture.json")["long"][name]
    e = L["edge"]
    params = cb.make_params(L["maxCellState"], L["flags"], L["birth"], L["survival"])
    return L, e, params


def test_long_tiled_193(ctx):
    L, e, params = _long("tiled193")
    with cb.Batch(ctx) as b:
        b.set_options(tiled_only=True)
        ix = b.add_init_seeded(e, e, e, (e, e, e), cb.threshold_from_fill(L["fill"]), L["seed"], L["maxCellState"])
        b.add_sims([cb.SimDesc(params, ix, L["maxTicks"], 0, 0)])
        b.launch()
        res = b.results_array()
    assert cb.result_records(res, [0])[0].tolist() == L["record"]


def _request(L, e, params, tag=0):
    r = cb.request_sims(1)
    r[0]["X"] = r[0]["Y"] = r[0]["Z"] = e
    r[0]["maxTicks"] = L["maxTicks"]
    r[0]["birth"], r[0]["survival"] = params.birthAndMaxCellStateRules, params.survivalAndNeighborhoodRules
    r[0]["spawnX"] = r[0]["spawnY"] = r[0]["spawnZ"] = e
    r[0]["runSeedIndex"] = L["seed"]
    r[0]["threshold"] = cb.threshold_from_fill(L["fill"])
    r[0]["tag"] = tag
    return r


def test_long_served_256_alone_and_in_mix(ctx):
    L, e, params = _long("served256")
    with cb.Server(ctx, hbm_budget=8 << 30) as s:
        rid = s.submit(_request(L, e, params))
        assert s.wait(rid, 300.0)
        alone, _ = s.fetch(rid)
    assert cb.result_records(alone, [0])[0].tolist() == L["record"]
    others = [req for _, req in bench.serve_requests(6, 200.0, seed=99)]
    with cb.Server(ctx, hbm_budget=8 << 30, ticks_per_round=4) as s:
        ids = [s.submit(others[0]), s.submit(others[1])]
        time.sleep(0.01)  # arrives while the first requests are on the GPU
        pid = s.submit(_request(L, e, params))
        ids += [s.submit(o) for o in others[2:]]
        for rid in ids + [pid]:
            assert s.wait(rid, 600.0)
        mixed, _ = s.fetch(pid)
        for rid in ids:
            res, _ = s.fetch(rid)
            assert int(res["error"].max()) == 0
    assert cb.result_records(mixed, [0])[0].tolist() == L["record"]
