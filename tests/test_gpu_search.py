"""Search driver (cave_search_run) vs the oracle's literal SearchSystem pipeline
(oracle_run_slot: searchSystem.cpp:480-713 + searchManager.slang), and the full reference
benchmark sweep vs the committed golden fixture."""
import glob
import hashlib
import json
import os

import numpy as np
import pytest

import cave_b200 as cb
import oracle as O

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
NB = {1: 6, 2: 12, 3: 18, 4: 8, 5: 14, 6: 20, 7: 26}


def jsonl_line(r, maxcs):
    return json.dumps({
        "birthAndMaxCellStateRules": int(r.birthAndMaxCellStateRules),
        "survivalAndNeighborhoodRules": int(r.survivalAndNeighborhoodRules),
        "shapeAndGridConfiguration": 0,
        "ticksSurvived": r.info.ticks, "totalBirths": r.info.totalBorn, "totalDeaths": r.info.totalDied,
        "maxAliveCount": r.info.maxAlive, "finalAliveCount": r.info.finalAlive,
    }, sort_keys=True, separators=(",", ":"))


def oracle_chunk(G, flags_list, cs_range, K, T, spawn, seed=0, random=False, density_index=0, part=(0, 1)):
    """Expected {category: set(lines)} of one chunk, by running every slot through oracle_run_slot."""
    out = {0: set(), 1: set(), 2: set()}
    thr = O.threshold_from_index(density_index) if random else 1 << 32
    for mcs in cs_range:
        init = O.seed(G, G, G, spawn=(spawn,) * 3, random=random, threshold=thr, run_seed=seed, max_cell_state=mcs)
        for flags in flags_list:
            n = NB[flags & 7]
            vb = O.valid_bitmasks(n, K) if K else None
            maxp = len(vb) if K else (1 << n) - 1
            pi, pc = part
            hi = (pi + 1) * maxp // pc if pc > 1 else maxp
            lo = 1 + pi * maxp // pc if pc > 1 else 1
            if lo > hi:
                continue
            res = O.run_slot(G, G, G, ((mcs - 1) << 60) | 1, (flags << 60) | lo, maxp, hi, init, T, valid=vb,
                             max_rule_bits=K, fast=True)
            for r in res:
                out[r.category].add(jsonl_line(r, mcs))
    return out


def read_chunk_files(folder, prefix):
    out = {}
    for cat, name in enumerate(("viable", "possible", "unviable")):
        path = os.path.join(folder, "cube", f"{prefix}_{name}.jsonl")
        with open(path) as f:
            lines = [l.rstrip("\n") for l in f if l.strip()]
        assert len(lines) == len(set(lines))
        out[cat] = set(lines)
    return out


@pytest.mark.parametrize("plain", [False, True])
def test_small_sweep_matches_oracle_pipeline(ctx, tmp_path, plain):
    G, T, K = 9, 8, 2
    out = str(tmp_path) + "/"
    cfg = cb.search_config(grid=G, spawn=5, spawn_mode="filled", neighborhood="FE", min_cs=2, max_cs=3, ticks=T,
                           max_rule_bits=K, output=out)
    s = cb.search_run(ctx, cfg, plain=plain)
    expect = oracle_chunk(G, [1, 2, 3], (2, 3), K, T, 5)
    got = read_chunk_files(out, f"cs2-3_FE_t{T}_b{K}_c1_g{G}x{G}x{G}_d7_s0_gpu0")
    assert got == expect
    n = (21 * 21 + 78 * 78 + 171 * 171) * 2
    assert s.sims == n and s.viable + s.possible + s.unviable == n and s.chunks == 1
    assert s.viable == len(expect[0]) and s.possible == len(expect[1])
    # aggregate: one line per distinct rule; keys in the reference's order
    agg = open(os.path.join(out, "cube", f"cs2-3_FE_t{T}_b{K}_aggregate.jsonl")).read().splitlines()
    assert len(agg) == n == s.uniqueRules
    first = json.loads(agg[0])
    assert list(first) == ["birth", "survival", "maxCellState", "neighborhoodFlags", "shapeId", "totalRuns",
                           "viableRuns", "possibleRuns", "unviableRuns", "viabilityRate", "minTicksSurvived",
                           "maxTicksSurvived", "avgTicksSurvived"]


def test_partitions_and_seed_density_sweep(ctx, tmp_path):
    """--chunks-per-config partitions split each slot's survival range (searchSystem.cpp:84-96);
    seeds and a density sweep create more chunks with random spawns."""
    G, T = 7, 6
    out = str(tmp_path) + "/"
    cfg = cb.search_config(grid=G, spawn=5, spawn_mode="random", density=0.5, neighborhood="F", min_cs=3, max_cs=3,
                           ticks=T, chunks_per_config=4, seed_runs=2, density_sweep=(0.25, 0.5, 0.25), output=out)
    cb.search_run(ctx, cfg)
    files = sorted(glob.glob(os.path.join(out, "cube", "*_viable.jsonl")))
    assert len(files) == 2 * 2 * 4  # densities x seeds x partitions
    ordinal = 1
    for di in (3, 7):
        for seed in range(2):
            for p in range(4):
                prefix = f"cs3-3_F_t{T}_c{ordinal}_g{G}x{G}x{G}_d{di}_s{seed}_gpu0"
                got = read_chunk_files(out, prefix)
                exp = oracle_chunk(G, [1], (3,), 0, T, 5, seed=seed, random=True, density_index=di, part=(p, 4))
                assert got == exp, prefix
                ordinal += 1


def test_batch_plain_equals_resident(ctx):
    G = 21
    rng = np.random.default_rng(4)
    descs = []
    with cb.Batch(ctx) as b1, cb.Batch(ctx) as b2:
        for mcs in (2, 4):
            init = O.seed(G, G, G, spawn=(9, 9, 9), random=True, threshold=O.threshold_from_float(0.35), run_seed=mcs,
                          max_cell_state=mcs)
            i1, i2 = b1.add_init(G, G, G, init), b2.add_init(G, G, G, init)
            assert i1 == i2
            for _ in range(30):
                flags = int(rng.integers(1, 8))
                B, S = int(rng.integers(1, 1 << 12)), int(rng.integers(1, 1 << 12))
                descs.append(cb.SimDesc(cb.make_params(mcs, flags, B, S), i1, int(rng.integers(1, 25)), 0, len(descs)))
        b1.add_sims(descs)
        b2.add_sims(descs)
        b1.launch()
        b2.run_plain(7)
        r1, r2 = b1.results(), b2.results()
    for a, c in zip(r1, r2):
        assert a.info.as_tuple() == c.info.as_tuple() and a.category == c.category
        assert (a.population, a.totalChanged, a.activeTicks) == (c.population, c.totalChanged, c.activeTicks)
        assert tuple(a.bbox_min) == tuple(c.bbox_min) and tuple(a.bbox_max) == tuple(c.bbox_max)


@pytest.mark.parametrize("G", [25, 49])
def test_reference_benchmark_sweep_vs_fixture(ctx, G):
    """The published benchmark sweep (bench_chunks.ps1:21-32): all 71,532 rules, every GridInfo
    checked through a hash against the oracle-generated fixture."""
    fx = json.load(open(os.path.join(HERE, "golden", "sweep_fixture.json")))[str(G)]
    descs, tabs = [], {}
    with cb.Batch(ctx) as b:
        for mcs in (2, 3):
            init = O.seed(G, G, G, spawn=(11, 11, 11), random=False, max_cell_state=mcs)
            ix = b.add_init(G, G, G, init)
            for flags in (1, 2, 3):
                vb = O.valid_bitmasks(NB[flags], 2)
                if flags not in tabs:
                    tabs[flags] = b.add_table(vb)
                n = len(vb)
                for si in range(n):
                    for bi in range(n):
                        descs.append(cb.SimDesc(cb.make_params(mcs, flags, bi + 1, si + 1), ix, 20, tabs[flags],
                                                len(descs)))
        b.add_sims(descs, max_rule_bits=2)
        b.launch()
        res = b.results()
    arr = np.array([r.info.as_tuple() for r in res], dtype="<u4")
    cats = np.array([r.category for r in res])
    assert len(res) == fx["rules"] == 71532
    assert (int((cats == 0).sum()), int((cats == 1).sum()), int((cats == 2).sum())) == (
        fx["viable"], fx["possible"], fx["unviable"])
    assert hashlib.sha256(arr.tobytes()).hexdigest() == fx["gridinfo_sha256"]


def oracle_chunk_results(G, flags_list, cs_range, K, T, spawn, seed=0, random=False, density_index=0):
    """(birth field, survival field, ticks, category) of every rule of one chunk (oracle_run_slot)."""
    out = []
    thr = O.threshold_from_index(density_index) if random else 1 << 32
    for mcs in cs_range:
        init = O.seed(G, G, G, spawn=(spawn,) * 3, random=random, threshold=thr, run_seed=seed, max_cell_state=mcs)
        for flags in flags_list:
            n = NB[flags & 7]
            vb = O.valid_bitmasks(n, K) if K else None
            maxp = len(vb) if K else (1 << n) - 1
            for r in O.run_slot(G, G, G, ((mcs - 1) << 60) | 1, (flags << 60) | 1, maxp, maxp, init, T, valid=vb,
                                max_rule_bits=K, fast=True):
                out.append((r.birthAndMaxCellStateRules, r.survivalAndNeighborhoodRules, r.info.ticks, r.category))
    return out


@pytest.mark.parametrize("plain", [False, True])
def test_aggregate_values_match_oracle(ctx, tmp_path, plain):
    """Every aggregate line -- runs per category, viabilityRate, min / max / avg ticks -- equals the
    oracle's RuleAggregator restatement over the oracle pipeline's results, across seeds and
    densities (each rule aggregated over four chunks)."""
    G, T = 8, 12
    out = str(tmp_path) + "/"
    cfg = cb.search_config(grid=G, spawn=6, spawn_mode="random", neighborhood="F", min_cs=2, max_cs=4, ticks=T,
                           seed_runs=2, density_sweep=(0.25, 0.5, 0.25), output=out)
    s = cb.search_run(ctx, cfg, plain=plain)
    results = []
    for di in (3, 7):
        for seed in range(2):
            results += oracle_chunk_results(G, [1], (2, 3, 4), 0, T, 6, seed=seed, random=True, density_index=di)
    want = O.aggregate_lines(results)
    got = open(os.path.join(out, "cube", f"cs2-4_F_t{T}_aggregate.jsonl")).read().splitlines()
    assert len(got) == len(want) == s.uniqueRules == 3 * 63 * 63
    assert sorted(got) == sorted(want.values())
    assert s.sims == len(results) and not s.stopped


def test_stop_keeps_written_results_and_writes_partial_aggregate(ctx, tmp_path, monkeypatch):
    """A stop request mid-sweep (searchMode.cpp:437-449): results written so far stay in their
    files (each line flushed as its wave finished), the aggregate of what ran goes to
    _aggregate_partial.jsonl, and no full aggregate is written."""
    import threading
    import time

    monkeypatch.setenv("CAVE_SEARCH_WAVE_SIMS", "256")
    G, T, K = 9, 8, 2
    out = str(tmp_path) + "/"
    cfg = cb.search_config(grid=G, spawn=5, spawn_mode="filled", neighborhood="FE", min_cs=2, max_cs=3, ticks=T,
                           max_rule_bits=K, seed_runs=3, output=out)
    box = {}
    th = threading.Thread(target=lambda: box.setdefault("s", cb.search_run(ctx, cfg)))
    th.start()
    first = os.path.join(out, "cube", f"cs2-3_FE_t{T}_b{K}_c1_g{G}x{G}x{G}_d7_s0_gpu0_unviable.jsonl")
    t0 = time.time()
    while not (os.path.exists(first) and os.path.getsize(first) > 0) and th.is_alive() and time.time() - t0 < 120:
        time.sleep(0.001)
    cb.search_stop(ctx)
    th.join(300)
    s = box["s"]
    assert s.stopped == 1
    total = (21 * 21 + 78 * 78 + 171 * 171) * 2 * 3
    assert 0 < s.sims < total
    cube = os.path.join(out, "cube")
    assert not os.path.exists(os.path.join(cube, f"cs2-3_FE_t{T}_b{K}_aggregate.jsonl"))
    partial = open(os.path.join(cube, f"cs2-3_FE_t{T}_b{K}_aggregate_partial.jsonl")).read().splitlines()
    # every written line is one of the oracle's, and the partial aggregate is the aggregate of them
    written = []
    expect = oracle_chunk(G, [1, 2, 3], (2, 3), K, T, 5)  # the spawn is filled: every seed has the same cells
    for f in sorted(glob.glob(os.path.join(cube, "*.jsonl"))):
        if "aggregate" in f:
            continue
        cat = 0 if f.endswith("_viable.jsonl") else 1 if f.endswith("_possible.jsonl") else 2
        for line in open(f).read().splitlines():
            assert line in expect[cat], f
            d = json.loads(line)
            written.append((d["birthAndMaxCellStateRules"], d["survivalAndNeighborhoodRules"], d["ticksSurvived"], cat))
    assert len(written) == s.sims
    assert sorted(partial) == sorted(O.aggregate_lines(written).values())


def test_unwritable_output_folder_is_an_io_error(ctx, tmp_path):
    blocker = tmp_path / "not_a_folder"
    blocker.write_text("x")
    cfg = cb.search_config(grid=7, spawn=5, neighborhood="F", min_cs=2, max_cs=2, ticks=4,
                           output=str(blocker) + "/out/")
    with pytest.raises(cb.CaveError) as e:
        cb.search_run(ctx, cfg)
    assert e.value.code == cb.ERR_IO


@pytest.mark.parametrize("plain", [False, True])
def test_resume_reads_complete_chunks_and_reruns_the_rest(ctx, tmp_path, monkeypatch, plain):
    """resume: a sweep cut short (a simulation limit in the middle of a chunk) left complete,
    partial and missing chunk files; run again into the same folder with resume, it reads the
    complete chunks back instead of running them, rewrites the partial one, runs the missing
    ones, and every file -- the aggregate included -- equals a fresh run's."""
    monkeypatch.setenv("CAVE_SEARCH_WAVE_SIMS", "512")
    G, T = 7, 6
    kw = dict(grid=G, spawn=5, spawn_mode="random", neighborhood="F", min_cs=2, max_cs=3, ticks=T, seed_runs=3)
    fresh, part = str(tmp_path / "fresh") + "/", str(tmp_path / "part") + "/"
    full = cb.search_run(ctx, cb.search_config(output=fresh, **kw), plain=plain)
    per_chunk = full.sims // full.chunks
    cut = cb.search_run(ctx, cb.search_config(output=part, **kw), plain=plain, sim_limit=per_chunk + per_chunk // 2)
    assert per_chunk < cut.sims < full.sims
    again = cb.search_run(ctx, cb.search_config(output=part, resume=True, **kw), plain=plain)
    assert again.resumedSims >= per_chunk and again.resumedSims % per_chunk == 0
    assert again.resumedSims < full.sims
    for k in ("sims", "viable", "possible", "unviable", "ticks", "uniqueRules"):
        assert getattr(again, k) == getattr(full, k), k
    names = sorted(os.path.relpath(p, fresh) for p in glob.glob(os.path.join(fresh, "**", "*.jsonl"), recursive=True))
    assert names == sorted(os.path.relpath(p, part) for p in glob.glob(os.path.join(part, "**", "*.jsonl"),
                                                                       recursive=True))
    for n in names:
        assert open(os.path.join(part, n)).read() == open(os.path.join(fresh, n)).read(), n
