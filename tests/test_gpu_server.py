"""The request server (continuous batching): each request's results equal the oracle's and do
not depend on what else is on the GPU -- alone, in a mix submitted while others run, and
under an HBM budget small enough that simulations queue for memory. Integer work: exact."""
import time

import numpy as np
import pytest

import cave_b200 as cb
import oracle as O

pytestmark = pytest.mark.gpu


def make_request(rng, n, edges=(24, 33, 40, 70, 100)):
    r = cb.request_sims(n)
    for i in range(n):
        e = int(rng.choice(edges))
        flags = int(rng.choice([1, 3, 7]))
        nb = {1: 6, 3: 18, 7: 26}[flags]
        maxcs = int(rng.integers(1, 16))
        B = sum(1 << int(v) for v in rng.choice(nb, size=int(rng.integers(1, 5)), replace=False))
        S = sum(1 << int(v) for v in rng.choice(nb, size=int(rng.integers(1, 5)), replace=False))
        p = O.make_params(maxcs, flags, B, S)
        r[i]["X"] = r[i]["Y"] = r[i]["Z"] = e
        r[i]["maxTicks"] = int(rng.integers(1, 20))
        r[i]["birth"], r[i]["survival"] = int(p[0]), int(p[1])
        r[i]["spawnX"] = r[i]["spawnY"] = r[i]["spawnZ"] = e
        r[i]["runSeedIndex"] = int(rng.integers(0, 1000))
        r[i]["threshold"] = O.threshold_from_float(float(rng.uniform(0.2, 0.5)))
        r[i]["tag"] = i
    return r


def oracle_result(sim):
    X, Y, Z = int(sim["X"]), int(sim["Y"]), int(sim["Z"])
    params = np.array([sim["birth"], sim["survival"], 0], dtype=np.uint64)
    maxcs = int((int(sim["birth"]) >> 60) & 0xF) + 1
    init = O.seed(X, Y, Z, spawn=(int(sim["spawnX"]),) * 3, random=True, threshold=int(sim["threshold"]),
                  run_seed=int(sim["runSeedIndex"]), max_cell_state=maxcs)
    info, ticks, _ = O.run_sim(X, Y, Z, params, init, int(sim["maxTicks"]), fast=True, per_tick=True)
    last = ticks[-1]
    return (info.as_tuple(), O.classify(info, maxcs), last.population, sum(t.changed for t in ticks),
            sum(1 for t in ticks if t.changed), tuple(last.bbox_min), tuple(last.bbox_max))


def as_tuple(r):
    return (tuple(int(v) for v in r["info"]), int(r["category"]), int(r["population"]), int(r["totalChanged"]),
            int(r["activeTicks"]), tuple(int(v) for v in r["bbox_min"]), tuple(int(v) for v in r["bbox_max"]))


def run_alone(ctx, req, **kw):
    with cb.Server(ctx, **kw) as s:
        rid = s.submit(req)
        assert s.wait(rid, 120.0)
        res, lat = s.fetch(rid)
    assert lat > 0
    return res


def test_request_matches_oracle(ctx):
    rng = np.random.default_rng(3)
    req = make_request(rng, 10)
    res = run_alone(ctx, req, hbm_budget=1 << 30)
    for i in range(req.size):
        assert int(res[i]["error"]) == 0
        assert as_tuple(res[i]) == oracle_result(req[i]), f"sim {i}"
        assert int(res[i]["birth"]) == int(req[i]["birth"])


def test_same_result_alone_and_in_mix(ctx):
    rng = np.random.default_rng(17)
    probe = make_request(rng, 12)
    alone = run_alone(ctx, probe, hbm_budget=1 << 30)
    others = [make_request(rng, int(rng.integers(1, 30))) for _ in range(6)]
    with cb.Server(ctx, hbm_budget=1 << 30, ticks_per_round=2) as s:
        ids = [s.submit(others[0]), s.submit(others[1])]
        time.sleep(0.005)  # the probe arrives while the first requests are on the GPU
        pid = s.submit(probe)
        ids += [s.submit(o) for o in others[2:]]
        for rid in ids + [pid]:
            assert s.wait(rid, 300.0)
        mixed, _ = s.fetch(pid)
        outs = [s.fetch(rid)[0] for rid in ids]
        st = s.stats()
    for i in range(probe.size):
        assert as_tuple(mixed[i]) == as_tuple(alone[i]), f"probe sim {i}"
    # spot-check the other requests against the oracle
    for o, r in zip(others[:2], outs[:2]):
        for i in range(min(3, o.size)):
            assert as_tuple(r[i]) == oracle_result(o[i])
    assert st.completed == 7 and st.simsCompleted == probe.size + sum(o.size for o in others)
    assert st.p99LatencySeconds >= st.p50LatencySeconds > 0


def test_small_budget_queues_and_completes(ctx):
    """Budget of a few 100^3 grids: simulations wait for memory, results stay exact."""
    rng = np.random.default_rng(23)
    req = make_request(rng, 16, edges=(100,))
    alone = run_alone(ctx, req, hbm_budget=1 << 30)
    per_sim = 2 * 4 * 100 * 100 * 16
    with cb.Server(ctx, hbm_budget=3 * per_sim + (1 << 16), tiled_only=True) as s:
        rid = s.submit(req)
        assert s.wait(rid, 300.0)
        res, _ = s.fetch(rid)
        st = s.stats()
    assert st.peakBytes <= 3 * per_sim + (1 << 16)
    for i in range(req.size):
        assert as_tuple(res[i]) == as_tuple(alone[i]), f"sim {i}"


def test_one_at_a_time_admission_gives_same_results(ctx):
    """An active-cell cap of one cell admits a single simulation at a time (FIFO)."""
    rng = np.random.default_rng(31)
    req = make_request(rng, 6)
    alone = run_alone(ctx, req, hbm_budget=1 << 30)
    capped = run_alone(ctx, req, hbm_budget=1 << 30, max_active_cells=1)
    for i in range(req.size):
        assert as_tuple(capped[i]) == as_tuple(alone[i]), f"sim {i}"


def test_oversized_simulation_is_rejected(ctx):
    rng = np.random.default_rng(1)
    req = make_request(rng, 1, edges=(100,))
    with cb.Server(ctx, hbm_budget=1 << 16, tiled_only=True) as s:
        with pytest.raises(cb.CaveError) as ei:
            s.submit(req)
        assert ei.value.code == cb.ERR_OUT_OF_MEMORY


def test_poll_reports_each_request_once(ctx):
    rng = np.random.default_rng(29)
    reqs = [make_request(rng, 3, edges=(24, 33)) for _ in range(5)]
    with cb.Server(ctx, hbm_budget=1 << 28) as s:
        ids = [s.submit(r) for r in reqs]
        seen = []
        t0 = time.time()
        while len(seen) < len(ids) and time.time() - t0 < 60:
            seen += s.poll()
            time.sleep(0.001)
        for rid in ids:
            s.fetch(rid)
    assert sorted(seen) == sorted(ids)


def test_cancel_queued_and_running_requests(ctx):
    """cave_server_cancel: a request queued behind others leaves the queue without running; a
    request cancelled while on the device finishes unreported; the others complete with the
    results they have alone, and the server's accounting stays consistent."""
    rng = np.random.default_rng(41)
    first = make_request(rng, 6, edges=(100,))
    queued = make_request(rng, 5, edges=(70,))
    later = make_request(rng, 4, edges=(40,))
    alone_first = run_alone(ctx, first, hbm_budget=1 << 30)
    alone_later = run_alone(ctx, later, hbm_budget=1 << 30)
    with cb.Server(ctx, hbm_budget=1 << 30, max_active_cells=1, ticks_per_round=1) as s:  # one simulation at a time
        a = s.submit(first)
        q = s.submit(queued)
        s.cancel(q)  # still behind `first`: dropped from the queue
        with pytest.raises(cb.CaveError) as e:
            s.wait(q, 1.0)
        assert e.value.code == cb.ERR_INVALID_ARG
        c = s.submit(later)
        assert s.wait(a, 300.0) and s.wait(c, 300.0)
        ra, _ = s.fetch(a)
        rc_, _ = s.fetch(c)
        st = s.stats()
        assert st.completed == 2 and st.simsCompleted == first.size + later.size
        # a request cancelled while it runs
        b = s.submit(make_request(rng, 6, edges=(100,)))
        time.sleep(0.02)
        s.cancel(b)
        d = s.submit(later)
        assert s.wait(d, 300.0)
        rd, _ = s.fetch(d)
    for i in range(first.size):
        assert as_tuple(ra[i]) == as_tuple(alone_first[i]), f"first sim {i}"
    for i in range(later.size):
        assert as_tuple(rc_[i]) == as_tuple(alone_later[i]), f"later sim {i}"
        assert as_tuple(rd[i]) == as_tuple(alone_later[i]), f"later (again) sim {i}"


def test_cancel_unknown_request_is_an_error(ctx):
    with cb.Server(ctx, hbm_budget=1 << 28) as s:
        with pytest.raises(cb.CaveError) as e:
            s.cancel(12345)
        assert e.value.code == cb.ERR_INVALID_ARG


def long_request(n, edge=256, ticks=300):
    """n copies of a simulation that stays alive for all its ticks (Moore S{4,5} B{5}, C = 16)."""
    r = cb.request_sims(n)
    p = O.make_params(15, 0x7, 1 << 4, (1 << 3) | (1 << 4))
    for i in range(n):
        r[i]["X"] = r[i]["Y"] = r[i]["Z"] = edge
        r[i]["maxTicks"] = ticks
        r[i]["birth"], r[i]["survival"] = int(p[0]), int(p[1])
        r[i]["spawnX"] = r[i]["spawnY"] = r[i]["spawnZ"] = edge
        r[i]["runSeedIndex"] = 11
        r[i]["threshold"] = O.threshold_from_float(0.35)
        r[i]["tag"] = i
    return r


def test_request_deadline_expires_and_later_requests_run(ctx):
    """requestDeadlineSeconds: a request still running past its deadline expires -- wait stops
    waiting, poll reports it, fetch returns CAVE_ERR_TIMEOUT and releases it, its queued
    simulations never run -- while a request submitted afterwards completes with the results it
    has alone."""
    rng = np.random.default_rng(43)
    small = make_request(rng, 4, edges=(24, 33))
    alone = run_alone(ctx, small, hbm_budget=1 << 30)
    big = long_request(400)  # one simulation at a time, one tick per round: seconds of work
    with cb.Server(ctx, hbm_budget=1 << 30, max_active_cells=1, ticks_per_round=1, request_deadline=1.0) as s:
        t0 = time.time()
        rid = s.submit(big)
        assert not s.wait(rid, 60.0)
        waited = time.time() - t0
        assert 1.0 <= waited < 10.0, waited
        assert rid in s.poll()
        with pytest.raises(cb.CaveError) as e:
            s.fetch(rid)
        assert e.value.code == cb.ERR_TIMEOUT and "deadline" in str(e.value)
        with pytest.raises(cb.CaveError) as e:  # released: the id is unknown now
            s.cancel(rid)
        assert e.value.code == cb.ERR_INVALID_ARG
        q = s.submit(small)
        assert s.wait(q, 60.0)
        res, _ = s.fetch(q)
        st = s.stats()
        assert st.expired == 1 and st.completed == 1
        assert st.simsCompleted < big.size + small.size  # the expired request's queue was dropped
    for i in range(small.size):
        assert as_tuple(res[i]) == as_tuple(alone[i]), f"sim {i}"


def test_cancel_of_an_expired_request_releases_it(ctx):
    with cb.Server(ctx, hbm_budget=1 << 30, max_active_cells=1, ticks_per_round=1, request_deadline=0.2) as s:
        rid = s.submit(long_request(50))
        assert not s.wait(rid, 60.0)
        s.cancel(rid)
        with pytest.raises(cb.CaveError) as e:
            s.wait(rid, 1.0)
        assert e.value.code == cb.ERR_INVALID_ARG
        assert s.stats().expired == 1


def test_injected_scheduler_failure_reaches_every_waiter(ctx, monkeypatch):
    """A scheduler thread that stops (failure injected on the host between rounds, with device
    work still queued) is reported to wait, poll, submit and fetch instead of leaving them
    blocked; the server shuts down cleanly and the context serves a new server."""
    monkeypatch.setenv("CAVE_TEST_SERVER_FAIL_AFTER_ROUNDS", "3")
    rng = np.random.default_rng(47)
    with cb.Server(ctx, hbm_budget=1 << 30, max_active_cells=1, ticks_per_round=1) as s:
        rid = s.submit(long_request(6, edge=100, ticks=50))  # needs hundreds of rounds
        for call in (lambda: s.wait(rid, 60.0), lambda: s.poll(), lambda: s.submit(make_request(rng, 2)),
                     lambda: s.fetch(rid)):
            with pytest.raises(cb.CaveError) as e:
                call()
            assert e.value.code == cb.ERR_INTERNAL and "failure injected after 3 rounds" in str(e.value)
    monkeypatch.delenv("CAVE_TEST_SERVER_FAIL_AFTER_ROUNDS")
    req = make_request(rng, 3, edges=(24, 40))
    res = run_alone(ctx, req, hbm_budget=1 << 30)
    for i in range(req.size):
        assert as_tuple(res[i]) == oracle_result(req[i]), f"sim {i}"


def test_progress_counts_results_as_they_arrive(ctx):
    """cave_server_progress (SearchProgress per request): done rises to the request's size, the
    categories so far add up to it and, at the end, equal the fetched results'."""
    req = long_request(24, edge=64, ticks=60)
    with cb.Server(ctx, hbm_budget=1 << 30, max_active_cells=1, ticks_per_round=1) as s:
        rid = s.submit(req)
        seen = []
        while True:
            p = s.progress(rid)
            assert p.total == req.size and p.viable + p.possible + p.unviable == p.done
            seen.append(p.done)
            if p.complete:
                break
            time.sleep(0.002)
        assert seen == sorted(seen) and seen[-1] == req.size and not p.expired
        res, _ = s.fetch(rid)
        cats = np.bincount(np.asarray(res["category"], dtype=np.int64), minlength=3)
        assert (p.viable, p.possible, p.unviable) == tuple(int(c) for c in cats)
        with pytest.raises(cb.CaveError) as e:  # fetched: the id is released
            s.progress(rid)
        assert e.value.code == cb.ERR_INVALID_ARG
