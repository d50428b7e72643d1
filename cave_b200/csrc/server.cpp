// server.cpp -- cave_server_*: sweep requests served as they arrive (continuous batching).
//
// The reference runs one sweep per process: SearchMode admits chunks into a pool of
// SearchSystems against a VRAM budget and steps them frame by frame (searchMode.cpp:252-459,
// :349-404). The server keeps that admission idea but across requests: each submitted request
// (a list of simulations) joins the engine's queue; the scheduler thread admits simulations as
// completion frees slots and HBM, runs them alongside whatever is already on the device (grid
// state stays in HBM or in shared memory between ticks), and a request completes when its
// last simulation has reported. A simulation's result does not depend on what it shares the
// GPU with: every simulation has its own cells and record.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cave_ca.h"
#include "context.h"
#include "engine.h"
#include "rules.h"

using namespace cave;

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kIndexBits = 24;  // engine key = request id << 24 | simulation index

struct Request {
    uint64_t n = 0, done = 0;
    std::vector<cave_sim_result> results;
    std::vector<cave_sim_params> params;
    Clock::time_point submitted, finished;
    bool complete = false;
    bool cancelled = false;  // cave_server_cancel: results are dropped as they arrive
    bool expired = false;    // past the deadline: results are dropped, wait / fetch time out
    uint64_t cat[3] = {0, 0, 0};  // categories of the results so far (viable, possible, unviable)
};

}  // namespace

struct cave_server {
    cave_ctx* ctx = nullptr;
    std::unique_ptr<Engine> engine;
    std::thread loop;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    cave_status loop_rc = CAVE_OK;
    std::string loop_msg;             // why the scheduler thread stopped
    double deadline_s = 0;            // requestDeadlineSeconds (0 = none)
    uint64_t fail_after_rounds = 0;   // CAVE_TEST_SERVER_FAIL_AFTER_ROUNDS (0 = never)
    uint64_t rounds = 0;
    uint64_t next_id = 1;
    std::map<uint64_t, Request> requests;
    std::vector<uint64_t> ready;      // completed or expired, not yet reported by poll
    std::vector<double> latencies;    // seconds, per completed request
    uint64_t submitted = 0, completed = 0, sims_completed = 0, cell_updates = 0, expired = 0;
    uint64_t outstanding = 0;         // simulations submitted and not finished
    double busy_s = 0;
    Clock::time_point busy_since;
};

// The scheduler thread's error, as the caller's status and last error text.
static cave_status loop_error(cave_server* s) { return set_error(s->ctx, s->loop_rc, s->loop_msg); }

static void server_loop(cave_server* s) {
    cudaSetDevice(s->ctx->device);
    std::vector<EngineResult> res;
    std::vector<uint64_t> expire;
    for (;;) {
        {
            std::unique_lock<std::mutex> lock(s->mu);
            if (s->stop) break;
            if (s->outstanding == 0) {
                s->cv_work.wait_for(lock, std::chrono::milliseconds(2));
                if (s->stop) break;
                if (s->outstanding == 0) continue;
            }
        }
        if (s->fail_after_rounds && s->rounds >= s->fail_after_rounds) {
            // host-side failure injection (tests): the scheduler stops between rounds with the
            // device work of earlier rounds still queued; destroy waits for it
            std::lock_guard<std::mutex> lock(s->mu);
            s->loop_rc = CAVE_ERR_INTERNAL;
            s->loop_msg = "scheduler thread stopped: failure injected after " + std::to_string(s->rounds) + " rounds";
            s->cv_done.notify_all();
            break;
        }
        bool idle = false;
        const cave_status rc = s->engine->step(&idle);
        s->rounds++;
        res.clear();
        s->engine->take_results(res);
        expire.clear();
        std::unique_lock<std::mutex> lock(s->mu);
        if (rc) {
            s->loop_rc = rc;
            s->loop_msg = std::string("scheduler thread stopped: ") + cave_last_error(s->ctx);
            s->cv_done.notify_all();
            break;
        }
        const auto now = Clock::now();
        for (const EngineResult& r : res) {
            const uint64_t id = r.key >> kIndexBits, ix = r.key & ((1ull << kIndexBits) - 1);
            auto it = s->requests.find(id);
            if (it == s->requests.end() || ix >= it->second.n) continue;
            Request& q = it->second;
            if (q.cancelled || q.expired) {  // dropped, or running when cancelled / expired
                q.done++;
                s->outstanding--;
                if (!(r.result.error & kErrCancelled)) s->sims_completed++;
                if (q.done == q.n && q.cancelled) s->requests.erase(it);
                continue;
            }
            q.results[ix] = r.result;
            q.results[ix].params = q.params[ix];
            q.cat[std::min<uint32_t>(r.result.category, 2u)]++;
            q.done++;
            s->sims_completed++;
            s->outstanding--;
            if (q.done == q.n) {
                q.complete = true;
                q.finished = now;
                s->completed++;
                s->latencies.push_back(std::chrono::duration<double>(q.finished - q.submitted).count());
                s->ready.push_back(id);
            }
        }
        if (s->deadline_s > 0) {  // watchdog: requests past their deadline expire
            for (auto& [id, q] : s->requests) {
                if (q.complete || q.cancelled || q.expired ||
                    std::chrono::duration<double>(now - q.submitted).count() <= s->deadline_s)
                    continue;
                q.expired = true;
                q.results.clear();
                s->expired++;
                s->ready.push_back(id);
                expire.push_back(id);
            }
        }
        if (s->outstanding == 0) s->busy_s += std::chrono::duration<double>(now - s->busy_since).count();
        if (!res.empty() || !expire.empty()) s->cv_done.notify_all();
        lock.unlock();
        for (const uint64_t id : expire) s->engine->cancel(id << kIndexBits, (id + 1) << kIndexBits);
    }
}

extern "C" {

cave_status cave_server_create(cave_ctx* ctx, const cave_server_options* opt, cave_server** out) {
    if (!ctx || !out) return CAVE_ERR_INVALID_ARG;
    *out = nullptr;
    cave_server_options o{};
    if (opt) o = *opt;
    CAVE_CUDA(ctx, cudaSetDevice(ctx->device));
    uint64_t budget = o.hbmBudget;
    if (!budget) {
        size_t fr = 0, tot = 0;
        CAVE_CUDA(ctx, cudaMemGetInfo(&fr, &tot));
        budget = fr / 2;
    }
    cave_server* s = new (std::nothrow) cave_server();
    if (!s) return CAVE_ERR_OUT_OF_MEMORY;
    s->ctx = ctx;
    s->deadline_s = o.requestDeadlineSeconds > 0 ? o.requestDeadlineSeconds : 0;
    if (const char* e = std::getenv("CAVE_TEST_SERVER_FAIL_AFTER_ROUNDS")) s->fail_after_rounds = std::strtoull(e, nullptr, 10);
    EngineConfig ec;
    ec.pool_bytes = budget;
    ec.max_slots = o.maxInFlight ? o.maxInFlight : (1u << 14);
    ec.ticks_per_round = o.ticksPerRound ? o.ticksPerRound : 8u;
    ec.tiled_only = o.tiledOnly;
    ec.autotune = o.autotune;
    ec.max_active_cells = o.maxActiveCells ? o.maxActiveCells : (1ull << 31);
    s->engine = std::make_unique<Engine>(ctx);
    const cave_status rc = s->engine->init(ec);
    if (rc) {
        delete s;
        return rc;
    }
    s->loop = std::thread(server_loop, s);
    *out = s;
    return CAVE_OK;
}

void cave_server_destroy(cave_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->loop.joinable()) s->loop.join();
    s->engine.reset();  // waits for the device work still in flight
    delete s;
}

cave_status cave_server_submit(cave_server* s, const cave_request_sim* sims, uint64_t n, uint64_t* requestId) {
    if (!s || !requestId || n == 0 || !sims || n >= (1ull << kIndexBits)) return CAVE_ERR_INVALID_ARG;
    Request q;
    q.n = n;
    q.results.assign(n, cave_sim_result{});
    q.params.resize(n);
    std::vector<EngineSim> es(n);
    uint64_t id;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->loop_rc) return loop_error(s);
        id = s->next_id++;
    }
    for (uint64_t i = 0; i < n; i++) {
        const cave_request_sim& r = sims[i];
        if (r.threshold > (1ull << 32)) return set_error(s->ctx, CAVE_ERR_INVALID_ARG, "fill threshold above 2^32");
        DecodedRule d;
        decode_params(r.params, nullptr, 0, 0, d);
        EngineSim& e = es[i];
        e.key = (id << kIndexBits) | i;
        e.rule = make_device_rule(d);
        e.nb = d.flags & 7u;
        e.nt = e.rule.nterms;
        e.X = r.X;
        e.Y = r.Y;
        e.Z = r.Z;
        e.max_ticks = r.maxTicks;
        e.init = nullptr;
        e.seed = make_seed_spec(r.X, r.Y, r.Z, r.spawnX, r.spawnY, r.spawnZ, 0, r.threshold,
                                r.threshold == (1ull << 32), r.runSeedIndex, d.maxcs);
        q.params[i] = r.params;
    }
    q.submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->requests.emplace(id, std::move(q));
        if (s->outstanding == 0) s->busy_since = Clock::now();
        s->outstanding += n;
        s->submitted++;
    }
    const cave_status rc = s->engine->submit(es);
    if (rc) {
        std::lock_guard<std::mutex> lock(s->mu);
        s->requests.erase(id);
        s->outstanding -= n;
        s->submitted--;
        return rc;
    }
    s->cv_work.notify_all();
    *requestId = id;
    return CAVE_OK;
}

cave_status cave_server_poll(cave_server* s, uint64_t* requestIds, uint64_t cap, uint64_t* n) {
    if (!s || !n || (cap && !requestIds)) return CAVE_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    const uint64_t k = std::min<uint64_t>(cap, s->ready.size());
    std::copy(s->ready.begin(), s->ready.begin() + k, requestIds);
    s->ready.erase(s->ready.begin(), s->ready.begin() + k);
    *n = k;
    return s->loop_rc ? loop_error(s) : CAVE_OK;
}

cave_status cave_server_wait(cave_server* s, uint64_t requestId, double timeoutSeconds) {
    if (!s) return CAVE_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lock(s->mu);
    auto done = [&]() {
        auto it = s->requests.find(requestId);
        return s->loop_rc != CAVE_OK || it == s->requests.end() || it->second.complete || it->second.cancelled ||
               it->second.expired;
    };
    if (timeoutSeconds > 0) {
        if (!s->cv_done.wait_for(lock, std::chrono::duration<double>(timeoutSeconds), done)) return CAVE_ERR_TIMEOUT;
    } else {
        s->cv_done.wait(lock, done);
    }
    auto it = s->requests.find(requestId);
    if (it == s->requests.end() || it->second.cancelled) return s->loop_rc ? loop_error(s) : CAVE_ERR_INVALID_ARG;
    if (it->second.complete) return CAVE_OK;  // results that arrived before a scheduler failure stand
    if (it->second.expired) return set_error(s->ctx, CAVE_ERR_TIMEOUT, "request passed its deadline");
    return loop_error(s);
}

cave_status cave_server_cancel(cave_server* s, uint64_t requestId) {
    if (!s) return CAVE_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = s->requests.find(requestId);
        if (it == s->requests.end() || it->second.cancelled) return CAVE_ERR_INVALID_ARG;
        Request& q = it->second;
        s->ready.erase(std::remove(s->ready.begin(), s->ready.end(), requestId), s->ready.end());
        if (q.complete || (q.expired && q.done == q.n)) {  // nothing still to arrive
            s->requests.erase(it);
            return CAVE_OK;
        }
        const bool was_expired = q.expired;  // its queue was cancelled when it expired
        q.cancelled = true;
        q.results.clear();
        if (was_expired) return CAVE_OK;
    }
    s->engine->cancel(requestId << kIndexBits, (requestId + 1) << kIndexBits);
    s->cv_done.notify_all();
    s->cv_work.notify_all();
    return CAVE_OK;
}

cave_status cave_server_fetch(cave_server* s, uint64_t requestId, cave_sim_result* out, uint64_t n,
                              double* latencySeconds) {
    if (!s) return CAVE_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(requestId);
    if (it == s->requests.end() || it->second.cancelled) return CAVE_ERR_INVALID_ARG;
    if (it->second.expired) {  // released: results still in flight are dropped as they arrive
        s->ready.erase(std::remove(s->ready.begin(), s->ready.end(), requestId), s->ready.end());
        if (it->second.done == it->second.n) s->requests.erase(it);
        else it->second.cancelled = true;
        return set_error(s->ctx, CAVE_ERR_TIMEOUT, "request passed its deadline");
    }
    if (!it->second.complete) return s->loop_rc ? loop_error(s) : CAVE_ERR_NOT_READY;
    if (n != it->second.n || !out) return CAVE_ERR_INVALID_ARG;
    std::memcpy(out, it->second.results.data(), sizeof(cave_sim_result) * n);
    if (latencySeconds)
        *latencySeconds = std::chrono::duration<double>(it->second.finished - it->second.submitted).count();
    s->ready.erase(std::remove(s->ready.begin(), s->ready.end(), requestId), s->ready.end());
    s->requests.erase(it);
    uint32_t err = 0;
    for (uint64_t i = 0; i < n; i++) err |= out[i].error;
    if (err & kErrBounds) return set_error(s->ctx, CAVE_ERR_INTERNAL, "a served simulation failed an index check");
    if (err) return set_error(s->ctx, CAVE_ERR_TIMEOUT, "a served simulation raised a device error flag");
    return CAVE_OK;
}

cave_status cave_server_progress(cave_server* s, uint64_t requestId, cave_request_progress* out) {
    if (!s || !out) return CAVE_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->requests.find(requestId);
    if (it == s->requests.end() || it->second.cancelled) return CAVE_ERR_INVALID_ARG;
    const Request& q = it->second;
    cave_request_progress p{};
    p.total = q.n;
    p.done = q.done;
    p.viable = q.cat[0];
    p.possible = q.cat[1];
    p.unviable = q.cat[2];
    p.complete = q.complete ? 1u : 0u;
    p.expired = q.expired ? 1u : 0u;
    *out = p;
    return CAVE_OK;
}

cave_status cave_server_get_stats(cave_server* s, cave_server_stats* out) {
    if (!s || !out) return CAVE_ERR_INVALID_ARG;
    const EngineStats es = s->engine->stats();
    std::lock_guard<std::mutex> lock(s->mu);
    cave_server_stats st{};
    st.submitted = s->submitted;
    st.completed = s->completed;
    st.simsCompleted = s->sims_completed;
    st.cellUpdates = es.cell_updates;
    std::vector<double> l = s->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) {
        if (l.empty()) return 0.0;
        const size_t i = std::min(l.size() - 1, (size_t)(p * (double)(l.size() - 1) + 0.5));
        return l[i];
    };
    st.p50LatencySeconds = pct(0.50);
    st.p99LatencySeconds = pct(0.99);
    st.busySeconds = s->busy_s + (s->outstanding ? std::chrono::duration<double>(Clock::now() - s->busy_since).count() : 0);
    st.peakBytes = es.peak_pool_bytes;
    st.rounds = es.rounds;
    st.tickLaunches = es.tick_launches;
    st.residentLaunches = es.resident_launches;
    st.tuneMs = es.tune_ms;
    st.expired = s->expired;
    *out = st;
    return s->loop_rc ? loop_error(s) : CAVE_OK;
}

}  // extern "C"
