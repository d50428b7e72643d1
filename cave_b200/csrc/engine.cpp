// engine.cpp -- see engine.h.
#include "engine.h"
#include "trace.h"

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <new>
#include <thread>
#include <tuple>

namespace cave {

// ---------------------------------------------------------------- geometry helpers
static uint64_t align_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }
static uint64_t grid_strips(uint32_t X, uint32_t Y, uint32_t Z) { return (uint64_t)((X + 31u) / 32u) * Y * Z; }
// Layout of one resident launch's descriptors: a 16-byte queue counter, the ResSim array,
// then the DeviceRule array on a 16-byte boundary (the kernel copies rules with 16-byte loads).
static uint64_t desc_rules_offset(uint64_t n) { return align_up(16 + n * sizeof(ResSim), 16); }
static uint64_t desc_bytes_for(uint64_t n) { return align_up(desc_rules_offset(n) + n * sizeof(DeviceRule), 256); }


constexpr size_t kMaxResidentSmem = 220 * 1024;

bool resident_fits(uint32_t X, uint32_t Y, uint32_t Z) {
    const uint32_t SX = (X + 31u) / 32u;
    uint32_t SXp = 1;
    while (SXp < SX) SXp <<= 1;
    if (SX > 32 || (uint64_t)Y * SXp > 1024) return false;
    return resident_smem_bytes(X, Y, Z, 1) <= kMaxResidentSmem;
}

// Registers a resident-kernel thread holds (its __launch_bounds__(1024) caps it at 64).
constexpr uint32_t kResidentRegs = 64;

static uint32_t resident_threads(uint32_t cols, uint32_t nseg) { return (nseg * cols + 31u) / 32u * 32u; }

// CTAs of a resident geometry that fit one SM together: by shared memory (228 KB per SM, about
// 3 KB of static shared memory and reserve per CTA), registers (64K per SM) and threads.
static uint32_t resident_fit(uint32_t X, uint32_t Y, uint32_t Z, uint32_t nseg, uint32_t threads) {
    const size_t smem = resident_smem_bytes(X, Y, Z, nseg);
    const uint32_t by_smem = (uint32_t)((228u * 1024u) / (smem + 3 * 1024u));
    const uint32_t by_regs = 65536u / (threads * kResidentRegs);
    const uint32_t by_threads = 2048u / threads;
    return std::max(1u, std::min({by_smem, by_regs, by_threads, 32u}));
}

// z-segments of a resident launch (or nseg_hint; CAVE_RESIDENT_NSEG overrides for tuning runs),
// within 1024 threads and the shared-memory cap: preferring counts that fit two or more CTAs per
// SM (each CTA waits at a barrier every plane; a second one fills those waits), then the most
// threads resident per SM, then the most segments (the shortest march per tick).
ResLaunch resident_geometry(uint32_t X, uint32_t Y, uint32_t Z, uint32_t nseg_hint, uint32_t& threads) {
    ResLaunch P{};
    P.X = X;
    P.Y = Y;
    P.Z = Z;
    P.SX = (X + 31u) / 32u;
    uint32_t SXp = 1, lg = 0;
    while (SXp < P.SX) {
        SXp <<= 1;
        lg++;
    }
    P.sxp_log2 = lg;
    const uint32_t cols = Y * SXp;
    const uint32_t most = std::max(1u, std::min<uint32_t>(1024u / cols, Z));
    if (!nseg_hint) {
        if (const char* v = std::getenv("CAVE_RESIDENT_NSEG")) nseg_hint = (uint32_t)std::max(0, std::atoi(v));
    }
    uint32_t nseg = 1;
    if (nseg_hint) {
        nseg = std::min(nseg_hint, most);
    } else {
        uint64_t best = 0;
        for (uint32_t k = 1; k <= most; k++) {
            if (k > 1 && resident_smem_bytes(X, Y, Z, k) > kMaxResidentSmem) break;
            const uint32_t t = resident_threads(cols, k);
            const uint32_t fit = resident_fit(X, Y, Z, k, t);
            const uint64_t score = ((uint64_t)std::min(fit, 2u) << 32) | ((uint64_t)(fit * t) << 8) | k;
            if (score >= best) {
                best = score;
                nseg = k;
            }
        }
    }
    while (nseg > 1 && resident_smem_bytes(X, Y, Z, nseg) > kMaxResidentSmem) nseg--;
    P.nseg = nseg;
    P.seg_len = (Z + nseg - 1) / nseg;
    threads = resident_threads(cols, nseg);
    return P;
}

uint32_t resident_ctas_per_sm(const ResLaunch& P, uint32_t threads) {
    return resident_fit(P.X, P.Y, P.Z, P.nseg, threads);
}

bool plan_tiled(uint32_t sim_index, uint32_t X, uint32_t Y, uint32_t Z, const ExecChoice& c, StreamPlan& plan) {
    const uint32_t lg = c.cells ? c.cells : 18u;
    const uint64_t vol = (uint64_t)X * Y * Z;
    const uint32_t target = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((vol + (1ull << lg) - 1) >> lg, 4096));
    return plan_stream(sim_index, X, Y, Z, target, c.rows, plan);
}

// ---------------------------------------------------------------- engine records
struct Engine::TiledClass {
    uint32_t SXp = 0, nb = 0, nt = 0, rows = 0;
    std::vector<uint32_t> slots;  // active simulations
    uint32_t stream = 0;
};

struct Engine::ResGroup {
    cudaEvent_t done = nullptr;
    uint64_t mem_off = 0, mem_bytes = 0;  // descriptors in the pool
};

struct Engine::Slot {
    uint64_t key = 0;
    uint32_t resident = 0;
    uint64_t mem_off = 0, mem_bytes = 0;  // cell memory in the pool (0 bytes: none)
    uint64_t volume = 0;
    TiledClass* cls = nullptr;
    // tiled: grid, the class's rows per CTA, the preferred and the current CTAs per tick
    uint32_t X = 0, Y = 0, Z = 0, rows_hint = 0;
    uint32_t pref_ctas = 0, cur_ctas = 0;
    std::vector<StreamItem> items;
};

struct Engine::Round {
    cudaEvent_t done = nullptr;
    int stage = 0;
};

Engine::Engine(cave_ctx* ctx) : ctx_(ctx) {}

Engine::~Engine() {
    if (!ctx_) return;
    cudaSetDevice(ctx_->device);
    if (main_) cudaStreamSynchronize(main_);
    if (copy_) cudaStreamSynchronize(copy_);
    for (cudaStream_t s : class_streams_) cudaStreamSynchronize(s);
    for (cudaStream_t s : res_streams_) cudaStreamSynchronize(s);
    for (Round* r : rounds_) {
        cudaEventDestroy(r->done);
        delete r;
    }
    for (ResGroup* g : groups_) {
        cudaEventDestroy(g->done);
        delete g;
    }
    for (Slot* s : slots_) delete s;
    for (auto& kv : classes_) delete kv.second;
    for (cudaStream_t s : class_streams_) cudaStreamDestroy(s);
    for (cudaStream_t s : res_streams_) cudaStreamDestroy(s);
    if (main_) cudaStreamDestroy(main_);
    if (copy_) cudaStreamDestroy(copy_);
    cudaFree(pool_);
    cudaFree(desc_);
    cudaFree(recs_);
    cudaFree(ring_);
    if (stage_cap_) {  // keep the pinned staging for the context's next engine
        std::lock_guard<std::mutex> lock(ctx_->staging_mu);
        ctx_->staging_free.push_back(StagingPair{{stage_h_[0], stage_h_[1]}, {stage_d_[0], stage_d_[1]}, stage_cap_});
    }
    cudaFreeHost(host_entries_);
    if (ev_first_) cudaEventDestroy(ev_first_);
    if (ev_last_) cudaEventDestroy(ev_last_);
    if (trace_) fclose(trace_);
}

double Engine::trace_us() const {
    return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - trace_t0_).count();
}

cave_status Engine::init(const EngineConfig& cfg) {
    cfg_ = cfg;
    cfg_.max_slots = std::max(1u, cfg_.max_slots);
    cfg_.ticks_per_round = std::max(1u, cfg_.ticks_per_round);
    CAVE_CUDA(ctx_, cudaSetDevice(ctx_->device));
    CAVE_CUDA(ctx_, cudaStreamCreateWithFlags(&main_, cudaStreamNonBlocking));
    CAVE_CUDA(ctx_, cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
    class_streams_.resize(8);
    for (auto& s : class_streams_) CAVE_CUDA(ctx_, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    res_streams_.resize(4);
    for (auto& s : res_streams_) CAVE_CUDA(ctx_, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    if (cfg_.pool_bytes) {
        cfg_.pool_bytes = align_up(cfg_.pool_bytes, 256);
        CAVE_CUDA(ctx_, cudaMalloc(&pool_, cfg_.pool_bytes));
    }
    cells_.reset(cfg_.pool_bytes);
    // Every simulation of a resident launch holds a slot, so the descriptors in flight never
    // exceed desc_bytes_for(1) = 512 bytes per slot (one launch per simulation is the worst
    // case); the heap is four times that, leaving room for fragmentation.
    const uint64_t desc_heap = (uint64_t)cfg_.max_slots * desc_bytes_for(1) * 4;
    CAVE_CUDA(ctx_, cudaMalloc(&desc_, desc_heap));
    descs_.reset(desc_heap);
    CAVE_CUDA(ctx_, cudaMalloc(&recs_, sizeof(StripSim) * cfg_.max_slots));
    CAVE_CUDA(ctx_, cudaMalloc(&ring_, sizeof(DoneRing)));
    CAVE_CUDA(ctx_, cudaHostAlloc(&host_entries_, sizeof(DoneEntry) * cfg_.max_slots, cudaHostAllocMapped));
    std::memset(host_entries_, 0, sizeof(DoneEntry) * cfg_.max_slots);
    DoneEntry* dev_entries = nullptr;
    CAVE_CUDA(ctx_, cudaHostGetDevicePointer((void**)&dev_entries, host_entries_, 0));
    DoneRing hr{0, cfg_.max_slots, dev_entries};
    CAVE_CUDA(ctx_, cudaMemcpyAsync(ring_, &hr, sizeof(hr), cudaMemcpyHostToDevice, main_));
    CAVE_CUDA(ctx_, cudaStreamSynchronize(main_));
    slots_.resize(cfg_.max_slots, nullptr);
    free_slots_.reserve(cfg_.max_slots);
    for (uint32_t i = cfg_.max_slots; i-- > 0;) free_slots_.push_back(i);
    CAVE_CUDA(ctx_, cudaEventCreate(&ev_first_));
    CAVE_CUDA(ctx_, cudaEventCreate(&ev_last_));
    {  // reuse pinned staging left by an earlier engine of this context (page-locking is slow)
        std::lock_guard<std::mutex> lock(ctx_->staging_mu);
        if (!ctx_->staging_free.empty()) {
            const StagingPair sp = ctx_->staging_free.back();
            ctx_->staging_free.pop_back();
            for (int i = 0; i < 2; i++) {
                stage_h_[i] = sp.h[i];
                stage_d_[i] = sp.d[i];
            }
            stage_cap_ = sp.cap;
        }
    }
    if (const char* path = std::getenv("CAVE_ENGINE_TRACE")) {
        trace_ = std::fopen(path, "a");
        trace_t0_ = std::chrono::steady_clock::now();
    }
    ready_ = true;
    return CAVE_OK;
}

void FreeList::reset(uint64_t size) {
    free_.clear();
    if (size) free_[0] = size;
    used_ = peak_ = 0;
}

bool FreeList::alloc(uint64_t bytes, uint64_t& off) {
    bytes = align_up(std::max<uint64_t>(bytes, 1), 256);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
        if (it->second < bytes) continue;
        off = it->first;
        const uint64_t rest = it->second - bytes;
        free_.erase(it);
        if (rest) free_[off + bytes] = rest;
        used_ += bytes;
        peak_ = std::max(peak_, used_);
        return true;
    }
    return false;
}

void FreeList::free(uint64_t off, uint64_t bytes) {
    bytes = align_up(std::max<uint64_t>(bytes, 1), 256);
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
        it->second += nx->second;
        free_.erase(nx);
    }
    if (it != free_.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) {
            pv->second += it->second;
            free_.erase(it);
        }
    }
}

cave_status Engine::submit(std::vector<EngineSim>& sims) {
    if (!ready_) return CAVE_ERR_INVALID_ARG;
    for (const EngineSim& s : sims) {
        if (s.X == 0 || s.Y == 0 || s.Z == 0 || s.X > 1024 || s.Y > 65535 || s.Z > 65535 ||
            (uint64_t)s.X * s.Y * s.Z >= (1ull << 32))
            return set_error(ctx_, CAVE_ERR_INVALID_ARG, "simulation grid shape outside X <= 1024, Y, Z <= 65535");
        // worst case footprint: two tiled copies
        const uint64_t need = align_up(2 * grid_strips(s.X, s.Y, s.Z) * 16, 256);
        const bool res_ok = !cfg_.tiled_only && resident_fits(s.X, s.Y, s.Z);
        const uint64_t need_res = s.init ? 0 : align_up(grid_strips(s.X, s.Y, s.Z) * 16, 256);
        if ((res_ok ? std::min(need, need_res) : need) > cfg_.pool_bytes)
            return set_error(ctx_, CAVE_ERR_OUT_OF_MEMORY,
                             "a simulation needs more cell memory than the engine's budget");
    }
    std::lock_guard<std::mutex> lock(mu_);
    for (EngineSim& s : sims) incoming_.push_back(s);
    return CAVE_OK;
}

void Engine::cancel(uint64_t key_lo, uint64_t key_hi) {
    std::lock_guard<std::mutex> lock(mu_);
    cancels_.push_back({key_lo, key_hi});
}

void Engine::take_results(std::vector<EngineResult>& out) {
    std::lock_guard<std::mutex> lock(mu_);
    out.insert(out.end(), results_.begin(), results_.end());
    results_.clear();
}

EngineStats Engine::stats() {
    std::lock_guard<std::mutex> lock(mu_);
    return stats_;
}

float Engine::device_ms() {
    if (!first_recorded_) return 0.f;
    float ms = 0;
    cudaEventSynchronize(ev_last_);
    cudaEventElapsedTime(&ms, ev_first_, ev_last_);
    return ms;
}

std::string Engine::plan_json() {
    std::string s = "[";
    bool first = true;
    for (const auto& [k, c] : plan_used_) {
        if (!first) s += ",";
        first = false;
        s += "{\"grid\":[" + std::to_string(k.X) + "," + std::to_string(k.Y) + "," + std::to_string(k.Z) +
             "],\"nb\":" + std::to_string(k.nb) + ",\"path\":\"" + (c.resident ? "resident" : "tiled") + "\"";
        if (c.resident)
            s += ",\"nseg\":" + std::to_string(c.nseg);
        else
            s += ",\"rows\":" + std::to_string(c.rows) + ",\"log2_cells_per_cta\":" + std::to_string(c.cells ? c.cells : 18);
        s += "}";
    }
    return s + "]";
}

// ---------------------------------------------------------------- choice + autotuning
ExecChoice choose_exec(cave_ctx* ctx, cudaStream_t st, const EngineSim& s, bool tiled_only, bool autotune,
                       double* tune_ms) {
    const TuneKey key{s.X, s.Y, s.Z, s.nb};
    const bool can_res = !tiled_only && resident_fits(s.X, s.Y, s.Z);
    ExecChoice c;
    bool have = false;
    {
        std::lock_guard<std::mutex> lock(ctx->tune_mu);
        auto it = ctx->tune_cache.find(key);
        if (it != ctx->tune_cache.end()) {
            c = it->second;
            have = true;
        }
    }
    if (!have && autotune) {
        const auto t0 = std::chrono::steady_clock::now();
        if (tune_class(ctx, st, s, false, c) == CAVE_OK) {
            have = true;
            std::lock_guard<std::mutex> lock(ctx->tune_mu);
            ctx->tune_cache[key] = c;
        }
        if (tune_ms)
            *tune_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    if (!have) {
        c = ExecChoice{};
        c.resident = can_res ? 1u : 0u;
    }
    if (c.resident && !can_res) c = ExecChoice{};  // tiled only
    return c;
}

ExecChoice Engine::choose(const EngineSim& s) {
    double ms = 0;
    const ExecChoice c = choose_exec(ctx_, main_, s, cfg_.tiled_only != 0, cfg_.autotune != 0, &ms);
    plan_used_[TuneKey{s.X, s.Y, s.Z, s.nb}] = c;
    if (ms > 0) {
        std::lock_guard<std::mutex> lock(mu_);
        stats_.tune_ms += ms;
    }
    return c;
}

// Candidates: the resident kernel with the default and with one z-segment per CTA (when the
// grid fits), and the tiled kernel with 256 / 512 / 1024 threads per CTA at 2^18 cells per
// CTA and with 2^16 / 2^20 cells per CTA at 512 threads. Each is timed on replicas of `s`
// (its rule and initial cells) for four ticks, enough replicas to fill the GPU; the one with
// the most cell updates per second wins. Scratch is allocated here and freed after (the
// trials run once per class and context).
cave_status tune_class(cave_ctx* ctx, cudaStream_t st, const EngineSim& s, bool tiled_only, ExecChoice& out) {
    constexpr uint32_t kTrialTicks = 4;
    constexpr uint32_t kMaxRep = 1024;       // resident replicas (one wave: SMs x CTAs per SM)
    constexpr uint64_t kMaxTiledRep = 256;   // tiled replicas
    const uint32_t sms = (uint32_t)ctx->sm_count;
    const uint64_t strips = grid_strips(s.X, s.Y, s.Z);
    const uint64_t grid_bytes = strips * 16;
    const uint64_t vol = (uint64_t)s.X * s.Y * s.Z;
    std::vector<ExecChoice> cands;
    if (!tiled_only && resident_fits(s.X, s.Y, s.Z)) {
        ExecChoice a;
        a.resident = 1;
        cands.push_back(a);
        a.nseg = 1;
        cands.push_back(a);
    }
    StreamPlan p0;
    if (!plan_tiled(0, s.X, s.Y, s.Z, ExecChoice{}, p0)) return CAVE_ERR_INVALID_ARG;
    {
        const uint32_t step = std::max(1u, 32u / p0.SXp);
        for (uint32_t th : {512u, 256u, 1024u}) {
            ExecChoice t;
            t.rows = std::max(3u * step, th / p0.SXp);
            t.cells = 18;
            cands.push_back(t);
        }
        for (uint32_t lg : {16u, 20u}) {
            ExecChoice t;
            t.cells = lg;
            cands.push_back(t);
        }
    }
    // Tiled candidates all run the same replicas: enough that the candidate with the fewest
    // CTAs per grid still has about four waves of CTAs (two per SM per wave), within 2 GB.
    const uint64_t tiled_bytes = align_up(2 * grid_bytes, 256);
    uint64_t fewest = p0.items.size();
    for (const ExecChoice& c : cands) {
        StreamPlan p;
        if (!c.resident && plan_tiled(0, s.X, s.Y, s.Z, c, p)) fewest = std::min<uint64_t>(fewest, p.items.size());
    }
    const uint32_t reps_tiled = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>({kMaxTiledRep, (8ull * sms + fewest - 1) / fewest, (2ull << 30) / tiled_bytes}));
    const uint64_t init_bytes = align_up(grid_bytes, 256);
    const uint64_t desc_bytes = desc_bytes_for(kMaxRep);
    unsigned char* base = nullptr;
    StripSim* trecs = nullptr;
    StreamItem* titems = nullptr;
    cave_sim_result* tres = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    constexpr uint32_t kMaxItems = 1u << 18;
    cudaError_t e = cudaMalloc(&base, init_bytes + desc_bytes + reps_tiled * tiled_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&trecs, sizeof(StripSim) * reps_tiled);
    if (e == cudaSuccess) e = cudaMalloc(&titems, sizeof(StreamItem) * kMaxItems);
    if (e == cudaSuccess) e = cudaMalloc(&tres, sizeof(cave_sim_result) * kMaxRep);
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    uint4* init = reinterpret_cast<uint4*>(base);
    unsigned char* desc = base + init_bytes;
    uint4* tpool = reinterpret_cast<uint4*>(base + init_bytes + desc_bytes);
    if (e == cudaSuccess) {
        if (s.init)
            e = cudaMemcpyAsync(init, s.init, grid_bytes, cudaMemcpyDeviceToDevice, st);
        else
            e = launch_seed_strips(init, s.seed, st);
    }
    // Each candidate runs twice, for kTrialTicks and 3 * kTrialTicks ticks; the rate compared is
    // the marginal one, (updates difference) / (time difference), so that one-off costs (the
    // resident kernel loading a whole grid into shared memory, the first launch) do not count
    // against a candidate in runs of hundreds of ticks.
    auto run = [&](const ExecChoice& c, uint32_t T, uint64_t& updates, float& ms) {
        updates = 0;
        ms = 0;
        if (c.resident) {
            uint32_t threads = 0;
            ResLaunch P = resident_geometry(s.X, s.Y, s.Z, c.nseg, threads);
            const uint32_t per_sm = resident_ctas_per_sm(P, threads);
            const uint32_t n = std::min<uint32_t>(kMaxRep, sms * per_sm);
            P.n_sims = n;
            std::vector<ResSim> rs(n);
            for (uint32_t i = 0; i < n; i++) rs[i] = ResSim{init, 0u, T, i, 0u};
            uint32_t* queue = reinterpret_cast<uint32_t*>(desc);
            ResSim* dsims = reinterpret_cast<ResSim*>(desc + 16);
            DeviceRule* drule = reinterpret_cast<DeviceRule*>(desc + desc_rules_offset(kMaxRep));
            e = cudaMemcpyAsync(dsims, rs.data(), sizeof(ResSim) * n, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(drule, &s.rule, sizeof(DeviceRule), cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaMemsetAsync(queue, 0, 4, st);
            if (e == cudaSuccess) e = cudaEventRecord(t0, st);
            if (e == cudaSuccess)
                e = launch_resident((int)s.nb, (int)s.nt, P, dsims, drule, tres, queue, nullptr, n, threads, st);
            if (e == cudaSuccess) e = cudaEventRecord(t1, st);
            std::vector<cave_sim_result> hr(n);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(hr.data(), tres, sizeof(cave_sim_result) * n, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return;
            cudaEventElapsedTime(&ms, t0, t1);
            for (const auto& r : hr) updates += (uint64_t)r.info.numberOfSimulationTicksSurvived * vol;
        } else {
            std::vector<StreamItem> items;
            std::vector<StripSim> recs(reps_tiled);
            uint32_t SXp = 1, threads = 0;
            bool ok = true;
            for (uint32_t i = 0; i < reps_tiled; i++) {
                StreamPlan p;
                ok = ok && plan_tiled(i, s.X, s.Y, s.Z, c, p);
                SXp = p.SXp;
                threads = p.threads;
                items.insert(items.end(), p.items.begin(), p.items.end());
                StripSim& r = recs[i];
                std::memset(&r, 0, sizeof(r));
                r.rule = s.rule;
                r.X = s.X;
                r.Y = s.Y;
                r.Z = s.Z;
                r.SX = p.SX;
                r.buf[0] = (uint64_t)i * tiled_bytes;
                r.buf[1] = r.buf[0] + grid_bytes;
                r.max_ticks = T;
                r.tick_limit = T;
                r.stop_on_status = 1;
                r.n_items = (uint32_t)p.items.size();
                for (int k = 0; k < 3; k++) r.acc_bmin[k] = 0xFFFFFFFFu;
            }
            if (!ok || items.size() > kMaxItems) {
                ms = -1;
                return;
            }
            for (uint32_t i = 0; i < reps_tiled && e == cudaSuccess; i++)
                e = cudaMemcpyAsync(reinterpret_cast<unsigned char*>(tpool) + recs[i].buf[0], init, grid_bytes,
                                    cudaMemcpyDeviceToDevice, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(trecs, recs.data(), sizeof(StripSim) * reps_tiled, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(titems, items.data(), sizeof(StreamItem) * items.size(), cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaEventRecord(t0, st);
            for (uint32_t k = 0; k < T && e == cudaSuccess; k++)
                e = launch_stream_tick((int)s.nb, (int)s.nt, nullptr, titems, (uint32_t)items.size(), trecs, tpool, SXp,
                                       SXp, threads, st, k > 0);
            if (e == cudaSuccess) e = cudaEventRecord(t1, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(recs.data(), trecs, sizeof(StripSim) * reps_tiled, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return;
            cudaEventElapsedTime(&ms, t0, t1);
            for (const auto& r : recs) updates += (uint64_t)r.tick * vol;
        }
    };
    double best = -1;
    ExecChoice best_c = cands[0];
    for (size_t ci = 0; ci < cands.size() && e == cudaSuccess; ci++) {
        const ExecChoice& c = cands[ci];
        uint64_t u1 = 0, u2 = 0;
        float m1 = 0, m2 = 0;
        run(c, kTrialTicks, u1, m1);
        if (e == cudaSuccess && m1 >= 0) run(c, 3 * kTrialTicks, u2, m2);
        if (e != cudaSuccess) break;
        if (m1 < 0 || m2 < 0) continue;
        const double rate = (m2 > m1 && u2 > u1) ? (double)(u2 - u1) / (m2 - m1) : (m2 > 0 ? (double)u2 / m2 : 0);
        if (rate > best) {
            best = rate;
            best_c = c;
        }
    }
    cudaStreamSynchronize(st);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    cudaFree(base);
    cudaFree(trecs);
    cudaFree(titems);
    cudaFree(tres);
    if (e != cudaSuccess) return check_cuda(ctx, e, "autotune trial");
    out = best_c;
    return CAVE_OK;
}

// ---------------------------------------------------------------- scheduling
cave_status Engine::consume_ring(bool* any) {
    *any = false;
    for (;;) {
        volatile DoneEntry* e = host_entries_ + (consumed_ % cfg_.max_slots);
        const uint32_t seq = e->seq;
        if (seq != consumed_ + 1u) break;
        std::atomic_thread_fence(std::memory_order_acquire);
        cave_sim_result r;
        std::memcpy(&r, const_cast<const cave_sim_result*>(&e->result), sizeof(r));
        const uint32_t slot = e->slot;
        consumed_++;
        *any = true;
        if (slot >= slots_.size() || !slots_[slot])
            return set_error(ctx_, CAVE_ERR_INTERNAL, "engine: completion for an unknown slot");
        Slot* s = slots_[slot];
        active_cells_ -= s->volume;
        if (s->mem_bytes) cells_.free(s->mem_off, s->mem_bytes);
        if (s->cls) {
            auto& v = s->cls->slots;
            v.erase(std::remove(v.begin(), v.end(), slot), v.end());
        }
        {
            std::lock_guard<std::mutex> lock(mu_);
            results_.push_back(EngineResult{s->key, r});
            stats_.finished++;
            stats_.cell_updates += (uint64_t)r.info.numberOfSimulationTicksSurvived * s->volume;
        }
        delete s;
        slots_[slot] = nullptr;
        free_slots_.push_back(slot);
    }
    return CAVE_OK;
}

cave_status Engine::retire(bool block) {
    while (!rounds_.empty()) {
        Round* r = rounds_.front();
        const double w0 = (trace_ && block) ? trace_us() : 0;
        const cudaError_t q = block ? cudaEventSynchronize(r->done) : cudaEventQuery(r->done);
        if (trace_ && block) std::fprintf(trace_, "{\"ev\":\"wait\",\"t_us\":%.1f,\"us\":%.1f}\n", w0, trace_us() - w0);
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) return check_cuda(ctx_, q, "engine round");
        cudaEventDestroy(r->done);
        delete r;
        rounds_.pop_front();
        block = false;
    }
    for (size_t i = 0; i < groups_.size();) {
        const cudaError_t q = cudaEventQuery(groups_[i]->done);
        if (q == cudaErrorNotReady) {
            i++;
            continue;
        }
        if (q != cudaSuccess) return check_cuda(ctx_, q, "engine resident launch");
        descs_.free(groups_[i]->mem_off, groups_[i]->mem_bytes);
        cudaEventDestroy(groups_[i]->done);
        delete groups_[i];
        groups_.erase(groups_.begin() + i);
    }
    return CAVE_OK;
}

// Admits pending simulations in order while slots and cell memory last.
cave_status Engine::admit(std::vector<EngineSim>& admitted) {
    {
        std::lock_guard<std::mutex> lock(mu_);
        while (!incoming_.empty()) {
            pending_.push_back(incoming_.front());
            incoming_.pop_front();
        }
        // cancelled simulations leave the queue, reported with the cancelled flag
        if (!cancels_.empty()) {
            std::deque<EngineSim> keep;
            for (EngineSim& s : pending_) {
                bool drop = false;
                for (const auto& [lo, hi] : cancels_) drop = drop || (s.key >= lo && s.key < hi);
                if (!drop) {
                    keep.push_back(s);
                    continue;
                }
                EngineResult r{};
                r.key = s.key;
                r.result.error = kErrCancelled;
                results_.push_back(r);
            }
            pending_.swap(keep);
            cancels_.clear();
        }
    }
    while (!pending_.empty() && !free_slots_.empty()) {
        EngineSim& s = pending_.front();
        const uint64_t vol = (uint64_t)s.X * s.Y * s.Z;
        if (cfg_.max_active_cells && active_cells_ && active_cells_ + vol > cfg_.max_active_cells) break;
        const ExecChoice c = choose(s);
        const uint64_t strips = grid_strips(s.X, s.Y, s.Z);
        uint64_t bytes = c.resident ? (s.init ? 0 : strips * 16) : 2 * strips * 16;
        uint64_t off = 0;
        if (bytes && !cells_.alloc(bytes, off)) break;
        const uint32_t slot = free_slots_.back();
        free_slots_.pop_back();
        Slot* sl = new Slot();
        sl->key = s.key;
        sl->resident = c.resident;
        sl->mem_off = off;
        sl->mem_bytes = bytes;
        sl->volume = vol;
        active_cells_ += vol;
        if (!c.resident) {
            StreamPlan p;
            plan_tiled(slot, s.X, s.Y, s.Z, c, p);
            sl->X = s.X;
            sl->Y = s.Y;
            sl->Z = s.Z;
            sl->rows_hint = c.rows;
            sl->pref_ctas = sl->cur_ctas = (uint32_t)p.items.size();
            sl->items = std::move(p.items);
            const auto ck = std::make_tuple(p.SXp, s.nb, s.nt, p.rows);
            TiledClass*& cls = classes_[ck];
            if (!cls) {
                cls = new TiledClass();
                cls->SXp = p.SXp;
                cls->nb = s.nb;
                cls->nt = s.nt;
                cls->rows = p.rows;
                cls->stream = (uint32_t)((classes_.size() - 1) % class_streams_.size());
            }
            cls->slots.push_back(slot);
            sl->cls = cls;
        }
        slots_[slot] = sl;
        admitted.push_back(s);
        admitted.back().key = slot;  // from here on `key` carries the slot
        admitted.back().max_ticks = s.max_ticks;
        // remember the choice for the round builder through nseg/resident
        pending_.pop_front();
        std::lock_guard<std::mutex> lock(mu_);
        stats_.admitted++;
        stats_.peak_pool_bytes = cells_.peak();
    }
    return CAVE_OK;
}

cave_status Engine::launch_round(std::vector<EngineSim>& admitted) {
    const int b = (int)(round_no_ & 1u);
    const double trace_start = trace_ ? trace_us() : 0;
    // ---- tiling for this round: each simulation's preferred CTA count (its class's cells
    // per CTA), scaled up when all active tiled simulations together would give fewer than
    // two CTAs per SM (the tail of a batch), down to 2^14 cells per CTA
    {
        uint64_t pref = 0;
        for (auto& kv : classes_)
            for (uint32_t sl : kv.second->slots) pref += slots_[sl]->pref_ctas;
        const uint64_t want = 2ull * (uint64_t)ctx_->sm_count;
        for (auto& kv : classes_)
            for (uint32_t sl : kv.second->slots) {
                Slot* s = slots_[sl];
                uint64_t t = s->pref_ctas;
                if (pref && pref < want)
                    t = std::min<uint64_t>((t * want + pref - 1) / pref, std::max<uint64_t>(t, s->volume >> 14));
                if (t != s->cur_ctas) {
                    StreamPlan p;
                    if (plan_stream(sl, s->X, s->Y, s->Z, (uint32_t)t, s->rows_hint, p) && p.rows == kv.second->rows) {
                        s->items = std::move(p.items);
                        s->cur_ctas = (uint32_t)t;
                    }
                }
            }
    }
    // ---- staging layout
    size_t n_items = 0;
    for (auto& kv : classes_)
        for (uint32_t sl : kv.second->slots) n_items += slots_[sl]->items.size();
    struct GroupKey {
        uint32_t X, Y, Z, nb, nt, nseg;
        bool operator<(const GroupKey& o) const {
            return std::tie(X, Y, Z, nb, nt, nseg) < std::tie(o.X, o.Y, o.Z, o.nb, o.nt, o.nseg);
        }
    };
    std::map<GroupKey, std::vector<size_t>> res_groups;
    std::vector<size_t> tiled_new;
    for (size_t i = 0; i < admitted.size(); i++) {
        const Slot* sl = slots_[admitted[i].key];
        if (sl->resident) {
            const ExecChoice c = plan_used_[TuneKey{admitted[i].X, admitted[i].Y, admitted[i].Z, admitted[i].nb}];
            res_groups[GroupKey{admitted[i].X, admitted[i].Y, admitted[i].Z, admitted[i].nb, admitted[i].nt,
                                c.nseg}].push_back(i);
        } else {
            tiled_new.push_back(i);
        }
    }
    const uint64_t off_recs = 0;
    const uint64_t off_slots = align_up(off_recs + sizeof(StripSim) * tiled_new.size(), 16);
    const uint64_t off_jobs = align_up(off_slots + 4 * tiled_new.size(), 16);
    const uint64_t off_res = align_up(off_jobs + sizeof(EngineJob) * admitted.size(), 16);
    uint64_t res_bytes = 0;
    for (auto& kv : res_groups) res_bytes += desc_bytes_for(kv.second.size());
    const uint64_t off_items = align_up(off_res + res_bytes, 16);
    const uint64_t total = align_up(off_items + sizeof(StreamItem) * n_items, 256);
    if (total > stage_cap_) {
        // grow both staging pairs once nothing in flight reads them
        while (!rounds_.empty())
            if (cave_status rc = retire(true); rc) return rc;
        CAVE_CUDA(ctx_, cudaStreamSynchronize(copy_));
        CAVE_CUDA(ctx_, cudaStreamSynchronize(main_));
        const uint64_t cap = std::max<uint64_t>(total * 2, 4u << 20);
        for (int i = 0; i < 2; i++) {
            cudaFreeHost(stage_h_[i]);
            cudaFree(stage_d_[i]);
            stage_h_[i] = nullptr;
            stage_d_[i] = nullptr;
            CAVE_CUDA(ctx_, cudaHostAlloc(&stage_h_[i], cap, cudaHostAllocDefault));
            CAVE_CUDA(ctx_, cudaMalloc(&stage_d_[i], cap));
        }
        stage_cap_ = cap;
    }
    unsigned char* H = stage_h_[b];
    unsigned char* D = stage_d_[b];
    // ---- records + jobs of the admitted simulations
    StripSim* hrec = reinterpret_cast<StripSim*>(H + off_recs);
    uint32_t* hslot = reinterpret_cast<uint32_t*>(H + off_slots);
    EngineJob* hjob = reinterpret_cast<EngineJob*>(H + off_jobs);
    uint32_t n_jobs = 0;
    uint64_t max_strips = 0;
    for (size_t k = 0; k < tiled_new.size(); k++) {
        const EngineSim& s = admitted[tiled_new[k]];
        const uint32_t slot = (uint32_t)s.key;
        const Slot* sl = slots_[slot];
        const uint64_t strips = grid_strips(s.X, s.Y, s.Z);
        StripSim& r = hrec[k];
        std::memset(&r, 0, sizeof(r));
        r.rule = s.rule;
        r.X = s.X;
        r.Y = s.Y;
        r.Z = s.Z;
        r.SX = (s.X + 31u) / 32u;
        r.buf[0] = sl->mem_off;
        r.buf[1] = sl->mem_off + strips * 16;
        r.max_ticks = s.max_ticks;
        r.tick_limit = s.max_ticks;
        r.stop_on_status = 1;
        r.n_items = (uint32_t)sl->items.size();
        for (int q = 0; q < 3; q++) r.acc_bmin[q] = 0xFFFFFFFFu;
        r.ring = ring_;
        r.slot = slot;
        hslot[k] = slot;
    }
    for (size_t i = 0; i < admitted.size(); i++) {
        const EngineSim& s = admitted[i];
        const Slot* sl = slots_[s.key];
        if (sl->resident && s.init) continue;  // read in place
        EngineJob& j = hjob[n_jobs++];
        j.src = s.init;
        j.dst = sl->mem_off;
        j.n_strips = grid_strips(s.X, s.Y, s.Z);
        j.seed = s.seed;
        max_strips = std::max(max_strips, j.n_strips);
    }
    // ---- resident descriptors: [queue counter | ResSim x n | DeviceRule x n] per group
    struct PendingLaunch {
        GroupKey k;
        uint64_t pool_off, bytes, stage_off;
        uint32_t n;
    };
    std::vector<PendingLaunch> launches;
    uint64_t ro = off_res;
    for (auto& [gk, idx] : res_groups) {
        const uint64_t bytes = desc_bytes_for(idx.size());
        uint64_t poff = 0;
        if (!descs_.alloc(bytes, poff))
            return set_error(ctx_, CAVE_ERR_INTERNAL, "engine: resident descriptor heap exhausted");
        unsigned char* g = H + ro;
        std::memset(g, 0, 16);
        ResSim* rs = reinterpret_cast<ResSim*>(g + 16);
        DeviceRule* rr = reinterpret_cast<DeviceRule*>(g + desc_rules_offset(idx.size()));
        for (size_t q = 0; q < idx.size(); q++) {
            const EngineSim& s = admitted[idx[q]];
            const Slot* sl = slots_[s.key];
            const uint4* init = s.init ? s.init : reinterpret_cast<const uint4*>(reinterpret_cast<unsigned char*>(pool_) + sl->mem_off);
            rs[q] = ResSim{init, (uint32_t)q, s.max_ticks, (uint32_t)s.key, 0u};
            rr[q] = s.rule;
        }
        launches.push_back(PendingLaunch{gk, poff, bytes, ro, (uint32_t)idx.size()});
        ro += bytes;
    }
    // ---- work items of every active tiled simulation, per class
    struct ClassLaunch {
        TiledClass* cls;
        uint64_t off;
        uint32_t n;
    };
    std::vector<ClassLaunch> cl;
    StreamItem* hitem = reinterpret_cast<StreamItem*>(H + off_items);
    size_t ni = 0;
    for (auto& kv : classes_) {
        TiledClass* c = kv.second;
        if (c->slots.empty()) continue;
        const size_t first = ni;
        for (uint32_t sl : c->slots) {
            const auto& it = slots_[sl]->items;
            std::memcpy(hitem + ni, it.data(), it.size() * sizeof(StreamItem));
            ni += it.size();
        }
        cl.push_back(ClassLaunch{c, off_items + first * sizeof(StreamItem), (uint32_t)(ni - first)});
    }
    if (cl.empty() && launches.empty() && n_jobs == 0 && tiled_new.empty()) return CAVE_OK;

    // ---- enqueue
    // The staging upload runs on its own stream, overlapping the previous round. When this
    // round admits simulations, their set-up (records, initial cells, resident descriptors)
    // runs on the main stream after the previous round's class work -- a slot or cell range
    // freed by a finished simulation may still be named by that round's launches -- and every
    // launch of this round waits for it. Otherwise the class streams only wait for the upload.
    cudaError_t e = cudaSuccess;
    if (!first_recorded_) {
        e = cudaEventRecord(ev_first_, main_);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(copy_, ev_first_, 0);
        first_recorded_ = true;
    }
    cudaEvent_t up = nullptr, setup = nullptr;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&up, cudaEventDisableTiming);
    if (e == cudaSuccess && total) e = cudaMemcpyAsync(D, H, total, cudaMemcpyHostToDevice, copy_);
    if (e == cudaSuccess) e = cudaEventRecord(up, copy_);
    const bool has_setup = !tiled_new.empty() || n_jobs || !launches.empty();
    if (has_setup) {
        if (e == cudaSuccess) e = cudaStreamWaitEvent(main_, up, 0);
        if (e == cudaSuccess)
            e = launch_engine_setup(reinterpret_cast<const EngineJob*>(D + off_jobs), n_jobs, max_strips, pool_,
                                    reinterpret_cast<const StripSim*>(D + off_recs),
                                    reinterpret_cast<const uint32_t*>(D + off_slots), (uint32_t)tiled_new.size(),
                                    recs_, main_);
        for (const PendingLaunch& L : launches)
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(desc_ + L.pool_off, D + L.stage_off, L.bytes, cudaMemcpyDeviceToDevice, main_);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&setup, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(setup, main_);
    }
    cudaEvent_t gate = has_setup ? setup : up;
    // resident groups: persistent launches on the resident streams
    for (const PendingLaunch& L : launches) {
        if (e != cudaSuccess) break;
        cudaStream_t st = res_streams_[res_rr_++ % res_streams_.size()];
        e = cudaStreamWaitEvent(st, gate, 0);
        uint32_t threads = 0;
        ResLaunch P = resident_geometry(L.k.X, L.k.Y, L.k.Z, L.k.nseg, threads);
        P.n_sims = L.n;
        const uint32_t ctas = std::min<uint32_t>(L.n, (uint32_t)ctx_->sm_count * resident_ctas_per_sm(P, threads));
        unsigned char* g = desc_ + L.pool_off;
        if (e == cudaSuccess)
            e = launch_resident((int)L.k.nb, (int)L.k.nt, P, reinterpret_cast<const ResSim*>(g + 16),
                                reinterpret_cast<const DeviceRule*>(g + desc_rules_offset(L.n)), nullptr,
                                reinterpret_cast<uint32_t*>(g), ring_, ctas, threads, st);
        ResGroup* rg = new ResGroup();
        rg->mem_off = L.pool_off;
        rg->mem_bytes = L.bytes;
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&rg->done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(rg->done, st);
        groups_.push_back(rg);
        std::lock_guard<std::mutex> lock(mu_);
        stats_.resident_launches++;
    }
    // tiled classes: ticks_per_round launches each; the first on each stream after the event
    // wait is launched without programmatic dependent launch
    std::vector<bool> used(class_streams_.size(), false);
    for (const ClassLaunch& c : cl) {
        if (e != cudaSuccess) break;
        cudaStream_t st = class_streams_[c.cls->stream];
        const bool first = !used[c.cls->stream];
        if (first) e = cudaStreamWaitEvent(st, gate, 0);
        used[c.cls->stream] = true;
        const StreamItem* items = reinterpret_cast<const StreamItem*>(D + c.off);
        for (uint32_t k = 0; k < cfg_.ticks_per_round && e == cudaSuccess; k++)
            e = launch_stream_tick((int)c.cls->nb, (int)c.cls->nt, nullptr, items, c.n, recs_, pool_, c.cls->SXp,
                                   c.cls->SXp, c.cls->rows * c.cls->SXp, st, !(first && k == 0));
        std::lock_guard<std::mutex> lock(mu_);
        stats_.tick_launches += cfg_.ticks_per_round;
    }
    Round* rd = new Round();
    rd->stage = b;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&rd->done, cudaEventDisableTiming);
    if (e == cudaSuccess && !has_setup) e = cudaStreamWaitEvent(main_, up, 0);
    for (size_t i = 0; i < class_streams_.size() && e == cudaSuccess; i++) {
        if (!used[i]) continue;
        cudaEvent_t j;
        e = cudaEventCreateWithFlags(&j, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(j, class_streams_[i]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(main_, j, 0);
        cudaEventDestroy(j);
    }
    if (e == cudaSuccess) e = cudaEventRecord(rd->done, main_);
    if (up) cudaEventDestroy(up);
    if (setup) cudaEventDestroy(setup);
    rounds_.push_back(rd);
    round_no_++;
    {
        std::lock_guard<std::mutex> lock(mu_);
        stats_.rounds++;
    }
    if (trace_) {
        size_t active = 0;
        for (auto& kv : classes_) active += kv.second->slots.size();
        std::fprintf(trace_,
                     "{\"ev\":\"round\",\"no\":%llu,\"t_us\":%.1f,\"enqueue_us\":%.1f,\"admitted\":%zu,"
                     "\"tiled_active\":%zu,\"classes\":%zu,\"items\":%zu,\"resident_launches\":%zu,"
                     "\"pool_bytes\":%llu}\n",
                     (unsigned long long)round_no_, trace_start, trace_us() - trace_start, admitted.size(), active,
                     cl.size(), ni, launches.size(), (unsigned long long)cells_.used());
    }
    if (e != cudaSuccess) return check_cuda(ctx_, e, "engine round");
    return CAVE_OK;
}

// Records the end of all work issued so far (for device_ms()).
cave_status Engine::finish_timing() {
    if (!first_recorded_) return CAVE_OK;
    std::vector<cudaStream_t> all = class_streams_;
    all.insert(all.end(), res_streams_.begin(), res_streams_.end());
    all.push_back(copy_);
    for (cudaStream_t st : all) {
        cudaEvent_t j;
        CAVE_CUDA(ctx_, cudaEventCreateWithFlags(&j, cudaEventDisableTiming));
        cudaEventRecord(j, st);
        cudaStreamWaitEvent(main_, j, 0);
        cudaEventDestroy(j);
    }
    CAVE_CUDA(ctx_, cudaEventRecord(ev_last_, main_));
    return CAVE_OK;
}

cave_status Engine::step(bool* idle) {
    TraceRange trace("engine_round");
    *idle = false;
    if (!ready_) return CAVE_ERR_INVALID_ARG;
    CAVE_CUDA(ctx_, cudaSetDevice(ctx_->device));
    bool any = false;
    cave_status rc = consume_ring(&any);
    if (rc) return rc;
    rc = retire(false);
    if (rc) return rc;
    bool active_tiled = false;
    for (auto& kv : classes_)
        if (!kv.second->slots.empty()) active_tiled = true;
    bool have_pending;
    {
        std::lock_guard<std::mutex> lock(mu_);
        have_pending = !incoming_.empty() || !pending_.empty();
    }
    if (rounds_.size() < 2 && (active_tiled || have_pending)) {
        std::vector<EngineSim> admitted;
        rc = admit(admitted);
        if (rc) return rc;
        for (auto& kv : classes_)
            if (!kv.second->slots.empty()) active_tiled = true;
        if (!admitted.empty() || active_tiled) {
            // rounds only start when fewer than two are in flight, so the staging pair about
            // to be written was last used by a retired round
            rc = launch_round(admitted);
            if (rc) return rc;
            return CAVE_OK;
        }
    }
    const bool busy = !rounds_.empty() || !groups_.empty() || free_slots_.size() < cfg_.max_slots;
    if (!busy) {
        std::lock_guard<std::mutex> lock(mu_);
        *idle = incoming_.empty() && pending_.empty();
        return CAVE_OK;
    }
    if (!any) {
        if (rounds_.size() >= 2)
            return retire(true);
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    return CAVE_OK;
}

cave_status Engine::after(cudaEvent_t ev) {
    CAVE_CUDA(ctx_, cudaStreamWaitEvent(main_, ev, 0));
    CAVE_CUDA(ctx_, cudaStreamWaitEvent(copy_, ev, 0));
    return CAVE_OK;
}

cave_status Engine::record_end(cudaEvent_t ev) {
    if (cave_status rc = finish_timing(); rc) return rc;
    CAVE_CUDA(ctx_, cudaEventRecord(ev, main_));
    return CAVE_OK;
}

cave_status Engine::run_until_idle() {
    for (;;) {
        bool idle = false;
        const cave_status rc = step(&idle);
        if (rc) return rc;
        if (idle) return finish_timing();
    }
}

}  // namespace cave
