// cave_ca.cpp -- C ABI of libcave_ca.so: contexts, grids, the plain path, the streaming path.
#include "../../include/cave_ca.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "context.h"
#include "jit.h"
#include "kernels.h"
#include "rules.h"
#include "trace.h"

namespace cave {

cave_status set_error(cave_ctx* ctx, cave_status code, const std::string& msg) {
    if (ctx) {
        std::lock_guard<std::mutex> lk(ctx->mu);
        ctx->last_error = msg;
    }
    return code;
}

cave_status check_cuda(cave_ctx* ctx, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return CAVE_OK;
    const cave_status code = (e == cudaErrorMemoryAllocation) ? CAVE_ERR_OUT_OF_MEMORY : CAVE_ERR_CUDA;
    return set_error(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

// Timing events of one call: 0 start, 1 before conversion, 2 first tick, 3 after the last
// tick, 4 after conversion back, 5 end.
static void record(cave_ctx* ctx, int i) {
    if (ctx->timing) cudaEventRecord(ctx->ev[i], ctx->stream);
}

static void finish_timing(cave_ctx* ctx, uint32_t ticks, uint32_t launches, bool converted) {
    if (!ctx->timing) return;
    cave_timing t{};
    t.ticks = ticks;
    t.launches = launches;
    float a = 0, b = 0, c = 0;
    cudaEventElapsedTime(&a, ctx->ev[2], ctx->ev[3]);
    if (converted) {
        cudaEventElapsedTime(&b, ctx->ev[1], ctx->ev[2]);
        cudaEventElapsedTime(&c, ctx->ev[3], ctx->ev[4]);
    }
    t.tick_ms = a;
    t.convert_ms = b + c;
    cudaEventElapsedTime(&t.total_ms, ctx->ev[0], ctx->ev[5]);
    ctx->last_timing = t;
}

static uint32_t resolve_spawn(uint32_t axis, uint32_t sizeIndex) {  // searchSystem.cpp:226-232
    if (sizeIndex == 0) return axis;
    uint32_t scaled = (uint32_t)(((uint64_t)axis * (sizeIndex + 1) + 15) / 16);
    return std::max(1u, std::min(axis, scaled));
}

SeedSpec make_seed_spec(uint32_t X, uint32_t Y, uint32_t Z, uint32_t sx, uint32_t sy, uint32_t sz,
                        uint32_t spawnSizeIndex, uint64_t threshold, bool fill_all, uint32_t seed,
                        uint32_t maxcs) {
    SeedSpec sp;
    sp.X = X;
    sp.Y = Y;
    sp.Z = Z;
    const uint32_t dims[3] = {X, Y, Z};
    const uint32_t sp_in[3] = {std::min(sx, X), std::min(sy, Y), std::min(sz, Z)};
    for (int k = 0; k < 3; k++) {
        const uint32_t e = resolve_spawn(sp_in[k], spawnSizeIndex);
        sp.lo[k] = (dims[k] - e) / 2;  // searchSystem.cpp:270-273
        sp.hi[k] = (dims[k] + e) / 2;
    }
    sp.threshold = threshold;
    sp.fill_all = fill_all ? 1u : 0u;
    sp.seed = seed;
    sp.maxcs = maxcs;
    return sp;
}

bool plan_stream(uint32_t sim_index, uint32_t X, uint32_t Y, uint32_t Z, uint32_t target_ctas, uint32_t rows_hint,
                 StreamPlan& plan, uint32_t spt, uint32_t halo, uint32_t max_threads) {
    const uint32_t SX = (X + 31u) / 32u;
    if (SX == 0 || SX > 32 || Y == 0 || Z == 0 || Y > 65535 || Z > 65535 || spt < 1 || spt > 3 || halo < 1 ||
        halo > 2)
        return false;
    uint32_t SXp = 1;
    while (SXp < SX) SXp <<= 1;
    const uint32_t step = std::max(1u, 32u / SXp) * spt;  // rows must keep threads a multiple of 32
    const uint32_t most_threads =
        max_threads ? max_threads : (halo == 2 ? (uint32_t)kJit2MaxThreads : spt == 1 ? 1024u : (uint32_t)kJitMaxThreads);
    uint32_t rows = rows_hint ? rows_hint : std::max((spt == 1 ? 512u : most_threads) * spt / SXp, 2 * halo + 1);
    rows = std::min(rows, most_threads * spt / SXp);
    rows = std::min(rows, Y + 2u * halo);
    rows = (rows + step - 1) / step * step;
    while (rows < 2 * halo + 1) rows += step;
    const uint32_t TY = rows - 2 * halo;
    const uint32_t ny = (Y + TY - 1) / TY;
    const uint32_t ty = (Y + ny - 1) / ny;
    uint32_t nz = std::max(1u, target_ctas / ny);
    nz = std::min(nz, Z);
    const uint32_t slab = (Z + nz - 1) / nz;
    nz = (Z + slab - 1) / slab;
    plan.SX = SX;
    plan.SXp = SXp;
    plan.rows = rows;
    plan.threads = rows * SXp / spt;
    plan.ny = ny;
    plan.nz = nz;
    plan.items.clear();
    for (uint32_t iz = 0; iz < nz; iz++) {
        for (uint32_t iy = 0; iy < ny; iy++) {
            StreamItem it;
            it.sim = sim_index;
            it.y0 = (uint16_t)(iy * ty);
            it.ty = (uint16_t)std::min(ty, Y - iy * ty);
            it.z0 = (uint16_t)(iz * slab);
            it.z1 = (uint16_t)std::min(Z, (iz + 1) * slab);
            it.dir_items = iz & 1u;
            plan.items.push_back(it);
        }
    }
    for (StreamItem& it : plan.items) it.dir_items |= (uint32_t)plan.items.size() << 1;
    return true;
}

}  // namespace cave

using namespace cave;

extern "C" {

const char* cave_status_string(cave_status s) {
    switch (s) {
        case CAVE_OK: return "ok";
        case CAVE_ERR_INVALID_ARG: return "invalid argument";
        case CAVE_ERR_CUDA: return "CUDA error";
        case CAVE_ERR_OUT_OF_MEMORY: return "out of device memory";
        case CAVE_ERR_NOT_READY: return "not ready";
        case CAVE_ERR_TIMEOUT: return "device-side wait timed out";
        case CAVE_ERR_IO: return "I/O error";
        case CAVE_ERR_INTERNAL: return "internal error";
        default: return "unknown status";
    }
}

const char* cave_last_error(const cave_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "no context"; }

cave_status cave_ctx_create(int device, cave_ctx** out) {
    if (!out) return CAVE_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || device < 0 || device >= n) return CAVE_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return CAVE_ERR_CUDA;
    if (prop.major != 10) return CAVE_ERR_CUDA;  // the kernels are built for sm_100a only
    cave_ctx* c = new (std::nothrow) cave_ctx();
    if (!c) return CAVE_ERR_OUT_OF_MEMORY;
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    c->smem_optin = (int)prop.sharedMemPerBlockOptin;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return CAVE_ERR_CUDA;
    }
    *out = c;
    return CAVE_OK;
}

void cave_ctx_destroy(cave_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
    }
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (const cave::StagingPair& sp : ctx->staging_free)
        for (int i = 0; i < 2; i++) {
            cudaFreeHost(sp.h[i]);
            cudaFree(sp.d[i]);
        }
    delete ctx;
}

cave_status cave_ctx_synchronize(cave_ctx* ctx) {
    if (!ctx) return CAVE_ERR_INVALID_ARG;
    CAVE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CAVE_OK;
}

uint64_t cave_grid_words(uint32_t X, uint32_t Y, uint32_t Z) { return (uint64_t)((X + 7u) / 8u) * Y * Z; }

static cave::PlainSlot fresh_slot() {
    cave::PlainSlot s;
    std::memset(&s, 0, sizeof(s));
    for (int k = 0; k < 3; k++) {
        s.bmin[k] = 0xFFFFFFFFu;
        s.bmax[k] = 0;
    }
    return s;
}

cave_status cave_grid_create(cave_ctx* ctx, uint32_t X, uint32_t Y, uint32_t Z, cave_grid** out) {
    if (!ctx || !out) return CAVE_ERR_INVALID_ARG;
    *out = nullptr;
    if (X == 0 || Y == 0 || Z == 0 || (uint64_t)X * Y * Z >= (1ull << 32))
        return set_error(ctx, CAVE_ERR_INVALID_ARG, "grid volume must be in [1, 2^32)");
    CAVE_CUDA(ctx, cudaSetDevice(ctx->device));
    cave_grid* g = new (std::nothrow) cave_grid();
    if (!g) return CAVE_ERR_OUT_OF_MEMORY;
    g->ctx = ctx;
    g->X = X;
    g->Y = Y;
    g->Z = Z;
    g->words = cave_grid_words(X, Y, Z);
    cudaError_t e = cudaMalloc(&g->nib[0], g->words * 4 * 2);
    if (e == cudaSuccess) {
        g->nib[1] = g->nib[0] + g->words;
        e = cudaMalloc(&g->slot, sizeof(cave::PlainSlot));
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(g->nib[0], 0, g->words * 4 * 2, ctx->stream);
    if (e == cudaSuccess) {
        cave::PlainSlot s = fresh_slot();
        e = cudaMemcpyAsync(g->slot, &s, sizeof(s), cudaMemcpyHostToDevice, ctx->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(g->nib[0]);
        cudaFree(g->slot);
        delete g;
        return check_cuda(ctx, e, "cave_grid_create");
    }
    *out = g;
    return CAVE_OK;
}

void cave_grid_destroy(cave_grid* g) {
    if (!g) return;
    cudaSetDevice(g->ctx->device);
    cudaStreamSynchronize(g->ctx->stream);
    cudaFree(g->nib[0]);
    cudaFree(g->slot);
    cudaFree(g->strips);
    cudaFree(g->sim);
    delete g;
}

cave_status cave_grid_upload(cave_grid* g, const uint32_t* words, uint64_t nwords) {
    if (!g || !words || nwords != g->words) return CAVE_ERR_INVALID_ARG;
    cave_ctx* ctx = g->ctx;
    CAVE_CUDA(ctx, cudaSetDevice(ctx->device));
    CAVE_CUDA(ctx, cudaMemcpyAsync(g->nib[g->cur], words, nwords * 4, cudaMemcpyHostToDevice, ctx->stream));
    CAVE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CAVE_OK;
}

cave_status cave_grid_download(cave_grid* g, uint32_t* words, uint64_t nwords) {
    if (!g || !words || nwords != g->words) return CAVE_ERR_INVALID_ARG;
    cave_ctx* ctx = g->ctx;
    CAVE_CUDA(ctx, cudaSetDevice(ctx->device));
    CAVE_CUDA(ctx, cudaMemcpyAsync(words, g->nib[g->cur], nwords * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CAVE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CAVE_OK;
}

static cave_status seed_grid(cave_grid* g, const SeedSpec& sp) {
    cave_ctx* ctx = g->ctx;
    CAVE_CUDA(ctx, cudaSetDevice(ctx->device));
    CAVE_CUDA(ctx, launch_seed_nib(g->nib[g->cur], sp, ctx->stream));
    CAVE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CAVE_OK;
}

cave_status cave_grid_seed(cave_grid* g, const cave_chunk_config* c, uint32_t maxCellState) {
    if (!g || !c || c->spawnDensityIndex > 15) return CAVE_ERR_INVALID_ARG;
    if (c->gridDimensionX != g->X || c->gridDimensionY != g->Y || c->gridDimensionZ != g->Z)
        return set_error(g->ctx, CAVE_ERR_INVALID_ARG, "chunk grid dimensions differ from the grid's");
    const bool random = c->spawnRegionShapeId == 0;  // searchSystem.cpp:238
    const float density = ((float)c->spawnDensityIndex + 1.0f) / 16.0f;  // :240
    const bool all = !random || density >= 1.0f;
    const uint64_t thr = all ? (1ull << 32) : (uint64_t)(uint32_t)(density * 4294967296.0);  // :260-262
    SeedSpec sp = make_seed_spec(g->X, g->Y, g->Z, c->spawnAreaDimensionX, c->spawnAreaDimensionY,
                                 c->spawnAreaDimensionZ, c->spawnSizeIndex, thr, all, c->runSeedIndex, maxCellState);
    return seed_grid(g, sp);
}

cave_status cave_grid_seed_threshold(cave_grid* g, uint32_t spawnX, uint32_t spawnY, uint32_t spawnZ,
                                     uint64_t threshold, uint32_t runSeedIndex, uint32_t maxCellState) {
    if (!g || threshold > (1ull << 32)) return CAVE_ERR_INVALID_ARG;
    SeedSpec sp = make_seed_spec(g->X, g->Y, g->Z, spawnX, spawnY, spawnZ, 0, threshold, threshold == (1ull << 32),
                                 runSeedIndex, maxCellState);
    return seed_grid(g, sp);
}

// Device copy of the K-index table (nullptr when not used).
struct DevTable {
    uint64_t* p = nullptr;
    ~DevTable() { cudaFree(p); }
};

cave_status cave_step(cave_grid* g, const cave_sim_params* params, const uint64_t* validBitmasks, uint32_t nValid,
                      uint32_t maxRuleBits, uint32_t nticks, cave_tick_stats* per_tick) {
    if (!g || !params) return CAVE_ERR_INVALID_ARG;
    TraceRange trace("cave_step");
    cave_ctx* ctx = g->ctx;
    DecodedRule d;
    if (!decode_params(*params, validBitmasks, nValid, maxRuleBits, d))
        return set_error(ctx, CAVE_ERR_INVALID_ARG, "rule index outside the valid-bitmask table");
    if (nticks == 0) return CAVE_OK;
    CAVE_CUDA(ctx, cudaSetDevice(ctx->device));
    DevTable tab;
    if (maxRuleBits > 0) {
        CAVE_CUDA(ctx, cudaMalloc(&tab.p, sizeof(uint64_t) * nValid));
        CAVE_CUDA(ctx, cudaMemcpyAsync(tab.p, validBitmasks, sizeof(uint64_t) * nValid, cudaMemcpyHostToDevice, ctx->stream));
    }
    cave_tick_stats* dticks = nullptr;
    if (per_tick) CAVE_CUDA(ctx, cudaMalloc(&dticks, sizeof(cave_tick_stats) * nticks));
    PlainSlot s = fresh_slot();
    s.perms = *params;
    s.run_manager = 0;
    s.per_tick = dticks;
    cudaError_t e = cudaMemcpyAsync(g->slot, &s, sizeof(s), cudaMemcpyHostToDevice, ctx->stream);
    record(ctx, 0);
    record(ctx, 2);
    for (uint32_t t = 0; t < nticks && e == cudaSuccess; t++) {
        e = launch_plain_step(g->nib[g->cur], g->nib[g->cur ^ 1], g->X, g->Y, g->Z, g->slot, tab.p, nValid,
                              maxRuleBits, ctx->stream);
        g->cur ^= 1;
    }
    record(ctx, 3);
    if (e == cudaSuccess && per_tick)
        e = cudaMemcpyAsync(per_tick, dticks, sizeof(cave_tick_stats) * nticks, cudaMemcpyDeviceToHost, ctx->stream);
    PlainSlot back;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&back, g->slot, sizeof(back), cudaMemcpyDeviceToHost, ctx->stream);
    record(ctx, 5);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(dticks);
    if (e != cudaSuccess) return check_cuda(ctx, e, "cave_step");
    finish_timing(ctx, nticks, nticks, false);
    if (back.error) return set_error(ctx, CAVE_ERR_INTERNAL, "plain kernel raised an error flag");
    return CAVE_OK;
}

static cave_status run_impl(cave_grid* g, const uint32_t* host_in, uint32_t* host_out, const cave_sim_params* params,
                            const uint64_t* validBitmasks, uint32_t nValid, uint32_t maxRuleBits, uint32_t nticks,
                            uint32_t maxTicks, cave_tick_stats* per_tick, cave_grid_info* info);

cave_status cave_run(cave_grid* g, const cave_sim_params* params, const uint64_t* validBitmasks, uint32_t nValid,
                     uint32_t maxRuleBits, uint32_t nticks, uint32_t maxTicks, cave_tick_stats* per_tick,
                     cave_grid_info* info) {
    return run_impl(g, nullptr, nullptr, params, validBitmasks, nValid, maxRuleBits, nticks, maxTicks, per_tick, info);
}

cave_status cave_run_host(cave_grid* g, const uint32_t* in_words, uint32_t* out_words, uint64_t nwords,
                          const cave_sim_params* params, const uint64_t* validBitmasks, uint32_t nValid,
                          uint32_t maxRuleBits, uint32_t nticks, uint32_t maxTicks, cave_tick_stats* per_tick,
                          cave_grid_info* info) {
    if (!g || !in_words || !out_words || nwords != g->words) return CAVE_ERR_INVALID_ARG;
    return run_impl(g, in_words, out_words, params, validBitmasks, nValid, maxRuleBits, nticks, maxTicks, per_tick,
                    info);
}

cave_status cave_prepare_rule(cave_ctx* ctx, const cave_sim_params* params, const uint64_t* validBitmasks,
                              uint32_t nValid, uint32_t maxRuleBits) {
    if (!ctx || !params) return CAVE_ERR_INVALID_ARG;
    DecodedRule d;
    if (!decode_params(*params, validBitmasks, nValid, maxRuleBits, d))
        return set_error(ctx, CAVE_ERR_INVALID_ARG, "rule index outside the valid-bitmask table");
    const JitMode jm = jit_mode();
    if (jm == JitMode::Off) return CAVE_OK;
    CAVE_CUDA(ctx, cudaSetDevice(ctx->device));
    const JitKey k = jit_key(make_device_rule(d));
    if (jit_stream_kernel(k, JitMode::Sync, true)) return CAVE_OK;
    std::string log;
    jit_compile(k, &log);
    return set_error(ctx, CAVE_ERR_INTERNAL, "rule-specialised kernel unavailable: " + log.substr(0, 2000));
}

cave_status cave_jit_compile_async(const cave_sim_params* params, const uint64_t* validBitmasks, uint32_t nValid,
                                   uint32_t maxRuleBits) {
    if (!params) return CAVE_ERR_INVALID_ARG;
    DecodedRule d;
    if (!decode_params(*params, validBitmasks, nValid, maxRuleBits, d)) return CAVE_ERR_INVALID_ARG;
    if (jit_mode() != JitMode::Off) jit_compile_async(jit_key(make_device_rule(d)));
    return CAVE_OK;
}

cave_status cave_jit_compile(const cave_sim_params* params, const uint64_t* validBitmasks, uint32_t nValid,
                             uint32_t maxRuleBits, char* log, size_t log_size) {
    if (!params) return CAVE_ERR_INVALID_ARG;
    DecodedRule d;
    if (!decode_params(*params, validBitmasks, nValid, maxRuleBits, d)) return CAVE_ERR_INVALID_ARG;
    std::string text;
    const bool ok = jit_compile(jit_key(make_device_rule(d)), &text);
    if (log && log_size) {
        const size_t n = std::min(text.size(), log_size - 1);
        std::memcpy(log, text.data(), n);
        log[n] = '\0';
    }
    return ok ? CAVE_OK : CAVE_ERR_INTERNAL;
}

cave_status cave_ctx_set_timing(cave_ctx* ctx, int enable) {
    if (!ctx) return CAVE_ERR_INVALID_ARG;
    CAVE_CUDA(ctx, cudaSetDevice(ctx->device));
    if (enable && !ctx->ev[0]) {
        for (auto& e : ctx->ev) CAVE_CUDA(ctx, cudaEventCreate(&e));
    }
    ctx->timing = enable != 0;
    return CAVE_OK;
}

cave_status cave_ctx_last_timing(const cave_ctx* ctx, cave_timing* out) {
    if (!ctx || !out) return CAVE_ERR_INVALID_ARG;
    *out = ctx->last_timing;
    return CAVE_OK;
}

}  // extern "C"

// Rows per CTA for cave_run's tick launches. The default (512 threads' worth of rows) is usually
// best, but the last row tile of a grid can waste most of its CTA (256^3: 5 tiles of 62 rows for
// 256), and no closed rule picked the fastest shape for every size measured. So the first long
// run of a grid shape times a few candidates -- the default and the seven with the least total
// row work (tiles x rows per tile) at up to 576 threads, the most that keeps two CTAs per SM --
// for five launches each and keeps the fastest per context (the default unless another is more
// than 2% faster: short trials are noisy). With the rule-specialised kernels the candidates stay
// within those kernels' thread limit (kJitMaxThreads, kJit2MaxThreads) and, for the two-tick
// kernels, within the shared memory of one CTA. The trial launches read the run's input copy and
// write the other one, which the first real launch overwrites, and add to the first statistics
// slots, which are cleared afterwards; results do not depend on the tile shape.
constexpr uint32_t kTuneMinTicks = 100;

// The tick kernels cave_run can use: the library's own (rule read at run time), the
// rule-specialised single-tick kernels, and the rule-specialised two-tick kernels.
enum RunKind : uint32_t { kRunGeneric = 0, kRunJit = 1, kRunJitPair = 2 };

static uint32_t kind_spt(uint32_t kind) {
    return kind == kRunGeneric ? 1u : kind == kRunJit ? (uint32_t)kJitRowsPerThread : tick2_geometry().rows_per_thread;
}
static uint32_t kind_halo(uint32_t kind) { return kind == kRunJitPair ? 2u : 1u; }
static uint32_t kind_max_threads(uint32_t kind) {
    return kind == kRunGeneric ? 1024u : kind == kRunJit ? (uint32_t)kJitMaxThreads : tick2_geometry().max_threads;
}
// Dynamic shared memory the two-tick kernels may take (their static share is a few KB).
static bool pair_smem_fits(const cave_ctx* ctx, const StreamPlan& p, uint32_t per_sm = 1) {
    const size_t need = tick2_smem_bytes(p.rows, p.SX, p.SXp) + 4096;
    // one CTA: the opt-in limit; several: their share of the SM's 228 KB
    return per_sm <= 1 ? need <= (size_t)ctx->smem_optin : need * per_sm <= 228u * 1024u;
}

// The plan of one cave_run tile shape: `rows` per CTA (0 = default) for tick kernels of `kind`.
// Generic kernels: `cps` CTAs per SM (default 2). Rule-specialised kernels (one CTA of up to
// their thread limit per SM, by registers): as many CTAs per SM as limit-sized equivalents,
// unless `cps` was given. Two-tick kernels: rows shrink until the CTA's shared memory fits.
static bool run_plan(const cave_ctx* ctx, const cave_grid* g, uint32_t rows, uint32_t kind, uint32_t cps,
                     bool cps_given, StreamPlan& plan) {
    const uint32_t sms = (uint32_t)ctx->sm_count;
    const uint32_t spt = kind_spt(kind), halo = kind_halo(kind), most = kind_max_threads(kind);
    if (kind == kRunGeneric) return plan_stream(0, g->X, g->Y, g->Z, sms * cps, rows, plan, 1);
    // CTAs per SM the kernels are built for (the two-tick kernels may be built for several)
    const uint32_t per_sm = cps_given ? cps : kind == kRunJitPair ? tick2_geometry().ctas_per_sm : 1u;
    if (!plan_stream(0, g->X, g->Y, g->Z, sms * per_sm, rows, plan, spt, halo, most)) return false;
    if (kind == kRunJitPair) {
        const uint32_t step = std::max(1u, 32u / plan.SXp) * spt;
        while (!pair_smem_fits(ctx, plan, per_sm)) {
            if (plan.rows < 2 * halo + 1 + step) return false;
            if (!plan_stream(0, g->X, g->Y, g->Z, sms * per_sm, plan.rows - step, plan, spt, halo, most)) return false;
        }
    }
    if (!cps_given && plan.threads < most)
        return plan_stream(0, g->X, g->Y, g->Z, sms * per_sm * (most / plan.threads), plan.rows, plan, spt, halo,
                           most);
    return true;
}

static std::vector<uint32_t> row_candidates(const cave_ctx* ctx, uint32_t X, uint32_t Y, uint32_t rows0,
                                            uint32_t kind) {
    const uint32_t SX = (X + 31u) / 32u;
    uint32_t SXp = 1;
    while (SXp < SX) SXp <<= 1;
    const uint32_t spt = kind_spt(kind), halo = kind_halo(kind);
    const uint32_t step = std::max(1u, 32u / SXp) * spt;
    const uint32_t hi = std::min((kind == kRunGeneric ? 576u : kind_max_threads(kind)) * spt / SXp, Y + 2u * halo);
    std::vector<std::pair<uint64_t, uint32_t>> scored;
    for (uint32_t r = std::max((2 * halo + 1) * step, (rows0 / 2 + step - 1) / step * step); r <= hi; r += step) {
        if (r == rows0 || r < 2 * halo + 1) continue;
        if (kind == kRunJitPair) {
            StreamPlan p;
            p.rows = r;
            p.SX = SX;
            p.SXp = SXp;
            if (!pair_smem_fits(ctx, p, tick2_geometry().ctas_per_sm)) continue;
        }
        const uint64_t tiles = (Y + (r - 2 * halo) - 1) / (r - 2 * halo);
        scored.push_back({tiles * r, r});
    }
    std::sort(scored.begin(), scored.end());
    std::vector<uint32_t> out{rows0};
    for (size_t i = 0; i < scored.size() && out.size() < 8; i++) out.push_back(scored[i].second);
    return out;
}

// One launch of cave_run's tick loop: ticks `tick` (and tick + 1 for the two-tick kernels),
// reading cell copy `sel` (the single-tick kernels take it from the tick's parity).
static cudaError_t launch_run_tick(cave_ctx* ctx, cave_grid* g, uint32_t kind, const DeviceRule& rule,
                                   const JitKernels& jk, const StreamPlan& plan, const StreamItem* ditems, bool first,
                                   bool pdl, uint32_t tick, uint32_t sel) {
    const uint32_t n = (uint32_t)plan.items.size();
    const bool dense = plan.SX == plan.SXp;
    switch (kind) {
        case kRunJitPair:
            return launch_stream_tick2_jit(jk.pick2(first, dense), ditems, n, g->sim, g->strips, plan.SX, plan.SXp,
                                           plan.threads, ctx->stream, pdl, (int)tick, (int)sel);
        case kRunJit:
            return launch_stream_tick_jit(jk.pick(first, dense), ditems, n, g->sim, g->strips, plan.SX, plan.SXp,
                                          plan.threads, ctx->stream, pdl, (int)tick);
        default:
            return launch_stream_tick((int)(rule.flags & 7u), (int)rule.nterms, &rule, ditems, n, g->sim, g->strips,
                                      plan.SX, plan.SXp, plan.threads, ctx->stream, pdl, (int)tick);
    }
}

// Times one candidate plan: one untimed launch then five timed ones (tick index 0 each time).
static cudaError_t time_plan(cave_ctx* ctx, cave_grid* g, uint32_t kind, const DeviceRule& rule, const JitKernels& jk,
                             const StreamPlan& plan, StreamItem* ditems, cudaEvent_t e0, cudaEvent_t e1, float* ms) {
    cudaError_t e = cudaMemcpyAsync(ditems, plan.items.data(), sizeof(StreamItem) * plan.items.size(),
                                    cudaMemcpyHostToDevice, ctx->stream);
    for (int i = 0; i < 6 && e == cudaSuccess; i++) {
        if (i == 1) e = cudaEventRecord(e0, ctx->stream);
        if (e == cudaSuccess) e = launch_run_tick(ctx, g, kind, rule, jk, plan, ditems, true, i > 0, 0, 0);
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, ctx->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    return e;
}

// cave_run's tick kernels by default use two ticks per launch when the rule-specialised kernels
// are ready and the run has two ticks or more; CAVE_TICK2=0 keeps one tick per launch.
static bool pair_ticks_enabled() {
    const char* v = std::getenv("CAVE_TICK2");
    return !(v && (!std::strcmp(v, "0") || !std::strcmp(v, "off")));
}


static cave_status run_impl(cave_grid* g, const uint32_t* host_in, uint32_t* host_out, const cave_sim_params* params,
                            const uint64_t* validBitmasks, uint32_t nValid, uint32_t maxRuleBits, uint32_t nticks,
                            uint32_t maxTicks, cave_tick_stats* per_tick, cave_grid_info* info) {
    if (!g || !params) return CAVE_ERR_INVALID_ARG;
    TraceRange trace(host_in ? "cave_run_host" : "cave_run");
    cave_ctx* ctx = g->ctx;
    DecodedRule d;
    if (!decode_params(*params, validBitmasks, nValid, maxRuleBits, d))
        return set_error(ctx, CAVE_ERR_INVALID_ARG, "rule index outside the valid-bitmask table");
    StreamPlan plan;
    // Tile-shape overrides for tuning sweeps: CAVE_STREAM_ROWS (rows per CTA incl. halo) and
    // CAVE_STREAM_CTAS_PER_SM (CTAs per tick per SM).
    const char* env_rows = std::getenv("CAVE_STREAM_ROWS");
    const char* env_cps = std::getenv("CAVE_STREAM_CTAS_PER_SM");
    const uint32_t rows_hint = env_rows ? (uint32_t)std::atoi(env_rows) : 0u;
    const uint32_t cps = env_cps ? std::max(1, std::atoi(env_cps)) : 2u;
    if (!plan_stream(0, g->X, g->Y, g->Z, (uint32_t)ctx->sm_count * cps, rows_hint, plan))
        return set_error(ctx, CAVE_ERR_INVALID_ARG,
                         "grid shape not supported by the streaming kernel (X <= 1024, Y, Z <= 65535)");
    CAVE_CUDA(ctx, cudaSetDevice(ctx->device));
    const uint64_t nstrips = (uint64_t)plan.SX * g->Y * g->Z;
    if (!g->strips) {
        CAVE_CUDA(ctx, cudaMalloc(&g->strips, nstrips * 16 * 2));
        CAVE_CUDA(ctx, cudaMalloc(&g->sim, sizeof(StripSim)));
        g->strip_count = nstrips;
    }
    StripSim s;
    std::memset(&s, 0, sizeof(s));
    s.rule = make_device_rule(d);
    s.X = g->X;
    s.Y = g->Y;
    s.Z = g->Z;
    s.SX = plan.SX;
    s.buf[0] = 0;
    s.buf[1] = nstrips * 16;
    s.max_ticks = maxTicks;
    s.tick_limit = nticks;
    s.stop_on_status = 0;
    s.n_items = (uint32_t)plan.items.size();
    for (int k = 0; k < 3; k++) s.acc_bmin[k] = 0xFFFFFFFFu;
    cave_tick_stats* dticks = nullptr;
    StreamItem* ditems = nullptr;
    TickTotals* dtt = nullptr;  // per-tick totals: the statistics are folded after the last tick
    if (per_tick && nticks) CAVE_CUDA(ctx, cudaMalloc(&dticks, sizeof(cave_tick_stats) * nticks));
    s.per_tick = dticks;
    cudaError_t e = nticks ? cudaMalloc(&dtt, sizeof(TickTotals) * nticks) : cudaSuccess;
    if (e == cudaSuccess && nticks) e = cudaMemsetAsync(dtt, 0, sizeof(TickTotals) * nticks, ctx->stream);
    s.deferred = dtt;
    if (e == cudaSuccess) e = cudaMemcpyAsync(g->sim, &s, sizeof(s), cudaMemcpyHostToDevice, ctx->stream);
    record(ctx, 0);
    if (e == cudaSuccess && host_in)
        e = cudaMemcpyAsync(g->nib[g->cur], host_in, g->words * 4, cudaMemcpyHostToDevice, ctx->stream);
    record(ctx, 1);
    if (e == cudaSuccess) e = launch_nib_to_strips(g->nib[g->cur], g->strips, g->X, g->Y, g->Z, ctx->stream);
    record(ctx, 2);
    // the rule-specialised kernels when they are ready (jit.h), else the generic one; with them
    // two ticks per launch unless disabled (the run's first launch counts every statistic; later
    // ones leave the zero cells to the fold)
    const JitMode jm = jit_mode();
    const JitKernels jk = nticks ? jit_stream_kernel(jit_key(s.rule), jm, (uint64_t)g->X * g->Y * g->Z >= kJitMinCells)
                                 : JitKernels{};
    uint32_t kind = !jk ? kRunGeneric : (nticks >= 2 && jk.pair[0] && pair_ticks_enabled()) ? kRunJitPair : kRunJit;
    if (e == cudaSuccess && !run_plan(ctx, g, rows_hint, kind, cps, env_cps != nullptr, plan)) {
        if (kind != kRunJitPair) return set_error(ctx, CAVE_ERR_INTERNAL, "streaming plan failed");
        kind = kRunJit;  // the grid's rows do not fit the two-tick kernel's shared memory
        if (!run_plan(ctx, g, rows_hint, kind, cps, env_cps != nullptr, plan))
            return set_error(ctx, CAVE_ERR_INTERNAL, "streaming plan failed");
    }
    // tile shape (and, with the rule-specialised kernels, one or two ticks per launch): an
    // override, the context's earlier choice for this shape, or a timing pass
    if (e == cudaSuccess && !rows_hint && nticks >= kTuneMinTicks && (uint64_t)g->X * g->Y * g->Z >= kJitMinCells) {
        const TuneKey key{g->X, g->Y, g->Z, (d.flags & 7u) + 8u * kind};
        RunChoice choice{};
        {
            std::lock_guard<std::mutex> lk(ctx->tune_mu);
            auto it = ctx->run_rows.find(key);
            if (it != ctx->run_rows.end()) choice = it->second;
        }
        if (!choice.rows) {
            // candidates of the kernel kind in use and, when that is the two-tick kind, of the
            // single-tick specialised kernels too; compared per tick
            struct Cand {
                uint32_t kind;
                StreamPlan plan;
            };
            std::vector<Cand> cands;
            size_t most = 0;
            const uint32_t kinds[2] = {kind, kind == kRunJitPair ? (uint32_t)kRunJit : kind};
            for (int ki = 0; ki < (kinds[1] != kinds[0] ? 2 : 1); ki++) {
                StreamPlan base;
                if (!run_plan(ctx, g, 0, kinds[ki], cps, env_cps != nullptr, base)) continue;
                for (uint32_t r : row_candidates(ctx, g->X, g->Y, base.rows, kinds[ki])) {
                    Cand c{kinds[ki], {}};
                    if (!run_plan(ctx, g, r, kinds[ki], cps, env_cps != nullptr, c.plan)) continue;
                    most = std::max(most, c.plan.items.size());
                    cands.push_back(std::move(c));
                }
            }
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            StreamItem* titems = nullptr;
            e = cudaEventCreate(&e0);
            if (e == cudaSuccess) e = cudaEventCreate(&e1);
            if (e == cudaSuccess) e = cudaMalloc(&titems, sizeof(StreamItem) * std::max<size_t>(most, 1));
            float best = 1e30f;
            choice = RunChoice{kind, plan.rows};
            for (const Cand& c : cands) {
                float ms = 0;
                if (e == cudaSuccess) e = time_plan(ctx, g, c.kind, s.rule, jk, c.plan, titems, e0, e1, &ms);
                if (c.kind == kRunJitPair) ms *= 0.5f;  // two ticks per launch
                if (e == cudaSuccess && c.kind == kind && c.plan.rows == plan.rows)
                    ms *= 0.98f;  // a challenger must beat the default by 2%
                if (e == cudaSuccess && ms < best) {
                    best = ms;
                    choice = RunChoice{c.kind, c.plan.rows};
                }
            }
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            cudaFree(titems);
            if (e == cudaSuccess) e = cudaMemsetAsync(dtt, 0, sizeof(TickTotals) * 2, ctx->stream);
            if (e == cudaSuccess) {
                std::lock_guard<std::mutex> lk(ctx->tune_mu);
                ctx->run_rows[key] = choice;
            }
        }
        if (e == cudaSuccess && (choice.kind != kind || choice.rows != plan.rows)) {
            kind = choice.kind;
            if (!run_plan(ctx, g, choice.rows, kind, cps, env_cps != nullptr, plan))
                return set_error(ctx, CAVE_ERR_INTERNAL, "tile shape chosen by the timing pass could not be planned");
        }
    }
    // an odd tick count with the two-tick kernels: tick 0 alone first, with the single-tick plan
    StreamPlan plan1;
    const bool lead = kind == kRunJitPair && (nticks & 1u);
    if (e == cudaSuccess && lead && !run_plan(ctx, g, 0, kRunJit, cps, env_cps != nullptr, plan1))
        return set_error(ctx, CAVE_ERR_INTERNAL, "streaming plan failed");
    const size_t n_main = plan.items.size(), n_lead = lead ? plan1.items.size() : 0;
    if (e == cudaSuccess) e = cudaMalloc(&ditems, sizeof(StreamItem) * (n_main + n_lead));
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ditems, plan.items.data(), sizeof(StreamItem) * n_main, cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess && lead)
        e = cudaMemcpyAsync(ditems + n_main, plan1.items.data(), sizeof(StreamItem) * n_lead, cudaMemcpyHostToDevice,
                            ctx->stream);
    // The tick launches. A launch reads cell copy `sel` and writes the other one.
    // CAVE_RUN_GRAPH=1 (a measurement mode) captures them into a CUDA graph and replays it; the
    // tick timing then covers the replay alone (instantiation falls in convert_ms).
    const char* env_graph = std::getenv("CAVE_RUN_GRAPH");
    const bool use_graph = env_graph && !std::strcmp(env_graph, "1") && nticks > 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    if (use_graph && e == cudaSuccess) e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed);
    uint32_t sel = 0, launches = 0;
    nvtxRangePushA("ticks");
    if (kind == kRunJitPair) {
        uint32_t t = 0;
        if (lead && e == cudaSuccess) {
            e = launch_run_tick(ctx, g, kRunJit, s.rule, jk, plan1, ditems + n_main, true, true, 0, 0);
            t = 1;
            sel = 1;
            launches++;
        }
        for (; t + 1 < nticks && e == cudaSuccess; t += 2) {
            e = launch_run_tick(ctx, g, kind, s.rule, jk, plan, ditems, t == 0, true, t, sel);
            sel ^= 1u;
            launches++;
        }
    } else {
        for (uint32_t t = 0; t < nticks && e == cudaSuccess; t++)
            e = launch_run_tick(ctx, g, kind, s.rule, jk, plan, ditems, t == 0, true, t, t & 1u);
        sel = nticks & 1u;
        launches = nticks;
    }
    if (use_graph) {
        const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &graph);
        if (e == cudaSuccess) e = ec;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&gexec, graph, 0);
        record(ctx, 2);
        if (e == cudaSuccess) e = cudaGraphLaunch(gexec, ctx->stream);
    }
    nvtxRangePop();
    if (e == cudaSuccess && nticks && jk)  // the last tick's population comes from the final grid
        e = launch_strip_stats(g->strips + (uint64_t)sel * nstrips, g->Y, g->Z, plan.SX, dtt + (nticks - 1),
                               (uint32_t)ctx->sm_count, ctx->stream);
    if (e == cudaSuccess && nticks) e = launch_fold_deferred(g->sim, dtt, nticks, (bool)jk, ctx->stream);
    record(ctx, 3);
    // Raw stepping never stops early, so the result is in copy `sel`.
    if (e == cudaSuccess)
        e = launch_strips_to_nib(g->strips + (uint64_t)sel * nstrips, g->nib[g->cur], g->X, g->Y, g->Z, ctx->stream);
    record(ctx, 4);
    if (e == cudaSuccess && host_out)
        e = cudaMemcpyAsync(host_out, g->nib[g->cur], g->words * 4, cudaMemcpyDeviceToHost, ctx->stream);
    StripSim back;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&back, g->sim, sizeof(back), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && per_tick && nticks)
        e = cudaMemcpyAsync(per_tick, dticks, sizeof(cave_tick_stats) * nticks, cudaMemcpyDeviceToHost, ctx->stream);
    record(ctx, 5);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    cudaFree(dticks);
    cudaFree(ditems);
    cudaFree(dtt);
    if (e != cudaSuccess) return check_cuda(ctx, e, "cave_run");
    finish_timing(ctx, nticks, launches + (jk ? 4 : 3), true);
    ctx->last_run_kind = kind;
    if (back.error & kErrBounds) return set_error(ctx, CAVE_ERR_INTERNAL, "streaming kernel: an index check failed");
    if (back.error & kErrWaitTimeout) return set_error(ctx, CAVE_ERR_TIMEOUT, "streaming kernel: bulk-copy wait timed out");
    if (back.error) return set_error(ctx, CAVE_ERR_INTERNAL, "streaming kernel raised an error flag");
    if (back.tick != nticks) return set_error(ctx, CAVE_ERR_INTERNAL, "streaming run stopped early");
    if (info) *info = back.info;
    return CAVE_OK;
}

extern "C" {

void cave_manager_update(const cave_grid_snapshot* snapshot, cave_grid_info* info, cave_sim_params* perms,
                         uint64_t maxPermutation, uint64_t survivalEndPermutation, uint32_t maxTicks,
                         cave_grid_info* infoCopy, cave_sim_params* permsCopy) {
    if (!snapshot || !info || !perms || !infoCopy || !permsCopy) return;
    manager_update(*snapshot, *info, *perms, maxPermutation, survivalEndPermutation, maxTicks, *infoCopy, *permsCopy);
}

uint64_t cave_enumerate_valid_bitmasks(uint32_t neighborCount, uint32_t maxBits, uint64_t* out, uint64_t cap) {
    std::vector<uint64_t> v = enumerate_valid_bitmasks(neighborCount, maxBits);
    if (out) std::memcpy(out, v.data(), sizeof(uint64_t) * std::min<uint64_t>(cap, v.size()));
    return v.size();
}

}  // extern "C"
