// kernels_stream.cu -- the z-streaming tick kernel (body in stream_tick.cuh), the fold of
// deferred-fold runs, and the launch helpers of both the library's kernels and the
// rule-specialised ones compiled at run time (jit.cpp).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <utility>

#include "jit.h"
#include "kernels.h"
#include "stream_tick.cuh"
#include "stream_tick2.cuh"

namespace cave {

template <int NB, int NT, bool PR>
__global__ void __launch_bounds__(1024) k_stream_tick(const StreamItem* __restrict__ items, StripSim* sims,
                                                      uint4* pool, uint32_t sxp_log2, int tick_arg,
                                                      const __grid_constant__ DeviceRule prule) {
    stream_tick_body<NB, NT, PR, RuntimeRule>(items, sims, pool, sxp_log2, tick_arg, prule);
}

// The fold of a deferred-fold run, after its last tick: every tick's statistics from its
// slot, and the record's GridInfo and totals as nticks sequential folds (fold_values) would
// leave them -- in raw stepping nothing the fold computes feeds back into the stepping.
// One block; the record must be fresh (tick 0, zero GridInfo and totals).
__global__ void __launch_bounds__(256) k_fold_deferred(StripSim* sim, const TickTotals* __restrict__ tt,
                                                       uint32_t nticks, uint32_t derive_zero) {
    __shared__ uint32_t s_died[256], s_born[256], s_maxs[256], s_nchg[256];
    __shared__ unsigned long long s_chg[256];
    const uint32_t volume = sim->X * sim->Y * sim->Z;
    cave_tick_stats* per_tick = sim->per_tick;
    uint32_t died = 0, born_sum = 0, maxs = 0, nchg = 0;
    unsigned long long chg = 0;
    for (uint32_t t = threadIdx.x; t < nticks; t += blockDim.x) {
        TickTotals v = tt[t];
        // a tick that did not count its zero cells: they are the cells that were 0 after the
        // previous tick (every cell outside the population)
        if (derive_zero && t > 0) v.zero = volume - tt[t - 1].pop;
        cave_tick_stats st;
        st.snapshot.numberOfDeadCells = v.zero - v.born;
        st.snapshot.numberOfCellsBorn = v.born;
        st.snapshot.numberOfSurvivingCells = v.surv;
        st.snapshot.numberOfDyingCells = volume - (v.zero - v.born) - v.born - v.surv;
        st.population = v.pop;
        st.changed = v.born + st.snapshot.numberOfDyingCells;
        for (int q = 0; q < 3; q++) {
            st.bbox_min[q] = ~v.nbmin[q];
            st.bbox_max[q] = v.bmax[q];
        }
        if (per_tick) per_tick[t] = st;
        if (t + 1 == nticks) sim->last = st;
        died += st.snapshot.numberOfDeadCells;
        born_sum += v.born;
        maxs = max(maxs, v.surv);
        chg += st.changed;
        nchg += st.changed ? 1u : 0u;
    }
    s_died[threadIdx.x] = died;
    s_born[threadIdx.x] = born_sum;
    s_maxs[threadIdx.x] = maxs;
    s_nchg[threadIdx.x] = nchg;
    s_chg[threadIdx.x] = chg;
    __syncthreads();
    for (uint32_t o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s_died[threadIdx.x] += s_died[threadIdx.x + o];
            s_born[threadIdx.x] += s_born[threadIdx.x + o];
            s_maxs[threadIdx.x] = max(s_maxs[threadIdx.x], s_maxs[threadIdx.x + o]);
            s_nchg[threadIdx.x] += s_nchg[threadIdx.x + o];
            s_chg[threadIdx.x] += s_chg[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && nticks) {
        const TickTotals last = tt[nticks - 1];
        cave_grid_info info = sim->info;  // searchManager.slang:115-139 over all ticks
        info.numberOfSimulationTicksSurvived += nticks;
        info.totalNumberOfCellsThatDied += s_died[0];
        info.totalNumberOfCellsThatWereBorn += s_born[0];
        info.finalAliveCount = last.surv;
        info.maxAliveCount = max(info.maxAliveCount, s_maxs[0]);
        if (last.surv == 0u && last.born == 0u)
            info.status = 1;
        else if (info.numberOfSimulationTicksSurvived >= sim->max_ticks)
            info.status = 2;
        else
            info.status = 0;
        sim->info = info;
        sim->total_changed += s_chg[0];
        sim->pop_change_ticks += s_nchg[0];
        sim->tick += nticks;
        if (sim->tick >= sim->tick_limit) sim->done = 1;
    }
}

// Population and bounding box of a whole strip grid, added to one tick slot: the last tick of a
// deferred-fold run whose ticks count their input's (every tick's but the last comes from the
// tick after it). Cells past X are 0 in the strip layout.
__global__ void __launch_bounds__(256) k_strip_stats(const uint4* __restrict__ strips, uint32_t Y, uint32_t Z,
                                                     uint32_t SX, TickTotals* slot) {
    __shared__ uint32_t red[8][7];
    uint32_t v[7] = {0u, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};  // pop, min xyz, max xyz
    const uint64_t n = (uint64_t)SX * Y * Z;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint4 st = strips[i];
        const uint32_t nz = st.x | st.y | st.z | st.w;
        if (!nz) continue;
        const uint32_t sx = (uint32_t)(i % SX);
        const uint64_t row = i / SX;
        const uint32_t y = (uint32_t)(row % Y), z = (uint32_t)(row / Y);
        v[0] += __popc(nz);
        v[1] = min(v[1], sx * 32u + (uint32_t)(__ffs(nz) - 1));
        v[4] = max(v[4], sx * 32u + 31u - (uint32_t)__clz(nz));
        v[2] = min(v[2], y);
        v[5] = max(v[5], y);
        v[3] = min(v[3], z);
        v[6] = max(v[6], z);
    }
    v[0] = warp_add(v[0]);
#pragma unroll
    for (int q = 1; q < 4; q++) v[q] = warp_min(v[q]);
#pragma unroll
    for (int q = 4; q < 7; q++) v[q] = warp_max(v[q]);
    const uint32_t warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31u) == 0) {
        for (int q = 0; q < 7; q++) red[warp][q] = v[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t w = 1; w < (blockDim.x >> 5); w++) {
            red[0][0] += red[w][0];
            for (int q = 1; q < 4; q++) red[0][q] = min(red[0][q], red[w][q]);
            for (int q = 4; q < 7; q++) red[0][q] = max(red[0][q], red[w][q]);
        }
        if (red[0][0]) {
            atomicAdd(&slot->pop, red[0][0]);
            for (int q = 0; q < 3; q++) {
                atomicMax(&slot->nbmin[q], ~red[0][1 + q]);
                atomicMax(&slot->bmax[q], red[0][4 + q]);
            }
        }
    }
}

cudaError_t launch_strip_stats(const uint4* strips, uint32_t Y, uint32_t Z, uint32_t SX, TickTotals* slot,
                               uint32_t sm_count, cudaStream_t st) {
    k_strip_stats<<<sm_count * 4u, 256, 0, st>>>(strips, Y, Z, SX, slot);
    return cudaGetLastError();
}

cudaError_t launch_fold_deferred(StripSim* sim, const TickTotals* tt, uint32_t nticks, bool derive_zero,
                                 cudaStream_t st) {
    k_fold_deferred<<<1, 256, 0, st>>>(sim, tt, nticks, derive_zero ? 1u : 0u);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ launch helpers
// CAVE_STREAM_PDL=0 launches the ticks without programmatic dependent launch (tuning runs).
static uint32_t env_flag(const char* name, uint32_t dflt) {
    const char* v = std::getenv(name);
    return v ? (uint32_t)std::atoi(v) : dflt;
}
static bool stream_pdl() {
    static const bool v = env_flag("CAVE_STREAM_PDL", 1) != 0;
    return v;
}
template <int NB, int NT, bool PR>
static cudaError_t launch_stream_inst(const StreamItem* items, uint32_t n_items, StripSim* sims, uint4* pool,
                                     uint32_t sxp_log2, uint32_t threads, size_t smem, const DeviceRule& rule,
                                     cudaStream_t st, bool pdl, int tick_arg) {
    auto k = k_stream_tick<NB, NT, PR>;
    static size_t configured = 0;  // largest dynamic shared memory set for this instance
    static std::mutex mu;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (smem > configured) {
            cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            configured = smem;
        }
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(n_items);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = (pdl && stream_pdl()) ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, items, sims, pool, sxp_log2, tick_arg, rule);
}

template <int NB, bool PR>
static cudaError_t launch_stream_nt(int nt, const StreamItem* items, uint32_t n_items, StripSim* sims, uint4* pool,
                                   uint32_t sxp_log2, uint32_t threads, size_t smem, const DeviceRule& rule,
                                   cudaStream_t st, bool pdl, int tick_arg) {
    switch (nt) {
        case 0: return launch_stream_inst<NB, 0, PR>(items, n_items, sims, pool, sxp_log2, threads, smem, rule, st, pdl, tick_arg);
        case 1: return launch_stream_inst<NB, 1, PR>(items, n_items, sims, pool, sxp_log2, threads, smem, rule, st, pdl, tick_arg);
        case 2: return launch_stream_inst<NB, 2, PR>(items, n_items, sims, pool, sxp_log2, threads, smem, rule, st, pdl, tick_arg);
        case 3: return launch_stream_inst<NB, 3, PR>(items, n_items, sims, pool, sxp_log2, threads, smem, rule, st, pdl, tick_arg);
        case 4: return launch_stream_inst<NB, 4, PR>(items, n_items, sims, pool, sxp_log2, threads, smem, rule, st, pdl, tick_arg);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_stream_tick_jit(cudaKernel_t k, const StreamItem* items, uint32_t n_items, StripSim* sims,
                                   uint4* pool, uint32_t SX, uint32_t SXp, uint32_t threads, cudaStream_t st,
                                   bool pdl, int tick_arg) {
    uint32_t lg = 0;
    while ((1u << lg) < SXp) lg++;
    const size_t smem = stream_smem_bytes(kJitRowsPerThread * threads / SXp, SX, SXp);
    {
        // the largest dynamic shared memory set so far, per kernel and device
        static std::mutex mu;
        static std::map<std::pair<const void*, int>, size_t> configured;
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        std::lock_guard<std::mutex> lock(mu);
        size_t& c = configured[{(const void*)k, dev}];
        if (smem > c) {
            e = cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            c = smem;
        }
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(n_items);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = (pdl && stream_pdl()) ? 1 : 0;
    void* args[] = {(void*)&items, (void*)&sims, (void*)&pool, (void*)&lg, (void*)&tick_arg};
    const cudaError_t e = cudaLaunchKernelExC(&cfg, (const void*)k, args);
    if (e == cudaSuccess) jit_count_launch();
    return e;
}

size_t tick2_smem_bytes(uint32_t rows, uint32_t SX, uint32_t SXp) { return stream2_smem_bytes(rows, SX, SXp); }

cudaError_t launch_stream_tick2_jit(cudaKernel_t k, const StreamItem* items, uint32_t n_items, StripSim* sims,
                                    uint4* pool, uint32_t SX, uint32_t SXp, uint32_t threads, cudaStream_t st,
                                    bool pdl, int tick_arg, int src_sel) {
    uint32_t lg = 0;
    while ((1u << lg) < SXp) lg++;
    const size_t smem = stream2_smem_bytes(tick2_geometry().rows_per_thread * threads / SXp, SX, SXp);
    {
        static std::mutex mu;
        static std::map<std::pair<const void*, int>, size_t> configured;
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        std::lock_guard<std::mutex> lock(mu);
        size_t& c = configured[{(const void*)k, dev}];
        if (smem > c) {
            e = cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            c = smem;
        }
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(n_items);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = (pdl && stream_pdl()) ? 1 : 0;
    void* args[] = {(void*)&items, (void*)&sims, (void*)&pool, (void*)&lg, (void*)&tick_arg, (void*)&src_sel};
    const cudaError_t e = cudaLaunchKernelExC(&cfg, (const void*)k, args);
    if (e == cudaSuccess) jit_count_launch();
    return e;
}

cudaError_t launch_stream_tick(int nb, int nt, const DeviceRule* param_rule, const StreamItem* items,
                               uint32_t n_items, StripSim* sims, uint4* pool, uint32_t SX, uint32_t SXp,
                               uint32_t threads, cudaStream_t st, bool pdl, int tick_arg) {
    uint32_t lg = 0;
    while ((1u << lg) < SXp) lg++;
    const uint32_t rows = threads / SXp;
    const size_t smem = stream_smem_bytes(rows, SX, SXp);
    DeviceRule dummy{};
    const DeviceRule& r = param_rule ? *param_rule : dummy;
#define CAVE_NB_CASE(N)                                                                                        \
    case N:                                                                                                    \
        return param_rule ? launch_stream_nt<N, true>(nt, items, n_items, sims, pool, lg, threads, smem, r, st, pdl, tick_arg) \
                          : launch_stream_nt<N, false>(nt, items, n_items, sims, pool, lg, threads, smem, r, st, pdl, tick_arg);
    switch (nb & 7) {
        CAVE_NB_CASE(0)
        CAVE_NB_CASE(1)
        CAVE_NB_CASE(2)
        CAVE_NB_CASE(3)
        CAVE_NB_CASE(4)
        CAVE_NB_CASE(5)
        CAVE_NB_CASE(6)
        CAVE_NB_CASE(7)
    }
#undef CAVE_NB_CASE
    return cudaErrorInvalidValue;
}

}  // namespace cave
