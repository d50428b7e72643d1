// kernels_strip.cu -- kernels on the bit-plane ("strip") layout: conversion from/to the
// reference's nibble layout, on-device seeding, and the z-streaming tick kernel.
//
// The streaming tick kernel covers the hot loop of searchSimulationCube.slang:117-247 for
// grids held in HBM/L2. Each CTA owns a tile of full x-rows [y0, y0+ty) and marches a
// z-range [z0, z1), reading each input plane tile exactly once: the tile's rows of the next
// plane (contiguous in memory) arrive by one cp.async.bulk (TMA bulk copy, no multicast)
// into a ring of shared-memory slots, completion tracked by mbarriers. A thread owns one
// strip column (sx, y); x-neighbour alive bits come from warp shuffles, y-neighbour column
// sums from a shared-memory exchange, z-neighbours from the thread's own rolling registers.
// The per-tick statistics (GridSnapshot + derived) are reduced per CTA and folded, with the
// search manager update (searchManager.slang:98-139), by the last CTA of each simulation.
#include <cuda_runtime.h>

#include <algorithm>

#include "ca_core.cuh"
#include "cave_internal.h"
#include "kernels.h"

namespace cave {

__device__ void fold_tick(StripSim* sim);

// ------------------------------------------------------------------ layout conversion
__device__ __forceinline__ uint32_t gather_nibble_bit(uint32_t w, int b) {
    uint32_t e = (w >> b) & 0x11111111u;
    e = (e | (e >> 3)) & 0x03030303u;
    e = (e | (e >> 6)) & 0x000F000Fu;
    e = (e | (e >> 12)) & 0x000000FFu;
    return e;
}
__device__ __forceinline__ uint32_t scatter_nibble_bit(uint32_t e8) {
    uint32_t e = e8 & 0xFFu;
    e = (e | (e << 12)) & 0x000F000Fu;
    e = (e | (e << 6)) & 0x03030303u;
    e = (e | (e << 3)) & 0x11111111u;
    return e;
}

// One thread per strip: nibble words 4*sx .. 4*sx+3 of a row -> four bit-planes.
__global__ void k_nib_to_strips(const uint32_t* __restrict__ nib, uint4* __restrict__ strips, uint32_t X,
                                uint32_t Y, uint32_t Z) {
    const uint32_t W = (X + 7u) / 8u, SX = (X + 31u) / 32u;
    const uint64_t n = (uint64_t)SX * Y * Z;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t sx = (uint32_t)(i % SX);
        const uint64_t row = i / SX;
        const uint32_t* r = nib + row * W;
        uint32_t w[4];
#pragma unroll
        for (int k = 0; k < 4; k++) w[k] = (4u * sx + k < W) ? r[4u * sx + k] : 0u;
        const uint32_t valid = strip_valid(sx, X);
        uint32_t p[4];
#pragma unroll
        for (int b = 0; b < 4; b++) {
            p[b] = gather_nibble_bit(w[0], b) | (gather_nibble_bit(w[1], b) << 8) |
                   (gather_nibble_bit(w[2], b) << 16) | (gather_nibble_bit(w[3], b) << 24);
            p[b] &= valid;
        }
        strips[i] = make_uint4(p[0], p[1], p[2], p[3]);
    }
}

// One thread per nibble word: the inverse of k_nib_to_strips (padding nibbles come out 0).
__global__ void k_strips_to_nib(const uint4* __restrict__ strips, uint32_t* __restrict__ nib, uint32_t X,
                                uint32_t Y, uint32_t Z) {
    const uint32_t W = (X + 7u) / 8u, SX = (X + 31u) / 32u;
    const uint64_t n = (uint64_t)W * Y * Z;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t ux = (uint32_t)(i % W);
        const uint64_t row = i / W;
        const uint4 s = strips[row * SX + ux / 4u];
        const uint32_t sh = 8u * (ux & 3u);
        uint32_t w = scatter_nibble_bit(s.x >> sh) | (scatter_nibble_bit(s.y >> sh) << 1) |
                     (scatter_nibble_bit(s.z >> sh) << 2) | (scatter_nibble_bit(s.w >> sh) << 3);
        nib[i] = w;
    }
}

// ------------------------------------------------------------------ seeding
// searchSystem.cpp:244-259 (wangHash, cellHash).
__device__ __forceinline__ uint32_t wang_hash(uint32_t s) {
    s = (s ^ 61u) ^ (s >> 16);
    s *= 9u;
    s = s ^ (s >> 4);
    s *= 0x27d4eb2du;
    s = s ^ (s >> 15);
    return s;
}
__device__ __forceinline__ uint32_t cell_hash(uint32_t x, uint32_t y, uint32_t z, uint32_t seed) {
    uint32_t h = wang_hash(x * 73856093u + seed);
    h = wang_hash(h ^ (y * 19349663u));
    h = wang_hash(h ^ (z * 83492791u));
    return h;
}

// searchSystem.cpp:264-305 in the nibble layout; one thread per word. box = [lo, hi) per axis.
__global__ void k_seed_nib(uint32_t* __restrict__ nib, SeedSpec sp) {
    const uint32_t W = (sp.X + 7u) / 8u;
    const uint64_t n = (uint64_t)W * sp.Y * sp.Z;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t ux = (uint32_t)(i % W);
        const uint64_t r = i / W;
        const uint32_t y = (uint32_t)(r % sp.Y), z = (uint32_t)(r / sp.Y);
        uint32_t w = 0;
        const bool inyz = y >= sp.lo[1] && y < sp.hi[1] && z >= sp.lo[2] && z < sp.hi[2];
        if (inyz) {
#pragma unroll
            for (uint32_t k = 0; k < 8; k++) {
                const uint32_t x = ux * 8u + k;
                if (x >= sp.X || x < sp.lo[0] || x >= sp.hi[0]) continue;
                const bool alive = sp.fill_all || (uint64_t)cell_hash(x, y, z, sp.seed) < sp.threshold;
                if (alive) w |= (sp.maxcs & 0xFu) << (4u * k);
            }
        }
        nib[i] = w;
    }
}

// The same cells directly in the strip layout; one thread per strip.
__global__ void k_seed_strips(uint4* __restrict__ strips, SeedSpec sp) {
    const uint32_t SX = (sp.X + 31u) / 32u;
    const uint64_t n = (uint64_t)SX * sp.Y * sp.Z;
    const uint32_t v = sp.maxcs & 0xFu;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t sx = (uint32_t)(i % SX);
        const uint64_t r = i / SX;
        const uint32_t y = (uint32_t)(r % sp.Y), z = (uint32_t)(r / sp.Y);
        uint32_t bits = 0;
        if (y >= sp.lo[1] && y < sp.hi[1] && z >= sp.lo[2] && z < sp.hi[2]) {
            for (uint32_t j = 0; j < 32; j++) {
                const uint32_t x = sx * 32u + j;
                if (x >= sp.X || x < sp.lo[0] || x >= sp.hi[0]) continue;
                if (sp.fill_all || (uint64_t)cell_hash(x, y, z, sp.seed) < sp.threshold) bits |= 1u << j;
            }
        }
        strips[i] = make_uint4((v & 1u) ? bits : 0u, (v & 2u) ? bits : 0u, (v & 4u) ? bits : 0u,
                               (v & 8u) ? bits : 0u);
    }
}

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bulk global->shared copy (no multicast), completion signalled on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ------------------------------------------------------------------ streaming tick
constexpr int kRing = 4;  // plane slots in flight per CTA

template <int N>
__device__ __forceinline__ uint4 pack_planes(const uint32_t* p) {
    uint4 v = make_uint4(p[0], 0u, 0u, 0u);
    if constexpr (N > 1) v.y = p[1];
    if constexpr (N > 2) v.z = p[2];
    if constexpr (N > 3) v.w = p[3];
    return v;
}


// Shared-memory layout of k_stream_tick (dynamic): ring[kRing][rows*SX] uint4,
// xch[2][rows*SXp] uint4, then kRing mbarriers.
__host__ __device__ inline size_t stream_smem_bytes(uint32_t rows, uint32_t SX, uint32_t SXp) {
    return (size_t)kRing * rows * SX * 16 + (size_t)2 * rows * SXp * 16 + kRing * 8 + 16;
}
size_t stream_smem_bytes_host(uint32_t rows, uint32_t SX, uint32_t SXp) { return stream_smem_bytes(rows, SX, SXp); }

template <int NB, bool SPARSE>
__global__ void __launch_bounds__(1024) k_stream_tick(const StreamItem* __restrict__ items, StripSim* sims,
                                                      uint4* pool, uint32_t SXp) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ DeviceRule rule;
    __shared__ uint32_t s_skip;
    const StreamItem it = items[blockIdx.x];
    StripSim* sim = sims + it.sim;
    const uint32_t SX = sim->SX, X = sim->X, Y = sim->Y, Z = sim->Z;
    const uint32_t rows = blockDim.x / SXp;  // incl. the two halo rows

    if (threadIdx.x == 0) s_skip = sim->done;
    // rule -> shared memory (each thread copies 16 B)
    {
        const uint4* src = reinterpret_cast<const uint4*>(&sim->rule);
        uint4* dst = reinterpret_cast<uint4*>(&rule);
        for (uint32_t i = threadIdx.x; i < sizeof(DeviceRule) / 16; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    if (s_skip) return;

    const uint32_t tick = sim->tick;
    const uint4* src = reinterpret_cast<const uint4*>(reinterpret_cast<unsigned char*>(pool) + sim->buf[tick & 1u]);
    uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(pool) + sim->buf[(tick + 1u) & 1u]);

    uint4* ring = reinterpret_cast<uint4*>(smem_raw);
    uint4* xch = ring + (size_t)kRing * rows * SX;
    uint64_t* bars = reinterpret_cast<uint64_t*>(xch + (size_t)2 * rows * SXp);

    const uint32_t sx = threadIdx.x % SXp, yy = threadIdx.x / SXp;
    const int y = (int)it.y0 - 1 + (int)yy;
    const bool has = sx < SX && y >= 0 && y < (int)Y && yy < (uint32_t)it.ty + 2u;
    const bool outp = has && yy >= 1 && yy <= it.ty;
    const uint32_t valid = has ? strip_valid(sx, X) : 0u;

    // rows of the tile present in memory: [ylo, yhi)
    const int ylo = max((int)it.y0 - 1, 0), yhi = min((int)it.y0 + (int)it.ty + 1, (int)Y);
    const uint32_t tile_bytes = (uint32_t)(yhi - ylo) * SX * 16u;
    const uint32_t slot_row0 = (uint32_t)(ylo - ((int)it.y0 - 1));  // first present row in a slot
    const int L = (int)it.z1 - (int)it.z0;                           // output planes
    const int nfetch = L + 2;
    auto plane_of = [&](int f) -> int { return it.dir ? (int)it.z1 - f : (int)it.z0 - 1 + f; };
    auto in_range = [&](int p) -> bool { return p >= 0 && p < (int)Z; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kRing; s++) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](int f) {
        if (f >= nfetch) return;
        const int p = plane_of(f);
        if (!in_range(p)) return;
        const int s = f % kRing;
        uint4* slot = ring + (size_t)s * rows * SX + (size_t)slot_row0 * SX;
        const uint4* g = src + ((size_t)p * Y + (size_t)ylo) * SX;
        mbar_expect_tx(&bars[s], tile_bytes);
        bulk_g2s(slot, g, tile_bytes, &bars[s]);
    };
    if (threadIdx.x == 0) {
        for (int f = 0; f < kRing; f++) issue(f);
    }

    uint32_t phase = 0;  // bit s: parity to wait for on slot s
    uint32_t err = 0;
    auto fetch = [&](int f) -> uint4 {
        const int p = plane_of(f);
        if (!in_range(p)) return make_uint4(0, 0, 0, 0);
        const int s = f % kRing;
        const uint32_t par = (phase >> s) & 1u;
        uint32_t spins = 0;
        while (!mbar_try_wait(&bars[s], par)) {
            if (++spins > kSpinLimit) {
                err = kErrWaitTimeout;
                break;
            }
        }
        phase ^= 1u << s;
        if (!has) return make_uint4(0, 0, 0, 0);
        return ring[(size_t)s * rows * SX + (size_t)yy * SX + sx];
    };
    auto row_of = [&](uint4 st) -> Row {
        const uint32_t a = has ? alive_plane(st, rule) : 0u;
        uint32_t al = __shfl_up_sync(0xFFFFFFFFu, a, 1, SXp);
        uint32_t ar = __shfl_down_sync(0xFFFFFFFFu, a, 1, SXp);
        if (sx == 0) al = 0u;
        if (sx + 1 >= SX) ar = 0u;
        return make_row(a, al, ar);
    };

    // warm-up: planes before and at the first output plane
    uint4 s_prev = fetch(0);
    Row r_m = row_of(s_prev);
    uint4 s_c = fetch(1);
    Row r_c = row_of(s_c);
    __syncthreads();  // slots 0 and 1 consumed
    if (threadIdx.x == 0) {
        fence_proxy_async();
        issue(kRing);
        issue(kRing + 1);
    }

    using P = Partials<NB>;
    TickAcc acc;
    acc.reset();
    for (int k = 0; k < L; k++) {
        const int zo = plane_of(k + 1);
        const uint4 s_in = fetch(k + 2);
        const Row r_p = row_of(s_in);
        uint32_t pc[P::NC], ps[P::NS];
        P::make(r_m, r_c, r_p, pc, ps);
        uint4* xb = xch + (size_t)(k & 1) * rows * SXp;
        xb[threadIdx.x] = pack_planes<P::NS>(ps);
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_proxy_async();
            issue(k + 2 + kRing);
        }
        if (outp) {
            const uint4 qm = xb[threadIdx.x - SXp], qp = xb[threadIdx.x + SXp];
            const uint32_t psm[4] = {qm.x, qm.y, qm.z, qm.w}, psp[4] = {qp.x, qp.y, qp.z, qp.w};
            uint32_t cnt[count_bits(NB)];
            combine<NB>(pc, psm, psp, cnt);
            const uint4 n = update_strip<NB, SPARSE>(s_c, r_c.a, cnt, valid, rule, acc, sx * 32u, (uint32_t)y,
                                                     (uint32_t)zo);
            dst[((size_t)zo * Y + (size_t)y) * SX + sx] = n;
        }
        r_m = r_c;
        r_c = r_p;
        s_c = s_in;
    }

    // ---- per-CTA reduction of the tick statistics
    __shared__ uint32_t red[32][11];
    uint32_t v[11] = {acc.surviving, acc.born, acc.zero, acc.population, acc.bmin[0], acc.bmin[1], acc.bmin[2],
                      acc.bmax[0], acc.bmax[1], acc.bmax[2], err};
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int q = 0; q < 4; q++) v[q] += __shfl_xor_sync(0xFFFFFFFFu, v[q], o);
#pragma unroll
        for (int q = 4; q < 7; q++) v[q] = min(v[q], __shfl_xor_sync(0xFFFFFFFFu, v[q], o));
#pragma unroll
        for (int q = 7; q < 10; q++) v[q] = max(v[q], __shfl_xor_sync(0xFFFFFFFFu, v[q], o));
        v[10] |= __shfl_xor_sync(0xFFFFFFFFu, v[10], o);
    }
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 11; q++) red[warp][q] = v[q];
    }
    __syncthreads();
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
        const uint32_t nw = blockDim.x >> 5;
        for (uint32_t w = 1; w < nw; w++) {
            for (int q = 0; q < 4; q++) red[0][q] += red[w][q];
            for (int q = 4; q < 7; q++) red[0][q] = min(red[0][q], red[w][q]);
            for (int q = 7; q < 10; q++) red[0][q] = max(red[0][q], red[w][q]);
            red[0][10] |= red[w][10];
        }
        if (red[0][0]) atomicAdd(&sim->acc_surv, red[0][0]);
        if (red[0][1]) atomicAdd(&sim->acc_born, red[0][1]);
        if (red[0][2]) atomicAdd(&sim->acc_zero, red[0][2]);
        if (red[0][3]) {
            atomicAdd(&sim->acc_pop, red[0][3]);
            for (int q = 0; q < 3; q++) {
                atomicMin(&sim->acc_bmin[q], red[0][4 + q]);
                atomicMax(&sim->acc_bmax[q], red[0][7 + q]);
            }
        }
        if (red[0][10]) atomicOr(&sim->error, red[0][10]);
        __threadfence();
        s_last = atomicAdd(&sim->ticket, 1u) == sim->n_items - 1u;
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_last) {
        __threadfence();
        fold_tick(sim);
    }
}

// Folds the accumulated statistics of one tick into the simulation record (last CTA).
__device__ void fold_tick(StripSim* sim) {
    volatile StripSim* vs = sim;
    const uint32_t surv = vs->acc_surv, born = vs->acc_born, zero = vs->acc_zero, pop = vs->acc_pop;
    const uint32_t volume = sim->X * sim->Y * sim->Z;
    cave_tick_stats st;
    st.snapshot.numberOfDeadCells = zero - born;
    st.snapshot.numberOfCellsBorn = born;
    st.snapshot.numberOfSurvivingCells = surv;
    st.snapshot.numberOfDyingCells = volume - (zero - born) - born - surv;
    st.population = pop;
    st.changed = born + st.snapshot.numberOfDyingCells;
    for (int q = 0; q < 3; q++) {
        st.bbox_min[q] = vs->acc_bmin[q];
        st.bbox_max[q] = vs->acc_bmax[q];
    }
    sim->acc_surv = sim->acc_born = sim->acc_zero = sim->acc_pop = 0;
    for (int q = 0; q < 3; q++) {
        sim->acc_bmin[q] = 0xFFFFFFFFu;
        sim->acc_bmax[q] = 0;
    }
    sim->ticket = 0;
    const uint32_t t = sim->tick;
    if (sim->per_tick) sim->per_tick[t] = st;
    sim->last = st;
    sim->total_changed += st.changed;
    if (st.changed) sim->pop_change_ticks++;
    // searchManager.slang:115-139
    cave_grid_info info = sim->info;
    info.numberOfSimulationTicksSurvived++;
    info.totalNumberOfCellsThatDied += st.snapshot.numberOfDeadCells;
    info.totalNumberOfCellsThatWereBorn += born;
    info.finalAliveCount = surv;
    if (surv > info.maxAliveCount) info.maxAliveCount = surv;
    if (surv == 0u && born == 0u)
        info.status = 1;
    else if (info.numberOfSimulationTicksSurvived >= sim->max_ticks)
        info.status = 2;
    else
        info.status = 0;
    sim->info = info;
    sim->tick = t + 1;
    if ((sim->stop_on_status && info.status > 0) || t + 1 >= sim->tick_limit) sim->done = 1;
    __threadfence();
}

// ------------------------------------------------------------------ launch helpers
template <int NB, bool SPARSE>
static cudaError_t launch_stream_nb(const StreamItem* items, uint32_t n_items, StripSim* sims, uint4* pool,
                                    uint32_t SXp, uint32_t threads, size_t smem, cudaStream_t st) {
    auto k = k_stream_tick<NB, SPARSE>;
    static size_t configured = 0;
    if (smem > configured) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = smem;
    }
    k<<<n_items, threads, smem, st>>>(items, sims, pool, SXp);
    return cudaGetLastError();
}

cudaError_t launch_stream_tick(int nb, bool sparse, const StreamItem* items, uint32_t n_items, StripSim* sims,
                               uint4* pool, uint32_t SX, uint32_t SXp, uint32_t threads, cudaStream_t st) {
    const uint32_t rows = threads / SXp;
    const size_t smem = stream_smem_bytes(rows, SX, SXp);
#define CAVE_NB_CASE(N)                                                                               \
    case N:                                                                                           \
        return sparse ? launch_stream_nb<N, true>(items, n_items, sims, pool, SXp, threads, smem, st) \
                      : launch_stream_nb<N, false>(items, n_items, sims, pool, SXp, threads, smem, st);
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

cudaError_t launch_nib_to_strips(const uint32_t* nib, uint4* strips, uint32_t X, uint32_t Y, uint32_t Z,
                                 cudaStream_t st) {
    const uint64_t n = (uint64_t)((X + 31) / 32) * Y * Z;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    k_nib_to_strips<<<blocks ? blocks : 1, 256, 0, st>>>(nib, strips, X, Y, Z);
    return cudaGetLastError();
}

cudaError_t launch_strips_to_nib(const uint4* strips, uint32_t* nib, uint32_t X, uint32_t Y, uint32_t Z,
                                 cudaStream_t st) {
    const uint64_t n = (uint64_t)((X + 7) / 8) * Y * Z;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    k_strips_to_nib<<<blocks ? blocks : 1, 256, 0, st>>>(strips, nib, X, Y, Z);
    return cudaGetLastError();
}

cudaError_t launch_seed_nib(uint32_t* nib, const SeedSpec& sp, cudaStream_t st) {
    const uint64_t n = (uint64_t)((sp.X + 7) / 8) * sp.Y * sp.Z;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    k_seed_nib<<<blocks ? blocks : 1, 256, 0, st>>>(nib, sp);
    return cudaGetLastError();
}

cudaError_t launch_seed_strips(uint4* strips, const SeedSpec& sp, cudaStream_t st) {
    const uint64_t n = (uint64_t)((sp.X + 31) / 32) * sp.Y * sp.Z;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    k_seed_strips<<<blocks ? blocks : 1, 256, 0, st>>>(strips, sp);
    return cudaGetLastError();
}

}  // namespace cave
