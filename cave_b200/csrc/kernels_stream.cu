// kernels_stream.cu -- the z-streaming tick kernel on the strip layout (grids in HBM / L2).
//
// Covers the hot loop of searchSimulationCube.slang:117-247 for one tick. Each CTA owns a
// tile of full x-rows [y0, y0+ty) and marches a z-range [z0, z1), reading each input plane
// tile once: the tile's rows of the next plane (contiguous in memory) arrive by one
// cp.async.bulk (TMA bulk copy, no multicast) into a ring of shared-memory slots, completion
// tracked by mbarriers. A thread owns one strip column (sx, y): x-neighbour alive bits come
// from warp shuffles, y-neighbour column sums from a shared-memory exchange, z-neighbours
// from the thread's rolling registers.
//
// The march is software-pipelined: between two CTA barriers a thread finishes plane k
// (y-exchange read, count, rule, update, store) and starts plane k+1 (fetch, alive bits,
// column sums, y-exchange write). The two halves are independent, so the scheduler can
// overlap them, and each barrier interval carries a full plane of arithmetic.
//
// Ticks are chained with programmatic dependent launch: a tick's CTAs set up their shared
// memory while the previous tick drains, then wait for it before touching the grid.
// The tick statistics (GridSnapshot + derived) are reduced per CTA and folded, with the
// search manager update (searchManager.slang:98-139), by the last CTA of each simulation.
//
// The rule reaches the kernel as a __grid_constant__ parameter when every work item of the
// launch belongs to one simulation (its fields are then constant-bank operands), or is read
// once per CTA from the simulation record otherwise.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "ca_core.cuh"
#include "cave_internal.h"
#include "kernels.h"
#include "ptx.cuh"
#include "ring.cuh"
#include "stream_common.cuh"

namespace cave {

__device__ void fold_tick(StripSim* sim);

template <int NB, int NT, bool PR>
__global__ void __launch_bounds__(1024) k_stream_tick(const StreamItem* __restrict__ items, StripSim* sims,
                                                      uint4* pool, uint32_t sxp_log2, uint32_t pipe, int tick_arg,
                                                      const __grid_constant__ DeviceRule prule) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint32_t s_skip;
    __shared__ uint32_t red[32][11];
    __shared__ bool s_last;
    const StreamItem it = items[blockIdx.x];
    const uint32_t SXp = 1u << sxp_log2;
    const uint32_t rows = blockDim.x >> sxp_log2;  // incl. the two halo rows
    uint64_t* bars;
    {
        const uint32_t SXc = sims[it.sim].SX;  // geometry is fixed for the run
        bars = reinterpret_cast<uint64_t*>(reinterpret_cast<uint4*>(smem_raw) + (size_t)kRing * rows * SXc +
                                           (size_t)kXch * rows * SXp);
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kRing; s++) mbar_init(&bars[s], 1);
        mbar_init_fence();
    }
    // Everything below reads the previous tick's results.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    StripSim* sim = sims + it.sim;
    if (threadIdx.x == 0) s_skip = sim->done;
    __syncthreads();
    if (s_skip) return;
    asm volatile("griddepcontrol.launch_dependents;");

    DeviceRule lr;
    if constexpr (!PR) {
        const DeviceRule& g = sim->rule;
#pragma unroll
        for (int i = 0; i < 4; i++) lr.m[i] = g.m[i];
        lr.alive_ok = g.alive_ok;
        lr.lut_s = g.lut_s;
        lr.lut_b = g.lut_b;
#pragma unroll
        for (int t = 0; t < NT; t++) lr.terms[t] = g.terms[t];
    }
    const DeviceRule& R = PR ? prule : lr;

    const uint32_t SX = sim->SX, X = sim->X, Y = sim->Y, Z = sim->Z;
    // A deferred-fold run (sim->deferred) passes the tick index; otherwise the record counts.
    const uint32_t tick = tick_arg >= 0 ? (uint32_t)tick_arg : sim->tick;
    const uint4* src = reinterpret_cast<const uint4*>(reinterpret_cast<unsigned char*>(pool) + sim->buf[tick & 1u]);
    uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(pool) + sim->buf[(tick + 1u) & 1u]);
    uint4* ring = reinterpret_cast<uint4*>(smem_raw);
    uint4* xch = ring + (size_t)kRing * rows * SX;

    const uint32_t sx = threadIdx.x & (SXp - 1u), yy = threadIdx.x >> sxp_log2;
    const int y = (int)it.y0 - 1 + (int)yy;
    const bool has = sx < SX && y >= 0 && y < (int)Y && yy < (uint32_t)it.ty + 2u;
    const bool outp = has && yy >= 1 && yy <= it.ty;
    const uint32_t valid = has ? strip_valid(sx, X) : 0u;
    const bool left_edge = sx == 0, right_edge = sx + 1 >= SX;

    // rows of the tile present in memory: [ylo, yhi)
    const int ylo = max((int)it.y0 - 1, 0), yhi = min((int)it.y0 + (int)it.ty + 1, (int)Y);
    const uint32_t tile_bytes = (uint32_t)(yhi - ylo) * SX * 16u;
    const uint32_t slot_row0 = (uint32_t)(ylo - ((int)it.y0 - 1));
    const uint32_t slot_stride = rows * SX;
    const int L = (int)it.z1 - (int)it.z0;  // output planes
    const int nfetch = L + 2;
    const bool down = (it.dir_items & 1u) != 0;
    const int zstep = down ? -1 : 1;
    const int zfirst = down ? (int)it.z1 : (int)it.z0 - 1;  // plane of fetch 0

    // Thread 0 fills ring slot f % kRing with input plane f. A plane outside the grid is not
    // copied; with `complete` set its slot's phase is completed by a plain arrive, so that every
    // fetch advances its slot by exactly one phase (the grouped march relies on that).
    auto issue = [&](int f, bool complete = false) {
        if (f >= nfetch) return;
        const int p = zfirst + f * zstep;
        const int s = f & (kRing - 1);
        if (p < 0 || p >= (int)Z) {
            if (complete) mbar_arrive(&bars[s]);
            return;
        }
        uint4* slot = ring + (size_t)s * slot_stride + (size_t)slot_row0 * SX;
        const uint4* g = src + ((size_t)p * Y + (size_t)ylo) * SX;
        mbar_expect_tx(&bars[s], tile_bytes);
        bulk_g2s(slot, g, tile_bytes, &bars[s]);
    };
    const uint32_t producer = 0;  // the thread that issues the plane copies
    const bool grouped = pipe == 2u;
    if (threadIdx.x == producer) {
        for (int f = 0; f < kRing; f++) issue(f, grouped);
    }

    const uint4* my_ring = ring + (size_t)yy * SX + sx;
    uint32_t phase = 0;  // bit s: parity to wait for on slot s
    uint32_t err = 0;
    auto fetch = [&](int f) -> uint4 {
        const int p = zfirst + f * zstep;
        if (p < 0 || p >= (int)Z) return make_uint4(0, 0, 0, 0);
        const int s = f & (kRing - 1);
        if (!mbar_wait_bounded(&bars[s], (phase >> s) & 1u, kWaitLimitNs)) err = kErrWaitTimeout;
        phase ^= 1u << s;
        return has ? my_ring[(size_t)s * slot_stride] : make_uint4(0, 0, 0, 0);
    };
    auto row_of = [&](uint4 st) -> Row {
        const uint32_t a = alive_plane(st, R);  // zero for absent strips: state 0 is never alive
        uint32_t al = __shfl_up_sync(0xFFFFFFFFu, a, 1, SXp);
        uint32_t ar = __shfl_down_sync(0xFFFFFFFFu, a, 1, SXp);
        al = left_edge ? 0u : al;
        ar = right_edge ? 0u : ar;
        return make_row(a, al, ar);
    };

    using P = Partials<NB>;
    TickAcc acc;
    acc.reset();
    uint32_t xbits = 0u;
    uint4* my_x = xch + threadIdx.x;
    uint4* my_dst = dst + ((size_t)max(y, 0) * SX + sx);
    const size_t plane_stride = (size_t)Y * SX;
    const size_t xpar = (size_t)rows * SXp;

    int zo = zfirst + zstep;
    if (grouped) {
        // Grouped order: the plain order below, unrolled by kUnroll so that exchange buffers
        // and slot offsets are fixed within a group and the plane rotation needs no register
        // moves. Every warp waits for the copy of the plane it reads; fetch f is the
        // (f / kRing)-th use of slot f % kRing, so the phase parity to wait for is (f / kRing) & 1.
        auto read = [&](int f, int s) -> uint4 {  // s == f % kRing
            const int p = zfirst + f * zstep;
            if (f >= nfetch || (unsigned)p >= Z) return make_uint4(0, 0, 0, 0);
            if (!mbar_wait_bounded(&bars[s], (uint32_t)(f >> kRingLog2) & 1u, kWaitLimitNs)) err = kErrWaitTimeout;
            return has ? my_ring[(size_t)s * slot_stride] : make_uint4(0, 0, 0, 0);
        };
        Row r_m = row_of(read(0, 0));
        uint4 s_c = read(1, 1);
        Row r_c = row_of(s_c);
        __syncthreads();  // slots 0 and 1 consumed
        if (threadIdx.x == producer) {
            fence_proxy_async();
            issue(kRing, true);
            issue(kRing + 1, true);
        }
        auto body = [&]<int U>(int k) {  // k % kUnroll == U
            const uint4 s_in = read(k + 2, (k + 2) & (kRing - 1));
            const Row r_p = row_of(s_in);
            uint32_t pc[P::NC], ps[P::NS];
            P::make(r_m, r_c, r_p, pc, ps);
            uint4* xb = my_x + (size_t)(U & 1) * xpar;
            *xb = pack_planes<P::NS>(ps);
            __syncthreads();
            if (threadIdx.x == producer) {
                fence_proxy_async();
                issue(k + 2 + kRing, true);
            }
            if (outp) {
                const uint4 qm = *(xb - SXp), qp = *(xb + SXp);
                const uint32_t psm[4] = {qm.x, qm.y, qm.z, qm.w}, psp[4] = {qp.x, qp.y, qp.z, qp.w};
                uint32_t cnt[count_bits(NB)];
                combine<NB>(pc, psm, psp, cnt);
                my_dst[(size_t)zo * plane_stride] =
                    update_strip<NB, NT>(s_c, r_c.a, cnt, valid, R, acc, xbits, (uint32_t)zo);
            }
            r_m = r_c;
            r_c = r_p;
            s_c = s_in;
            zo += zstep;
        };
        static_assert(kUnroll == 4, "the grouped march is unrolled four times");
        for (int k = 0; k < L; k += kUnroll) {
            body.template operator()<0>(k);
            if (k + 1 < L) body.template operator()<1>(k + 1);
            if (k + 2 < L) body.template operator()<2>(k + 2);
            if (k + 3 < L) body.template operator()<3>(k + 3);
        }
    } else if (!pipe) {
        // Plain order: per plane, column sums -> barrier -> count, rule, update, store.
        Row r_m = row_of(fetch(0));
        uint4 s_c = fetch(1);
        Row r_c = row_of(s_c);
        __syncthreads();  // slots 0 and 1 consumed
        if (threadIdx.x == 0) {
            fence_proxy_async();
            issue(kRing);
            issue(kRing + 1);
        }
        for (int k = 0; k < L; k++) {
            const uint4 s_in = fetch(k + 2);
            const Row r_p = row_of(s_in);
            uint32_t pc[P::NC], ps[P::NS];
            P::make(r_m, r_c, r_p, pc, ps);
            uint4* xb = my_x + (size_t)(k & 1) * xpar;
            *xb = pack_planes<P::NS>(ps);
            __syncthreads();
            if (threadIdx.x == 0) {
                fence_proxy_async();
                issue(k + 2 + kRing);
            }
            if (outp) {
                const uint4 qm = *(xb - SXp), qp = *(xb + SXp);
                const uint32_t psm[4] = {qm.x, qm.y, qm.z, qm.w}, psp[4] = {qp.x, qp.y, qp.z, qp.w};
                uint32_t cnt[count_bits(NB)];
                combine<NB>(pc, psm, psp, cnt);
                my_dst[(size_t)zo * plane_stride] =
                    update_strip<NB, NT>(s_c, r_c.a, cnt, valid, R, acc, xbits, (uint32_t)zo);
            }
            r_m = r_c;
            r_c = r_p;
            s_c = s_in;
            zo += zstep;
        }
    } else {
    // Software-pipelined order (see the file comment).
    // prologue: rows of fetches 0..2 and the column sums of plane 0
    Row r_a = row_of(fetch(0));          // plane before the first output
    uint4 s_b = fetch(1);                 // first output plane
    Row r_b = row_of(s_b);
    uint4 s_c = fetch(2);
    Row r_c = row_of(s_c);
    uint32_t pc[P::NC];
    {
        uint32_t ps[P::NS];
        P::make(r_a, r_b, r_c, pc, ps);
        my_x[0] = pack_planes<P::NS>(ps);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        fence_proxy_async();
        for (int f = kRing; f < kRing + 3; f++) issue(f);
    }

    for (int k = 0; k < L; k++) {
        // (1) finish plane k: rows (a, b, c), centre state s_b, column sums pc, exchange slot k&1
        uint4 nout;
        {
            // Only output rows (1 <= yy <= ty <= rows-2) read their y-neighbours: the halo rows'
            // neighbours would lie outside the exchange buffer.
            const uint4* xb = my_x + (size_t)(k & 1) * xpar;
            uint4 qm = make_uint4(0, 0, 0, 0), qp = qm;
            if (outp) {
                qm = *(xb - SXp);
                qp = *(xb + SXp);
            }
            const uint32_t psm[4] = {qm.x, qm.y, qm.z, qm.w}, psp[4] = {qp.x, qp.y, qp.z, qp.w};
            uint32_t cnt[count_bits(NB)];
            combine<NB>(pc, psm, psp, cnt);
            nout = update_strip<NB, NT>(s_b, r_b.a, cnt, valid, R, acc, xbits, (uint32_t)zo, outp);
        }
        // (2) start plane k+1: fetch k+3, rows (b, c, d), column sums into exchange slot (k+1)&1
        const bool more = k + 1 < L;
        uint4 s_d = make_uint4(0, 0, 0, 0);
        Row r_d = r_c;
        if (more) {
            s_d = fetch(k + 3);
            r_d = row_of(s_d);
            uint32_t ps[P::NS];
            P::make(r_b, r_c, r_d, pc, ps);
            my_x[(size_t)((k + 1) & 1) * xpar] = pack_planes<P::NS>(ps);
        }
        if (outp) my_dst[(size_t)zo * plane_stride] = nout;
        if (more) {
            __syncthreads();
            if (threadIdx.x == 0) {
                fence_proxy_async();
                issue(k + 3 + kRing);
            }
        }
        r_b = r_c;
        r_c = r_d;
        s_b = s_c;
        s_c = s_d;
        zo += zstep;
    }

    }

    // ---- per-CTA reduction of the tick statistics
    uint32_t bx0 = 0xFFFFFFFFu, bx1 = 0u, by0 = 0xFFFFFFFFu, by1 = 0u;
    if (xbits) {
        bx0 = sx * 32u + (uint32_t)(__ffs(xbits) - 1);
        bx1 = sx * 32u + 31u - (uint32_t)__clz(xbits);
        by0 = by1 = (uint32_t)y;
    }
    uint32_t v[11] = {acc.surviving, acc.born, acc.zero, acc.population, bx0, by0, acc.zmin, bx1, by1, acc.zmax, err};
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
    if (threadIdx.x == 0) {
        const uint32_t nw = blockDim.x >> 5;
        for (uint32_t w = 1; w < nw; w++) {
            for (int q = 0; q < 4; q++) red[0][q] += red[w][q];
            for (int q = 4; q < 7; q++) red[0][q] = min(red[0][q], red[w][q]);
            for (int q = 7; q < 10; q++) red[0][q] = max(red[0][q], red[w][q]);
            red[0][10] |= red[w][10];
        }
        if (tick_arg >= 0) {
            // deferred fold: add this CTA's totals to the tick's slot (no ticket, no fence:
            // the next launch starts after this one has completed and flushed)
            TickTotals* d = sim->deferred + tick;
            if (red[0][0]) atomicAdd(&d->surv, red[0][0]);
            if (red[0][1]) atomicAdd(&d->born, red[0][1]);
            if (red[0][2]) atomicAdd(&d->zero, red[0][2]);
            if (red[0][3]) {
                atomicAdd(&d->pop, red[0][3]);
                for (int q = 0; q < 3; q++) {
                    atomicMax(&d->nbmin[q], ~red[0][4 + q]);
                    atomicMax(&d->bmax[q], red[0][7 + q]);
                }
            }
            if (red[0][10]) atomicOr(&sim->error, red[0][10]);
            return;
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
        s_last = atomicAdd(&sim->ticket, 1u) == (it.dir_items >> 1) - 1u;
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_last) {
        __threadfence();
        fold_tick(sim);
    }
}

// The fold of a deferred-fold run, after its last tick: every tick's statistics from its
// slot, and the record's GridInfo and totals as nticks sequential folds (fold_values) would
// leave them -- in raw stepping nothing the fold computes feeds back into the stepping.
// One block; the record must be fresh (tick 0, zero GridInfo and totals).
__global__ void __launch_bounds__(256) k_fold_deferred(StripSim* sim, const TickTotals* __restrict__ tt,
                                                       uint32_t nticks) {
    __shared__ uint32_t s_died[256], s_born[256], s_maxs[256], s_nchg[256];
    __shared__ unsigned long long s_chg[256];
    const uint32_t volume = sim->X * sim->Y * sim->Z;
    cave_tick_stats* per_tick = sim->per_tick;
    uint32_t died = 0, born_sum = 0, maxs = 0, nchg = 0;
    unsigned long long chg = 0;
    for (uint32_t t = threadIdx.x; t < nticks; t += blockDim.x) {
        const TickTotals v = tt[t];
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

cudaError_t launch_fold_deferred(StripSim* sim, const TickTotals* tt, uint32_t nticks, cudaStream_t st) {
    k_fold_deferred<<<1, 256, 0, st>>>(sim, tt, nticks);
    return cudaGetLastError();
}

// Folds the accumulated statistics of one tick into the simulation record (last CTA).
__device__ void fold_tick(StripSim* sim) {
    volatile StripSim* vs = sim;
    const uint32_t surv = vs->acc_surv, born = vs->acc_born, zero = vs->acc_zero, pop = vs->acc_pop;
    uint32_t bmin[3], bmax[3];
    for (int q = 0; q < 3; q++) {
        bmin[q] = vs->acc_bmin[q];
        bmax[q] = vs->acc_bmax[q];
    }
    sim->acc_surv = sim->acc_born = sim->acc_zero = sim->acc_pop = 0;
    for (int q = 0; q < 3; q++) {
        sim->acc_bmin[q] = 0xFFFFFFFFu;
        sim->acc_bmax[q] = 0;
    }
    sim->ticket = 0;
    fold_values(sim, surv, born, zero, pop, bmin, bmax);
}

// ------------------------------------------------------------------ launch helpers
// Variant switches for tuning runs: CAVE_STREAM_PIPE (march order: 2 grouped, the default;
// 0 plain; 1 software-pipelined) and CAVE_STREAM_PDL (programmatic dependent launch between
// ticks, default 1).
static uint32_t env_flag(const char* name, uint32_t dflt) {
    const char* v = std::getenv(name);
    return v ? (uint32_t)std::atoi(v) : dflt;
}
static uint32_t stream_pipe() {
    static const uint32_t v = env_flag("CAVE_STREAM_PIPE", 2);
    return v;
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
    return cudaLaunchKernelEx(&cfg, k, items, sims, pool, sxp_log2, stream_pipe(), tick_arg, rule);
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
