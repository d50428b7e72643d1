// stream_tick.cuh -- body of the z-streaming tick kernel on the strip layout (grids in HBM / L2).
//
// Covers the hot loop of searchSimulationCube.slang:117-247 for one tick. Each CTA owns a
// tile of full x-rows [y0, y0+ty) and marches a z-range [z0, z1), reading each input plane
// tile once: the tile's rows of the next plane (contiguous in memory) arrive by one
// cp.async.bulk (TMA bulk copy, no multicast) into a ring of shared-memory slots, completion
// tracked by mbarriers. A thread owns one strip column (sx, y): x-neighbour alive bits come
// from warp shuffles, y-neighbour column sums from a shared-memory exchange, z-neighbours
// from the thread's rolling registers.
//
// Three march orders exist (`pipe`): grouped (2, the default: unrolled by four, every warp
// waits on its slot's mbarrier), plain (0: one CTA barrier per plane) and software-pipelined
// (1: a thread finishes plane k and starts plane k+1 between two barriers).
//
// Ticks are chained with programmatic dependent launch: a tick's CTAs set up their shared
// memory while the previous tick drains, then wait for it before touching the grid.
// The tick statistics (GridSnapshot + derived) are reduced per CTA and folded, with the
// search manager update (searchManager.slang:98-139), by the last CTA of each simulation,
// or added to the tick's slot of a deferred-fold run.
//
// The rule comes from one of three places: a __grid_constant__ kernel parameter (PR: every
// work item of the launch belongs to one simulation), the simulation record (read once per
// CTA), or -- in the rule-specialised kernel compiled at run time -- a Fixed::rule() made of
// compile-time constants, which lets the compiler fold the alive test, the rule tables and
// the state update into the fewest logic operations for that rule.
//
// This header is compiled twice: by nvcc into the library (kernels_stream.cu) and by NVRTC
// into the rule-specialised kernels (jit.cpp), so it includes nothing but device headers.
#pragma once
#include "cave_stdint.h"

#include "ca_core.cuh"
#include "cave_internal.h"
#include "ptx.cuh"
#include "ring.cuh"
#include "stream_common.cuh"

namespace cave {

// Fixed-rule policy of the library's own kernels: the rule is read at run time.
struct RuntimeRule {
    static constexpr bool kFixed = false;
    __device__ static DeviceRule rule() { return DeviceRule{}; }
};

template <int NB, int NT, bool PR, class Fixed>
__device__ __forceinline__ void stream_tick_body(const StreamItem* __restrict__ items, StripSim* sims, uint4* pool,
                                                 uint32_t sxp_log2, uint32_t pipe, int tick_arg,
                                                 const DeviceRule& prule) {
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
    if constexpr (Fixed::kFixed) {
        lr = Fixed::rule();  // compile-time constants: every rule field folds into the logic
    } else if constexpr (!PR) {
        const DeviceRule& g = sim->rule;
#pragma unroll
        for (int i = 0; i < 4; i++) lr.m[i] = g.m[i];
        lr.alive_ok = g.alive_ok;
        lr.lut_s = g.lut_s;
        lr.lut_b = g.lut_b;
#pragma unroll
        for (int t = 0; t < NT; t++) lr.terms[t] = g.terms[t];
    }
    const DeviceRule& R = (PR && !Fixed::kFixed) ? prule : lr;

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

}  // namespace cave
