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
// The march is unrolled by four so that exchange buffers and slot offsets are fixed within a
// group; every warp waits on the mbarrier of the slot it reads, and one CTA barrier per plane
// separates the y-exchange write from its reads.
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
    static constexpr bool kFullRange = false;  // alive state known to be 15
    __device__ static DeviceRule rule() { return DeviceRule{}; }
};

// kCountZero: count the cells that were 0 before the tick; a deferred-fold run may instead derive
// them from the previous tick's population (all ticks after its first).
// kDense: the launch guarantees SX == SXp (every lane of a row holds a strip); ring positions of
// rows outside the tile are then zeroed once and read like the others.
// kPop (deferred-fold runs only; see update_strip): kPopInput counts the population and bounding
// box of the tick's input into the previous tick's slot, kPopNone leaves them out (the first
// tick of such a run; a pass over the final grid supplies the last tick's).
template <int NB, int NT, bool PR, class Fixed, bool kCountZero = true, bool kDense = false,
          int kPop = kPopOutput, int kStrips = 1>
__device__ __forceinline__ void stream_tick_body(const StreamItem* __restrict__ items, StripSim* sims, uint4* pool,
                                                 uint32_t sxp_log2, int tick_arg, const DeviceRule& prule) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint32_t s_state[2];  // done, tick (records that count their own ticks)
    __shared__ uint32_t red[32][11];
    const StreamItem it = items[blockIdx.x];
    StripSim* sim = sims + it.sim;
    const uint32_t SXp = 1u << sxp_log2;
    const uint32_t rows = kStrips * (blockDim.x >> sxp_log2);  // incl. the two halo rows
    // A record's geometry, cell buffers and rule stay fixed while its simulation runs, so they
    // are read while the previous tick drains, before griddepcontrol.wait. (A launch that may
    // start early is never the first one after the record was written: those are launched
    // without programmatic dependent launch.)
    const uint32_t SX = sim->SX, X = sim->X, Y = sim->Y, Z = sim->Z;
    const uint64_t buf0 = sim->buf[0], buf1 = sim->buf[1];
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
    uint4* ring = reinterpret_cast<uint4*>(smem_raw);
    uint4* xch = ring + (size_t)kRing * rows * SX;
    uint64_t* bars = reinterpret_cast<uint64_t*>(xch + (size_t)kXch * rows * SXp);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kRing; s++) mbar_init(&bars[s], 1);
        mbar_init_fence();
    }
    __syncthreads();
    // Everything below reads the previous tick's results.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    uint32_t tick;
    if (tick_arg >= 0) {
        tick = (uint32_t)tick_arg;  // a deferred-fold run: the record is not updated between ticks
    } else {
        if (threadIdx.x == 0) {
            s_state[0] = sim->done;
            s_state[1] = sim->tick;
        }
        __syncthreads();
        if (s_state[0]) return;
        tick = s_state[1];
    }
    asm volatile("griddepcontrol.launch_dependents;");
    const uint4* src =
        reinterpret_cast<const uint4*>(reinterpret_cast<unsigned char*>(pool) + ((tick & 1u) ? buf1 : buf0));
    uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(pool) + ((tick & 1u) ? buf0 : buf1));

    const uint32_t sx = threadIdx.x & (SXp - 1u), yy0 = kStrips * (threadIdx.x >> sxp_log2);
    int y[kStrips];
    bool has[kStrips], outp[kStrips];
#pragma unroll
    for (int q = 0; q < kStrips; q++) {
        const uint32_t yy = yy0 + q;
        y[q] = (int)it.y0 - 1 + (int)yy;
        has[q] = sx < SX && y[q] >= 0 && y[q] < (int)Y && yy < (uint32_t)it.ty + 2u;
        outp[q] = has[q] && yy >= 1 && yy <= it.ty;
    }
    // valid cells of this column's strips (the rows a thread outputs are all present)
    const uint32_t valid = (kStrips == 1 ? has[0] : sx < SX) ? strip_valid(sx, X) : 0u;
    // x-neighbour bits travel by rotation inside the warp: lane - 1 (mod 32) holds the previous
    // strip of the row or, for a row's first strip, the last lane of the previous row (or of the
    // warp), which is a right edge or an absent strip; symmetrically for lane + 1. Each thread
    // sends its alive plane with bit 31 cleared when it ends its row and bit 0 cleared when it
    // starts it, so the bits that wrap across rows are zero (outside the grid is dead).
    const bool left_edge = sx == 0, right_edge = sx + 1 >= SX;
    const uint32_t send_mask = (left_edge ? ~1u : ~0u) & (right_edge ? 0x7FFFFFFFu : ~0u);
    const int lane_l = (int)((threadIdx.x + 31u) & 31u), lane_r = (int)((threadIdx.x + 1u) & 31u);

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
    uint32_t err = 0;
    // extents (uint4 units) that the checked build tests every index against; a layout that does
    // not fit the launch's shared memory fails every shared-memory check
    const size_t xpar = (size_t)rows * SXp;
    size_t ring_n = (size_t)kRing * slot_stride, xch_n = (size_t)kXch * xpar;
    const size_t copy_n = (size_t)Z * Y * SX;
#ifdef CAVE_CHECKED
    if (!CAVE_IN_BOUNDS((ring_n + xch_n) * 16 + kRing * 8 - 1, dynamic_smem_bytes(), err)) ring_n = xch_n = 0;
#endif
    const size_t ring_off = (size_t)yy0 * SX + sx, x_off = (size_t)yy0 * SXp + sx;

    // Thread 0 fills ring slot f % kRing with input plane f. A plane outside the grid is not
    // copied; its slot's phase is completed by a plain arrive instead, so that every fetch
    // advances its slot by exactly one phase (the waits rely on that).
    auto issue = [&](int f) {
        if (f >= nfetch) return;
        const int p = zfirst + f * zstep;
        const int s = f & (kRing - 1);
        if (p < 0 || p >= (int)Z) {
            mbar_arrive(&bars[s]);
            return;
        }
        const size_t slot_i = (size_t)s * slot_stride + (size_t)slot_row0 * SX, g_i = ((size_t)p * Y + (size_t)ylo) * SX;
        if (!CAVE_IN_BOUNDS(slot_i + tile_bytes / 16u - 1u, ring_n, err) ||
            !CAVE_IN_BOUNDS(g_i + tile_bytes / 16u - 1u, copy_n, err)) {
            mbar_arrive(&bars[s]);  // checked build: the copy is skipped, its phase completed
            return;
        }
        mbar_expect_tx(&bars[s], tile_bytes);
        bulk_g2s(ring + slot_i, src + g_i, tile_bytes, &bars[s]);
    };
    const uint32_t producer = 0;  // the thread that issues the plane copies
    if (threadIdx.x == producer) {
        for (int f = 0; f < kRing; f++) issue(f);
    }

    const uint4* my_ring = ring + (size_t)yy0 * SX + sx;  // row q at + q * SX
    if constexpr (kDense) {
        // rows the plane copies never write (outside the grid or the tile) read as dead cells
#pragma unroll
        for (int q = 0; q < kStrips; q++) {
            if (!has[q]) {
#pragma unroll
                for (int s = 0; s < kRing; s++)
                    if (CAVE_IN_BOUNDS(ring_off + (size_t)s * slot_stride + (size_t)q * SX, ring_n, err))
                        const_cast<uint4*>(my_ring)[(size_t)s * slot_stride + (size_t)q * SX] = make_uint4(0, 0, 0, 0);
            }
        }
    }
    auto ring_ok = [&](int s, int q) {
        return CAVE_IN_BOUNDS(ring_off + (size_t)s * slot_stride + (size_t)q * SX, ring_n, err);
    };
    auto x_ok = [&](size_t rel) { return CAVE_IN_BOUNDS(x_off + rel, xch_n, err); };
    auto row_of = [&](uint4 st) -> Row {
        const uint32_t a = alive_plane(st, R);  // zero for absent strips: state 0 is never alive
        const uint32_t v = a & send_mask;
        return make_row(a, __shfl_sync(0xFFFFFFFFu, v, lane_l), __shfl_sync(0xFFFFFFFFu, v, lane_r));
    };

    using P = typename ColumnsFor<NB, Fixed::kFixed>::type;  // carry-save Moore columns when specialised
    TickAcc acc;
    acc.reset(SX != 0u ? 1u : 0u);  // SX >= 1: a 1 the compiler cannot fold
    uint32_t xbits[kStrips];
    // strip index of each row in a plane of the output copy (a copy holds at most 2^25 strips)
    uint32_t dst_row[kStrips];
#pragma unroll
    for (int q = 0; q < kStrips; q++) {
        xbits[q] = 0u;
        dst_row[q] = (uint32_t)max(y[q], 0) * SX + sx;
    }
    uint4* my_x = xch + (size_t)yy0 * SXp + sx;  // row q at + q * SXp
    const uint32_t plane_strips = Y * SX;

    int zo = zfirst + zstep;
    // Fetch f is the (f / kRing)-th use of slot f % kRing, so the phase parity to wait for is
    // (f / kRing) & 1.
    auto read = [&](int f, int s, uint4* out) {  // s == f % kRing
        const int p = zfirst + f * zstep;
        if (f >= nfetch || (unsigned)p >= Z) {
#pragma unroll
            for (int q = 0; q < kStrips; q++) out[q] = make_uint4(0, 0, 0, 0);
            return;
        }
        if (!mbar_wait_bounded(&bars[s], (uint32_t)(f >> kRingLog2) & 1u, kWaitLimitNs)) err = kErrWaitTimeout;
#pragma unroll
        for (int q = 0; q < kStrips; q++)
            out[q] = has[q] && ring_ok(s, q) ? my_ring[(size_t)s * slot_stride + (size_t)q * SX] : make_uint4(0, 0, 0, 0);
    };
    Row r_m[kStrips], r_c[kStrips];
    uint4 s_c[kStrips];
    {
        uint4 t0[kStrips];
        read(0, 0, t0);
        read(1, 1, s_c);
#pragma unroll
        for (int q = 0; q < kStrips; q++) {
            r_m[q] = row_of(t0[q]);
            r_c[q] = row_of(s_c[q]);
        }
    }
    __syncthreads();  // slots 0 and 1 consumed
    if (threadIdx.x == producer) {
        fence_proxy_async();
        issue(kRing);
        issue(kRing + 1);
    }
    auto body = [&](int k, const int U, const bool checked) {
        const int f = k + 2, s = f & (kRing - 1);
        uint4 s_in[kStrips];
        if (checked) {
            read(f, s, s_in);
        } else {
            if (!mbar_wait_bounded(&bars[s], (uint32_t)(f >> kRingLog2) & 1u, kWaitLimitNs)) err = kErrWaitTimeout;
#pragma unroll
            for (int q = 0; q < kStrips; q++)
                s_in[q] = (kDense || has[q]) && ring_ok(s, q) ? my_ring[(size_t)s * slot_stride + (size_t)q * SX]
                                                              : make_uint4(0, 0, 0, 0);
        }
        Row r_p[kStrips];
        uint32_t pc[kStrips][P::NC], ps[kStrips][P::NS];
#pragma unroll
        for (int q = 0; q < kStrips; q++) {
            r_p[q] = row_of(s_in[q]);
            P::make(r_m[q], r_c[q], r_p[q], pc[q], ps[q]);
        }
        uint4* xb = my_x + (size_t)(U & 1) * xpar;
        const size_t xb_rel = (size_t)(U & 1) * xpar;
        if (x_ok(xb_rel)) xb[0] = pack_planes<P::NS>(ps[0]);
        if constexpr (kStrips > 1)
            if (x_ok(xb_rel + (size_t)(kStrips - 1) * SXp)) xb[(size_t)(kStrips - 1) * SXp] = pack_planes<P::NS>(ps[kStrips - 1]);
        __syncthreads();
        if (threadIdx.x == producer) {
            fence_proxy_async();
            issue(f + kRing);
        }
        uint32_t zany = 0u;  // the counted cells' non-zero masks of this plane (its z-extent)
#pragma unroll
        for (int q = 0; q < kStrips; q++) {
            if (outp[q]) {
                uint32_t psm[4], psp[4];
                if (q == 0) {
                    const uint4 t = x_ok(xb_rel - SXp) ? *(xb - SXp) : make_uint4(0, 0, 0, 0);
                    psm[0] = t.x; psm[1] = t.y; psm[2] = t.z; psm[3] = t.w;
                } else {
#pragma unroll
                    for (int i = 0; i < P::NS; i++) psm[i] = ps[q - 1][i];
                }
                if (q == kStrips - 1) {
                    const uint4 t = x_ok(xb_rel + (size_t)kStrips * SXp) ? *(xb + (size_t)kStrips * SXp)
                                                                          : make_uint4(0, 0, 0, 0);
                    psp[0] = t.x; psp[1] = t.y; psp[2] = t.z; psp[3] = t.w;
                } else {
#pragma unroll
                    for (int i = 0; i < P::NS; i++) psp[i] = ps[q + 1][i];
                }
                uint32_t cnt[count_bits(NB)];
                P::combine(pc[q], psm, psp, cnt);
                const uint4 n = update_strip<NB, NT, kCountZero, Fixed::kFullRange, kPop, false>(
                    s_c[q], r_c[q].a, cnt, valid, R, acc, xbits[q], (uint32_t)zo, true, &zany);
                const uint32_t di = (uint32_t)zo * plane_strips + dst_row[q];
                if (CAVE_IN_BOUNDS(di, copy_n, err)) dst[di] = n;
            }
        }
        if (zany) {
            acc.zmin = min(acc.zmin, (uint32_t)zo);
            acc.zmax = max(acc.zmax, (uint32_t)zo);
        }
#pragma unroll
        for (int q = 0; q < kStrips; q++) {
            r_m[q] = r_c[q];
            r_c[q] = r_p[q];
            s_c[q] = s_in[q];
        }
        zo += zstep;
    };
    static_assert(kUnroll == 6, "the march is unrolled six times");
    int k = 0;
    for (; k + kUnroll < L; k += kUnroll) {  // every fetch inside the grid
        body(k, 0, false);
        body(k + 1, 1, false);
        body(k + 2, 2, false);
        body(k + 3, 3, false);
        body(k + 4, 4, false);
        body(k + 5, 5, false);
    }
    for (; k < L; k++) body(k, k & 1, k + 1 == L);

    // ---- per-CTA reduction of the tick statistics
    uint32_t bx0 = 0xFFFFFFFFu, bx1 = 0u, by0 = 0xFFFFFFFFu, by1 = 0u;
    uint32_t xall = xbits[0];
    if (xbits[0]) by0 = by1 = (uint32_t)y[0];
#pragma unroll
    for (int q = 1; q < kStrips; q++) {  // rows in increasing y
        xall |= xbits[q];
        if (xbits[q]) {
            by0 = min(by0, (uint32_t)y[q]);
            by1 = (uint32_t)y[q];
        }
    }
    if (xall) {
        bx0 = sx * 32u + (uint32_t)(__ffs(xall) - 1);
        bx1 = sx * 32u + 31u - (uint32_t)__clz(xall);
    }
    bool slots_ok = true;
#ifdef CAVE_CHECKED
    if (tick_arg >= 0) {  // the deferred-fold slots this launch adds to: tick, and tick - 1 for kPopInput
        const uint32_t tick_limit = sim->tick_limit;
        slots_ok = CAVE_IN_BOUNDS(tick, tick_limit, err) &&
                   (kPop != kPopInput || CAVE_IN_BOUNDS(tick - 1u, tick_limit, err));
    }
#endif
    uint32_t v[11] = {acc.surviving, acc.born, acc.zero, acc.population, bx0, by0, acc.zmin, bx1, by1, acc.zmax, err};
    warp_reduce_tick(v);
    v[10] = warp_or(v[10]);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 11; q++) red[warp][q] = v[q];
    }
    __syncthreads();
    if (warp != 0) return;
    // Lane 0 of warp 0 folds the per-warp values (measured faster than a parallel fold by 11
    // lanes); then lane q (< 11) applies column q to the record with one atomic -- 0..3 sums,
    // 4..6 bounding-box minimum, 7..9 maximum, 10 error flags.
    if (lane == 0) {
        const uint32_t nw = blockDim.x >> 5;
        for (uint32_t w = 1; w < nw; w++) {
            for (int q = 0; q < 4; q++) red[0][q] += red[w][q];
            for (int q = 4; q < 7; q++) red[0][q] = min(red[0][q], red[w][q]);
            for (int q = 7; q < 10; q++) red[0][q] = max(red[0][q], red[w][q]);
            red[0][10] |= red[w][10];
        }
    }
    __syncwarp();
    const uint32_t x = red[0][lane < 11u ? lane : 10u];
    const uint32_t pop = __shfl_sync(0xFFFFFFFFu, x, 3);
    if (tick_arg >= 0) {
        // deferred fold: add this CTA's totals to the tick's slot (no ticket, no fence: the next
        // launch starts after this one has completed and flushed)
        if (!slots_ok) {  // checked build: only the error flags are applied
            if (lane == 10u && x) atomicOr(&sim->error, x);
            return;
        }
        TickTotals* d = sim->deferred + tick;
        TickTotals* dp = kPop == kPopInput ? d - 1 : d;  // the slot the population belongs to
        if (lane < 3u && x) atomicAdd(&d->surv + lane, x);
        if (kPop != kPopNone) {
            if (lane == 3u && x) atomicAdd(&dp->pop, x);
            if (lane >= 4u && lane < 7u && pop) atomicMax(&dp->nbmin[lane - 4u], ~x);
            if (lane >= 7u && lane < 10u && pop) atomicMax(&dp->bmax[lane - 7u], x);
        }
        if (lane == 10u && x) atomicOr(&sim->error, x);
        return;
    }
    if (lane < 4u && x) atomicAdd(&sim->acc_surv + lane, x);
    if (lane >= 4u && lane < 7u && pop) atomicMin(&sim->acc_bmin[lane - 4u], x);
    if (lane >= 7u && lane < 10u && pop) atomicMax(&sim->acc_bmax[lane - 7u], x);
    if (lane == 10u && x) atomicOr(&sim->error, x);
    __threadfence();  // each lane's update is visible before the ticket is taken
    __syncwarp();
    bool last = false;
    if (lane == 0) last = atomicAdd(&sim->ticket, 1u) == (it.dir_items >> 1) - 1u;
    if (__shfl_sync(0xFFFFFFFFu, last, 0) && lane == 0) {
        __threadfence();
        fold_tick(sim);
    }
}

}  // namespace cave
