// stream_tick2.cuh -- two ticks per launch on the strip layout (temporal blocking), for the
// rule-specialised kernels compiled at run time (jit.cpp).
//
// The same arithmetic as stream_tick.cuh (searchSimulationCube.slang:117-247 per tick), with
// two ticks fused in one march so that a grid crosses HBM once per two ticks: each input plane
// tile arrives once (cp.async.bulk into the plane ring), the first tick ("stage A") is computed
// for the tile's rows plus one halo row on each side, its result stays on chip, and the second
// tick ("stage B") is computed from it one plane behind and written to HBM. The tile therefore
// carries two halo rows on each side (rows = ty + 4) and a z-slab reads two halo planes on each
// side. Stage A's rows and planes outside the grid are held at state 0 (outside the grid is
// dead), so stage B sees exactly the first tick's grid.
//
// Per step f of the march (fetch f = input plane zfirst + f * zstep, f = 0 .. L + 3):
//   stage A, f in [2, L + 3]: output A(f - 1) from input planes f - 2, f - 1, f;
//   stage B, f in [5, L + 4]: output B(f - 3) from A(f - 4), A(f - 3), A(f - 2);
// both stages write their y-exchange column sums before one CTA barrier and read their
// neighbours' after it. B's output planes are the item's [z0, z1); A(j) is needed for
// j in [1, L + 2].
//
// Statistics (deferred-fold runs only): stage A is tick `tick`, stage B tick `tick + 1`. Each
// counts its surviving and born cells over the item's own rows and planes into its slot, and the
// population and bounding box of its input (the previous tick's result) into the previous
// tick's slot; the run's first launch (kFirst) counts the cells that were 0 instead of the
// previous population (there is none), exactly as the single-tick counting / derived kernels.
#pragma once
#include "cave_stdint.h"

#include "ca_core.cuh"
#include "cave_internal.h"
#include "ptx.cuh"
#include "stream_common.cuh"

namespace cave {

// Shared-memory layout (dynamic): ring[kRing][rows*SX] uint4, xch[2 stages][kXch][rows*SXp] uint4,
// mbarriers.
__host__ __device__ inline size_t stream2_smem_bytes(uint32_t rows, uint32_t SX, uint32_t SXp) {
    return (size_t)kRing * rows * SX * 16 + (size_t)2 * kXch * rows * SXp * 16 + kRing * 8 + 16;
}

// NB: neighbourhood bits. Fixed: the rule as compile-time constants (kFixed must be true).
// kFirst: the run's first launch (ticks 0 and 1). kDense: the launch guarantees SX == SXp.
// kStrips: rows per thread. src_sel: the cell copy (0 / 1) holding the input; the output goes to
// the other one.
template <int NB, class Fixed, bool kFirst, bool kDense, int kStrips>
__device__ __forceinline__ void stream_tick2_body(const StreamItem* __restrict__ items, StripSim* sims, uint4* pool,
                                                  uint32_t sxp_log2, int tick_arg, int src_sel) {
    static_assert(Fixed::kFixed, "the two-tick kernel is compiled for one rule");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ uint32_t red[32][21];
    const StreamItem it = items[blockIdx.x];
    StripSim* sim = sims + it.sim;
    const uint32_t SXp = 1u << sxp_log2;
    const uint32_t rows = kStrips * (blockDim.x >> sxp_log2);  // incl. two halo rows on each side
    // fixed while the simulation runs: read while the previous launch drains
    const uint32_t SX = sim->SX, X = sim->X, Y = sim->Y, Z = sim->Z;
    const uint64_t buf0 = sim->buf[0], buf1 = sim->buf[1];
    TickTotals* const deferred = sim->deferred;
    const DeviceRule R = Fixed::rule();
    uint4* ring = reinterpret_cast<uint4*>(smem_raw);
    uint4* xch = ring + (size_t)kRing * rows * SX;
    uint64_t* bars = reinterpret_cast<uint64_t*>(xch + (size_t)2 * kXch * rows * SXp);
    if (threadIdx.x == 0) {
        for (int s = 0; s < kRing; s++) mbar_init(&bars[s], 1);
        mbar_init_fence();
    }
    __syncthreads();
    // Everything below reads the previous launch's results.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;");

    const uint32_t sx = threadIdx.x & (SXp - 1u), yy0 = kStrips * (threadIdx.x >> sxp_log2);
    const uint32_t ty = it.ty;
    int y[kStrips];
    bool has[kStrips], own[kStrips];
#pragma unroll
    for (int q = 0; q < kStrips; q++) {
        const uint32_t yy = yy0 + q;
        y[q] = (int)it.y0 - 2 + (int)yy;
        has[q] = sx < SX && y[q] >= 0 && y[q] < (int)Y && yy < ty + 4u;
        own[q] = has[q] && yy >= 2 && yy <= ty + 1u;   // stage B computes it; both count it
    }
    const uint32_t valid = sx < SX ? strip_valid(sx, X) : 0u;
    const bool left_edge = sx == 0, right_edge = sx + 1 >= SX;
    const uint32_t send_mask = (left_edge ? ~1u : ~0u) & (right_edge ? 0x7FFFFFFFu : ~0u);
    const int lane_l = (int)((threadIdx.x + 31u) & 31u), lane_r = (int)((threadIdx.x + 1u) & 31u);

    // rows of the tile present in memory: [ylo, yhi)
    const int ylo = max((int)it.y0 - 2, 0), yhi = min((int)it.y0 + (int)ty + 2, (int)Y);
    const uint32_t tile_bytes = (uint32_t)(yhi - ylo) * SX * 16u;
    const uint32_t slot_row0 = (uint32_t)(ylo - ((int)it.y0 - 2));
    const uint32_t slot_stride = rows * SX;
    const int L = (int)it.z1 - (int)it.z0;  // stage B output planes
    const int nfetch = L + 4;
    const bool down = (it.dir_items & 1u) != 0;
    const int zstep = down ? -1 : 1;
    const int zfirst = down ? (int)it.z1 + 1 : (int)it.z0 - 2;  // plane of fetch 0
    uint32_t err = 0;
    // extents (uint4 units) that the checked build tests every index against; a layout that does
    // not fit the launch's shared memory fails every shared-memory check
    const size_t xpar = (size_t)rows * SXp;
    size_t ring_n = (size_t)kRing * slot_stride, xch_n = (size_t)2 * kXch * xpar;
    const size_t copy_n = (size_t)Z * Y * SX;
#ifdef CAVE_CHECKED
    if (!CAVE_IN_BOUNDS((ring_n + xch_n) * 16 + kRing * 8 - 1, dynamic_smem_bytes(), err)) ring_n = xch_n = 0;
    const uint32_t tick_limit = sim->tick_limit;
#endif
    const size_t ring_off = (size_t)yy0 * SX + sx, x_off = (size_t)yy0 * SXp + sx;

    const uint32_t tick = (uint32_t)tick_arg;
    const uint4* src = reinterpret_cast<const uint4*>(reinterpret_cast<unsigned char*>(pool) + (src_sel ? buf1 : buf0));
    uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(pool) + (src_sel ? buf0 : buf1));

    // Thread 0 fills ring slot f % kRing with input plane f; a plane outside the grid completes
    // its slot's phase with a plain arrive (every fetch advances its slot by one phase).
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
    if (threadIdx.x == 0) {
        for (int f = 0; f < kRing; f++) issue(f);
    }
    const uint4* my_ring = ring + (size_t)yy0 * SX + sx;  // row q at + q * SX
    if constexpr (kDense) {
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
    auto row_of = [&](uint4 st) -> Row {
        const uint32_t a = alive_plane(st, R);
        const uint32_t v = a & send_mask;
        return make_row(a, __shfl_sync(0xFFFFFFFFu, v, lane_l), __shfl_sync(0xFFFFFFFFu, v, lane_r));
    };
    // A fetch outside the slab or the grid has no copy: nothing to wait for, and it reads as dead
    // cells. Otherwise each warp waits for the fetch itself (phase parity (f / kRing) & 1 of slot
    // f % kRing) when it reads it. (Waiting one step ahead, before the previous step's barrier,
    // measured 3.5% slower.)
    auto no_copy = [&](int f) { return f >= nfetch || (unsigned)(zfirst + f * zstep) >= Z; };
    auto read = [&](int f, uint4* out, bool checked) {
        if (checked && no_copy(f)) {
#pragma unroll
            for (int q = 0; q < kStrips; q++) out[q] = make_uint4(0, 0, 0, 0);
            return;
        }
        const int s = f & (kRing - 1);
        if (!mbar_wait_bounded(&bars[s], (uint32_t)(f >> kRingLog2) & 1u, kWaitLimitNs)) err = kErrWaitTimeout;
#pragma unroll
        for (int q = 0; q < kStrips; q++)
            out[q] = (kDense || has[q]) &&
                             CAVE_IN_BOUNDS(ring_off + (size_t)s * slot_stride + (size_t)q * SX, ring_n, err)
                         ? my_ring[(size_t)s * slot_stride + (size_t)q * SX]
                         : make_uint4(0, 0, 0, 0);
    };

    using P = typename ColumnsFor<NB, true>::type;
    TickAcc accA, accB;
    accA.reset(SX != 0u ? 1u : 0u);  // SX >= 1: a 1 the compiler cannot fold (see mad_add)
    accB.reset(accA.one);
    uint32_t xbA[kStrips], xbB[kStrips];
    // strip index of each row in a plane of the output copy (a copy holds at most 2^25 strips),
    // and stage A's valid mask per row: 0 on rows outside the grid, whose input is all 0, so
    // that their stage-A result is 0 (outside the grid is dead) without a select
    uint32_t dst_row[kStrips], validA[kStrips];
#pragma unroll
    for (int q = 0; q < kStrips; q++) {
        xbA[q] = xbB[q] = 0u;
        dst_row[q] = (uint32_t)max(y[q], 0) * SX + sx;
        validA[q] = has[q] ? valid : 0u;
    }
    const uint32_t plane_strips = Y * SX;
    uint4* my_x = xch + (size_t)yy0 * SXp + sx;  // row q at + q * SXp; stage B at + kXch * xpar
    // offsets of the rows above and below this thread's rows in an exchange buffer, clamped to
    // its own row at the tile's first and last thread rows (whose results are not used)
    const size_t x_dn = yy0 > 0 ? (size_t)SXp : 0, x_up = yy0 + kStrips < rows ? (size_t)kStrips * SXp : 0;
    // the checked build's test of an exchange-buffer index, relative to my_x
    auto x_ok = [&](size_t rel) { return CAVE_IN_BOUNDS(x_off + rel, xch_n, err); };

    // rolling state: stage A input rows (planes f-2, f-1) and centre state; stage A outputs
    // A(f-2), A(f-3); stage B rows of A(f-4), A(f-3)
    Row rAm[kStrips], rAc[kStrips], rBm[kStrips], rBc[kStrips];
    uint4 sAc[kStrips], nA2[kStrips], nA3[kStrips];
    {
        uint4 t0[kStrips];
        read(0, t0, true);
        read(1, sAc, true);
#pragma unroll
        for (int q = 0; q < kStrips; q++) {
            rAm[q] = row_of(t0[q]);
            rAc[q] = row_of(sAc[q]);
            nA2[q] = nA3[q] = make_uint4(0, 0, 0, 0);
            rBm[q] = rBc[q] = Row{0u, 0u, 0u, 0u, 0u};
        }
    }
    __syncthreads();  // slots 0 and 1 consumed
    if (threadIdx.x == 0) {
        fence_proxy_async();
        issue(kRing);
        issue(kRing + 1);
    }

    // One step of the march. U: exchange-buffer parity; checked: the step may be at a slab end
    // (fetches outside the grid or past the slab, stage A or B inactive).
    auto step = [&](int f, int U, bool checked) {
        const bool actA = !checked || f <= L + 3;
        const bool actB = !checked || f >= 5;
        uint4* xa = my_x + (size_t)(U & 1) * xpar;
        uint4* xb = xa + (size_t)kXch * xpar;
        // ---- stage A: input plane f
        uint4 s_in[kStrips];
        Row rAp[kStrips];
        uint32_t pcA[kStrips][P::NC], psA[kStrips][P::NS];
        if (actA) {
            read(f, s_in, checked);
#pragma unroll
            for (int q = 0; q < kStrips; q++) {
                rAp[q] = row_of(s_in[q]);
                P::make(rAm[q], rAc[q], rAp[q], pcA[q], psA[q]);
            }
            const size_t xa_rel = (size_t)(U & 1) * xpar;
            if (x_ok(xa_rel)) xa[0] = pack_planes<P::NS>(psA[0]);
            if constexpr (kStrips > 1)
                if (x_ok(xa_rel + (size_t)(kStrips - 1) * SXp))
                    xa[(size_t)(kStrips - 1) * SXp] = pack_planes<P::NS>(psA[kStrips - 1]);
        }
        // ---- stage B: rows of A(f-2)
        Row rBp[kStrips];
        uint32_t pcB[kStrips][P::NC], psB[kStrips][P::NS];
#pragma unroll
        for (int q = 0; q < kStrips; q++) rBp[q] = row_of(nA2[q]);
        if (actB) {
#pragma unroll
            for (int q = 0; q < kStrips; q++) P::make(rBm[q], rBc[q], rBp[q], pcB[q], psB[q]);
            const size_t xb_rel = (size_t)(U & 1) * xpar + (size_t)kXch * xpar;
            if (x_ok(xb_rel)) xb[0] = pack_planes<P::NS>(psB[0]);
            if constexpr (kStrips > 1)
                if (x_ok(xb_rel + (size_t)(kStrips - 1) * SXp))
                    xb[(size_t)(kStrips - 1) * SXp] = pack_planes<P::NS>(psB[kStrips - 1]);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            fence_proxy_async();
            issue(f + kRing);
        }
        // ---- stage A: A(f - 1), plane zA. Every row is computed, branch-free (a branch per row
        // would split the step into blocks the compiler cannot interleave). Rows and planes
        // outside the grid have input 0 and valid mask 0, so their result is 0. The tile's two
        // outermost rows (0 and ty + 3) read clamped neighbour rows and come out wrong; they feed
        // only stage B's rows 1 and ty + 2, which are neither stored nor counted.
        uint4 nA1[kStrips];
        if (actA) {
            const int jA = f - 1;
            const int zA = zfirst + jA * zstep;
            const bool inA = !checked || (unsigned)zA < Z;
            const bool ownA = !checked || (jA >= 2 && jA <= L + 1);
            uint32_t zany = 0u;
#pragma unroll
            for (int q = 0; q < kStrips; q++) {
                uint32_t psm[4], psp[4];
                if (q == 0) {
                    const uint4 t = x_ok((size_t)(U & 1) * xpar - x_dn) ? *(xa - x_dn) : make_uint4(0, 0, 0, 0);
                    psm[0] = t.x; psm[1] = t.y; psm[2] = t.z; psm[3] = t.w;
                } else {
#pragma unroll
                    for (int i = 0; i < P::NS; i++) psm[i] = psA[q - 1][i];
                }
                if (q == kStrips - 1) {
                    const uint4 t = x_ok((size_t)(U & 1) * xpar + x_up) ? *(xa + x_up) : make_uint4(0, 0, 0, 0);
                    psp[0] = t.x; psp[1] = t.y; psp[2] = t.z; psp[3] = t.w;
                } else {
#pragma unroll
                    for (int i = 0; i < P::NS; i++) psp[i] = psA[q + 1][i];
                }
                uint32_t cnt[count_bits(NB)];
                P::combine(pcA[q], psm, psp, cnt);
                nA1[q] = update_strip<NB, 0, kFirst, Fixed::kFullRange, kFirst ? kPopNone : kPopInput, false>(
                    sAc[q], rAc[q].a, cnt, inA ? validA[q] : 0u, R, accA, xbA[q], (uint32_t)zA, own[q] && ownA,
                    &zany);
            }
            if (zany) {
                accA.zmin = min(accA.zmin, (uint32_t)zA);
                accA.zmax = max(accA.zmax, (uint32_t)zA);
            }
        }
        // ---- stage B: B(f - 3), plane zB, written to HBM (rows it owns; the others computed and
        // dropped, as in stage A)
        if (actB) {
            const int zB = zfirst + (f - 3) * zstep;
            uint32_t zany = 0u;
#pragma unroll
            for (int q = 0; q < kStrips; q++) {
                uint32_t psm[4], psp[4];
                if (q == 0) {
                    const uint4 t = x_ok((size_t)((U & 1) + kXch) * xpar - x_dn) ? *(xb - x_dn)
                                                                                   : make_uint4(0, 0, 0, 0);
                    psm[0] = t.x; psm[1] = t.y; psm[2] = t.z; psm[3] = t.w;
                } else {
#pragma unroll
                    for (int i = 0; i < P::NS; i++) psm[i] = psB[q - 1][i];
                }
                if (q == kStrips - 1) {
                    const uint4 t = x_ok((size_t)((U & 1) + kXch) * xpar + x_up) ? *(xb + x_up)
                                                                                   : make_uint4(0, 0, 0, 0);
                    psp[0] = t.x; psp[1] = t.y; psp[2] = t.z; psp[3] = t.w;
                } else {
#pragma unroll
                    for (int i = 0; i < P::NS; i++) psp[i] = psB[q + 1][i];
                }
                uint32_t cnt[count_bits(NB)];
                P::combine(pcB[q], psm, psp, cnt);
                const uint4 n = update_strip<NB, 0, false, Fixed::kFullRange, kPopInput, false>(
                    nA3[q], rBc[q].a, cnt, valid, R, accB, xbB[q], (uint32_t)zB, own[q], &zany);
                const uint32_t di = (uint32_t)zB * plane_strips + dst_row[q];
                if (own[q] && CAVE_IN_BOUNDS(di, copy_n, err)) dst[di] = n;
            }
            if (zany) {
                accB.zmin = min(accB.zmin, (uint32_t)zB);
                accB.zmax = max(accB.zmax, (uint32_t)zB);
            }
        }
        // ---- rotate
#pragma unroll
        for (int q = 0; q < kStrips; q++) {
            if (actA) {
                rAm[q] = rAc[q];
                rAc[q] = rAp[q];
                sAc[q] = s_in[q];
            }
            nA3[q] = nA2[q];
            nA2[q] = actA ? nA1[q] : make_uint4(0, 0, 0, 0);
            rBm[q] = rBc[q];
            rBc[q] = rBp[q];
        }
    };
    static_assert(kUnroll == 6, "the march is unrolled six times");
    int f = 2;
    for (; f < 5; f++) step(f, f & 1, true);
    // steps 5 .. L + 1 read planes inside the slab and run both stages
    for (; f + kUnroll <= L + 2; f += kUnroll) {
        step(f, 1, false);
        step(f + 1, 0, false);
        step(f + 2, 1, false);
        step(f + 3, 0, false);
        step(f + 4, 1, false);
        step(f + 5, 0, false);
    }
    for (; f <= L + 4; f++) step(f, f & 1, true);

    // ---- per-CTA reduction of both ticks' statistics
    uint32_t v[21];
    bool slots_ok = true;
    {
        uint32_t ax0 = 0xFFFFFFFFu, ax1 = 0u, ay0 = 0xFFFFFFFFu, ay1 = 0u, xa = 0u;
        uint32_t bx0 = 0xFFFFFFFFu, bx1 = 0u, by0 = 0xFFFFFFFFu, by1 = 0u, xb = 0u;
#pragma unroll
        for (int q = 0; q < kStrips; q++) {  // rows in increasing y
            xa |= xbA[q];
            xb |= xbB[q];
            if (xbA[q]) {
                ay0 = min(ay0, (uint32_t)y[q]);
                ay1 = (uint32_t)y[q];
            }
            if (xbB[q]) {
                by0 = min(by0, (uint32_t)y[q]);
                by1 = (uint32_t)y[q];
            }
        }
        if (xa) {
            ax0 = sx * 32u + (uint32_t)(__ffs(xa) - 1);
            ax1 = sx * 32u + 31u - (uint32_t)__clz(xa);
        }
        if (xb) {
            bx0 = sx * 32u + (uint32_t)(__ffs(xb) - 1);
            bx1 = sx * 32u + 31u - (uint32_t)__clz(xb);
        }
#ifdef CAVE_CHECKED
        // the statistics slots: stage A's input population goes to slot tick - 1 (none for the
        // run's first launch), stage B's to slot tick + 1
        slots_ok = CAVE_IN_BOUNDS(tick + 1u, tick_limit, err) && (kFirst || CAVE_IN_BOUNDS(tick - 1u, tick_limit, err));
#endif
        const uint32_t vv[21] = {accA.surviving, accA.born, accA.zero, accA.population, ax0, ay0, accA.zmin,
                                 ax1, ay1, accA.zmax,
                                 accB.surviving, accB.born, accB.zero, accB.population, bx0, by0, accB.zmin,
                                 bx1, by1, accB.zmax, err};
#pragma unroll
        for (int q = 0; q < 21; q++) v[q] = vv[q];
    }
    warp_reduce_tick(v);
    warp_reduce_tick(v + 10);
    v[20] = warp_or(v[20]);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 21; q++) red[warp][q] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
    if (lane == 0) {
        const uint32_t nw = blockDim.x >> 5;
        for (uint32_t w = 1; w < nw; w++) {
            for (int h = 0; h < 2; h++) {
                for (int q = 0; q < 4; q++) red[0][10 * h + q] += red[w][10 * h + q];
                for (int q = 4; q < 7; q++) red[0][10 * h + q] = min(red[0][10 * h + q], red[w][10 * h + q]);
                for (int q = 7; q < 10; q++) red[0][10 * h + q] = max(red[0][10 * h + q], red[w][10 * h + q]);
            }
            red[0][20] |= red[w][20];
        }
    }
    __syncwarp();
    // lane q applies column q: stage A (tick) 0..9, stage B (tick + 1) 10..19, error flags 20
    const uint32_t x = red[0][lane < 21u ? lane : 20u];
    const uint32_t popA = __shfl_sync(0xFFFFFFFFu, x, 3), popB = __shfl_sync(0xFFFFFFFFu, x, 13);
    if (slots_ok || lane >= 20u) {  // checked build: only the error flags when a slot is out of range
    TickTotals* dA = deferred + tick;  // stage A's slot; its input's population goes to dA - 1
    TickTotals* dB = dA + 1;           // stage B's slot; its input's population goes to dA
    if (lane < 3u) {
        if (x && (lane < 2u || kFirst)) atomicAdd(&dA->surv + lane, x);
    } else if (lane < 10u) {
        if (!kFirst) {
            if (lane == 3u && x) atomicAdd(&(dA - 1)->pop, x);
            if (lane >= 4u && lane < 7u && popA) atomicMax(&(dA - 1)->nbmin[lane - 4u], ~x);
            if (lane >= 7u && popA) atomicMax(&(dA - 1)->bmax[lane - 7u], x);
        }
    } else if (lane < 12u) {
        if (x) atomicAdd(&dB->surv + (lane - 10u), x);
    } else if (lane == 13u) {
        if (x) atomicAdd(&dA->pop, x);
    } else if (lane >= 14u && lane < 17u) {
        if (popB) atomicMax(&dA->nbmin[lane - 14u], ~x);
    } else if (lane >= 17u && lane < 20u) {
        if (popB) atomicMax(&dA->bmax[lane - 17u], x);
    } else if (lane == 20u) {
        if (x) atomicOr(&sim->error, x);
    }
    }
    }
}

}  // namespace cave
