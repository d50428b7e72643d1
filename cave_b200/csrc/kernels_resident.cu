// kernels_resident.cu -- persistent batched kernel: whole small grids resident in one CTA's
// shared memory for all their ticks.
//
// Each CTA takes a simulation from a work queue (atomic counter), copies its initial grid
// (strip layout) into shared memory with one TMA bulk copy, and runs the rule tick after
// tick until the search manager reports status > 0 (searchManager.slang:98-139: early death
// when nothing survives and nothing is born, or the tick limit) -- the per-rule lifecycle of
// a SearchSystem slot (searchSystem.cpp:496-526), with no host round trip per tick. Then it
// writes the result and takes the next simulation.
//
// Within a tick the grid is updated in place. The CTA's threads are split into `nseg`
// z-segments; in each, a thread owns one strip column (sx, y) and marches its segment's
// planes, all segments in lockstep (one CTA barrier per plane for the y-exchange of column
// sums). A thread reads the raw state of its own column only, one plane ahead of the plane
// it writes; the two segment-boundary planes it needs from its neighbouring segments are
// read before anyone writes (the upper one is held in registers), so in-place is safe.
#include <cuda_runtime.h>

#include <algorithm>

#include "ca_core.cuh"
#include "cave_internal.h"
#include "kernels.h"
#include "ptx.cuh"
#include "ring.cuh"

namespace cave {

template <int N>
__device__ __forceinline__ uint4 to_u4(const uint32_t* p) {
    uint4 v = make_uint4(p[0], 0u, 0u, 0u);
    if constexpr (N > 1) v.y = p[1];
    if constexpr (N > 2) v.z = p[2];
    if constexpr (N > 3) v.w = p[3];
    return v;
}

template <int NB, int NT>
__global__ void __launch_bounds__(1024) k_resident(ResLaunch P, const ResSim* __restrict__ sims,
                                                   const DeviceRule* __restrict__ rules,
                                                   cave_sim_result* __restrict__ results, uint32_t* queue,
                                                   DoneRing* ring) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(16) DeviceRule s_rule;  // filled with 16-byte copies
    __shared__ uint32_t s_sim, s_stop;
    __shared__ uint32_t red[32][11];
    __shared__ __align__(8) uint64_t s_bar;

    const uint32_t X = P.X, Y = P.Y, Z = P.Z, SX = P.SX;
    const uint32_t SXp = 1u << P.sxp_log2;
    const uint32_t cols = Y * SXp;                   // threads per segment
    uint4* grid = reinterpret_cast<uint4*>(smem_raw);
    const uint32_t plane = SX * Y;                   // strips per plane
    uint4* xch = grid + (size_t)plane * Z;           // [2][nseg][Y+2][SXp]
    const uint32_t xseg = (Y + 2) * SXp, xpar = xseg * P.nseg;

    const uint32_t tid = threadIdx.x;
    const uint32_t seg = tid / cols, rem = tid % cols;
    const uint32_t yy = rem >> P.sxp_log2, sx = rem & (SXp - 1u);
    const bool in_seg = seg < P.nseg;
    const bool has = in_seg && sx < SX;
    const uint32_t valid = has ? strip_valid(sx, X) : 0u;
    // x-neighbour bits by rotation inside the warp (as in the streaming kernel): lane - 1 (mod 32)
    // of a row's first strip is the last lane of the previous row, segment or warp -- a right
    // edge or an absent strip -- and each thread sends its alive plane with the bits that would
    // wrap across rows cleared.
    const bool left_edge = sx == 0, right_edge = sx + 1 >= SX;
    const uint32_t send_mask = (left_edge ? ~1u : ~0u) & (right_edge ? 0x7FFFFFFFu : ~0u);
    const int lane_l = (int)((tid + 31u) & 31u), lane_r = (int)((tid + 1u) & 31u);
    const int zs = in_seg ? (int)(seg * P.seg_len) : (int)Z;
    const int ze = min(zs + (int)P.seg_len, (int)Z);
    const int L = max(ze - zs, 0);
    const uint32_t volume = X * Y * Z;

    // zero the exchange buffers once: the halo rows (y = -1, y = Y) are never written
    for (uint32_t i = tid; i < 2 * xpar; i += blockDim.x) xch[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        mbar_init(&s_bar, 1);
        mbar_init_fence();
    }
    __syncthreads();
    uint32_t bar_phase = 0;
    const uint32_t grid_bytes = plane * Z * 16u;
    // extents (uint4 units) that the checked build tests every index against; a layout that does
    // not fit the launch's shared memory fails every shared-memory check
    uint32_t layout_err = 0;
    size_t grid_n = (size_t)plane * Z, xch_n = (size_t)2 * xpar;
#ifdef CAVE_CHECKED
    if (!CAVE_IN_BOUNDS((grid_n + xch_n) * 16 - 1, dynamic_smem_bytes(), layout_err)) grid_n = xch_n = 0;
#endif
    const size_t g_off = (size_t)yy * SX + sx, x_off = (size_t)seg * xseg + (size_t)(yy + 1) * SXp + sx;

    uint4* my_x = xch + (size_t)seg * xseg + (size_t)(yy + 1) * SXp + sx;
    uint4* my_g = grid + (size_t)yy * SX + sx;  // + z * plane

    while (true) {
        if (tid == 0) s_sim = atomicAdd(queue, 1u);
        __syncthreads();
        const uint32_t si = s_sim;
        if (si >= P.n_sims) break;
        const ResSim sd = sims[si];
        // rule and initial grid
        {
            const uint4* rsrc = reinterpret_cast<const uint4*>(rules + sd.rule);
            uint4* rdst = reinterpret_cast<uint4*>(&s_rule);
            for (uint32_t i = tid; i < sizeof(DeviceRule) / 16; i += blockDim.x) rdst[i] = rsrc[i];
        }
        uint32_t err = layout_err;
        if (tid == 0 && !P.hold_init) {
            fence_proxy_async();
            if (CAVE_IN_BOUNDS(grid_bytes / 16u - 1u, grid_n, err)) {
                mbar_expect_tx(&s_bar, grid_bytes);
                bulk_g2s(grid, sd.init, grid_bytes, &s_bar);
            } else {
                mbar_arrive(&s_bar);  // checked build: the copy is skipped, its phase completed
            }
        }
        if (!mbar_wait_bounded(&s_bar, bar_phase, P.wait_us ? (uint64_t)P.wait_us * 1000u : kWaitLimitNs))
            err = kErrWaitTimeout;
        bar_phase ^= 1u;
        __syncthreads();  // rule visible
        DeviceRule R;
#pragma unroll
        for (int i = 0; i < 4; i++) R.m[i] = s_rule.m[i];
        R.alive_ok = s_rule.alive_ok;
        R.lut_s = s_rule.lut_s;
        R.lut_b = s_rule.lut_b;
#pragma unroll
        for (int t = 0; t < NT; t++) R.terms[t] = s_rule.terms[t];

        auto load = [&](int z) -> uint4 {
            return (has && z >= 0 && z < (int)Z && CAVE_IN_BOUNDS(g_off + (size_t)z * plane, grid_n, err))
                       ? my_g[(size_t)z * plane]
                       : make_uint4(0, 0, 0, 0);
        };
        auto row_of = [&](uint4 st) -> Row {
            const uint32_t a = alive_plane(st, R);  // zero for absent strips
            const uint32_t v = a & send_mask;
            return make_row(a, __shfl_sync(0xFFFFFFFFu, v, lane_l), __shfl_sync(0xFFFFFFFFu, v, lane_r));
        };

        cave_grid_info info{0, 0, 0, 0, 0, 0};
        uint32_t active_ticks = 0, last_pop = 0;
        uint64_t total_changed = 0;
        uint32_t bmin[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, bmax[3] = {0, 0, 0};
        using PS = Partials<NB>;
        for (;;) {  // ends when the manager reports status > 0 (the tick limit included)
            // warm-up: planes zs-1 and zs, plus the upper boundary plane ze, before any write
            Row r_m = row_of(L > 0 ? load(zs - 1) : make_uint4(0, 0, 0, 0));
            uint4 s_c = L > 0 ? load(zs) : make_uint4(0, 0, 0, 0);
            Row r_c = row_of(s_c);
            const uint4 s_top = L > 0 ? load(ze) : make_uint4(0, 0, 0, 0);
            __syncthreads();
            TickAcc acc;
            acc.reset(P.nseg != 0u ? 1u : 0u);  // nseg >= 1: a 1 the compiler cannot fold (see mad_add)
            uint32_t xbits = 0u;
            // one plane; U = k & 1 (the exchange buffer half) is a constant of each call
            auto step = [&](int k, const int U) {
                const bool act = k < L;
                const int z = zs + k;
                const uint4 s_in = !act ? make_uint4(0, 0, 0, 0) : (z + 1 < ze ? load(z + 1) : s_top);
                const Row r_p = row_of(s_in);
                uint32_t pc[PS::NC], ps[PS::NS];
                PS::make(r_m, r_c, r_p, pc, ps);
                uint4* xb = my_x + (size_t)U * xpar;
                const size_t xi = x_off + (size_t)U * xpar;
                if (in_seg && CAVE_IN_BOUNDS(xi, xch_n, err)) *xb = to_u4<PS::NS>(ps);
                __syncthreads();
                if (act && has) {
                    const uint4 qm = CAVE_IN_BOUNDS(xi - SXp, xch_n, err) ? *(xb - SXp) : make_uint4(0, 0, 0, 0);
                    const uint4 qp = CAVE_IN_BOUNDS(xi + SXp, xch_n, err) ? *(xb + SXp) : make_uint4(0, 0, 0, 0);
                    const uint32_t psm[4] = {qm.x, qm.y, qm.z, qm.w}, psp[4] = {qp.x, qp.y, qp.z, qp.w};
                    uint32_t cnt[count_bits(NB)];
                    combine<NB>(pc, psm, psp, cnt);
                    const uint4 n = update_strip<NB, NT>(s_c, r_c.a, cnt, valid, R, acc, xbits, (uint32_t)z);
                    if (CAVE_IN_BOUNDS(g_off + (size_t)z * plane, grid_n, err)) my_g[(size_t)z * plane] = n;
                }
                r_m = r_c;
                r_c = r_p;
                s_c = s_in;
            };
            const int seg_len = (int)P.seg_len;  // the same for every thread: the barriers match
            int k = 0;
            for (; k + 1 < seg_len; k += 2) {
                step(k, 0);
                step(k + 1, 1);
            }
            if (k < seg_len) step(k, 0);
            // ---- tick statistics
            uint32_t bx0 = 0xFFFFFFFFu, bx1 = 0u, by0 = 0xFFFFFFFFu, by1 = 0u;
            if (xbits) {
                bx0 = sx * 32u + (uint32_t)(__ffs(xbits) - 1);
                bx1 = sx * 32u + 31u - (uint32_t)__clz(xbits);
                by0 = by1 = yy;
            }
            uint32_t v[11] = {acc.surviving, acc.born, acc.zero, acc.population, bx0, by0, acc.zmin, bx1, by1,
                              acc.zmax, err};
            warp_reduce_tick(v);
            v[10] = warp_or(v[10]);
            const uint32_t lane = tid & 31u, warp = tid >> 5;
            if (lane == 0) {
#pragma unroll
                for (int q = 0; q < 11; q++) red[warp][q] = v[q];
            }
            __syncthreads();
            if (warp == 0) {
                // lane w takes warp w's values; then a reduction over the lanes
                const uint32_t nw = (blockDim.x + 31) >> 5;
                const bool live = lane < nw;
#pragma unroll
                for (int q = 0; q < 11; q++) v[q] = live ? red[lane][q] : ((q >= 4 && q < 7) ? 0xFFFFFFFFu : 0u);
                warp_reduce_tick(v);
                v[10] = warp_or(v[10]);
            }
            if (tid == 0) {
                const uint32_t surv = v[0], born = v[1], zero = v[2], pop = v[3];
                const uint32_t dead = zero - born;
                const uint32_t dying = volume - dead - born - surv;
                // searchManager.slang:115-139
                info.numberOfSimulationTicksSurvived++;
                info.totalNumberOfCellsThatDied += dead;
                info.totalNumberOfCellsThatWereBorn += born;
                info.finalAliveCount = surv;
                if (surv > info.maxAliveCount) info.maxAliveCount = surv;
                if (surv == 0u && born == 0u)
                    info.status = 1;
                else if (info.numberOfSimulationTicksSurvived >= sd.max_ticks)
                    info.status = 2;
                else
                    info.status = 0;
                const uint32_t changed = born + dying;
                total_changed += changed;
                if (changed) active_ticks++;
                last_pop = pop;
                for (int q = 0; q < 3; q++) {
                    bmin[q] = v[4 + q];
                    bmax[q] = v[7 + q];
                }
                if (v[10]) err |= v[10];
                s_stop = info.status != 0;
            }
            __syncthreads();
            if (s_stop) break;
        }
        if (tid == 0) {
            cave_sim_result r;
            r.info = info;
            r.category = result_category(info, s_rule.maxcs);
            r.tag = 0;
            r.population = last_pop;
            r.activeTicks = active_ticks;
            r.totalChanged = total_changed;
            for (int q = 0; q < 3; q++) {
                r.bbox_min[q] = bmin[q];
                r.bbox_max[q] = bmax[q];
            }
            r.params = cave_sim_params{0, 0, 0};
            r.error = err;
            r.pad = 0;
            if (ring)
                ring_push(ring, sd.result, r);
            else
                results[sd.result] = r;
        }
        __syncthreads();  // grid and rule buffers are reused by the next simulation
    }
}

size_t resident_smem_bytes(uint32_t X, uint32_t Y, uint32_t Z, uint32_t nseg) {
    const uint32_t SX = (X + 31u) / 32u;
    uint32_t SXp = 1;
    while (SXp < SX) SXp <<= 1;
    return (size_t)SX * Y * Z * 16 + (size_t)2 * nseg * (Y + 2) * SXp * 16;
}

template <int NB, int NT>
static cudaError_t launch_res_inst(const ResLaunch& P, const ResSim* sims, const DeviceRule* rules,
                                   cave_sim_result* results, uint32_t* queue, DoneRing* ring, uint32_t ctas,
                                   uint32_t threads, size_t smem, cudaStream_t st) {
    auto k = k_resident<NB, NT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<ctas, threads, smem, st>>>(P, sims, rules, results, queue, ring);
    return cudaGetLastError();
}

template <int NB>
static cudaError_t launch_res_nb(int nt, const ResLaunch& P, const ResSim* sims, const DeviceRule* rules,
                                 cave_sim_result* results, uint32_t* queue, DoneRing* ring,
                                 uint32_t ctas, uint32_t threads, size_t smem, cudaStream_t st) {
    switch (nt) {
        case 0: return launch_res_inst<NB, 0>(P, sims, rules, results, queue, ring, ctas, threads, smem, st);
        case 1: return launch_res_inst<NB, 1>(P, sims, rules, results, queue, ring, ctas, threads, smem, st);
        case 2: return launch_res_inst<NB, 2>(P, sims, rules, results, queue, ring, ctas, threads, smem, st);
        case 3: return launch_res_inst<NB, 3>(P, sims, rules, results, queue, ring, ctas, threads, smem, st);
        case 4: return launch_res_inst<NB, 4>(P, sims, rules, results, queue, ring, ctas, threads, smem, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_resident(int nb, int nt, const ResLaunch& P, const ResSim* sims, const DeviceRule* rules,
                            cave_sim_result* results, uint32_t* queue, DoneRing* ring, uint32_t ctas,
                            uint32_t threads, cudaStream_t st) {
    const size_t smem = resident_smem_bytes(P.X, P.Y, P.Z, P.nseg);
    switch (nb & 7) {
        case 0: return launch_res_nb<0>(nt, P, sims, rules, results, queue, ring, ctas, threads, smem, st);
        case 1: return launch_res_nb<1>(nt, P, sims, rules, results, queue, ring, ctas, threads, smem, st);
        case 2: return launch_res_nb<2>(nt, P, sims, rules, results, queue, ring, ctas, threads, smem, st);
        case 3: return launch_res_nb<3>(nt, P, sims, rules, results, queue, ring, ctas, threads, smem, st);
        case 4: return launch_res_nb<4>(nt, P, sims, rules, results, queue, ring, ctas, threads, smem, st);
        case 5: return launch_res_nb<5>(nt, P, sims, rules, results, queue, ring, ctas, threads, smem, st);
        case 6: return launch_res_nb<6>(nt, P, sims, rules, results, queue, ring, ctas, threads, smem, st);
        case 7: return launch_res_nb<7>(nt, P, sims, rules, results, queue, ring, ctas, threads, smem, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace cave
