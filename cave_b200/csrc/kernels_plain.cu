// kernels_plain.cu -- the plain drop-in step: one launch per simulation per tick, on the
// reference's padded nibble layout, with the GridSnapshot reduction and the search
// manager fused into the epilogue of the last CTA to finish.
//
// Replaces searchSimulationCube.slang computeMain (:117-248) + searchManager.slang
// computeMain (:98-149) for one slot. One thread owns one packed word (8 cells along x),
// as in the reference, but each of the 27 neighbouring words is loaded once per word
// rather than once per cell, and neighbour counts are formed for all 8 cells at once
// with nibble-parallel (SWAR) adds in byte lanes.
#include <cuda_runtime.h>

#include "cave_internal.h"
#include "ptx.cuh"

namespace cave {

// Nibble n of the result is 1 (at bit 4n) iff nibble n of w equals m (m in 0..15).
__device__ __forceinline__ uint32_t nib_eq(uint32_t w, uint32_t m) {
    const uint32_t t = w ^ (m * 0x11111111u);
    const uint32_t nz = ((t & 0x77777777u) + 0x77777777u) | t;  // bit 4n+3 set iff nibble n != 0
    return (~nz & 0x88888888u) >> 3;
}

struct PlainArgs {
    const uint32_t* in;
    uint32_t* out;
    uint32_t X, Y, Z, W;          // W = words per row
    PlainSlot* slot;
    const uint64_t* valid;        // K-index table
    uint32_t nValid, maxRuleBits;
};

__global__ void __launch_bounds__(256) k_plain_step(PlainArgs A) {
    const uint64_t nwords = (uint64_t)A.W * A.Y * A.Z;
    const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    PlainSlot* slot = A.slot;

    // ---- decode the rule (slang:139-157)
    const cave_sim_params P = slot->perms;
    const uint32_t maxCS = (uint32_t)(P.birthAndMaxCellStateRules >> 60) + 1u;
    const uint32_t flags = (uint32_t)(P.survivalAndNeighborhoodRules >> 60);
    uint64_t B, S;
    bool bad = false, skip = false;
    if (A.maxRuleBits > 0) {
        // An exhausted slot (NULL permutation) is still dispatched for one tick after its last
        // rule, as in searchSystem.cpp:541-564; its K-indices are meaningless and the manager
        // ignores its snapshot (searchManager.slang:104-110), so nothing is computed.
        skip = P.birthAndMaxCellStateRules == 0 || P.survivalAndNeighborhoodRules == 0;
        const uint32_t bi = (uint32_t)(P.birthAndMaxCellStateRules & kPermMask) - 1u;
        const uint32_t si = (uint32_t)(P.survivalAndNeighborhoodRules & kPermMask) - 1u;
        bad = !skip && (bi >= A.nValid || si >= A.nValid);
        B = (bad || skip) ? 0 : A.valid[bi];
        S = (bad || skip) ? 0 : A.valid[si];
    } else {
        B = P.birthAndMaxCellStateRules & kPermMask;
        S = P.survivalAndNeighborhoodRules & kPermMask;
    }
    const bool fF = flags & 1u, fE = flags & 2u, fC = flags & 4u;

    uint32_t died = 0, dying = 0, born = 0, surv = 0, pop = 0;
    uint32_t bmin[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, bmax[3] = {0, 0, 0};

    if (idx < nwords && !bad && !skip) {
        const uint32_t ux = (uint32_t)(idx % A.W);
        const uint64_t r = idx / A.W;
        const uint32_t y = (uint32_t)(r % A.Y);
        const uint32_t z = (uint32_t)(r / A.Y);
        const uint32_t m = maxCS & 0xFu;
        const bool can_live = maxCS <= 15u;
        const uint32_t nvalid = min(8u, A.X - ux * 8u);
        const uint32_t vmask = nvalid >= 8u ? 0x11111111u : (0x11111111u & ((1u << (4u * nvalid)) - 1u));
        // Byte-lane neighbour counts: even nibbles in ce, odd nibbles in co.
        uint32_t ce = 0, co = 0;
#pragma unroll
        for (int dz = -1; dz <= 1; dz++) {
#pragma unroll
            for (int dy = -1; dy <= 1; dy++) {
                const int yy = (int)y + dy, zz = (int)z + dz;
                const int cls = (dy != 0) + (dz != 0);  // 0 centre row, 1 face row, 2 diagonal row
                // contribution of this row: which of {same x, x+-1} count
                const bool same = (cls == 1 && fF) || (cls == 2 && fE);
                const bool side = (cls == 0 && fF) || (cls == 1 && fE) || (cls == 2 && fC);
                if (!same && !side) continue;
                if (yy < 0 || yy >= (int)A.Y || zz < 0 || zz >= (int)A.Z || !can_live) continue;
                const uint32_t* row = A.in + ((uint64_t)zz * A.Y + (uint32_t)yy) * A.W;
                const uint32_t wc = row[ux];
                const uint32_t wl = ux > 0 ? row[ux - 1] : 0u;
                const uint32_t wr = ux + 1 < A.W ? row[ux + 1] : 0u;
                // Padding nibbles of the row's last word never count (slang:80-81 bounds
                // check); the neighbouring words' edge nibbles are always real cells.
                const uint32_t ac = nib_eq(wc, m) & vmask;
                const uint32_t al = ux > 0 ? nib_eq(wl, m) : 0u;
                const uint32_t ar = ux + 1 < A.W ? nib_eq(wr, m) : 0u;
                uint32_t c = 0;
                if (same) c += ac;
                if (side) c += ((ac << 4) | (al >> 28)) + ((ac >> 4) | (ar << 28));
                ce += c & 0x0F0F0F0Fu;
                co += (c >> 4) & 0x0F0F0F0Fu;
            }
        }
        const uint32_t inw = A.in[idx];
        uint32_t outw = 0;
#pragma unroll
        for (uint32_t nib = 0; nib < 8; nib++) {
            const uint32_t cx = ux * 8u + nib;
            if (cx >= A.X) break;
            const uint32_t cur = (inw >> (nib * 4u)) & 0xFu;
            const uint32_t n = (((nib & 1u) ? co : ce) >> (8u * (nib >> 1))) & 0xFFu;
            uint32_t ns;
            if (cur == maxCS) {
                if (n > 0 && ((S >> (n - 1)) & 1u)) { ns = maxCS; surv++; }
                else { ns = cur - 1u; dying++; }
            } else if (cur == 0u) {
                if (n > 0 && ((B >> (n - 1)) & 1u)) { ns = maxCS; born++; }
                else { ns = 0u; died++; }
            } else {
                ns = cur - 1u;
                dying++;
            }
            ns &= 0xFu;
            outw |= ns << (nib * 4u);
            if (ns) {
                pop++;
                bmin[0] = min(bmin[0], cx); bmax[0] = max(bmax[0], cx);
                bmin[1] = min(bmin[1], y);  bmax[1] = max(bmax[1], y);
                bmin[2] = min(bmin[2], z);  bmax[2] = max(bmax[2], z);
            }
        }
        A.out[idx] = outw;
    }

    // ---- block reduction of the counters (slang:219-247 does wave sums + atomics)
    __shared__ uint32_t red[8][11];
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t v[11] = {died, dying, born, surv, pop, bmin[0], bmin[1], bmin[2], bmax[0], bmax[1], bmax[2]};
#pragma unroll
    for (int k = 0; k < 5; k++) v[k] = warp_add(v[k]);
#pragma unroll
    for (int k = 5; k < 8; k++) v[k] = warp_min(v[k]);
#pragma unroll
    for (int k = 8; k < 11; k++) v[k] = warp_max(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 11; k++) red[warp][k] = v[k];
    }
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        const unsigned nw = blockDim.x >> 5;
        for (unsigned w = 1; w < nw; w++) {
            for (int k = 0; k < 5; k++) red[0][k] += red[w][k];
            for (int k = 5; k < 8; k++) red[0][k] = min(red[0][k], red[w][k]);
            for (int k = 8; k < 11; k++) red[0][k] = max(red[0][k], red[w][k]);
        }
        if (red[0][0]) atomicAdd(&slot->acc[0], red[0][0]);
        if (red[0][1]) atomicAdd(&slot->acc[1], red[0][1]);
        if (red[0][2]) atomicAdd(&slot->acc[2], red[0][2]);
        if (red[0][3]) atomicAdd(&slot->acc[3], red[0][3]);
        if (red[0][4]) atomicAdd(&slot->population, red[0][4]);
        if (red[0][4]) {
            for (int k = 0; k < 3; k++) {
                atomicMin(&slot->bmin[k], red[0][5 + k]);
                atomicMax(&slot->bmax[k], red[0][8 + k]);
            }
        }
        if (bad && blockIdx.x == 0) atomicOr(&slot->error, kErrBadRuleIndex);
        __threadfence();
        const uint32_t t = atomicAdd(&slot->ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;

    // ---- last CTA: fold the tick and run the manager (searchManager.slang:98-149)
    __threadfence();
    volatile PlainSlot* vs = slot;
    cave_tick_stats st;
    st.snapshot.numberOfDeadCells = vs->acc[0];
    st.snapshot.numberOfDyingCells = vs->acc[1];
    st.snapshot.numberOfCellsBorn = vs->acc[2];
    st.snapshot.numberOfSurvivingCells = vs->acc[3];
    st.population = vs->population;
    st.changed = st.snapshot.numberOfCellsBorn + st.snapshot.numberOfDyingCells;
    for (int k = 0; k < 3; k++) {
        st.bbox_min[k] = vs->bmin[k];
        st.bbox_max[k] = vs->bmax[k];
    }
    slot->acc[0] = slot->acc[1] = slot->acc[2] = slot->acc[3] = 0;
    slot->population = 0;
    for (int k = 0; k < 3; k++) {
        slot->bmin[k] = 0xFFFFFFFFu;
        slot->bmax[k] = 0;
    }
    slot->ticket = 0;
    slot->last = st;
    if (slot->per_tick) slot->per_tick[slot->tick_count] = st;
    slot->tick_count++;
    if (slot->run_manager) {
        cave_grid_info info = slot->info, ic;
        cave_sim_params perms = slot->perms, pc;
        manager_update(st.snapshot, info, perms, slot->maxPermutation, slot->survivalEnd, slot->maxTicks, ic, pc);
        slot->info = info;
        slot->perms = perms;
        slot->infoCopy = ic;
        slot->permsCopy = pc;
    }
    __threadfence();
}

cudaError_t launch_plain_step(const uint32_t* in, uint32_t* out, uint32_t X, uint32_t Y, uint32_t Z,
                              PlainSlot* slot, const uint64_t* valid, uint32_t nValid, uint32_t maxRuleBits,
                              cudaStream_t stream) {
    PlainArgs a;
    a.in = in;
    a.out = out;
    a.X = X;
    a.Y = Y;
    a.Z = Z;
    a.W = (X + 7u) / 8u;
    a.slot = slot;
    a.valid = valid;
    a.nValid = nValid;
    a.maxRuleBits = maxRuleBits;
    const uint64_t nwords = (uint64_t)a.W * Y * Z;
    const uint32_t blocks = (uint32_t)((nwords + 255) / 256);
    k_plain_step<<<blocks ? blocks : 1, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace cave
