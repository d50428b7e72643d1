// stream_common.cuh -- ring geometry, shared-memory layout and the per-tick fold of the
// streaming tick kernel (kernels_stream.cu).
#pragma once
#include "cave_stdint.h"

#include "cave_internal.h"
#include "ring.cuh"

namespace cave {

constexpr int kRing = 8;      // plane slots in flight per CTA (power of two)
constexpr int kRingLog2 = 3;
constexpr int kUnroll = 6;    // the march's unroll: a multiple of the row rotation (3) and of the exchange buffers (2)
static_assert((1 << kRingLog2) == kRing, "ring geometry");

template <int N>
__device__ __forceinline__ uint4 pack_planes(const uint32_t* p) {
    uint4 v = make_uint4(p[0], 0u, 0u, 0u);
    if constexpr (N > 1) v.y = p[1];
    if constexpr (N > 2) v.z = p[2];
    if constexpr (N > 3) v.w = p[3];
    return v;
}

constexpr int kXch = 2;       // y-exchange buffers (double-buffered)


// Shared-memory layout (dynamic): ring[kRing][rows*SX] uint4, xch[kXch][rows*SXp] uint4, mbarriers.
__host__ __device__ inline size_t stream_smem_bytes(uint32_t rows, uint32_t SX, uint32_t SXp) {
    return (size_t)kRing * rows * SX * 16 + (size_t)kXch * rows * SXp * 16 + kRing * 8 + 16;
}

// Folds one tick's totals (surviving, born, cells that were 0 before the tick, population
// and bounding box after it) into the simulation record: tick statistics, the search
// manager update (searchManager.slang:115-139), derived totals, and -- when the simulation
// is done and reports to a completion ring -- its result. Called by one thread.
__device__ __forceinline__ void fold_values(StripSim* sim, uint32_t surv, uint32_t born, uint32_t zero, uint32_t pop,
                                            const uint32_t* bmin, const uint32_t* bmax) {
    const uint32_t volume = sim->X * sim->Y * sim->Z;
    cave_tick_stats st;
    st.snapshot.numberOfDeadCells = zero - born;
    st.snapshot.numberOfCellsBorn = born;
    st.snapshot.numberOfSurvivingCells = surv;
    st.snapshot.numberOfDyingCells = volume - (zero - born) - born - surv;
    st.population = pop;
    st.changed = born + st.snapshot.numberOfDyingCells;
    for (int q = 0; q < 3; q++) {
        st.bbox_min[q] = bmin[q];
        st.bbox_max[q] = bmax[q];
    }
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
    const bool done = (sim->stop_on_status && info.status > 0) || t + 1 >= sim->tick_limit;
    if (done) sim->done = 1;
    __threadfence();
    if (done && sim->ring) {
        cave_sim_result r;
        r.info = info;
        r.category = result_category(info, sim->rule.maxcs);
        r.tag = 0;
        r.population = st.population;
        r.activeTicks = sim->pop_change_ticks;
        r.totalChanged = sim->total_changed;
        for (int q = 0; q < 3; q++) {
            r.bbox_min[q] = st.bbox_min[q];
            r.bbox_max[q] = st.bbox_max[q];
        }
        r.params = cave_sim_params{0, 0, 0};
        r.error = sim->error;
        r.pad = 0;
        ring_push(sim->ring, sim->slot, r);
    }
}

// Folds the accumulated statistics of one tick into the simulation record (last CTA).
__device__ inline void fold_tick(StripSim* sim) {
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

}  // namespace cave
