// ring.cuh -- device side of the completion ring (DoneRing, cave_internal.h).
#pragma once
#include "cave_internal.h"

namespace cave {

// Category of a finished rule (searchSystem.cpp:697-711): 0 viable (status 2), 1 possible
// (survived more than maxCellState + 1 ticks), 2 unviable.
__device__ __forceinline__ uint32_t result_category(const cave_grid_info& info, uint32_t maxcs) {
    return info.status == 2 ? 0u
                            : ((uint64_t)info.numberOfSimulationTicksSurvived > (uint64_t)maxcs + 1 ? 1u : 2u);
}

// Appends one finished simulation to the ring. Called by one thread.
__device__ __forceinline__ void ring_push(DoneRing* ring, uint32_t slot, const cave_sim_result& r) {
    const uint32_t idx = atomicAdd(&ring->count, 1u);
    DoneEntry* e = ring->entries + (idx % ring->cap);
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&r);
    volatile uint32_t* dst = reinterpret_cast<volatile uint32_t*>(&e->result);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(cave_sim_result) / 4); i++) dst[i] = src[i];
    reinterpret_cast<volatile uint32_t*>(&e->slot)[0] = slot;
    __threadfence_system();  // the payload reaches host memory before seq
    reinterpret_cast<volatile uint32_t*>(&e->seq)[0] = idx + 1u;
}

}  // namespace cave
