// cave_internal.h -- device-side records shared by the kernels and the host library.
#pragma once
#include "cave_stdint.h"

#include "../../include/cave_ca.h"
#include "ca_types.h"
#ifndef __CUDACC_RTC__
#include <vector_types.h>
#endif

namespace cave {

constexpr uint64_t kPermMask = (uint64_t(1) << 60) - 1;  // simulation.h:43

// Bounded device-side waits give up after this many nanoseconds and raise an error flag.
constexpr uint64_t kWaitLimitNs = 1000000000ull;

// Error flags a kernel may raise in its record (read back by the host).
enum : uint32_t { kErrNone = 0, kErrWaitTimeout = 1, kErrBadRuleIndex = 2, kErrCancelled = 4, kErrBounds = 8 };

// Index checks of the checked build (compiled with -DCAVE_CHECKED, libcave_ca_checked.so): the
// hot kernels test every shared- and global-memory index against the extent it must stay in.
// CAVE_IN_BOUNDS(i, n, err) is true when i < n; otherwise it raises kErrBounds in err (which
// reaches the simulation record like any other error flag) and is false, and the caller skips
// the access: a failed check neither faults nor traps. In the normal build it is the constant
// true and its arguments are never evaluated.
#ifdef CAVE_CHECKED
#define CAVE_IN_BOUNDS(i, n, err) (((uint64_t)(i) < (uint64_t)(n)) ? true : (((err) |= cave::kErrBounds), false))
#else
#define CAVE_IN_BOUNDS(i, n, err) true
#endif

// Per-grid device record of the plain path. It holds what the reference keeps in the
// per-slot permutation / snapshot / GridInfo / copy buffers (searchSystem.cpp:202-374).
struct PlainSlot {
    cave_sim_params perms;        // gridPermutationsBuffer (live; the manager advances it)
    uint32_t run_manager;         // 1: apply searchManager semantics after each tick
    uint32_t error;               // kErr* flags
    // tick accumulators (zeroed again by the last CTA of each tick)
    uint32_t acc[4];              // dead, dying, born, surviving (GridSnapshot order)
    uint32_t population;
    uint32_t bmin[3], bmax[3];
    uint32_t ticket;
    cave_grid_info info;          // gridInfoBuffer
    cave_grid_info infoCopy;      // gridInfoCopyBuffer
    cave_sim_params permsCopy;    // gridPermutationsCopyBuffer
    uint64_t maxPermutation;      // gridMaxPermutationBuffer
    uint64_t survivalEnd;         // gridSurvivalEndPermutationBuffer
    uint32_t maxTicks;            // MAX_NUMBER_OF_TICKS_TO_SURVIVE
    uint32_t tick_count;          // ticks folded since the slot was reset
    cave_tick_stats last;         // statistics of the most recent tick
    cave_tick_stats* per_tick;    // optional device array indexed by tick_count
};

// Host+device restatement of searchManager.slang:56-149 on plain structs.
CAVE_HD inline void manager_update(const cave_grid_snapshot& snap, cave_grid_info& info,
                                               cave_sim_params& perms, uint64_t maxPermutation,
                                               uint64_t survivalEnd, uint32_t maxTicks, cave_grid_info& infoCopy,
                                               cave_sim_params& permsCopy) {
    cave_sim_params p = perms;
    if (p.survivalAndNeighborhoodRules == 0 || p.birthAndMaxCellStateRules == 0) {
        infoCopy = info;
        permsCopy = p;
        return;
    }
    info.numberOfSimulationTicksSurvived++;
    info.totalNumberOfCellsThatDied += snap.numberOfDeadCells;
    info.totalNumberOfCellsThatWereBorn += snap.numberOfCellsBorn;
    info.finalAliveCount = snap.numberOfSurvivingCells;
    if (snap.numberOfSurvivingCells > info.maxAliveCount) info.maxAliveCount = snap.numberOfSurvivingCells;
    if (snap.numberOfSurvivingCells == 0u && snap.numberOfCellsBorn == 0u)
        info.status = 1;
    else if (info.numberOfSimulationTicksSurvived >= maxTicks)
        info.status = 2;
    else
        info.status = 0;
    infoCopy = info;
    permsCopy = p;
    if (info.status > 0) {
        // NextPermutation (searchManager.slang:56-96)
        if ((p.birthAndMaxCellStateRules & kPermMask) < maxPermutation) {
            p.birthAndMaxCellStateRules++;
        } else if ((p.survivalAndNeighborhoodRules & kPermMask) < survivalEnd) {
            p.survivalAndNeighborhoodRules++;
            p.birthAndMaxCellStateRules = (p.birthAndMaxCellStateRules & ~kPermMask) + 1;
        } else {
            p.survivalAndNeighborhoodRules = 0;
            p.birthAndMaxCellStateRules = 0;
            perms = p;
            return;
        }
        perms = p;
        info = cave_grid_info{0, 0, 0, 0, 0, 0};
    }
}

// ---- completion ring -------------------------------------------------------------------
// Finished simulations of the engine (batched and served runs) are reported through a ring
// whose entries live in host-mapped pinned memory: the device writes the result, fences at
// system scope and then writes `seq`; the host reads entries in order, an entry being ready
// once its seq equals its index + 1. Indices come from `count` (device memory). The engine
// never has more simulations in flight than the ring has entries, so no entry is overwritten
// before the host has read it.
struct DoneEntry {
    cave_sim_result result;
    uint32_t slot;             // engine slot of the simulation
    uint32_t seq;              // index + 1, written last
};
static_assert(sizeof(DoneEntry) == 112, "DoneEntry layout");
struct DoneRing {
    uint32_t count;            // next entry index (device memory, atomic)
    uint32_t cap;
    DoneEntry* entries;        // device alias of the host-mapped entry array
};

// One tick's totals of a raw-stepping run whose fold is deferred to the end of the run. The
// minimum of the bounding box is kept inverted (~min, combined with atomicMax) so that an
// all-zero slot is the empty state.
struct TickTotals {
    uint32_t surv, born, zero, pop;
    uint32_t nbmin[3], bmax[3];
    uint32_t pad[2];
};
static_assert(sizeof(TickTotals) == 48, "TickTotals layout");
// The tick kernel adds its four sums to surv + 0..3 (and acc_surv + 0..3 of StripSim).
// (Checked by nvcc and the host compiler; NVRTC has no offsetof.)
#ifndef __CUDACC_RTC__
static_assert(__builtin_offsetof(TickTotals, pop) == __builtin_offsetof(TickTotals, surv) + 12, "TickTotals sums");
#endif

// ---- bit-plane (strip) path -----------------------------------------------------------
// One CTA's share of one tick of one simulation in the streaming kernel.
struct StreamItem {
    uint32_t sim;            // index into the StripSim array
    uint16_t y0, ty;         // output rows [y0, y0 + ty)
    uint16_t z0, z1;         // output planes [z0, z1)
    uint32_t dir_items;      // bit 0: march towards +z (0) or -z (1); bits 1..31: the number of
                             // work items of `sim` in this launch (the last one to finish folds)
};

// Per-simulation device record of the strip kernels.
struct StripSim {
    DeviceRule rule;
    uint32_t X, Y, Z, SX;       // SX = strips per row
    uint64_t buf[2];            // byte offsets (into the strip pool) of the two cell copies
    uint32_t max_ticks;         // MAX_NUMBER_OF_TICKS_TO_SURVIVE
    uint32_t tick_limit;        // ticks to run in total (raw stepping) or max_ticks (search)
    uint32_t stop_on_status;    // 1: stop when the manager reports status > 0
    uint32_t n_items;           // work items per tick when the record was written (the kernel
                                // takes the count from each item, so launches may re-tile)
    uint32_t tick;              // ticks completed
    uint32_t done;              // no further ticks run
    uint32_t error;
    uint32_t ticket;
    cave_grid_info info;        // manager state (searchManager.slang GridInfo semantics)
    // per-tick accumulators
    uint32_t acc_surv, acc_born, acc_zero, acc_pop;
    uint32_t acc_bmin[3], acc_bmax[3];
    // derived totals
    uint32_t prev_pop;
    uint32_t pop_change_ticks;
    uint64_t total_changed;
    cave_tick_stats last;
    cave_tick_stats* per_tick;  // optional, tick_limit entries
    DoneRing* ring;             // optional: the final result is pushed here when done
    uint32_t slot;              // engine slot reported with the result
    uint32_t pad;
    TickTotals* deferred;       // raw stepping: per-tick totals, folded after the run (the
                                // tick launches then take their tick index as an argument)
};
#ifndef __CUDACC_RTC__
static_assert(__builtin_offsetof(StripSim, acc_pop) == __builtin_offsetof(StripSim, acc_surv) + 12, "StripSim sums");
#endif

}  // namespace cave
