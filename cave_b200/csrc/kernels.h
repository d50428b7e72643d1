// kernels.h -- launch entry points of the CUDA kernels (host-callable, C++ linkage).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "cave_internal.h"

namespace cave {

// Spawn box and fill of searchSystem.cpp:219-306, resolved on the host.
struct SeedSpec {
    uint32_t X, Y, Z;
    uint32_t lo[3], hi[3];   // box [lo, hi) per axis
    uint64_t threshold;      // alive iff cellHash < threshold
    uint32_t fill_all;       // density >= 1 (or filled spawn): every box cell alive
    uint32_t seed;           // runSeedIndex
    uint32_t maxcs;          // written as (maxcs & 0xF)
};

cudaError_t launch_plain_step(const uint32_t* in, uint32_t* out, uint32_t X, uint32_t Y, uint32_t Z,
                              PlainSlot* slot, const uint64_t* valid, uint32_t nValid, uint32_t maxRuleBits,
                              cudaStream_t stream);
cudaError_t launch_nib_to_strips(const uint32_t* nib, uint4* strips, uint32_t X, uint32_t Y, uint32_t Z,
                                 cudaStream_t st);
cudaError_t launch_strips_to_nib(const uint4* strips, uint32_t* nib, uint32_t X, uint32_t Y, uint32_t Z,
                                 cudaStream_t st);
cudaError_t launch_seed_nib(uint32_t* nib, const SeedSpec& sp, cudaStream_t st);
cudaError_t launch_seed_strips(uint4* strips, const SeedSpec& sp, cudaStream_t st);
// ---- resident batched kernel
struct ResLaunch {           // geometry shared by every simulation of one launch
    uint32_t X, Y, Z, SX;
    uint32_t sxp_log2;       // lanes per row = 1 << sxp_log2 >= SX
    uint32_t nseg, seg_len;  // z-segments per CTA and planes per segment
    uint32_t n_sims;
    uint32_t wait_us;        // limit of the wait for an initial grid's copy (0 = kWaitLimitNs)
    uint32_t hold_init;      // failure test: the initial-grid copy is never issued, so the wait
                             // runs out (only for launches of exactly one simulation)
};
struct ResSim {              // one simulation of a resident launch (24 bytes)
    const uint4* init;       // initial grid (strip layout, device memory, 16-byte aligned)
    uint32_t rule;           // index into the DeviceRule table
    uint32_t max_ticks;
    uint32_t result;         // index into the result array, or the slot reported to the ring
    uint32_t pad;
};
size_t resident_smem_bytes(uint32_t X, uint32_t Y, uint32_t Z, uint32_t nseg);
// nt: sparse term count of every rule in the launch (0 = mux tree), nb: neighbourhood bits.
// ring: when set, each finished simulation is pushed to it (slot = ResSim::result) instead of
// being written to results.
cudaError_t launch_resident(int nb, int nt, const ResLaunch& P, const ResSim* sims, const DeviceRule* rules,
                            cave_sim_result* results, uint32_t* queue, DoneRing* ring, uint32_t ctas,
                            uint32_t threads, cudaStream_t st);

// ---- engine set-up
// One initial grid to place at byte offset `dst` of the engine's cell pool: a copy of `src`
// (strip layout, n_strips strips) when src is set, else seeded by `seed`.
struct EngineJob {
    const uint4* src;
    uint64_t dst;
    uint64_t n_strips;
    SeedSpec seed;
};
// Installs n_recs staged records at recs[rec_slots[i]] and runs every job, in one launch.
cudaError_t launch_engine_setup(const EngineJob* jobs, uint32_t n_jobs, uint64_t max_strips, uint4* pool,
                                const StripSim* recs_in, const uint32_t* rec_slots, uint32_t n_recs, StripSim* recs,
                                cudaStream_t st);

// ---- render-mode layout (kernels_render.cu)
struct RenderGeom {
    uint32_t X, Y, Z, pad;        // cells; ghost shell thickness of the strip grid (wrap: 1)
    uint32_t Xp, Yp, Zp, SX;      // padded strip grid
    uint32_t W;                   // texels per row
    uint64_t elements;            // render buffer elements (8x8x8 texel blocks)
    uint32_t sdx, sdy, sdz;       // skip grid chunks per axis (8 cells)
    uint64_t skip_elements;
};
RenderGeom render_geometry(uint32_t X, uint32_t Y, uint32_t Z, uint32_t pad);
cudaError_t launch_render_to_strips(const uint32_t* render, uint4* strips, const RenderGeom& g, cudaStream_t st);
cudaError_t launch_strips_to_render(const uint4* strips, uint32_t* render, const RenderGeom& g, cudaStream_t st);
cudaError_t launch_ghost_fill(uint4* strips, const RenderGeom& g, cudaStream_t st);
cudaError_t launch_render_skip(const uint4* strips, uint32_t* skip, const RenderGeom& g, cudaStream_t st);

// threads = rows * SXp (rows includes the two halo rows), SXp = power of two >= SX, <= 32.
// nt: sparse term count of the rule (0 = mux tree). param_rule: the rule of every item's
// simulation when the launch holds one simulation only (passed as a kernel parameter), else null.
// Launches use programmatic dependent launch, so consecutive ticks overlap set-up and drain.
// pdl = false launches without the programmatic-dependent-launch attribute (the first tick
// after a cross-stream event wait).
// tick_arg >= 0: a deferred-fold run (the one simulation's record has `deferred` set); the
// launch is tick tick_arg and only adds its totals to deferred[tick_arg].
cudaError_t launch_stream_tick(int nb, int nt, const DeviceRule* param_rule, const StreamItem* items,
                               uint32_t n_items, StripSim* sims, uint4* pool, uint32_t SX, uint32_t SXp,
                               uint32_t threads, cudaStream_t st, bool pdl = true, int tick_arg = -1);
// Population and bounding box of a strip grid (SX strips per row), added to `slot`.
cudaError_t launch_strip_stats(const uint4* strips, uint32_t Y, uint32_t Z, uint32_t SX, TickTotals* slot,
                               uint32_t sm_count, cudaStream_t st);
// After the last tick of a deferred-fold run: per-tick statistics and the record's GridInfo.
// derive_zero: ticks after the first did not count their zero cells (volume - previous population).
cudaError_t launch_fold_deferred(StripSim* sim, const TickTotals* tt, uint32_t nticks, bool derive_zero,
                                 cudaStream_t st);

}  // namespace cave
