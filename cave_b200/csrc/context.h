// context.h -- host-side objects behind the opaque handles of cave_ca.h.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "cave_internal.h"
#include "kernels.h"

namespace cave {
// How one simulation class is executed (chosen by the autotuner or by defaults).
struct ExecChoice {
    uint32_t resident = 0;   // 1: resident kernel, 0: tiled
    uint32_t nseg = 0;       // resident: z-segments per CTA (0 = default geometry)
    uint32_t rows = 0;       // tiled: rows per CTA incl. the two halo rows (0 = default)
    uint32_t cells = 0;      // tiled: log2 of the target cells per CTA (0 = default)
    bool operator==(const ExecChoice& o) const {
        return resident == o.resident && nseg == o.nseg && rows == o.rows && cells == o.cells;
    }
};
// cave_run's choice for a grid shape: tick kernel kind (cave_ca.cpp RunKind) and rows per CTA.
struct RunChoice {
    uint32_t kind = 0, rows = 0;
};
// Tuning-cache key: grid shape and neighbourhood bits.
struct TuneKey {
    uint32_t X, Y, Z, nb;
    bool operator<(const TuneKey& o) const {
        if (X != o.X) return X < o.X;
        if (Y != o.Y) return Y < o.Y;
        if (Z != o.Z) return Z < o.Z;
        return nb < o.nb;
    }
};
// Pinned host staging plus its device mirror, two of each (the engine's upload buffers).
struct StagingPair {
    unsigned char* h[2];
    unsigned char* d[2];
    uint64_t cap;
};
}  // namespace cave

struct cave_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sm_count = 148;
    int smem_optin = 227 * 1024;  // largest shared memory one CTA may opt in to
    uint32_t last_run_kind = 0;   // tick kernels of the last cave_run (0 generic, 1 specialised, 2 two-tick)
    std::atomic<bool> search_stop{false};  // set by cave_search_stop (any thread), read between waves
    std::string last_error;
    std::mutex mu;  // guards last_error
    bool timing = false;
    cudaEvent_t ev[6] = {};  // created when timing is enabled
    cave_timing last_timing = {};
    // autotuner results, shared by every batch and server of the context
    std::mutex tune_mu;
    std::map<cave::TuneKey, cave::ExecChoice> tune_cache;
    // cave_run's tick kernel kind and tile (rows per CTA) per grid shape and the kernels available
    // (key nb: neighbourhood bits + 8 x the default kind), found by a short timing pass (cave_ca.cpp)
    std::map<cave::TuneKey, cave::RunChoice> run_rows;
    // engine staging buffers released by finished engines, reused by the next (freed with the context)
    std::mutex staging_mu;
    std::vector<cave::StagingPair> staging_free;
};

struct cave_grid {
    cave_ctx* ctx = nullptr;
    uint32_t X = 0, Y = 0, Z = 0;
    uint64_t words = 0;
    uint32_t* nib[2] = {nullptr, nullptr};  // ping-pong nibble copies
    int cur = 0;                             // index of the current copy
    cave::PlainSlot* slot = nullptr;         // plain-path record
    // strip path (allocated on first cave_run)
    uint4* strips = nullptr;                 // 2 copies back to back
    uint64_t strip_count = 0;                // strips per copy
    cave::StripSim* sim = nullptr;
};

namespace cave {

// Records `msg` as the context's last error and returns `code`.
cave_status set_error(cave_ctx* ctx, cave_status code, const std::string& msg);
// Checks a CUDA call; on failure records the error text.
cave_status check_cuda(cave_ctx* ctx, cudaError_t e, const char* what);

#define CAVE_CUDA(ctx, call)                                         \
    do {                                                             \
        cudaError_t _e = (call);                                     \
        if (_e != cudaSuccess) return ::cave::check_cuda(ctx, _e, #call); \
    } while (0)

// Tiling of one simulation for the streaming tick kernel.
struct StreamPlan {
    uint32_t SX, SXp, threads, rows;
    uint32_t ny, nz;       // y-tiles and z-slabs
    std::vector<StreamItem> items;
};
// Builds the work items of simulation `sim_index` with grid X*Y*Z; `target_ctas` is the
// number of CTAs one tick should spread over (a multiple of the SM count); rows_hint = rows
// per CTA including the two halo rows (0 = default); spt = rows per thread (1, or 2 for the
// rule-specialised kernels): threads = rows * SXp / spt, a whole number of warps. halo: halo rows
// on each side of a tile (1, or 2 for the two-tick kernels; rows_hint includes them), at most
// max_threads threads (0 = the kernel's own limit).
bool plan_stream(uint32_t sim_index, uint32_t X, uint32_t Y, uint32_t Z, uint32_t target_ctas,
                 uint32_t rows_hint, StreamPlan& plan, uint32_t spt = 1, uint32_t halo = 1,
                 uint32_t max_threads = 0);

SeedSpec make_seed_spec(uint32_t X, uint32_t Y, uint32_t Z, uint32_t sx, uint32_t sy, uint32_t sz,
                        uint32_t spawnSizeIndex, uint64_t threshold, bool fill_all, uint32_t seed,
                        uint32_t maxcs);

}  // namespace cave
