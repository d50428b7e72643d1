// kernels_engine.cu -- set-up kernels of the engine (engine.cpp): one launch seeds, copies or
// installs the records of every simulation admitted in a round, instead of one launch or one
// copy per simulation.
#include <cuda_runtime.h>

#include <algorithm>

#include "cave_internal.h"
#include "kernels.h"

namespace cave {

__device__ __forceinline__ uint32_t wang_hash_e(uint32_t s) {  // searchSystem.cpp:244-252
    s = (s ^ 61u) ^ (s >> 16);
    s *= 9u;
    s = s ^ (s >> 4);
    s *= 0x27d4eb2du;
    s = s ^ (s >> 15);
    return s;
}
__device__ __forceinline__ uint32_t cell_hash_e(uint32_t x, uint32_t y, uint32_t z, uint32_t seed) {
    uint32_t h = wang_hash_e(x * 73856093u + seed);  // searchSystem.cpp:253-259
    h = wang_hash_e(h ^ (y * 19349663u));
    h = wang_hash_e(h ^ (z * 83492791u));
    return h;
}

// blockIdx.y strides over the jobs; each job's strips are spread over gridDim.x blocks.
// Seeds the strip layout exactly as k_seed_strips does for one grid.
__global__ void k_engine_setup(const EngineJob* __restrict__ jobs, uint32_t n_jobs, uint4* __restrict__ pool,
                               const StripSim* __restrict__ recs_in, const uint32_t* __restrict__ rec_slots,
                               uint32_t n_recs, StripSim* __restrict__ recs) {
    // records first: block (x, 0) copies its share of the staged records
    if (blockIdx.y == 0) {
        const uint32_t words = sizeof(StripSim) / 8;
        const uint64_t total = (uint64_t)n_recs * words;
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
             i += (uint64_t)gridDim.x * blockDim.x) {
            const uint32_t r = (uint32_t)(i / words), w = (uint32_t)(i % words);
            reinterpret_cast<uint64_t*>(recs + rec_slots[r])[w] = reinterpret_cast<const uint64_t*>(recs_in + r)[w];
        }
    }
    for (uint32_t j = blockIdx.y; j < n_jobs; j += gridDim.y) {
        const EngineJob jb = jobs[j];
        uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(pool) + jb.dst);
        if (jb.src) {  // copy an initial grid (strip layout)
            for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < jb.n_strips;
                 i += (uint64_t)gridDim.x * blockDim.x)
                dst[i] = jb.src[i];
            continue;
        }
        const SeedSpec& sp = jb.seed;
        const uint32_t SX = (sp.X + 31u) / 32u;
        const uint32_t v = sp.maxcs & 0xFu;
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < jb.n_strips;
             i += (uint64_t)gridDim.x * blockDim.x) {
            const uint32_t sx = (uint32_t)(i % SX);
            const uint64_t r = i / SX;
            const uint32_t y = (uint32_t)(r % sp.Y), z = (uint32_t)(r / sp.Y);
            uint32_t bits = 0;
            if (y >= sp.lo[1] && y < sp.hi[1] && z >= sp.lo[2] && z < sp.hi[2]) {
                for (uint32_t b = 0; b < 32; b++) {
                    const uint32_t x = sx * 32u + b;
                    if (x >= sp.X || x < sp.lo[0] || x >= sp.hi[0]) continue;
                    if (sp.fill_all || (uint64_t)cell_hash_e(x, y, z, sp.seed) < sp.threshold) bits |= 1u << b;
                }
            }
            dst[i] = make_uint4((v & 1u) ? bits : 0u, (v & 2u) ? bits : 0u, (v & 4u) ? bits : 0u,
                                (v & 8u) ? bits : 0u);
        }
    }
}

cudaError_t launch_engine_setup(const EngineJob* jobs, uint32_t n_jobs, uint64_t max_strips, uint4* pool,
                                const StripSim* recs_in, const uint32_t* rec_slots, uint32_t n_recs, StripSim* recs,
                                cudaStream_t st) {
    if (n_jobs == 0 && n_recs == 0) return cudaSuccess;
    const uint32_t gy = std::max<uint32_t>(1u, std::min<uint32_t>(n_jobs, 65535u));
    // blocks per job: about 2,048 strips per block for the largest job, at least enough
    // blocks for the records when there are no jobs
    uint32_t gx = (uint32_t)std::min<uint64_t>(std::max<uint64_t>((max_strips + 2047) / 2048, 1), 512);
    if (n_jobs == 0) gx = std::max<uint32_t>(1u, std::min<uint32_t>((n_recs + 7) / 8, 148u));
    k_engine_setup<<<dim3(gx, gy), 256, 0, st>>>(jobs, n_jobs, pool, recs_in, rec_slots, n_recs, recs);
    return cudaGetLastError();
}

}  // namespace cave
