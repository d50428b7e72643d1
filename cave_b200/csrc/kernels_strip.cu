// kernels_strip.cu -- layout conversion between the reference's nibble layout and the
// bit-plane ("strip") layout, and on-device seeding in either layout.
#include <cuda_runtime.h>

#include <algorithm>

#include "ca_core.cuh"
#include "cave_internal.h"
#include "kernels.h"

namespace cave {

// ------------------------------------------------------------------ layout conversion
__device__ __forceinline__ uint32_t gather_nibble_bit(uint32_t w, int b) {
    uint32_t e = (w >> b) & 0x11111111u;
    e = (e | (e >> 3)) & 0x03030303u;
    e = (e | (e >> 6)) & 0x000F000Fu;
    e = (e | (e >> 12)) & 0x000000FFu;
    return e;
}
__device__ __forceinline__ uint32_t scatter_nibble_bit(uint32_t e8) {
    uint32_t e = e8 & 0xFFu;
    e = (e | (e << 12)) & 0x000F000Fu;
    e = (e | (e << 6)) & 0x03030303u;
    e = (e | (e << 3)) & 0x11111111u;
    return e;
}

// One thread per strip: nibble words 4*sx .. 4*sx+3 of a row -> four bit-planes.
__global__ void k_nib_to_strips(const uint32_t* __restrict__ nib, uint4* __restrict__ strips, uint32_t X,
                                uint32_t Y, uint32_t Z) {
    const uint32_t W = (X + 7u) / 8u, SX = (X + 31u) / 32u;
    const uint64_t n = (uint64_t)SX * Y * Z;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t sx = (uint32_t)(i % SX);
        const uint64_t row = i / SX;
        const uint32_t* r = nib + row * W;
        uint32_t w[4];
#pragma unroll
        for (int k = 0; k < 4; k++) w[k] = (4u * sx + k < W) ? r[4u * sx + k] : 0u;
        const uint32_t valid = strip_valid(sx, X);
        uint32_t p[4];
#pragma unroll
        for (int b = 0; b < 4; b++) {
            p[b] = gather_nibble_bit(w[0], b) | (gather_nibble_bit(w[1], b) << 8) |
                   (gather_nibble_bit(w[2], b) << 16) | (gather_nibble_bit(w[3], b) << 24);
            p[b] &= valid;
        }
        strips[i] = make_uint4(p[0], p[1], p[2], p[3]);
    }
}

// One thread per nibble word: the inverse of k_nib_to_strips (padding nibbles come out 0).
__global__ void k_strips_to_nib(const uint4* __restrict__ strips, uint32_t* __restrict__ nib, uint32_t X,
                                uint32_t Y, uint32_t Z) {
    const uint32_t W = (X + 7u) / 8u, SX = (X + 31u) / 32u;
    const uint64_t n = (uint64_t)W * Y * Z;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t ux = (uint32_t)(i % W);
        const uint64_t row = i / W;
        const uint4 s = strips[row * SX + ux / 4u];
        const uint32_t sh = 8u * (ux & 3u);
        uint32_t w = scatter_nibble_bit(s.x >> sh) | (scatter_nibble_bit(s.y >> sh) << 1) |
                     (scatter_nibble_bit(s.z >> sh) << 2) | (scatter_nibble_bit(s.w >> sh) << 3);
        nib[i] = w;
    }
}

// ------------------------------------------------------------------ seeding
// searchSystem.cpp:244-259 (wangHash, cellHash).
__device__ __forceinline__ uint32_t wang_hash(uint32_t s) {
    s = (s ^ 61u) ^ (s >> 16);
    s *= 9u;
    s = s ^ (s >> 4);
    s *= 0x27d4eb2du;
    s = s ^ (s >> 15);
    return s;
}
__device__ __forceinline__ uint32_t cell_hash(uint32_t x, uint32_t y, uint32_t z, uint32_t seed) {
    uint32_t h = wang_hash(x * 73856093u + seed);
    h = wang_hash(h ^ (y * 19349663u));
    h = wang_hash(h ^ (z * 83492791u));
    return h;
}

// searchSystem.cpp:264-305 in the nibble layout; one thread per word. box = [lo, hi) per axis.
__global__ void k_seed_nib(uint32_t* __restrict__ nib, SeedSpec sp) {
    const uint32_t W = (sp.X + 7u) / 8u;
    const uint64_t n = (uint64_t)W * sp.Y * sp.Z;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t ux = (uint32_t)(i % W);
        const uint64_t r = i / W;
        const uint32_t y = (uint32_t)(r % sp.Y), z = (uint32_t)(r / sp.Y);
        uint32_t w = 0;
        const bool inyz = y >= sp.lo[1] && y < sp.hi[1] && z >= sp.lo[2] && z < sp.hi[2];
        if (inyz) {
#pragma unroll
            for (uint32_t k = 0; k < 8; k++) {
                const uint32_t x = ux * 8u + k;
                if (x >= sp.X || x < sp.lo[0] || x >= sp.hi[0]) continue;
                const bool alive = sp.fill_all || (uint64_t)cell_hash(x, y, z, sp.seed) < sp.threshold;
                if (alive) w |= (sp.maxcs & 0xFu) << (4u * k);
            }
        }
        nib[i] = w;
    }
}

// The same cells directly in the strip layout; one thread per strip.
__global__ void k_seed_strips(uint4* __restrict__ strips, SeedSpec sp) {
    const uint32_t SX = (sp.X + 31u) / 32u;
    const uint64_t n = (uint64_t)SX * sp.Y * sp.Z;
    const uint32_t v = sp.maxcs & 0xFu;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t sx = (uint32_t)(i % SX);
        const uint64_t r = i / SX;
        const uint32_t y = (uint32_t)(r % sp.Y), z = (uint32_t)(r / sp.Y);
        uint32_t bits = 0;
        if (y >= sp.lo[1] && y < sp.hi[1] && z >= sp.lo[2] && z < sp.hi[2]) {
            for (uint32_t j = 0; j < 32; j++) {
                const uint32_t x = sx * 32u + j;
                if (x >= sp.X || x < sp.lo[0] || x >= sp.hi[0]) continue;
                if (sp.fill_all || (uint64_t)cell_hash(x, y, z, sp.seed) < sp.threshold) bits |= 1u << j;
            }
        }
        strips[i] = make_uint4((v & 1u) ? bits : 0u, (v & 2u) ? bits : 0u, (v & 4u) ? bits : 0u,
                               (v & 8u) ? bits : 0u);
    }
}

cudaError_t launch_nib_to_strips(const uint32_t* nib, uint4* strips, uint32_t X, uint32_t Y, uint32_t Z,
                                 cudaStream_t st) {
    const uint64_t n = (uint64_t)((X + 31) / 32) * Y * Z;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    k_nib_to_strips<<<blocks ? blocks : 1, 256, 0, st>>>(nib, strips, X, Y, Z);
    return cudaGetLastError();
}

cudaError_t launch_strips_to_nib(const uint4* strips, uint32_t* nib, uint32_t X, uint32_t Y, uint32_t Z,
                                 cudaStream_t st) {
    const uint64_t n = (uint64_t)((X + 7) / 8) * Y * Z;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    k_strips_to_nib<<<blocks ? blocks : 1, 256, 0, st>>>(strips, nib, X, Y, Z);
    return cudaGetLastError();
}

cudaError_t launch_seed_nib(uint32_t* nib, const SeedSpec& sp, cudaStream_t st) {
    const uint64_t n = (uint64_t)((sp.X + 7) / 8) * sp.Y * sp.Z;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    k_seed_nib<<<blocks ? blocks : 1, 256, 0, st>>>(nib, sp);
    return cudaGetLastError();
}

cudaError_t launch_seed_strips(uint4* strips, const SeedSpec& sp, cudaStream_t st) {
    const uint64_t n = (uint64_t)((sp.X + 31) / 32) * sp.Y * sp.Z;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    k_seed_strips<<<blocks ? blocks : 1, 256, 0, st>>>(strips, sp);
    return cudaGetLastError();
}

}  // namespace cave
