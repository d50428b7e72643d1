// kernels_render.cu -- the render mode's cell buffers on the strip kernels.
//
// Render mode keeps cells in a different layout (cellStateUtils.slang:18-54): two cells per
// texel along x (low nibble = even x), one texel per uint32 element, texels grouped in
// 8x8x8 blocks (block-major x, y, z) with Morton order inside a block. Its tick
// (rayMarchCompute.slang:211-280) is the search tick's rule with optional wrap-around on
// every axis (WRAP_AT_BOUNDARY, the W neighbourhood flag).
//
// These kernels convert a render buffer into the strip layout, optionally surrounded by a
// one-cell ghost shell that holds the opposite faces (wrap), refresh that shell between
// ticks, convert back, and build the skip grid the renderer reads (8-cell chunks within one
// cell of a non-zero cell, rayMarchCompute.slang:182-205).
#include <cuda_runtime.h>

#include <algorithm>

#include "ca_core.cuh"
#include "kernels.h"

namespace cave {

__device__ __forceinline__ uint32_t spread3(uint32_t v) {  // cellStateUtils.slang:19-26
    v &= 7u;
    v = (v | (v << 8u)) & 0x100Fu;
    v = (v | (v << 4u)) & 0x10C30C3u;
    v = (v | (v << 2u)) & 0x1249249u;
    return v;
}
__device__ __forceinline__ uint32_t gather3(uint32_t m) {  // inverse of spread3 on bits 0, 3, 6
    return (m & 1u) | ((m >> 2) & 2u) | ((m >> 4) & 4u);
}

struct RenderDims {
    uint32_t X, Y, Z;        // cells
    uint32_t W;              // texels per row, ceil(X / 2)
    uint32_t nbx, nby, nbz;  // 8x8x8 texel blocks per axis
    uint32_t pad;            // ghost shell thickness of the strip grid (0 or 1)
    uint32_t SX;             // strips per row of the (padded) strip grid
    uint32_t Yp, Zp;         // rows and planes of the padded strip grid
};

__device__ __forceinline__ uint64_t texel_index(const RenderDims& d, uint32_t tx, uint32_t ty, uint32_t tz) {
    const uint64_t block = ((uint64_t)(tz >> 3) * d.nby + (ty >> 3)) * d.nbx + (tx >> 3);
    return block * 512u + (spread3(tx) | (spread3(ty) << 1u) | (spread3(tz) << 2u));
}

// One thread per strip of the padded grid. Ghost rows and planes are written as zero; the
// ghost cells of interior rows as zero too (they are filled by the ghost kernels).
__global__ void k_render_to_strips(const uint32_t* __restrict__ render, uint4* __restrict__ strips, RenderDims d) {
    const uint64_t n = (uint64_t)d.SX * d.Yp * d.Zp;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t sx = (uint32_t)(i % d.SX);
        const uint64_t r = i / d.SX;
        const int y = (int)(r % d.Yp) - (int)d.pad, z = (int)(r / d.Yp) - (int)d.pad;
        uint32_t p[4] = {0u, 0u, 0u, 0u};
        if (y >= 0 && y < (int)d.Y && z >= 0 && z < (int)d.Z) {
            for (uint32_t j = 0; j < 32u; j += 2u) {
                // cells xp, xp + 1 of the padded row; x = xp - pad
                const int x0 = (int)(sx * 32u + j) - (int)d.pad;
                for (int c = 0; c < 2; c++) {
                    const int x = x0 + c;
                    if (x < 0 || x >= (int)d.X) continue;
                    const uint32_t t = render[texel_index(d, (uint32_t)x >> 1, (uint32_t)y, (uint32_t)z)];
                    const uint32_t s = (x & 1) ? ((t >> 4) & 0xFu) : (t & 0xFu);
                    const uint32_t bit = 1u << (j + c);
#pragma unroll
                    for (int b = 0; b < 4; b++)
                        if ((s >> b) & 1u) p[b] |= bit;
                }
            }
        }
        strips[i] = make_uint4(p[0], p[1], p[2], p[3]);
    }
}

// One thread per buffer element: the texel's two cells from the strip grid; elements outside
// the texel grid (block padding) become 0.
__global__ void k_strips_to_render(const uint4* __restrict__ strips, uint32_t* __restrict__ render, RenderDims d) {
    const uint64_t n = (uint64_t)d.nbx * d.nby * d.nbz * 512u;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t block = e >> 9;
        const uint32_t m = (uint32_t)(e & 511u);
        const uint32_t bx = (uint32_t)(block % d.nbx), by = (uint32_t)((block / d.nbx) % d.nby),
                       bz = (uint32_t)(block / ((uint64_t)d.nbx * d.nby));
        const uint32_t tx = bx * 8u + gather3(m), ty = by * 8u + gather3(m >> 1), tz = bz * 8u + gather3(m >> 2);
        uint32_t v = 0u;
        if (tx < d.W && ty < d.Y && tz < d.Z) {
            const uint64_t row = ((uint64_t)(tz + d.pad) * d.Yp + (ty + d.pad)) * d.SX;
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const uint32_t x = 2u * tx + c;
                if (x >= d.X) continue;
                const uint32_t xp = x + d.pad;
                const uint4 s = strips[row + xp / 32u];
                const uint32_t sh = xp % 32u;
                const uint32_t st = ((s.x >> sh) & 1u) | (((s.y >> sh) & 1u) << 1) | (((s.z >> sh) & 1u) << 2) |
                                    (((s.w >> sh) & 1u) << 3);
                v |= st << (4 * c);
            }
        }
        render[e] = v;
    }
}

// Ghost shell refresh for wrap-around, in three passes so that edges and corners take the
// wrapped values of all three axes. x: bit xp = 0 <- xp = X, bit xp = X + 1 <- xp = 1, one
// thread per interior row.
__device__ __forceinline__ uint32_t bit_of(const uint4& s, uint32_t b, int plane) {
    const uint32_t w = plane == 0 ? s.x : plane == 1 ? s.y : plane == 2 ? s.z : s.w;
    return (w >> b) & 1u;
}
__device__ __forceinline__ void set_bit(uint4& s, uint32_t b, int plane, uint32_t v) {
    uint32_t& w = plane == 0 ? s.x : plane == 1 ? s.y : plane == 2 ? s.z : s.w;
    w = (w & ~(1u << b)) | (v << b);
}

__global__ void k_ghost_x(uint4* __restrict__ strips, RenderDims d) {
    const uint64_t n = (uint64_t)d.Y * d.Z;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t y = (uint32_t)(i % d.Y) + 1u, z = (uint32_t)(i / d.Y) + 1u;
        uint4* row = strips + ((uint64_t)z * d.Yp + y) * d.SX;
        const uint32_t xl = d.X, xr = d.X + 1u;  // padded positions of cell X-1 and of the right ghost
        const uint4 last = row[xl / 32u], first = row[0];
        uint4 g0 = first;
        for (int b = 0; b < 4; b++) set_bit(g0, 0u, b, bit_of(last, xl % 32u, b));
        uint4 g1 = (xr / 32u == 0u) ? g0 : row[xr / 32u];
        for (int b = 0; b < 4; b++) set_bit(g1, xr % 32u, b, bit_of(first, 1u, b));
        if (xr / 32u == 0u) {
            row[0] = g1;
        } else {
            row[0] = g0;
            row[xr / 32u] = g1;
        }
    }
}

// y: row yp = 0 <- yp = Y and yp = Y + 1 <- yp = 1, for interior planes; one thread per strip.
__global__ void k_ghost_y(uint4* __restrict__ strips, RenderDims d) {
    const uint64_t n = (uint64_t)d.SX * d.Z * 2u;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t sx = (uint32_t)(i % d.SX);
        const uint64_t r = i / d.SX;
        const uint32_t z = (uint32_t)(r >> 1) + 1u, side = (uint32_t)(r & 1u);
        uint4* plane = strips + (uint64_t)z * d.Yp * d.SX;
        const uint32_t from = side ? 1u : d.Y, to = side ? d.Y + 1u : 0u;
        plane[(uint64_t)to * d.SX + sx] = plane[(uint64_t)from * d.SX + sx];
    }
}

// z: plane zp = 0 <- zp = Z and zp = Z + 1 <- zp = 1; one thread per strip.
__global__ void k_ghost_z(uint4* __restrict__ strips, RenderDims d) {
    const uint64_t plane = (uint64_t)d.SX * d.Yp;
    const uint64_t n = plane * 2u;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = i % plane;
        const uint32_t side = (uint32_t)(i / plane);
        const uint32_t from = side ? 1u : d.Z, to = side ? d.Z + 1u : 0u;
        strips[(uint64_t)to * plane + k] = strips[(uint64_t)from * plane + k];
    }
}

// Skip grid: chunk (i, j, k) of 8x8x8 cells is marked (1) iff a non-zero cell lies within one
// cell of it, clamped to the grid (rayMarchCompute.slang:182-205 scatter-writes exactly those
// chunks). One thread per skip-buffer element; block padding is 0.
__global__ void k_render_skip(const uint4* __restrict__ strips, uint32_t* __restrict__ skip, RenderDims d,
                              uint32_t sdx, uint32_t sdy, uint32_t sdz) {
    const uint32_t nbx = (sdx + 7u) / 8u, nby = (sdy + 7u) / 8u, nbz = (sdz + 7u) / 8u;
    const uint64_t n = (uint64_t)nbx * nby * nbz * 512u;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t block = e >> 9;
        const uint32_t m = (uint32_t)(e & 511u);
        const uint32_t ci = (uint32_t)(block % nbx) * 8u + gather3(m);
        const uint32_t cj = (uint32_t)((block / nbx) % nby) * 8u + gather3(m >> 1);
        const uint32_t ck = (uint32_t)(block / ((uint64_t)nbx * nby)) * 8u + gather3(m >> 2);
        uint32_t hit = 0u;
        if (ci < sdx && cj < sdy && ck < sdz) {
            const int x0 = max((int)(8u * ci) - 1, 0), x1 = min((int)(8u * ci) + 8, (int)d.X - 1);
            const int y0 = max((int)(8u * cj) - 1, 0), y1 = min((int)(8u * cj) + 8, (int)d.Y - 1);
            const int z0 = max((int)(8u * ck) - 1, 0), z1 = min((int)(8u * ck) + 8, (int)d.Z - 1);
            const uint32_t p0 = (uint32_t)x0 + d.pad, p1 = (uint32_t)x1 + d.pad;  // padded x range
            for (int z = z0; z <= z1 && !hit; z++)
                for (int y = y0; y <= y1 && !hit; y++) {
                    const uint4* row = strips + (((uint64_t)(z + d.pad) * d.Yp) + (uint64_t)(y + d.pad)) * d.SX;
                    for (uint32_t s = p0 / 32u; s <= p1 / 32u; s++) {
                        const uint4 v = row[s];
                        uint32_t nz = v.x | v.y | v.z | v.w;
                        const uint32_t lo = s == p0 / 32u ? p0 % 32u : 0u, hi = s == p1 / 32u ? p1 % 32u : 31u;
                        nz &= (hi == 31u ? 0xFFFFFFFFu : ((1u << (hi + 1u)) - 1u)) & ~((1u << lo) - 1u);
                        if (nz) hit = 1u;
                    }
                }
        }
        skip[e] = hit;
    }
}

static uint32_t blocks_for(uint64_t n) {
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, 148ull * 16));
}

RenderGeom render_geometry(uint32_t X, uint32_t Y, uint32_t Z, uint32_t pad) {
    RenderGeom g;
    g.X = X;
    g.Y = Y;
    g.Z = Z;
    g.pad = pad;
    g.Xp = X + 2 * pad;
    g.Yp = Y + 2 * pad;
    g.Zp = Z + 2 * pad;
    g.SX = (g.Xp + 31u) / 32u;
    g.W = (X + 1u) / 2u;
    g.elements = (uint64_t)((g.W + 7u) / 8u) * ((Y + 7u) / 8u) * ((Z + 7u) / 8u) * 512u;
    g.sdx = (X + 7u) / 8u;
    g.sdy = (Y + 7u) / 8u;
    g.sdz = (Z + 7u) / 8u;
    g.skip_elements = (uint64_t)((g.sdx + 7u) / 8u) * ((g.sdy + 7u) / 8u) * ((g.sdz + 7u) / 8u) * 512u;
    return g;
}

static RenderDims dims_of(const RenderGeom& g) {
    RenderDims d;
    d.X = g.X;
    d.Y = g.Y;
    d.Z = g.Z;
    d.W = g.W;
    d.nbx = (g.W + 7u) / 8u;
    d.nby = (g.Y + 7u) / 8u;
    d.nbz = (g.Z + 7u) / 8u;
    d.pad = g.pad;
    d.SX = g.SX;
    d.Yp = g.Yp;
    d.Zp = g.Zp;
    return d;
}

cudaError_t launch_render_to_strips(const uint32_t* render, uint4* strips, const RenderGeom& g, cudaStream_t st) {
    k_render_to_strips<<<blocks_for((uint64_t)g.SX * g.Yp * g.Zp), 256, 0, st>>>(render, strips, dims_of(g));
    return cudaGetLastError();
}

cudaError_t launch_strips_to_render(const uint4* strips, uint32_t* render, const RenderGeom& g, cudaStream_t st) {
    k_strips_to_render<<<blocks_for(g.elements), 256, 0, st>>>(strips, render, dims_of(g));
    return cudaGetLastError();
}

cudaError_t launch_ghost_fill(uint4* strips, const RenderGeom& g, cudaStream_t st) {
    const RenderDims d = dims_of(g);
    k_ghost_x<<<blocks_for((uint64_t)g.Y * g.Z), 256, 0, st>>>(strips, d);
    k_ghost_y<<<blocks_for((uint64_t)g.SX * g.Z * 2), 256, 0, st>>>(strips, d);
    k_ghost_z<<<blocks_for((uint64_t)g.SX * g.Yp * 2), 256, 0, st>>>(strips, d);
    return cudaGetLastError();
}

cudaError_t launch_render_skip(const uint4* strips, uint32_t* skip, const RenderGeom& g, cudaStream_t st) {
    k_render_skip<<<blocks_for(g.skip_elements), 256, 0, st>>>(strips, skip, dims_of(g), g.sdx, g.sdy, g.sdz);
    return cudaGetLastError();
}

}  // namespace cave
