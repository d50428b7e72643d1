// Checks the tiling of the streaming tick kernels (cave::plan_stream, cave_ca.cpp) on the host
// over many grid shapes, target CTA counts, row hints, rows per thread and halo widths:
//  * the plan accepts every grid the kernels support (1..1024 cells per row);
//  * SX = ceil(X / 32) strips per row, SXp the next power of two;
//  * threads = rows * SXp / spt, a whole number of warps within the kernel's limit, and
//    rows >= 2 * halo + 1 with every item's tile (ty rows) fitting rows - 2 * halo;
//  * the items cover every (y, z) of the grid exactly once, with in-range y and z ranges,
//    and each carries the item count of its simulation in dir_items >> 1;
//  * the tile's dynamic shared memory (the kernels' own size functions) fits one CTA (227 KB).
// And the resident kernel's geometry (cave::resident_geometry, engine.cpp) for every grid that
// resident_fits accepts, with and without a z-segment hint: whole warps of at most 1024 threads
// covering nseg segments of Y * SXp lanes, segments covering every plane, shared memory within
// the resident cap, and at least one CTA per SM.
// Built with nvcc (the size functions sit in the kernels' headers); needs no GPU. Exit status
// 0 = every check held.
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

#include "ca_types.h"
#include "engine.h"
#include "stream_common.cuh"
#include "stream_tick2.cuh"

namespace {
int check(uint32_t X, uint32_t Y, uint32_t Z, uint32_t target, uint32_t hint, uint32_t spt, uint32_t halo) {
    cave::StreamPlan p;
    if (!cave::plan_stream(7, X, Y, Z, target, hint, p, spt, halo)) {
        std::printf("rejected %u %u %u target %u hint %u spt %u halo %u\n", X, Y, Z, target, hint, spt, halo);
        return 1;
    }
    uint32_t sxp = 1;
    while (sxp < (X + 31) / 32) sxp <<= 1;
    const uint32_t limit = halo == 2 ? (uint32_t)cave::kJit2MaxThreads : spt == 1 ? 1024u : (uint32_t)cave::kJitMaxThreads;
    bool ok = p.SX == (X + 31) / 32 && p.SXp == sxp && (p.rows * p.SXp) % spt == 0 &&
              p.threads == p.rows * p.SXp / spt && p.threads % 32 == 0 && p.threads >= 32 && p.threads <= limit &&
              p.rows >= 2 * halo + 1 && !p.items.empty();
    const size_t smem = halo == 2 ? cave::stream2_smem_bytes(p.rows, p.SX, p.SXp)
                                  : cave::stream_smem_bytes(p.rows, p.SX, p.SXp);
    ok = ok && smem <= 227u * 1024u;
    std::vector<uint8_t> seen((size_t)Y * Z, 0);
    for (const cave::StreamItem& it : p.items) {
        ok = ok && it.sim == 7 && it.ty >= 1 && it.ty <= p.rows - 2 * halo && (uint32_t)it.y0 + it.ty <= Y &&
             it.z0 < it.z1 && it.z1 <= Z && (it.dir_items >> 1) == p.items.size();
        if (!ok) break;
        for (uint32_t z = it.z0; z < it.z1; z++)
            for (uint32_t y = it.y0; y < (uint32_t)it.y0 + it.ty; y++) ok = ok && ++seen[(size_t)z * Y + y] == 1;
    }
    for (uint8_t v : seen) ok = ok && v == 1;
    if (!ok) {
        std::printf("bad plan %u %u %u target %u hint %u spt %u halo %u: SX %u SXp %u rows %u threads %u items %zu\n", X,
                    Y, Z, target, hint, spt, halo, p.SX, p.SXp, p.rows, p.threads, p.items.size());
        return 1;
    }
    return 0;
}
int check_resident(uint32_t X, uint32_t Y, uint32_t Z, uint32_t hint) {
    if (!cave::resident_fits(X, Y, Z)) return 0;
    uint32_t threads = 0;
    const cave::ResLaunch P = cave::resident_geometry(X, Y, Z, hint, threads);
    uint32_t sxp = 1;
    while (sxp < (X + 31) / 32) sxp <<= 1;
    const uint32_t cols = Y * sxp;
    const bool ok = P.X == X && P.Y == Y && P.Z == Z && P.SX == (X + 31) / 32 && (1u << P.sxp_log2) == sxp &&
                    P.nseg >= 1 && P.nseg <= Z && (hint == 0 || P.nseg <= hint) &&
                    (uint64_t)P.seg_len * P.nseg >= Z && P.seg_len >= 1 && threads % 32 == 0 &&
                    threads >= P.nseg * cols && threads < P.nseg * cols + 32 && threads <= 1024 &&
                    cave::resident_smem_bytes(X, Y, Z, P.nseg) <= 220u * 1024u &&
                    cave::resident_ctas_per_sm(P, threads) >= 1;
    if (!ok) {
        std::printf("bad resident geometry %u %u %u hint %u: nseg %u seg_len %u threads %u\n", X, Y, Z, hint, P.nseg,
                    P.seg_len, threads);
        return 1;
    }
    return 0;
}
}  // namespace

int main() {
    std::mt19937 rng(12345);
    const uint32_t targets[] = {1, 148, 296, 592, 4096};
    int n = 0;
    // the benchmarked and tested shapes, then random ones
    const uint32_t fixed[][3] = {{512, 512, 512}, {1024, 1024, 1024}, {256, 256, 256}, {49, 49, 49},
                                 {1024, 40, 4},   {1, 1, 1},          {193, 193, 193}, {200, 9, 21}};
    for (const auto& d : fixed)
        for (uint32_t t : targets)
            for (uint32_t spt = 1; spt <= 3; spt++)
                for (uint32_t halo = 1; halo <= 2; halo++, n++)
                    if (check(d[0], d[1], d[2], t, 0, spt, halo)) return 1;
    for (int i = 0; i < 20000; i++, n++) {
        const uint32_t X = 1 + rng() % 1024, Y = 1 + rng() % 700, Z = 1 + rng() % 700;
        const uint32_t spt = 1 + rng() % 3, halo = 1 + rng() % 2;
        const uint32_t hint = rng() % 3 == 0 ? 0u : 1u + rng() % 1200;
        if (check(X, Y, Z, targets[rng() % 5], hint, spt, halo)) return 1;
    }
    int nres = 0;
    for (uint32_t X : {1u, 8u, 25u, 33u, 49u, 64u, 65u, 97u, 128u})
        for (uint32_t Y = 1; Y <= 130; Y += 3)
            for (uint32_t Z = 1; Z <= 130; Z += 7)
                for (uint32_t hint : {0u, 1u, 3u, 64u}) {
                    if (check_resident(X, Y, Z, hint)) return 1;
                    nres += cave::resident_fits(X, Y, Z) ? 1 : 0;
                }
    if (nres == 0) return 1;
    std::printf("ok %d plans, %d resident geometries\n", n, nres);
    return 0;
}
