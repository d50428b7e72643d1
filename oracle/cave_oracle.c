/*
 * cave_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of CAVE's search-mode cellular-automaton arithmetic, used as
 * the parity oracle for the CUDA path and as the timed CPU baseline. Nothing in the
 * product (cave_b200/) links or calls this file; only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it, and only to check results or to be timed.
 *
 * The reference has no CPU stepping (src/simulation/simulation.cpp:48-50: all cell
 * work happens in GPU shaders), so this file restates the shader and host arithmetic
 * directly. Every function cites the reference lines it follows:
 *   - shaders/slang/search/searchSimulationCube.slang:40-247   one tick + counters
 *   - shaders/slang/common/cube.slang:7-21                     neighbour deltas
 *   - shaders/slang/search/searchManager.slang:16-149          GridInfo, status, NextPermutation
 *   - src/vulkan/systems/searchSystem.cpp:219-306              initial cells / seeding
 *   - src/vulkan/systems/searchSystem.cpp:646-713              classification
 *   - src/common/permutationMath.h:101-128                     valid-bitmask enumeration
 *   - src/simulation/simulation.h:43-59                        field encodings
 *
 * Parity pin: the reference cannot run here (Vulkan + Slang). The restatement is pinned
 * by the reference's only exact-value test (cli-rules, src/testing/testRunner.cpp:231-260,
 * tests/test_rules.py) and by hand-derived known-answer tests (tests/test_oracle.py); the
 * historical aggregate counts of benchmarks/reference/debug/bench_results.csv:2-9 are a
 * partial cross-check only (they predate the shader's early-death rule).
 *
 * The render-mode step (oracle_render_step) restates shaders/slang/rendering/
 * rayMarchCompute.slang:60-280 with the packed, Morton-tiled buffer layout of
 * shaders/slang/common/cellStateUtils.slang:18-54.
 *
 * Two step implementations live here:
 *   oracle_step       -- literal per-cell restatement (up to 26 neighbour reads per cell)
 *   oracle_step_fast  -- the same arithmetic on an unpacked byte grid with separable
 *                        x-sums, parallelised over z with OpenMP; tests require it to be
 *                        bit-identical to oracle_step. It is the CPU baseline.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PERM_MASK ((((uint64_t)1) << 60) - 1) /* simulation.h:43 EXISTENCE_PERMUTATION_BIT_MASK */

/* cube.slang:7-21 -- delta tables in the shader's order. */
static const int kFace[6][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}};
static const int kEdge[12][3] = {{1, 1, 0},  {1, -1, 0}, {-1, 1, 0}, {-1, -1, 0}, {1, 0, 1},  {1, 0, -1},
                                 {-1, 0, 1}, {-1, 0, -1}, {0, 1, 1}, {0, 1, -1},  {0, -1, 1}, {0, -1, -1}};
static const int kCorner[8][3] = {{1, 1, 1},  {-1, 1, 1},  {1, -1, 1},  {-1, -1, 1},
                                  {1, 1, -1}, {-1, 1, -1}, {1, -1, -1}, {-1, -1, -1}};

uint32_t oracle_words_per_row(uint32_t X) { return (X + 7u) / 8u; } /* slang:52 */

uint64_t oracle_grid_words(uint32_t X, uint32_t Y, uint32_t Z) {
    return (uint64_t)oracle_words_per_row(X) * Y * Z; /* slang:52-53, searchSystem.cpp:140-143 */
}

/* ------------------------------------------------------------------------------------ */
/* permutationMath.h:101-128 -- bitmasks with 1..maxBits bits over the low N bits, sorted. */
static void emit_masks(uint64_t acc, uint32_t start, uint32_t remaining, uint32_t n, uint64_t *out,
                       size_t cap, size_t *count) {
    if (remaining == 0) {
        if (acc != 0) {
            if (*count < cap && out) out[*count] = acc;
            (*count)++;
        }
        return;
    }
    for (uint32_t i = start; i + remaining <= n; i++)
        emit_masks(acc | ((uint64_t)1 << i), i + 1, remaining - 1, n, out, cap, count);
}

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* Returns the number of masks; writes min(count, cap) of them, sorted ascending. */
size_t oracle_enumerate_valid_bitmasks(uint32_t neighborCount, uint32_t maxBits, uint64_t *out, size_t cap) {
    if (maxBits == 0 || neighborCount == 0) return 0;
    uint32_t eff = maxBits < neighborCount ? maxBits : neighborCount;
    size_t count = 0;
    for (uint32_t p = 1; p <= eff; p++) emit_masks(0, 0, p, neighborCount, NULL, 0, &count);
    if (!out) return count;
    uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * (count ? count : 1));
    size_t c2 = 0;
    for (uint32_t p = 1; p <= eff; p++) emit_masks(0, 0, p, neighborCount, tmp, count, &c2);
    qsort(tmp, count, sizeof(uint64_t), cmp_u64);
    memcpy(out, tmp, sizeof(uint64_t) * (count < cap ? count : cap));
    free(tmp);
    return count;
}

/* ------------------------------------------------------------------------------------ */
/* searchSystem.cpp:244-252 (wangHash) and :253-259 (cellHash). */
static uint32_t wang_hash(uint32_t seed) {
    seed = (seed ^ 61u) ^ (seed >> 16);
    seed *= 9u;
    seed = seed ^ (seed >> 4);
    seed *= 0x27d4eb2du;
    seed = seed ^ (seed >> 15);
    return seed;
}

uint32_t oracle_cell_hash(uint32_t x, uint32_t y, uint32_t z, uint32_t runSeedIndex) {
    uint32_t h = wang_hash(x * 73856093u + runSeedIndex);
    h = wang_hash(h ^ (y * 19349663u));
    h = wang_hash(h ^ (z * 83492791u));
    return h;
}

/* searchSystem.cpp:226-232: spawn size index 0 = full area, else scaled (i+1)/16. */
static uint32_t resolve_spawn(uint32_t axis, uint32_t sizeIndex) {
    if (sizeIndex == 0) return axis;
    uint32_t scaled = (uint32_t)(((uint64_t)axis * (sizeIndex + 1) + 15) / 16);
    if (scaled > axis) scaled = axis;
    return scaled < 1 ? 1 : scaled;
}

/* searchSystem.cpp:240 + :260-262 -- density index (0..15) to the uint32 threshold; the
 * value 2^32 stands for "density >= 1, every cell in the box alive" (the reference
 * short-circuits that case at :278 rather than comparing against the threshold). */
uint64_t oracle_density_threshold_from_index(uint32_t densityIndex) {
    float density = ((float)densityIndex + 1.0f) / 16.0f;
    if (density >= 1.0f) return (uint64_t)1 << 32;
    return (uint64_t)(uint32_t)(density * 4294967296.0);
}

/* Same expression for an arbitrary float density p (the harness form used for fills such
 * as 0.30 that the 1/16-quantised CLI cannot express). */
uint64_t oracle_density_threshold_from_float(float density) {
    if (density >= 1.0f) return (uint64_t)1 << 32;
    if (density <= 0.0f) return 0;
    return (uint64_t)(uint32_t)(density * 4294967296.0);
}

/* searchSystem.cpp:219-306 -- initial cells for one slot. spawnRandom != 0 is the random
 * spawn shape (spawnRegionShapeId == 0); otherwise every box cell is alive. Alive cells
 * get (maxCellState & 0xF) (:302), so maxCellState 16 seeds zeros. */
void oracle_seed(uint32_t X, uint32_t Y, uint32_t Z, uint32_t spawnX, uint32_t spawnY, uint32_t spawnZ,
                 uint32_t spawnSizeIndex, int spawnRandom, uint64_t threshold, uint32_t runSeedIndex,
                 uint32_t maxCellState, uint32_t *out) {
    uint32_t wpr = oracle_words_per_row(X);
    memset(out, 0, sizeof(uint32_t) * oracle_grid_words(X, Y, Z));
    uint32_t ex = resolve_spawn(spawnX, spawnSizeIndex);
    uint32_t ey = resolve_spawn(spawnY, spawnSizeIndex);
    uint32_t ez = resolve_spawn(spawnZ, spawnSizeIndex);
    uint32_t x0 = (X - ex) / 2, x1 = (X + ex) / 2;
    uint32_t y0 = (Y - ey) / 2, y1 = (Y + ey) / 2;
    uint32_t z0 = (Z - ez) / 2, z1 = (Z + ez) / 2;
    for (uint32_t x = 0; x < X; x++)
        for (uint32_t y = 0; y < Y; y++)
            for (uint32_t z = 0; z < Z; z++) {
                int in = x >= x0 && x < x1 && y >= y0 && y < y1 && z >= z0 && z < z1;
                if (!in) continue;
                int alive = spawnRandom ? ((uint64_t)oracle_cell_hash(x, y, z, runSeedIndex) < threshold) : 1;
                if (alive) {
                    uint64_t idx = (uint64_t)(x / 8u) + (uint64_t)y * wpr + (uint64_t)z * wpr * Y;
                    out[idx] |= (maxCellState & 0xFu) << ((x % 8u) * 4u);
                }
            }
}

/* ------------------------------------------------------------------------------------ */
/* searchSimulationCube.slang:139-157 -- decode params; K > 0 means 1-based indices into
 * validBitmasks. Returns -1 when an index falls outside the table (the shader would read
 * out of bounds; the oracle refuses). */
static int decode_rules(const uint64_t params[3], const uint64_t *validBitmasks, uint32_t nValid,
                        uint32_t maxRuleBits, uint32_t *maxCS, uint32_t *flags, uint64_t *birth,
                        uint64_t *survival) {
    *maxCS = (uint32_t)(params[0] >> 60) + 1u;
    *flags = (uint32_t)(params[1] >> 60);
    if (maxRuleBits > 0) {
        uint32_t bi = (uint32_t)(params[0] & PERM_MASK) - 1u;
        uint32_t si = (uint32_t)(params[1] & PERM_MASK) - 1u;
        if (bi >= nValid || si >= nValid) return -1;
        *birth = validBitmasks[bi];
        *survival = validBitmasks[si];
    } else {
        *birth = params[0] & PERM_MASK;
        *survival = params[1] & PERM_MASK;
    }
    return 0;
}

/* slang:78-94 -- out-of-grid is not alive; alive means state == maxCellState. */
static int is_alive(const uint32_t *cells, int x, int y, int z, uint32_t X, uint32_t Y, uint32_t Z,
                    uint32_t wpr, uint32_t maxCS) {
    if (x < 0 || x >= (int)X || y < 0 || y >= (int)Y || z < 0 || z >= (int)Z) return 0;
    uint64_t idx = (uint64_t)((uint32_t)x / 8u) + (uint64_t)y * wpr + (uint64_t)z * wpr * Y;
    uint32_t state = (cells[idx] >> (((uint32_t)x % 8u) * 4u)) & 0xFu;
    return state == maxCS;
}

/* slang:96-115 */
static int count_alive(const uint32_t *cells, int x, int y, int z, uint32_t X, uint32_t Y, uint32_t Z,
                       uint32_t wpr, uint32_t maxCS, uint32_t flags) {
    int n = 0;
    if (flags & 1u)
        for (int i = 0; i < 6; i++)
            n += is_alive(cells, x + kFace[i][0], y + kFace[i][1], z + kFace[i][2], X, Y, Z, wpr, maxCS);
    if (flags & 2u)
        for (int i = 0; i < 12; i++)
            n += is_alive(cells, x + kEdge[i][0], y + kEdge[i][1], z + kEdge[i][2], X, Y, Z, wpr, maxCS);
    if (flags & 4u)
        for (int i = 0; i < 8; i++)
            n += is_alive(cells, x + kCorner[i][0], y + kCorner[i][1], z + kCorner[i][2], X, Y, Z, wpr, maxCS);
    return n;
}

/* Per-tick statistics. The first four fields are the reference's GridSnapshot
 * (structs.h:130-136, same order). The rest are derived statistics the reference does
 * not compute: population = cells with a non-zero state after the tick; changed = cells
 * whose state differs from before the tick; bounding box of non-zero cells after the
 * tick (min = 0xFFFFFFFF and max = 0 when no cell is non-zero). */
typedef struct {
    uint32_t dead, dying, born, surviving;
    uint32_t population, changed;
    uint32_t bbox_min[3], bbox_max[3];
} oracle_tick_stats;

static void derived_stats(uint32_t X, uint32_t Y, uint32_t Z, const uint32_t *in, const uint32_t *out,
                          oracle_tick_stats *st) {
    uint32_t wpr = oracle_words_per_row(X);
    st->population = 0;
    st->changed = 0;
    st->bbox_min[0] = st->bbox_min[1] = st->bbox_min[2] = 0xFFFFFFFFu;
    st->bbox_max[0] = st->bbox_max[1] = st->bbox_max[2] = 0;
    for (uint32_t z = 0; z < Z; z++)
        for (uint32_t y = 0; y < Y; y++)
            for (uint32_t x = 0; x < X; x++) {
                uint64_t idx = (uint64_t)(x / 8u) + (uint64_t)y * wpr + (uint64_t)z * wpr * Y;
                uint32_t sh = (x % 8u) * 4u;
                uint32_t a = (in[idx] >> sh) & 0xFu, b = (out[idx] >> sh) & 0xFu;
                if (a != b) st->changed++;
                if (b) {
                    st->population++;
                    uint32_t c[3] = {x, y, z};
                    for (int k = 0; k < 3; k++) {
                        if (c[k] < st->bbox_min[k]) st->bbox_min[k] = c[k];
                        if (c[k] > st->bbox_max[k]) st->bbox_max[k] = c[k];
                    }
                }
            }
}

/* searchSimulationCube.slang:117-247, literally, one cell at a time. Writes the whole
 * packed word including zeroed padding nibbles (:213-216). Returns 0, or -1 on a bad
 * rule index. `stats` may be NULL. */
int oracle_step(uint32_t X, uint32_t Y, uint32_t Z, const uint64_t params[3], const uint64_t *validBitmasks,
                uint32_t nValid, uint32_t maxRuleBits, const uint32_t *in, uint32_t *out,
                oracle_tick_stats *stats) {
    uint32_t maxCS, flags;
    uint64_t B, S;
    if (decode_rules(params, validBitmasks, nValid, maxRuleBits, &maxCS, &flags, &B, &S)) return -1;
    uint32_t wpr = oracle_words_per_row(X);
    uint32_t died = 0, dying = 0, born = 0, survived = 0;
    for (uint32_t z = 0; z < Z; z++)
        for (uint32_t y = 0; y < Y; y++)
            for (uint32_t ux = 0; ux < wpr; ux++) {
                uint64_t idx = (uint64_t)ux + (uint64_t)y * wpr + (uint64_t)z * wpr * Y;
                uint32_t inPacked = in[idx], outPacked = 0;
                for (uint32_t nib = 0; nib < 8; nib++) {
                    uint32_t cx = ux * 8u + nib;
                    if (cx >= X) break;
                    uint32_t cur = (inPacked >> (nib * 4u)) & 0xFu;
                    int n = count_alive(in, (int)cx, (int)y, (int)z, X, Y, Z, wpr, maxCS, flags);
                    uint32_t ns;
                    if (cur == maxCS) {
                        if (n > 0 && ((S >> (uint64_t)(n - 1)) & 1u)) {
                            ns = maxCS;
                            survived++;
                        } else {
                            ns = cur - 1u;
                            dying++;
                        }
                    } else if (cur == 0u) {
                        if (n > 0 && ((B >> (uint64_t)(n - 1)) & 1u)) {
                            ns = maxCS;
                            born++;
                        } else {
                            ns = 0u;
                            died++;
                        }
                    } else {
                        ns = cur - 1u;
                        dying++;
                    }
                    outPacked |= (ns & 0xFu) << (nib * 4u);
                }
                out[idx] = outPacked;
            }
    if (stats) {
        stats->dead = died;
        stats->dying = dying;
        stats->born = born;
        stats->surviving = survived;
        derived_stats(X, Y, Z, in, out, stats);
    }
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/* The same arithmetic on an unpacked byte grid. alive[] is padded by one cell on every
 * side so that the zero boundary (slang:80-81) needs no branch; hx[] holds the x-direction
 * 3-sums of alive[]. The counts follow directly from the delta sets of cube.slang:7-21:
 *   faces   = (hx - a)(centre row) + sum over the 4 face rows  of a
 *   edges   = (hx - a)(4 face rows) + sum over the 4 diagonal rows of a
 *   corners = (hx - a)(4 diagonal rows)
 * where "face rows" are (y+-1, z) and (y, z+-1), "diagonal rows" are (y+-1, z+-1).       */
int oracle_step_fast(uint32_t X, uint32_t Y, uint32_t Z, const uint64_t params[3],
                     const uint64_t *validBitmasks, uint32_t nValid, uint32_t maxRuleBits, const uint32_t *in,
                     uint32_t *out, uint32_t snapshot[4], int nthreads) {
    uint32_t maxCS, flags;
    uint64_t B, S;
    if (decode_rules(params, validBitmasks, nValid, maxRuleBits, &maxCS, &flags, &B, &S)) return -1;
    const uint32_t wpr = oracle_words_per_row(X);
    const int64_t PX = (int64_t)X + 2, PY = (int64_t)Y + 2, PZ = (int64_t)Z + 2;
    const int64_t sy = PX, sz = PX * PY;
    uint8_t *a = (uint8_t *)calloc((size_t)(PX * PY * PZ), 1);
    uint8_t *hx = (uint8_t *)calloc((size_t)(PX * PY * PZ), 1);
    if (!a || !hx) {
        free(a);
        free(hx);
        return -2;
    }
    const int fF = (flags & 1u) != 0, fE = (flags & 2u) != 0, fC = (flags & 4u) != 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(static)
    for (int64_t z = 0; z < (int64_t)Z; z++)
        for (uint32_t y = 0; y < Y; y++) {
            const uint32_t *row = in + (uint64_t)y * wpr + (uint64_t)z * wpr * Y;
            uint8_t *ar = a + (z + 1) * sz + (int64_t)(y + 1) * sy + 1;
            for (uint32_t x = 0; x < X; x++) ar[x] = ((row[x >> 3] >> ((x & 7u) * 4u)) & 0xFu) == maxCS;
        }
#pragma omp parallel for schedule(static)
    for (int64_t z = 0; z < (int64_t)Z; z++)
        for (uint32_t y = 0; y < Y; y++) {
            int64_t base = (z + 1) * sz + (int64_t)(y + 1) * sy + 1;
            for (uint32_t x = 0; x < X; x++) hx[base + x] = a[base + x - 1] + a[base + x] + a[base + x + 1];
        }
    uint64_t died = 0, dying = 0, born = 0, survived = 0;
#pragma omp parallel for schedule(static) reduction(+ : died, dying, born, survived)
    for (int64_t z = 0; z < (int64_t)Z; z++)
        for (uint32_t y = 0; y < Y; y++) {
            const uint32_t *row = in + (uint64_t)y * wpr + (uint64_t)z * wpr * Y;
            uint32_t *orow = out + (uint64_t)y * wpr + (uint64_t)z * wpr * Y;
            int64_t c = (z + 1) * sz + (int64_t)(y + 1) * sy + 1;
            const int64_t f[4] = {c - sy, c + sy, c - sz, c + sz};
            const int64_t d[4] = {c - sy - sz, c - sy + sz, c + sy - sz, c + sy + sz};
            for (uint32_t w = 0; w < wpr; w++) orow[w] = 0;
            for (uint32_t x = 0; x < X; x++) {
                int n = 0;
                if (fF) {
                    n += hx[c + x] - a[c + x];
                    for (int k = 0; k < 4; k++) n += a[f[k] + x];
                }
                if (fE) {
                    for (int k = 0; k < 4; k++) n += hx[f[k] + x] - a[f[k] + x];
                    for (int k = 0; k < 4; k++) n += a[d[k] + x];
                }
                if (fC)
                    for (int k = 0; k < 4; k++) n += hx[d[k] + x] - a[d[k] + x];
                uint32_t cur = (row[x >> 3] >> ((x & 7u) * 4u)) & 0xFu, ns;
                if (cur == maxCS) {
                    if (n > 0 && ((S >> (uint64_t)(n - 1)) & 1u)) {
                        ns = maxCS;
                        survived++;
                    } else {
                        ns = cur - 1u;
                        dying++;
                    }
                } else if (cur == 0u) {
                    if (n > 0 && ((B >> (uint64_t)(n - 1)) & 1u)) {
                        ns = maxCS;
                        born++;
                    } else {
                        ns = 0;
                        died++;
                    }
                } else {
                    ns = cur - 1u;
                    dying++;
                }
                orow[x >> 3] |= (ns & 0xFu) << ((x & 7u) * 4u);
            }
        }
    free(a);
    free(hx);
    if (snapshot) {
        snapshot[0] = (uint32_t)died;
        snapshot[1] = (uint32_t)dying;
        snapshot[2] = (uint32_t)born;
        snapshot[3] = (uint32_t)survived;
    }
    return 0;
}

/* The derived statistics of derived_stats (population, changed cells, bounding box of the
 * non-zero cells after the tick) computed in parallel over z: bit-identical to derived_stats,
 * for the large fixtures (hundreds of ticks of 512^3). The snapshot fields are left as they are. */
void oracle_derived_stats_fast(uint32_t X, uint32_t Y, uint32_t Z, const uint32_t *in, const uint32_t *out,
                               oracle_tick_stats *st, int nthreads) {
    const uint32_t wpr = oracle_words_per_row(X);
    uint64_t pop = 0, chg = 0;
    uint32_t mnx = 0xFFFFFFFFu, mny = 0xFFFFFFFFu, mnz = 0xFFFFFFFFu, mxx = 0, mxy = 0, mxz = 0;
    int any = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(static) reduction(+ : pop, chg) reduction(min : mnx, mny, mnz) \
    reduction(max : mxx, mxy, mxz) reduction(| : any)
    for (int64_t z = 0; z < (int64_t)Z; z++)
        for (uint32_t y = 0; y < Y; y++) {
            const uint64_t base = (uint64_t)y * wpr + (uint64_t)z * wpr * Y;
            for (uint32_t w = 0; w < wpr; w++) {
                const uint32_t a = in[base + w], b = out[base + w];
                for (uint32_t k = 0; k < 8; k++) {
                    const uint32_t x = w * 8u + k;
                    if (x >= X) break;
                    const uint32_t ca = (a >> (4u * k)) & 0xFu, cb = (b >> (4u * k)) & 0xFu;
                    chg += ca != cb;
                    if (cb) {
                        pop++;
                        any = 1;
                        if (x < mnx) mnx = x;
                        if (x > mxx) mxx = x;
                        if (y < mny) mny = y;
                        if (y > mxy) mxy = y;
                        if ((uint32_t)z < mnz) mnz = (uint32_t)z;
                        if ((uint32_t)z > mxz) mxz = (uint32_t)z;
                    }
                }
            }
        }
    st->population = (uint32_t)pop;
    st->changed = (uint32_t)chg;
    st->bbox_min[0] = mnx;
    st->bbox_min[1] = mny;
    st->bbox_min[2] = mnz;
    st->bbox_max[0] = any ? mxx : 0;
    st->bbox_max[1] = any ? mxy : 0;
    st->bbox_max[2] = any ? mxz : 0;
}

/* ------------------------------------------------------------------------------------ */
/* GridInfo (structs.h:79-87) and GridPermutations (searchManager.slang:40-44). */
typedef struct {
    uint32_t totalDied, totalBorn, ticks, status, maxAlive, finalAlive;
} oracle_grid_info;

typedef struct {
    uint64_t birthAndMaxCellStateRules, survivalAndNeighborhoodRules;
} oracle_perms;

/* searchManager.slang:56-96 */
static void next_permutation(oracle_perms *p, oracle_grid_info *info, uint64_t maxPermutation,
                             uint64_t survivalEnd) {
    if (p->survivalAndNeighborhoodRules == 0 || p->birthAndMaxCellStateRules == 0) return;
    if ((p->birthAndMaxCellStateRules & PERM_MASK) < maxPermutation) {
        p->birthAndMaxCellStateRules++;
    } else if ((p->survivalAndNeighborhoodRules & PERM_MASK) < survivalEnd) {
        p->survivalAndNeighborhoodRules++;
        p->birthAndMaxCellStateRules = (p->birthAndMaxCellStateRules & ~PERM_MASK) + 1;
    } else {
        p->survivalAndNeighborhoodRules = 0;
        p->birthAndMaxCellStateRules = 0;
        return;
    }
    memset(info, 0, sizeof(*info));
}

/* searchManager.slang:98-149 -- one manager dispatch. infoCopy/permCopy receive what the
 * shader writes to its host-visible copy buffers. */
void oracle_manager(const uint32_t snapshot[4], oracle_grid_info *info, oracle_perms *perms,
                    uint64_t maxPermutation, uint64_t survivalEnd, uint32_t maxTicks,
                    oracle_grid_info *infoCopy, oracle_perms *permCopy) {
    oracle_perms p = *perms;
    if (p.survivalAndNeighborhoodRules == 0 || p.birthAndMaxCellStateRules == 0) {
        *infoCopy = *info;
        *permCopy = p;
        return;
    }
    info->ticks++;
    info->totalDied += snapshot[0];
    info->totalBorn += snapshot[2];
    info->finalAlive = snapshot[3];
    if (snapshot[3] > info->maxAlive) info->maxAlive = snapshot[3];
    if (snapshot[3] == 0u && snapshot[2] == 0u)
        info->status = 1;
    else if (info->ticks >= maxTicks)
        info->status = 2;
    else
        info->status = 0;
    *infoCopy = *info;
    *permCopy = p;
    if (info->status > 0) next_permutation(perms, info, maxPermutation, survivalEnd);
}

/* One rule from a fresh copy of the initial cells until the manager reports status > 0
 * (the per-rule lifecycle of searchSystem.cpp:496-526 + :608-616 + searchManager.slang).
 * Optional outputs: per_tick (maxTicks entries), final_cells. Returns ticks run, or -1. */
int oracle_run_sim(uint32_t X, uint32_t Y, uint32_t Z, const uint64_t params[3],
                   const uint64_t *validBitmasks, uint32_t nValid, uint32_t maxRuleBits,
                   const uint32_t *initial, uint32_t maxTicks, int fast, oracle_grid_info *info_out,
                   oracle_tick_stats *per_tick, uint32_t *final_cells) {
    uint64_t nw = oracle_grid_words(X, Y, Z);
    uint32_t *cur = (uint32_t *)malloc(sizeof(uint32_t) * (nw ? nw : 1));
    uint32_t *nxt = (uint32_t *)malloc(sizeof(uint32_t) * (nw ? nw : 1));
    if (!cur || !nxt) {
        free(cur);
        free(nxt);
        return -1;
    }
    memcpy(cur, initial, sizeof(uint32_t) * nw);
    oracle_grid_info info;
    memset(&info, 0, sizeof(info));
    oracle_perms perms = {params[0], params[1]};
    int t = 0;
    if (params[0] == 0 || params[1] == 0) {
        /* NULL permutation: the manager never counts a tick for it (searchManager.slang:104-110). */
        if (info_out) *info_out = info;
        if (final_cells) memcpy(final_cells, cur, sizeof(uint32_t) * nw);
        free(cur);
        free(nxt);
        return 0;
    }
    while (1) {
        oracle_tick_stats st;
        uint32_t snap[4];
        int rc;
        if (fast) {
            rc = oracle_step_fast(X, Y, Z, params, validBitmasks, nValid, maxRuleBits, cur, nxt, snap, 0);
            if (per_tick && !rc) {
                st.dead = snap[0];
                st.dying = snap[1];
                st.born = snap[2];
                st.surviving = snap[3];
                derived_stats(X, Y, Z, cur, nxt, &st);
            }
        } else {
            rc = oracle_step(X, Y, Z, params, validBitmasks, nValid, maxRuleBits, cur, nxt, &st);
            snap[0] = st.dead;
            snap[1] = st.dying;
            snap[2] = st.born;
            snap[3] = st.surviving;
        }
        if (rc) {
            free(cur);
            free(nxt);
            return -1;
        }
        if (per_tick) per_tick[t] = st;
        t++;
        oracle_grid_info ic;
        oracle_perms pc;
        /* maxPermutation/survivalEnd are irrelevant for a single rule: the lifecycle ends at
         * the first status > 0 regardless of what NextPermutation does afterwards. */
        oracle_manager(snap, &info, &perms, 0, 0, maxTicks, &ic, &pc);
        uint32_t *tmp = cur;
        cur = nxt;
        nxt = tmp;
        if (ic.status > 0) {
            info = ic;
            break;
        }
    }
    if (info_out) *info_out = info;
    if (final_cells) memcpy(final_cells, cur, sizeof(uint32_t) * nw);
    free(cur);
    free(nxt);
    return t;
}

/* searchSystem.cpp:697-711 -- 0 viable, 1 possible, 2 unviable. */
int oracle_classify(const oracle_grid_info *info, uint32_t maxCellState) {
    if (info->status == 2) return 0;
    if ((uint64_t)info->ticks > (uint64_t)maxCellState + 1) return 1;
    return 2;
}

/* A whole SearchSystem slot, literally as the reference pipelines it: every tick runs
 * Phase 0 (reset from initial cells when the host saw a finished rule), Phase 1 (sim),
 * Phase 2 (manager), Phase 3 (cellsOut -> cellsIn); the host then reads the copy buffers
 * and records each finished rule once (searchSystem.cpp:480-713). Results are written in
 * completion order as (birthField, survivalField, GridInfo) with the K-index translated
 * to bitmasks as in :668-685. Returns the number of results (may exceed cap). */
typedef struct {
    uint64_t birthAndMaxCellStateRules, survivalAndNeighborhoodRules;
    oracle_grid_info info;
    int32_t category;
    uint32_t pad;
} oracle_result;

int64_t oracle_run_slot(uint32_t X, uint32_t Y, uint32_t Z, uint64_t startBirthField, uint64_t startSurvivalField,
                        uint64_t maxPermutation, uint64_t survivalEnd, const uint64_t *validBitmasks,
                        uint32_t nValid, uint32_t maxRuleBits, const uint32_t *initial, uint32_t maxTicks, int fast,
                        oracle_result *out, size_t cap) {
    uint64_t nw = oracle_grid_words(X, Y, Z);
    uint32_t *cellsIn = (uint32_t *)malloc(sizeof(uint32_t) * (nw ? nw : 1));
    uint32_t *cellsOut = (uint32_t *)malloc(sizeof(uint32_t) * (nw ? nw : 1));
    memcpy(cellsIn, initial, sizeof(uint32_t) * nw);
    oracle_grid_info info;
    memset(&info, 0, sizeof(info));
    oracle_perms perms = {startBirthField, startSurvivalField};
    oracle_perms lastSaved = {0, 0};
    int needReset = 0;
    int64_t nres = 0;
    while (1) {
        if (needReset) {
            memcpy(cellsIn, initial, sizeof(uint32_t) * nw);
            needReset = 0;
        }
        uint32_t snap[4] = {0, 0, 0, 0};
        uint64_t params[3] = {perms.birthAndMaxCellStateRules, perms.survivalAndNeighborhoodRules, 0};
        int exhausted = (perms.birthAndMaxCellStateRules == 0 || perms.survivalAndNeighborhoodRules == 0);
        if (!exhausted) {
            int rc;
            if (fast)
                rc = oracle_step_fast(X, Y, Z, params, validBitmasks, nValid, maxRuleBits, cellsIn, cellsOut,
                                      snap, 0);
            else {
                oracle_tick_stats st;
                rc = oracle_step(X, Y, Z, params, validBitmasks, nValid, maxRuleBits, cellsIn, cellsOut, &st);
                snap[0] = st.dead;
                snap[1] = st.dying;
                snap[2] = st.born;
                snap[3] = st.surviving;
            }
            if (rc) {
                nres = -1;
                break;
            }
        }
        oracle_grid_info ic;
        oracle_perms pc;
        oracle_manager(snap, &info, &perms, maxPermutation, survivalEnd, maxTicks, &ic, &pc);
        if (!exhausted) memcpy(cellsIn, cellsOut, sizeof(uint32_t) * nw);
        /* host side: CacheCompletedResults (searchSystem.cpp:646-713) */
        if (ic.status != 0 && !(pc.birthAndMaxCellStateRules == 0 && pc.survivalAndNeighborhoodRules == 0) &&
            !(pc.birthAndMaxCellStateRules == lastSaved.birthAndMaxCellStateRules &&
              pc.survivalAndNeighborhoodRules == lastSaved.survivalAndNeighborhoodRules)) {
            lastSaved = pc;
            needReset = 1;
            oracle_result r;
            r.birthAndMaxCellStateRules = pc.birthAndMaxCellStateRules;
            r.survivalAndNeighborhoodRules = pc.survivalAndNeighborhoodRules;
            if (maxRuleBits > 0) {
                uint64_t bi = (pc.birthAndMaxCellStateRules & PERM_MASK) - 1;
                uint64_t si = (pc.survivalAndNeighborhoodRules & PERM_MASK) - 1;
                if (bi < nValid && si < nValid) {
                    r.birthAndMaxCellStateRules = (pc.birthAndMaxCellStateRules & ~PERM_MASK) | validBitmasks[bi];
                    r.survivalAndNeighborhoodRules =
                        (pc.survivalAndNeighborhoodRules & ~PERM_MASK) | validBitmasks[si];
                }
            }
            r.info = ic;
            r.category = oracle_classify(&ic, (uint32_t)((pc.birthAndMaxCellStateRules >> 60) & 0xF) + 1u);
            r.pad = 0;
            if ((size_t)nres < cap && out) out[nres] = r;
            nres++;
        }
        if (exhausted) break; /* IsRunning() false once the read-back permutation is NULL */
    }
    free(cellsIn);
    free(cellsOut);
    return nres;
}


/* ------------------------------------------------------------------ render-mode layout
 * cellStateUtils.slang:18-54 (buffer mode): texel (tx, ty, tz) holds cells x = 2tx (low
 * nibble) and 2tx + 1 (high nibble) in one uint32 element; texels are grouped in 8x8x8
 * blocks (block-major x, then y, then z), Morton order (x bit 0, y bit 1, z bit 2 of each
 * triplet) inside a block. Texel width = ceil(X / 2) (simulationRenderer.cpp:58). */
static uint32_t expand_bits3(uint32_t v) {
    v &= 7u;
    v = (v | (v << 8u)) & 0x100Fu;
    v = (v | (v << 4u)) & 0x10C30C3u;
    v = (v | (v << 2u)) & 0x1249249u;
    return v;
}

uint64_t oracle_render_index(uint32_t tx, uint32_t ty, uint32_t tz, uint32_t X, uint32_t Y, uint32_t Z) {
    const uint32_t nbx = ((X + 1u) / 2u + 7u) / 8u, nby = (Y + 7u) / 8u;
    (void)Z;
    const uint64_t block = (uint64_t)(tz / 8u) * nbx * nby + (uint64_t)(ty / 8u) * nbx + (tx / 8u);
    const uint32_t m = expand_bits3(tx % 8u) | (expand_bits3(ty % 8u) << 1u) | (expand_bits3(tz % 8u) << 2u);
    return block * 512u + m;
}

uint64_t oracle_render_elements(uint32_t X, uint32_t Y, uint32_t Z) {
    const uint64_t nbx = ((X + 1u) / 2u + 7u) / 8u, nby = (Y + 7u) / 8u, nbz = (Z + 7u) / 8u;
    return nbx * nby * nbz * 512u;
}

/* Skip grid of 8-cell chunks, tiled the same way (simulationRenderer.cpp:86-95). */
uint64_t oracle_render_skip_elements(uint32_t X, uint32_t Y, uint32_t Z) {
    const uint32_t sx = (X + 7u) / 8u, sy = (Y + 7u) / 8u, sz = (Z + 7u) / 8u;
    return (uint64_t)((sx + 7u) / 8u) * ((sy + 7u) / 8u) * ((sz + 7u) / 8u) * 512u;
}

static uint32_t render_cell(const uint32_t *buf, int x, int y, int z, uint32_t X, uint32_t Y, uint32_t Z) {
    const uint32_t packed = buf[oracle_render_index((uint32_t)x >> 1, (uint32_t)y, (uint32_t)z, X, Y, Z)];
    return (x & 1) == 0 ? (packed & 0xFu) : ((packed >> 4) & 0xFu);
}

/* rayMarchCompute.slang:80-113 -- with WRAP_AT_BOUNDARY every axis wraps (no domain
 * decomposition here), else out-of-grid is not alive. */
static int render_alive(const uint32_t *buf, int x, int y, int z, uint32_t X, uint32_t Y, uint32_t Z, int wrap,
                        uint32_t maxCS) {
    if (wrap) {
        x = ((x % (int)X) + (int)X) % (int)X;
        y = ((y % (int)Y) + (int)Y) % (int)Y;
        z = ((z % (int)Z) + (int)Z) % (int)Z;
    } else if (x < 0 || x >= (int)X || y < 0 || y >= (int)Y || z < 0 || z >= (int)Z) {
        return 0;
    }
    return render_cell(buf, x, y, z, X, Y, Z) == maxCS;
}

static uint32_t render_simulate(const uint32_t *buf, int x, int y, int z, uint32_t X, uint32_t Y, uint32_t Z,
                                int wrap, uint32_t cur, uint32_t maxCS, uint64_t survival, uint64_t birth,
                                uint32_t flags) {
    /* rayMarchCompute.slang:121-179 (cube: IsCellViable is always true) */
    uint32_t n = 0;
    if (flags & 1u)
        for (int i = 0; i < 6; i++)
            n += render_alive(buf, x + kFace[i][0], y + kFace[i][1], z + kFace[i][2], X, Y, Z, wrap, maxCS);
    if (flags & 2u)
        for (int i = 0; i < 12; i++)
            n += render_alive(buf, x + kEdge[i][0], y + kEdge[i][1], z + kEdge[i][2], X, Y, Z, wrap, maxCS);
    if (flags & 4u)
        for (int i = 0; i < 8; i++)
            n += render_alive(buf, x + kCorner[i][0], y + kCorner[i][1], z + kCorner[i][2], X, Y, Z, wrap, maxCS);
    if (cur == maxCS) return (n > 0u && ((survival >> (n - 1u)) & 1u)) ? maxCS : cur - 1u;
    if (cur == 0u) return (n > 0u && ((birth >> (n - 1u)) & 1u)) ? maxCS : 0u;
    return cur - 1u;
}

/* One tick of rayMarchCompute.slang:211-280 computeMain with compute skip disabled, over
 * every texel; elements outside the texel grid (block padding) are written as 0. When skip
 * is given it receives the skip grid the shader scatter-writes for the next frame
 * (:182-205, chunk size 8, neighbour reach 1 per axis; chunk indices are clamped, not
 * wrapped), cleared first as computeSystem.cpp:198-250 does. */
void oracle_render_step(uint32_t X, uint32_t Y, uint32_t Z, const uint64_t params[3], int wrap, const uint32_t *in,
                        uint32_t *out, uint32_t *skip) {
    const uint32_t maxCS = (uint32_t)(params[0] >> 60) + 1u;
    const uint64_t birth = params[0] & PERM_MASK, survival = params[1] & PERM_MASK;
    const uint32_t flags = (uint32_t)(params[1] >> 60);
    const uint32_t W = (X + 1u) / 2u;
    const uint32_t sdx = (X + 7u) / 8u, sdy = (Y + 7u) / 8u, sdz = (Z + 7u) / 8u;
    memset(out, 0, sizeof(uint32_t) * oracle_render_elements(X, Y, Z));
    if (skip) memset(skip, 0, sizeof(uint32_t) * oracle_render_skip_elements(X, Y, Z));
    for (uint32_t tz = 0; tz < Z; tz++)
        for (uint32_t ty = 0; ty < Y; ty++)
            for (uint32_t tx = 0; tx < W; tx++) {
                const uint32_t packed = in[oracle_render_index(tx, ty, tz, X, Y, Z)];
                const int xa = (int)(2u * tx), xb = xa + 1;
                const int bvalid = xb < (int)X;
                const uint32_t na = render_simulate(in, xa, (int)ty, (int)tz, X, Y, Z, wrap, packed & 0xFu, maxCS,
                                                    survival, birth, flags);
                const uint32_t nbv = bvalid ? render_simulate(in, xb, (int)ty, (int)tz, X, Y, Z, wrap,
                                                              (packed >> 4) & 0xFu, maxCS, survival, birth, flags)
                                            : 0u;
                out[oracle_render_index(tx, ty, tz, X, Y, Z)] = (nbv << 4) | (na & 0xFu);
                if (!skip) continue;
                for (int c = 0; c < 2; c++) {
                    const int x = c ? xb : xa;
                    if ((c ? nbv : na) == 0u || (c && !bvalid)) continue;
                    int lo[3] = {x - 1, (int)ty - 1, (int)tz - 1}, hi[3] = {x + 1, (int)ty + 1, (int)tz + 1};
                    const int dim[3] = {(int)sdx, (int)sdy, (int)sdz};
                    for (int a = 0; a < 3; a++) {
                        lo[a] = lo[a] < 0 ? 0 : lo[a] / 8;  /* floor for lo >= 0; clamp(-1 / 8) to 0 */
                        hi[a] = hi[a] / 8;
                        if (hi[a] > dim[a] - 1) hi[a] = dim[a] - 1;
                    }
                    for (int k = lo[2]; k <= hi[2]; k++)
                        for (int j = lo[1]; j <= hi[1]; j++)
                            for (int i = lo[0]; i <= hi[0]; i++) {
                                const uint32_t nbx = (sdx + 7u) / 8u, nby = (sdy + 7u) / 8u;
                                const uint64_t block = (uint64_t)((uint32_t)k / 8u) * nbx * nby +
                                                       (uint64_t)((uint32_t)j / 8u) * nbx + ((uint32_t)i / 8u);
                                const uint32_t m = expand_bits3((uint32_t)i % 8u) |
                                                   (expand_bits3((uint32_t)j % 8u) << 1u) |
                                                   (expand_bits3((uint32_t)k % 8u) << 2u);
                                skip[block * 512u + m] = 1u;
                            }
                }
            }
}
