// ca_types.h -- rule and geometry types shared by host code and the sm_100a kernels.
#pragma once
#include "cave_stdint.h"

#if defined(__CUDACC__)
#define CAVE_HD __host__ __device__
#else
#define CAVE_HD
#endif

namespace cave {

// One count value k that appears in the survival or birth table (sparse rule evaluation).
struct RuleTerm {
    uint32_t nk[5];    // nk[i] = ~0 if bit i of k is 0 else 0 (so (c_i ^ nk_i) is 1 where c_i == k_i)
    uint32_t sm, bm;   // ~0 if k is in lut_s / lut_b
    uint32_t pad;
};
static_assert(sizeof(RuleTerm) == 32, "RuleTerm is two 16-byte words");

// Rows per thread of the rule-specialised tick kernels (one CTA per SM: the rows' registers
// would not fit two). Several rows per thread share the per-plane work that does not depend on
// the rows (waits, barrier, loop and address arithmetic) and keep the pair's inner y-neighbours
// in registers: 512^3 tick 34.1 us at one row, 27.7 at two, 27.6 at three (256^3: 7.2 -> 6.9).
constexpr int kJitRowsPerThread = 3;
// Most threads per CTA of those kernels (their __launch_bounds__): the registers of
// kJitRowsPerThread rows (three: about 155) and the ring of rows x strips in shared memory must
// fit one CTA per SM.
constexpr int kJitMaxThreads = kJitRowsPerThread == 2 ? 512 : 384;
// The same for the two-tick kernels (stream_tick2.cuh), which hold two ticks' rolling rows per
// row of the thread.
#ifndef CAVE_TICK2_ROWS
#define CAVE_TICK2_ROWS 2
#endif
#ifndef CAVE_TICK2_THREADS
#define CAVE_TICK2_THREADS 384
#endif
#ifndef CAVE_TICK2_CTAS
#define CAVE_TICK2_CTAS 1
#endif
constexpr int kJit2RowsPerThread = CAVE_TICK2_ROWS;
constexpr int kJit2CtasPerSm = CAVE_TICK2_CTAS;  // CTAs per SM the kernels' registers are sized for
constexpr int kJit2MaxThreads = CAVE_TICK2_THREADS;

constexpr int kMaxTerms = 8;        // capacity of DeviceRule::terms
constexpr int kMaxSparseTerms = 4;  // the kernels' sparse evaluation handles up to this many terms

// Decoded rule for one simulation, in the form the kernels consume.
//   lut_s: bit b set  <=> an alive cell whose row-sum count is b survives
//   lut_b: bit b set  <=> a dead cell whose count is b is born
// (the reference's survival/birth masks shifted by 1, plus 1 more for an alive cell when
//  the neighbourhood contains faces, because the row sums then include the cell itself).
struct DeviceRule {
    uint32_t maxcs;        // 1..16 (16 = the encoded value 15: nothing is ever alive)
    uint32_t flags;        // neighbourhood bits F=1 E=2 C=4 (wrap bit 8 is ignored by the cube shader)
    uint32_t lut_s, lut_b;
    uint32_t m[4];         // m[i] = ~0 if bit i of maxcs is set (maxcs & 15)
    uint32_t alive_ok;     // ~0 unless maxcs == 16
    uint32_t nterms;       // number of entries in terms[] (0 => use the LUT tree)
    uint32_t pad[2];
    RuleTerm terms[kMaxTerms];
};

static_assert(sizeof(DeviceRule) % 16 == 0, "DeviceRule arrays keep 16-byte alignment (copied as uint4)");

// Count planes needed per neighbourhood (max count: F 7, E 12, FE 19, C 8, FC 15, EC 20,
// FEC 27, where the F-containing ones include the cell itself); nb = 0 counts nothing.
CAVE_HD constexpr int count_bits(int nb) {
    return nb == 0 ? 1 : nb == 1 ? 3 : (nb == 2 || nb == 4 || nb == 5) ? 4 : 5;
}
CAVE_HD constexpr bool counts_self(int nb) { return (nb & 1) != 0; }
CAVE_HD constexpr int max_count(int nb) {
    return nb == 0 ? 0 : nb == 1 ? 7 : nb == 2 ? 12 : nb == 3 ? 19 : nb == 4 ? 8 : nb == 5 ? 15 : nb == 6 ? 20 : 27;
}

// Logic operations of the rule table's mux tree for counts up to maxc (ca_core.cuh,
// lut_tree_bounded<bit, lo, maxc>): one per leaf above the first, i.e. maxc for lo = 0.
CAVE_HD constexpr int lut_tree_ops(int bit, int lo, int maxc) {
    return bit < 0 ? 0
           : lo + (1 << bit) > maxc ? lut_tree_ops(bit - 1, lo, maxc)
                                    : lut_tree_ops(bit - 1, lo + (1 << bit), maxc) + lut_tree_ops(bit - 1, lo, maxc) + 1;
}

// Valid-cell mask of strip sx in a row of X cells.
CAVE_HD inline uint32_t strip_valid(uint32_t sx, uint32_t X) {
    const uint32_t x0 = sx * 32u;
    if (x0 >= X) return 0u;
    const uint32_t n = X - x0;
    return n >= 32u ? 0xFFFFFFFFu : ((1u << n) - 1u);
}

}  // namespace cave
