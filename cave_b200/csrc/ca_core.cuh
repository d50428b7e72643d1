// ca_core.cuh -- bit-sliced arithmetic of one CA tick, shared by every sm_100a kernel.
//
// Reference semantics (shaders/slang/search/searchSimulationCube.slang:117-247):
//   * a neighbour is alive iff its state == maxCellState (:78-94); outside the grid is dead;
//   * alive cell: survives (stays maxCS) iff n > 0 and survival bit (n-1) is set, else -> maxCS-1;
//   * state 0: born (-> maxCS) iff n > 0 and birth bit (n-1) is set, else stays 0;
//   * any other state s -> s-1;
//   * counters: dead (0 stays 0), dying (every decrement), born, surviving (:178-211).
//
// Layout used here (the "strip" layout): a strip is 32 consecutive cells of one x-row held as
// four 32-bit bit-planes (uint4 .x = bit 0 of every cell's state ... .w = bit 3); bit j of a
// plane is cell x = 32*strip + j. A row has SX = ceil(X/32) strips; strip index
// = sx + y*SX + z*SX*Y. Cells past X are kept at state 0.
//
// Neighbour counting is done on alive bit-planes with full adders (XOR3 / MAJ, one LOP3
// each). The count is formed as Bn = sum over the 3x3 (y,z) rows of per-row terms, with
// the reference's delta sets (cube.slang:7-21) split by row class:
//   centre row (y,z)        : faces along x            -> L+R
//   face rows (y+-1,z),(y,z+-1): face (dx=0) + edges (dx=+-1)
//   diagonal rows (y+-1,z+-1)  : edge (dx=0) + corners (dx=+-1)
// For neighbourhoods that contain faces the centre row contributes H = L+A+R, so Bn counts
// the cell itself when it is alive; the survival table is shifted one more place for that
// case (Bn = n + 1 for an alive cell), so no subtraction is needed anywhere.
#pragma once
#include <cstdint>

#include "ca_types.h"

namespace cave {

// ---------------------------------------------------------------- bit-sliced adders
__device__ __forceinline__ uint32_t xor3(uint32_t a, uint32_t b, uint32_t c) { return a ^ b ^ c; }
__device__ __forceinline__ uint32_t maj3(uint32_t a, uint32_t b, uint32_t c) { return (a & b) | (c & (a | b)); }

// out[0..NO) = a + b + c (bit-sliced, LSB first). Widths are compile-time; the caller
// guarantees the true sum fits in NO bits. Missing input planes are zero.
template <int NA, int NB, int NC, int NO>
__device__ __forceinline__ void add3(const uint32_t* a, const uint32_t* b, const uint32_t* c, uint32_t* out) {
    constexpr int N = (NA > NB ? (NA > NC ? NA : NC) : (NB > NC ? NB : NC));
    uint32_t s[N + 1], k[N + 1];
#pragma unroll
    for (int i = 0; i < N; i++) {
        uint32_t x = i < NA ? a[i] : 0u, y = i < NB ? b[i] : 0u, z = i < NC ? c[i] : 0u;
        s[i] = xor3(x, y, z);
        k[i] = maj3(x, y, z);
    }
    s[N] = 0u;
    k[N] = 0u;
    // out = s + 2k
    uint32_t carry = 0u;
#pragma unroll
    for (int i = 0; i < NO; i++) {
        uint32_t x = i <= N ? s[i] : 0u;
        uint32_t y = (i >= 1 && i - 1 <= N) ? k[i - 1] : 0u;
        if (i == 0) {
            out[0] = x;
        } else {
            out[i] = xor3(x, y, carry);
            carry = maj3(x, y, carry);
        }
    }
}

// ---------------------------------------------------------------- rules
// LUT evaluation by a mux tree over the count planes; leaves are the table bits.
template <int NBITS>
__device__ __forceinline__ uint32_t lut_tree(const uint32_t* c, uint32_t lut) {
    constexpr int NL = 1 << NBITS;
    uint32_t v[NL / 2];
#pragma unroll
    for (int j = 0; j < NL / 2; j++) {
        uint32_t t0 = 0u - ((lut >> (2 * j)) & 1u);
        uint32_t t1 = 0u - ((lut >> (2 * j + 1)) & 1u);
        v[j] = (c[0] & t1) | (~c[0] & t0);
    }
#pragma unroll
    for (int lvl = 1; lvl < NBITS; lvl++) {
#pragma unroll
        for (int j = 0; j < (NL >> (lvl + 1)); j++) v[j] = (c[lvl] & v[2 * j + 1]) | (~c[lvl] & v[2 * j]);
    }
    return v[0];
}

// (survive-hit, birth-hit) planes for count planes c.
template <int NBITS, bool SPARSE>
__device__ __forceinline__ void eval_rule(const uint32_t* c, const DeviceRule& r, uint32_t& hs, uint32_t& hb) {
    if constexpr (SPARSE) {
        uint32_t as = 0u, ab = 0u;
#pragma unroll
        for (int t = 0; t < kMaxTerms; t++) {
            if (t < (int)r.nterms) {
                const RuleTerm& T = r.terms[t];
                uint32_t e = (c[0] ^ T.nk[0]) & (c[1] ^ T.nk[1]) & (c[2] ^ T.nk[2]);
                if (NBITS > 3) e &= (c[3] ^ T.nk[3]);
                if (NBITS > 4) e &= (c[4] ^ T.nk[4]);
                as |= e & T.sm;
                ab |= e & T.bm;
            }
        }
        hs = as;
        hb = ab;
    } else {
        hs = lut_tree<NBITS>(c, r.lut_s);
        hb = lut_tree<NBITS>(c, r.lut_b);
    }
}

// ---------------------------------------------------------------- per-row terms
__device__ __forceinline__ uint32_t alive_plane(uint4 s, const DeviceRule& r) {
    uint32_t d = (s.x ^ r.m[0]) | (s.y ^ r.m[1]) | (s.z ^ r.m[2]) | (s.w ^ r.m[3]);
    return ~d & r.alive_ok;
}

struct Row {           // alive bits and their x-neighbours for one strip of one row
    uint32_t a, l, r;  // l: bit j = alive(x-1), r: bit j = alive(x+1)
};

// H = l + a + r  (2 planes), LR = l + r (2 planes)
__device__ __forceinline__ void hsum(const Row& w, uint32_t* h) { h[0] = xor3(w.l, w.a, w.r); h[1] = maj3(w.l, w.a, w.r); }
__device__ __forceinline__ void lrsum(const Row& w, uint32_t* h) { h[0] = w.l ^ w.r; h[1] = w.l & w.r; }

// Column partial sums for neighbourhood NB from the column's rows at z-1 (m), z (c), z+1 (p):
//   pc: contribution when this column is the output's own column
//   ps: contribution when this column is a y-neighbour column (y-1 or y+1)
template <int NB> struct Partials;

template <> struct Partials<0> {  // no neighbourhood selected: every count is 0
    static constexpr int NC = 1, NS = 1;
    __device__ static void make(const Row&, const Row&, const Row&, uint32_t* pc, uint32_t* ps) {
        pc[0] = 0u;
        ps[0] = 0u;
    }
};

template <> struct Partials<1> {  // F: centre H, face rows A
    static constexpr int NC = 3, NS = 1;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        uint32_t h[2]; hsum(c, h);
        uint32_t am[1] = {m.a}, ap[1] = {p.a};
        add3<2, 1, 1, 3>(h, am, ap, pc);
        ps[0] = c.a;
    }
};
template <> struct Partials<2> {  // E: face rows LR, diagonal rows A
    static constexpr int NC = 3, NS = 3;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        uint32_t lm[2], lp[2], lc[2]; lrsum(m, lm); lrsum(p, lp); lrsum(c, lc);
        uint32_t z[1] = {0u};
        add3<2, 2, 1, 3>(lm, lp, z, pc);
        uint32_t am[1] = {m.a}, ap[1] = {p.a};
        add3<2, 1, 1, 3>(lc, am, ap, ps);
    }
};
template <> struct Partials<3> {  // FE: centre H, face rows H, diagonal rows A
    static constexpr int NC = 4, NS = 3;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        uint32_t hm[2], hc[2], hp[2]; hsum(m, hm); hsum(c, hc); hsum(p, hp);
        add3<2, 2, 2, 4>(hm, hc, hp, pc);
        uint32_t am[1] = {m.a}, ap[1] = {p.a};
        add3<2, 1, 1, 3>(hc, am, ap, ps);
    }
};
template <> struct Partials<4> {  // C: diagonal rows LR
    static constexpr int NC = 1, NS = 3;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        uint32_t lm[2], lp[2]; lrsum(m, lm); lrsum(p, lp);
        uint32_t z[1] = {0u};
        add3<2, 2, 1, 3>(lm, lp, z, ps);
        pc[0] = 0u;
    }
};
template <> struct Partials<5> {  // FC: centre H, face rows A, diagonal rows LR
    static constexpr int NC = 3, NS = 3;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        uint32_t hc[2]; hsum(c, hc);
        uint32_t am[1] = {m.a}, ap[1] = {p.a};
        add3<2, 1, 1, 3>(hc, am, ap, pc);
        uint32_t lm[2], lp[2]; lrsum(m, lm); lrsum(p, lp);
        uint32_t ac[1] = {c.a};
        add3<2, 2, 1, 3>(lm, lp, ac, ps);
    }
};
template <> struct Partials<6> {  // EC: face rows LR, diagonal rows H
    static constexpr int NC = 3, NS = 4;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        uint32_t lm[2], lp[2], lc[2]; lrsum(m, lm); lrsum(p, lp); lrsum(c, lc);
        uint32_t z[1] = {0u};
        add3<2, 2, 1, 3>(lm, lp, z, pc);
        uint32_t hm[2], hp[2]; hsum(m, hm); hsum(p, hp);
        add3<2, 2, 2, 4>(lc, hm, hp, ps);
    }
};
template <> struct Partials<7> {  // FEC: every row H (pc == ps)
    static constexpr int NC = 4, NS = 4;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        uint32_t hm[2], hc[2], hp[2]; hsum(m, hm); hsum(c, hc); hsum(p, hp);
        add3<2, 2, 2, 4>(hm, hc, hp, pc);
#pragma unroll
        for (int i = 0; i < 4; i++) ps[i] = pc[i];
    }
};

// Bn = pc(y) + ps(y-1) + ps(y+1), in count_bits(NB) planes.
template <int NB>
__device__ __forceinline__ void combine(const uint32_t* pc, const uint32_t* psm, const uint32_t* psp, uint32_t* cnt) {
    using P = Partials<NB>;
    add3<P::NC, P::NS, P::NS, count_bits(NB)>(pc, psm, psp, cnt);
}

// ---------------------------------------------------------------- state update + stats
struct TickAcc {  // per-thread accumulators for one tick
    uint32_t surviving, born, zero, population;
    uint32_t bmin[3], bmax[3];
    __device__ void reset() {
        surviving = born = zero = population = 0u;
        bmin[0] = bmin[1] = bmin[2] = 0xFFFFFFFFu;
        bmax[0] = bmax[1] = bmax[2] = 0u;
    }
};

// New state of one strip. s: current state planes; a: its alive plane; valid: cells < X.
template <int NB, bool SPARSE>
__device__ __forceinline__ uint4 update_strip(uint4 s, uint32_t a, const uint32_t* cnt, uint32_t valid,
                                              const DeviceRule& r, TickAcc& acc, uint32_t x0, uint32_t y,
                                              uint32_t z) {
    uint32_t hs, hb;
    eval_rule<count_bits(NB), SPARSE>(cnt, r, hs, hb);
    const uint32_t nz = s.x | s.y | s.z | s.w;
    const uint32_t zero = ~nz & valid;
    const uint32_t sv = a & hs;
    const uint32_t bn = zero & hb;
    const uint32_t set = sv | bn;
    const uint32_t keep = nz & ~set;
    // s - 1 for non-zero cells (borrow chain), maxcs where set, 0 for dead cells
    const uint32_t b1 = ~s.x;
    const uint32_t b2 = b1 & ~s.y;
    const uint32_t b3 = b2 & ~s.z;
    uint4 n;
    n.x = (set & r.m[0]) | (keep & ~s.x);
    n.y = (set & r.m[1]) | (keep & (s.y ^ b1));
    n.z = (set & r.m[2]) | (keep & (s.z ^ b2));
    n.w = (set & r.m[3]) | (keep & (s.w ^ b3));
    acc.surviving += __popc(sv);
    acc.born += __popc(bn);
    acc.zero += __popc(zero);
    const uint32_t nn = n.x | n.y | n.z | n.w;
    if (nn) {
        acc.population += __popc(nn);
        const uint32_t lo = x0 + (uint32_t)(__ffs(nn) - 1);
        const uint32_t hi = x0 + 31u - (uint32_t)__clz(nn);
        acc.bmin[0] = min(acc.bmin[0], lo);
        acc.bmax[0] = max(acc.bmax[0], hi);
        acc.bmin[1] = min(acc.bmin[1], y);
        acc.bmax[1] = max(acc.bmax[1], y);
        acc.bmin[2] = min(acc.bmin[2], z);
        acc.bmax[2] = max(acc.bmax[2], z);
    }
    return n;
}

// x-neighbour words for the alive plane of a strip, given the neighbouring strips' planes.
__device__ __forceinline__ Row make_row(uint32_t a, uint32_t a_left, uint32_t a_right) {
    Row w;
    w.a = a;
    w.l = (a << 1) | (a_left >> 31);
    w.r = (a >> 1) | (a_right << 31);
    return w;
}

}  // namespace cave
