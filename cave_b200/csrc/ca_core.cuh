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
//   centre row (y,z)           : faces along x (dx=+-1)
//   face rows (y+-1,z),(y,z+-1): face (dx=0) + edges (dx=+-1)
//   diagonal rows (y+-1,z+-1)  : edge (dx=0) + corners (dx=+-1)
// For neighbourhoods that contain faces the centre row contributes H = L+A+R, so Bn counts
// the cell itself when it is alive; the survival table is shifted one more place for that
// case (Bn = n + 1 for an alive cell), so no subtraction is needed anywhere.
#pragma once
#include "cave_stdint.h"

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
        const uint32_t x = i < NA ? a[i] : 0u, y = i < NB ? b[i] : 0u, z = i < NC ? c[i] : 0u;
        s[i] = xor3(x, y, z);
        k[i] = maj3(x, y, z);
    }
    s[N] = 0u;
    k[N] = 0u;
    // out = s + 2k
    uint32_t carry = 0u;
#pragma unroll
    for (int i = 0; i < NO; i++) {
        const uint32_t x = i <= N ? s[i] : 0u;
        const uint32_t y = (i >= 1 && i - 1 <= N) ? k[i - 1] : 0u;
        if (i == 0) {
            out[0] = x;
        } else {
            out[i] = xor3(x, y, carry);
            carry = maj3(x, y, carry);
        }
    }
}

// ---------------------------------------------------------------- rules
// Table bit `lut[k]` at count k = (c[0..BIT]) + LO, for counts up to MAXC: a mux tree over the
// count planes whose branches above MAXC are left out -- a count there never occurs, so a
// subtree whose upper half lies wholly above MAXC is its lower half alone: MAXC logic operations
// per table (lut_tree_ops) instead of 2^bits - 1, e.g. FE 19 instead of 31, C 8 instead of 15.
template <int BIT, int LO, int MAXC>
__device__ __forceinline__ uint32_t lut_tree_bounded(const uint32_t* c, uint32_t lut) {
    if constexpr (BIT < 0) {
        return 0u - ((lut >> LO) & 1u);
    } else if constexpr (LO + (1 << BIT) > MAXC) {
        return lut_tree_bounded<BIT - 1, LO, MAXC>(c, lut);
    } else {
        const uint32_t hi = lut_tree_bounded<BIT - 1, LO + (1 << BIT), MAXC>(c, lut);
        const uint32_t lo = lut_tree_bounded<BIT - 1, LO, MAXC>(c, lut);
        return (c[BIT] & hi) | (~c[BIT] & lo);
    }
}

// (survive-hit, birth-hit) planes for count planes c. NT = number of sparse terms the rule
// was built with (1..kMaxTerms), or 0 for the mux-tree evaluation of the two tables; MAXC = the
// largest count the planes can hold (the tree leaves out the branches above it).
template <int NBITS, int NT, int MAXC = (1 << NBITS) - 1>
__device__ __forceinline__ void eval_rule(const uint32_t* c, const DeviceRule& r, uint32_t& hs, uint32_t& hb) {
    if constexpr (NT > 0) {
        uint32_t as = 0u, ab = 0u;
#pragma unroll
        for (int t = 0; t < NT; t++) {
            const RuleTerm& T = r.terms[t];
            uint32_t e = (c[0] ^ T.nk[0]) & (c[1] ^ T.nk[1]) & (c[2] ^ T.nk[2]);
            if constexpr (NBITS > 3) e &= (c[3] ^ T.nk[3]);
            if constexpr (NBITS > 4) e &= (c[4] ^ T.nk[4]);
            as |= e & T.sm;
            ab |= e & T.bm;
        }
        hs = as;
        hb = ab;
    } else {
        hs = lut_tree_bounded<NBITS - 1, 0, MAXC>(c, r.lut_s);
        hb = lut_tree_bounded<NBITS - 1, 0, MAXC>(c, r.lut_b);
    }
}

// ---------------------------------------------------------------- per-row terms
__device__ __forceinline__ uint32_t alive_plane(uint4 s, const DeviceRule& r) {
    const uint32_t d = (s.x ^ r.m[0]) | (s.y ^ r.m[1]) | (s.z ^ r.m[2]) | (s.w ^ r.m[3]);
    return ~d & r.alive_ok;
}

// Sums of one strip of one row, formed once when the row is read: a = alive bits,
// h = l + a + r (2 planes), lr = l + r (2 planes), with l/r the x-1 / x+1 alive bits.
struct Row {
    uint32_t a, h0, h1, lr0, lr1;
};

__device__ __forceinline__ Row make_row(uint32_t a, uint32_t a_left, uint32_t a_right) {
    const uint32_t l = __funnelshift_l(a_left, a, 1);   // bit j = alive(x-1)
    const uint32_t r = __funnelshift_r(a, a_right, 1);  // bit j = alive(x+1)
    Row w;
    w.a = a;
    w.h0 = xor3(l, a, r);
    w.h1 = maj3(l, a, r);
    w.lr0 = l ^ r;
    w.lr1 = l & r;
    return w;
}

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
        const uint32_t h[2] = {c.h0, c.h1}, am[1] = {m.a}, ap[1] = {p.a};
        add3<2, 1, 1, 3>(h, am, ap, pc);
        ps[0] = c.a;
    }
};
template <> struct Partials<2> {  // E: face rows LR, diagonal rows A
    static constexpr int NC = 3, NS = 3;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        const uint32_t lm[2] = {m.lr0, m.lr1}, lp[2] = {p.lr0, p.lr1}, lc[2] = {c.lr0, c.lr1}, z[1] = {0u};
        add3<2, 2, 1, 3>(lm, lp, z, pc);
        const uint32_t am[1] = {m.a}, ap[1] = {p.a};
        add3<2, 1, 1, 3>(lc, am, ap, ps);
    }
};
template <> struct Partials<3> {  // FE: centre H, face rows H, diagonal rows A
    static constexpr int NC = 4, NS = 3;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        const uint32_t hm[2] = {m.h0, m.h1}, hc[2] = {c.h0, c.h1}, hp[2] = {p.h0, p.h1};
        add3<2, 2, 2, 4>(hm, hc, hp, pc);
        const uint32_t am[1] = {m.a}, ap[1] = {p.a};
        add3<2, 1, 1, 3>(hc, am, ap, ps);
    }
};
template <> struct Partials<4> {  // C: diagonal rows LR
    static constexpr int NC = 1, NS = 3;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        const uint32_t lm[2] = {m.lr0, m.lr1}, lp[2] = {p.lr0, p.lr1}, z[1] = {0u};
        add3<2, 2, 1, 3>(lm, lp, z, ps);
        pc[0] = 0u;
    }
};
template <> struct Partials<5> {  // FC: centre H, face rows A, diagonal rows LR
    static constexpr int NC = 3, NS = 3;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        const uint32_t hc[2] = {c.h0, c.h1}, am[1] = {m.a}, ap[1] = {p.a};
        add3<2, 1, 1, 3>(hc, am, ap, pc);
        const uint32_t lm[2] = {m.lr0, m.lr1}, lp[2] = {p.lr0, p.lr1}, ac[1] = {c.a};
        add3<2, 2, 1, 3>(lm, lp, ac, ps);
    }
};
template <> struct Partials<6> {  // EC: face rows LR, diagonal rows H
    static constexpr int NC = 3, NS = 4;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        const uint32_t lm[2] = {m.lr0, m.lr1}, lp[2] = {p.lr0, p.lr1}, lc[2] = {c.lr0, c.lr1}, z[1] = {0u};
        add3<2, 2, 1, 3>(lm, lp, z, pc);
        const uint32_t hm[2] = {m.h0, m.h1}, hp[2] = {p.h0, p.h1};
        add3<2, 2, 2, 4>(lc, hm, hp, ps);
    }
};
template <> struct Partials<7> {  // FEC: every row H (pc == ps)
    static constexpr int NC = 4, NS = 4;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        const uint32_t hm[2] = {m.h0, m.h1}, hc[2] = {c.h0, c.h1}, hp[2] = {p.h0, p.h1};
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

// Column sums of the FEC neighbourhood kept in carry-save form: the column's three H summed by
// two full adders and left unresolved, its sum (at most 9) being pc[0] + 2 (pc[1] + pc[2]) +
// 4 pc[3]; combine resolves three such columns at once (4 + 16 logic operations per strip
// against 8 + 15 for Partials<7> and combine<7>). Used by the rule-specialised tick kernels,
// where it measured faster; the generic kernels measured slower with it and keep Partials<7>.
struct MooreCarrySave {
    static constexpr int NC = 4, NS = 4;
    __device__ static void make(const Row& m, const Row& c, const Row& p, uint32_t* pc, uint32_t* ps) {
        pc[0] = xor3(m.h0, c.h0, p.h0);  // weight 1
        pc[1] = maj3(m.h0, c.h0, p.h0);  // weight 2
        pc[2] = xor3(m.h1, c.h1, p.h1);  // weight 2
        pc[3] = maj3(m.h1, c.h1, p.h1);  // weight 4
#pragma unroll
        for (int i = 0; i < 4; i++) ps[i] = pc[i];
    }
    // Three columns into the binary count (at most 27) with eight full adders and one half
    // adder: the bits of each weight are reduced in threes and their carries passed up.
    __device__ static void combine(const uint32_t* c, const uint32_t* m, const uint32_t* p, uint32_t* cnt) {
        cnt[0] = xor3(c[0], m[0], p[0]);  // weight 1: 3 bits
        const uint32_t c1 = maj3(c[0], m[0], p[0]);
        const uint32_t sa = xor3(c[1], c[2], m[1]), ka = maj3(c[1], c[2], m[1]);  // weight 2: 6 bits + carry
        const uint32_t sb = xor3(m[2], p[1], p[2]), kb = maj3(m[2], p[1], p[2]);
        cnt[1] = xor3(sa, sb, c1);
        const uint32_t kc = maj3(sa, sb, c1);
        const uint32_t sd = xor3(c[3], m[3], p[3]), k1 = maj3(c[3], m[3], p[3]);  // weight 4: 3 bits + 3 carries
        const uint32_t se = xor3(ka, kb, kc), k2 = maj3(ka, kb, kc);
        cnt[2] = sd ^ se;
        const uint32_t k3 = sd & se;
        cnt[3] = xor3(k1, k2, k3);  // weight 8: 3 carries
        cnt[4] = maj3(k1, k2, k3);  // weight 16
    }
};

// The column-sum policy of a kernel: P::make and P::combine.
template <int NB> struct BinaryColumns : Partials<NB> {
    __device__ static void combine(const uint32_t* pc, const uint32_t* psm, const uint32_t* psp, uint32_t* cnt) {
        cave::combine<NB>(pc, psm, psp, cnt);
    }
};
template <int NB, bool kCarrySave> struct ColumnsFor { using type = BinaryColumns<NB>; };
template <> struct ColumnsFor<7, true> { using type = MooreCarrySave; };

// ---------------------------------------------------------------- state update + stats
// acc + v as an integer multiply-add by `one`, so that the add issues on the FMA pipe instead of
// the integer ALU, which the cell logic keeps busy. `one` must be 1 at run time in a way the
// compiler cannot see (it would fold the product back into an add on the ALU).
__device__ __forceinline__ uint32_t mad_add(uint32_t acc, uint32_t v, uint32_t one) {
    uint32_t r;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(v), "r"(one), "r"(acc));
    return r;
}

struct TickAcc {  // per-thread accumulators for one tick
    uint32_t surviving, born, zero, population;
    uint32_t zmin, zmax;  // z-extent of the thread's non-zero strips
    uint32_t one;         // 1, opaque to the compiler (see mad_add)
    __device__ void reset(uint32_t opaque_one = 1u) {
        surviving = born = zero = population = 0u;
        zmin = 0xFFFFFFFFu;
        zmax = 0u;
        one = opaque_one;
    }
};

// New state of one strip. s: current state planes; a: its alive plane; valid: cells < X;
// xbits accumulates the OR of the strip's non-zero masks (its x-extent). The statistics are
// accumulated only when `count` is set (strips this thread owns, not halo copies); cells that
// were 0 only with kCountZero (a caller may derive them from the previous tick's population).
// kFullRange: the rule's alive state is 15 (all four planes set; a compile-time fact of the
// specialised kernels), which allows the shorter update below.
// kPop: where the population and bounding box come from -- kPopOutput: the strip's new state
// (the tick's own); kPopInput: its current state, i.e. the previous tick's result, whose
// non-zero mask the update computes anyway; kPopNone: not counted.
// kZPerStrip: the z-extent (acc.zmin / zmax) is updated here for this strip; otherwise the
// counted non-zero mask is ORed into *zany and the caller updates the extent once per plane.
enum : int { kPopNone = 0, kPopOutput = 1, kPopInput = 2 };
template <int NB, int NT, bool kCountZero = true, bool kFullRange = false, int kPop = kPopOutput,
          bool kZPerStrip = true>
__device__ __forceinline__ uint4 update_strip(uint4 s, uint32_t a, const uint32_t* cnt, uint32_t valid,
                                              const DeviceRule& r, TickAcc& acc, uint32_t& xbits, uint32_t z,
                                              bool count = true, uint32_t* zany = nullptr) {
    uint32_t hs, hb;
    eval_rule<count_bits(NB), NT, max_count(NB)>(cnt, r, hs, hb);
    const uint32_t nz = s.x | s.y | s.z | s.w;
    const uint32_t zero = ~nz & valid;
    const uint32_t sv = a & hs;
    const uint32_t bn = zero & hb;
    const uint32_t b2 = ~s.x & ~s.y;
    const uint32_t b3 = b2 & ~s.z;
    uint4 n;
    if constexpr (kFullRange) {
        // Alive state 15. A born cell (state 0) becomes 15 = 0 - 1 in four bits, so the borrow
        // chain of the decrement runs on every cell of t = non-zero or born; a surviving cell
        // (15) decrements to 14 and gets its low bit back from sv; every other cell is
        // s - 1, or stays 0 outside t.
        const uint32_t t = nz | bn;
        n.x = sv | (t & ~s.x);
        n.z = t & (s.z ^ b2);
        n.w = t & (s.w ^ b3);
        n.y = (s.x & s.y) | (~s.x & ~s.y & t);
    } else {
        // d = s - 1 for non-zero cells, 0 for zero cells (borrow chain masked by nz); then each
        // plane is set ? bit of maxcs : d (one 3-input select per plane)
        const uint32_t set = sv | bn;
        const uint32_t d0 = nz & ~s.x;
        const uint32_t d1 = nz & ~(s.y ^ s.x);
        const uint32_t d2 = nz & (s.z ^ b2);
        const uint32_t d3 = nz & (s.w ^ b3);
        n.x = (set & r.m[0]) | (~set & d0);
        n.y = (set & r.m[1]) | (~set & d1);
        n.z = (set & r.m[2]) | (~set & d2);
        n.w = (set & r.m[3]) | (~set & d3);
    }
    if (count) {
        acc.surviving = mad_add(acc.surviving, __popc(sv), acc.one);
        acc.born = mad_add(acc.born, __popc(bn), acc.one);
        if constexpr (kCountZero) acc.zero = mad_add(acc.zero, __popc(zero), acc.one);
        if constexpr (kPop != kPopNone) {
            const uint32_t nn = kPop == kPopInput ? nz : (n.x | n.y | n.z | n.w);
            acc.population = mad_add(acc.population, __popc(nn), acc.one);
            xbits |= nn;
            if constexpr (kZPerStrip) {
                const bool any = nn != 0u;
                acc.zmin = any ? min(acc.zmin, z) : acc.zmin;
                acc.zmax = any ? max(acc.zmax, z) : acc.zmax;
            } else {
                *zany |= nn;
            }
        }
    }
    return n;
}

}  // namespace cave
