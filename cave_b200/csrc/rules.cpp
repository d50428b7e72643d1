// rules.cpp -- host-side rule decoding (see rules.h).
#include "rules.h"

#include <algorithm>
#include <bit>
#include <cstring>
#include <functional>

namespace cave {

bool decode_params(const cave_sim_params& p, const uint64_t* valid, uint32_t nValid, uint32_t maxRuleBits,
                   DecodedRule& out) {
    out.maxcs = (uint32_t)(p.birthAndMaxCellStateRules >> 60) + 1u;
    out.flags = (uint32_t)(p.survivalAndNeighborhoodRules >> 60);
    if (maxRuleBits > 0) {
        const uint32_t bi = (uint32_t)(p.birthAndMaxCellStateRules & kPermMask) - 1u;
        const uint32_t si = (uint32_t)(p.survivalAndNeighborhoodRules & kPermMask) - 1u;
        if (!valid || bi >= nValid || si >= nValid) return false;
        out.birth = valid[bi];
        out.survival = valid[si];
    } else {
        out.birth = p.birthAndMaxCellStateRules & kPermMask;
        out.survival = p.survivalAndNeighborhoodRules & kPermMask;
    }
    return true;
}

DeviceRule make_device_rule(const DecodedRule& d) {
    DeviceRule r;
    std::memset(&r, 0, sizeof(r));
    const int nb = (int)(d.flags & 7u);
    r.maxcs = d.maxcs;
    r.flags = d.flags & 7u;
    const uint32_t m = d.maxcs & 0xFu;
    for (int i = 0; i < 4; i++) r.m[i] = ((m >> i) & 1u) ? 0xFFFFFFFFu : 0u;
    r.alive_ok = d.maxcs <= 15u ? 0xFFFFFFFFu : 0u;
    // Bn = n (+1 for an alive cell when faces are in the neighbourhood); rule bit (n-1)
    // applies at n >= 1, i.e. LUT bit n (+1).
    const int maxc = max_count(nb);
    const uint64_t keep = (maxc >= 63) ? ~0ull : ((1ull << (maxc + 1)) - 1ull);
    const uint64_t ls = (d.survival << (counts_self(nb) ? 2 : 1)) & keep;
    const uint64_t lb = (d.birth << 1) & keep;
    r.lut_s = (uint32_t)ls;
    r.lut_b = (uint32_t)lb;
    // Sparse evaluation costs ~9 logic ops per distinct count value; the mux tree costs one op
    // per table and reachable count (lut_tree_ops). Use whichever is cheaper.
    const uint32_t u = r.lut_s | r.lut_b;
    const int nterms = std::popcount(u);
    const int nbits = count_bits(nb);
    const int tree_cost = 2 * lut_tree_ops(nbits - 1, 0, maxc);
    if (nterms <= kMaxSparseTerms && nterms * 9 < tree_cost) {
        int t = 0;
        for (int k = 0; k < 32; k++) {
            if (!((u >> k) & 1u)) continue;
            RuleTerm& T = r.terms[t++];
            for (int i = 0; i < 5; i++) T.nk[i] = ((k >> i) & 1) ? 0u : 0xFFFFFFFFu;
            T.sm = ((r.lut_s >> k) & 1u) ? 0xFFFFFFFFu : 0u;
            T.bm = ((r.lut_b >> k) & 1u) ? 0xFFFFFFFFu : 0u;
        }
        r.nterms = (uint32_t)nterms;
        if (nterms == 0) {
            // an empty rule is cheapest as "sparse with zero terms"; mark it with one dead term
            RuleTerm& T = r.terms[0];
            for (int i = 0; i < 5; i++) T.nk[i] = 0xFFFFFFFFu;
            T.sm = T.bm = 0;
            r.nterms = 1;
        }
    } else {
        r.nterms = 0;
    }
    return r;
}

std::vector<uint64_t> enumerate_valid_bitmasks(uint32_t n, uint32_t maxBits) {
    std::vector<uint64_t> out;
    if (maxBits == 0 || n == 0) return out;
    const uint32_t eff = std::min(maxBits, n);
    std::function<void(uint64_t, uint32_t, uint32_t)> emit = [&](uint64_t acc, uint32_t start, uint32_t rem) {
        if (rem == 0) {
            if (acc) out.push_back(acc);
            return;
        }
        for (uint32_t i = start; i + rem <= n; i++) emit(acc | (1ull << i), i + 1, rem - 1);
    };
    for (uint32_t p = 1; p <= eff; p++) emit(0, 0, p);
    std::sort(out.begin(), out.end());
    return out;
}

}  // namespace cave
