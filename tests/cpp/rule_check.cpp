// Checks the rule compiler (cave::make_device_rule, rules.cpp) on the host: for random and edge
// rules over every neighbourhood and state count, the DeviceRule the kernels consume must give,
// for every neighbour count n a cell can see, the reference's decision
// (searchSimulationCube.slang:163-216): an alive cell survives iff n > 0 and survival bit n-1 is
// set; a dead cell is born iff n > 0 and birth bit n-1 is set. The kernels evaluate the count
// their row sums give -- n, plus 1 for an alive cell when faces are in the neighbourhood (the
// centre row's sum includes the cell) -- through the sparse terms when the rule has them (each
// term matches one count on the count's low count_bits(nb) bits; ca_core.cuh eval_rule) and
// through the two tables otherwise (the mux tree returns the table bit of the count). Also:
// the alive-state masks m[] and alive_ok, the term limit, and that nothing above the
// neighbourhood's largest count is set. Needs no GPU. Exit status 0 = every check held.
#include <cstdint>
#include <cstdio>
#include <random>

#include "rules.h"

namespace {
int neighbours(uint32_t nb) { return ((nb & 1) ? 6 : 0) + ((nb & 2) ? 12 : 0) + ((nb & 4) ? 8 : 0); }

// (survive, birth) decision of the DeviceRule for row-sum count c, as the kernels take it
void device_decision(const cave::DeviceRule& r, uint32_t nb, uint32_t c, bool& s, bool& b) {
    if (r.nterms > 0) {
        const int bits = cave::count_bits((int)nb);
        s = b = false;
        for (uint32_t t = 0; t < r.nterms; t++) {
            const cave::RuleTerm& T = r.terms[t];
            bool match = true;
            for (int i = 0; i < bits; i++) match = match && ((((c >> i) & 1u) ^ (T.nk[i] & 1u)) == 1u);
            s = s || (match && T.sm);
            b = b || (match && T.bm);
        }
    } else {
        s = (r.lut_s >> c) & 1u;
        b = (r.lut_b >> c) & 1u;
    }
}

int check(const cave::DecodedRule& d) {
    const cave::DeviceRule r = cave::make_device_rule(d);
    const uint32_t nb = d.flags & 7u;
    const uint32_t m = d.maxcs & 0xFu;
    bool ok = r.maxcs == d.maxcs && r.flags == nb && r.nterms <= (uint32_t)cave::kMaxSparseTerms &&
              r.alive_ok == (d.maxcs <= 15 ? 0xFFFFFFFFu : 0u);
    for (int i = 0; i < 4; i++) ok = ok && r.m[i] == (((m >> i) & 1u) ? 0xFFFFFFFFu : 0u);
    const uint32_t maxc = (uint32_t)cave::max_count((int)nb);
    ok = ok && (maxc >= 31 || ((r.lut_s | r.lut_b) >> (maxc + 1)) == 0);
    const int N = neighbours(nb);
    for (int n = 0; n <= N && ok; n++) {
        const bool want_s = n > 0 && ((d.survival >> (n - 1)) & 1u);
        const bool want_b = n > 0 && ((d.birth >> (n - 1)) & 1u);
        bool s = false, b = false, s2 = false, b2 = false;
        device_decision(r, nb, (uint32_t)n + (cave::counts_self((int)nb) ? 1u : 0u), s, b2);  // alive cell
        device_decision(r, nb, (uint32_t)n, s2, b);                                            // dead cell
        ok = s == want_s && b == want_b;
        if (!ok)
            std::printf("maxcs %u flags %u birth %llx survival %llx: n %d survive %d/%d birth %d/%d (terms %u)\n",
                        d.maxcs, d.flags, (unsigned long long)d.birth, (unsigned long long)d.survival, n, s, want_s,
                        b, want_b, r.nterms);
    }
    if (!ok && r.nterms == 0) std::printf("  tables s %x b %x\n", r.lut_s, r.lut_b);
    return ok ? 0 : 1;
}
}  // namespace

int main() {
    std::mt19937_64 rng(2024);
    int n = 0;
    for (uint32_t flags = 0; flags < 16; flags++)
        for (uint32_t maxcs = 1; maxcs <= 16; maxcs++) {
            // edge rules: empty, full, single counts, the highest counts
            const uint64_t edge[] = {0, (1ull << 26) - 1, 1, 1ull << 5, 1ull << 17, 1ull << 25, ~0ull >> 4, 0x5555555};
            for (uint64_t bm : edge)
                for (uint64_t sm : edge) {
                    n++;
                    if (check(cave::DecodedRule{maxcs, flags, bm, sm})) return 1;
                }
            for (int i = 0; i < 400; i++, n++) {
                // sparse rules (1..4 counts each) half of the time, dense 27-bit masks otherwise
                auto draw = [&]() -> uint64_t {
                    if (rng() & 1) return rng() & ((1ull << 27) - 1);
                    uint64_t v = 0;
                    for (int k = 1 + (int)(rng() % 4); k > 0; k--) v |= 1ull << (rng() % 26);
                    return v;
                };
                if (check(cave::DecodedRule{maxcs, flags, draw(), draw()})) return 1;
            }
        }
    std::printf("ok %d rules\n", n);
    return 0;
}
