// Drives the engine's device-pool allocator (cave::FreeList, engine.cpp) through seeded random
// alloc / free sequences on the host and compares it with a model: a map of the pool's 256-byte
// units, allocated first fit. Every offset must be the model's, no two live ranges may overlap,
// used() and peak() must match, and once everything is freed the whole pool must be one range
// again. Needs no GPU (the allocator is host code). Exit status 0 = every check held.
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>

#include "engine.h"

namespace {
constexpr uint64_t kUnit = 256;

struct Model {
    std::vector<uint8_t> busy;  // one entry per unit
    uint64_t used = 0, peak = 0;
    explicit Model(uint64_t units) : busy(units, 0) {}
    bool alloc(uint64_t bytes, uint64_t& off) {
        const uint64_t n = (bytes ? bytes + kUnit - 1 : kUnit) / kUnit;
        uint64_t run = 0;
        for (uint64_t u = 0; u < busy.size(); u++) {
            run = busy[u] ? 0 : run + 1;
            if (run == n) {
                const uint64_t first = u + 1 - n;
                for (uint64_t k = first; k <= u; k++) busy[k] = 1;
                off = first * kUnit;
                used += n * kUnit;
                if (used > peak) peak = used;
                return true;
            }
        }
        return false;
    }
    void free(uint64_t off, uint64_t bytes) {
        const uint64_t n = (bytes ? bytes + kUnit - 1 : kUnit) / kUnit;
        for (uint64_t k = off / kUnit; k < off / kUnit + n; k++) busy[k] = 0;
        used -= n * kUnit;
    }
};

int run(uint32_t seed, uint64_t pool_units, int steps) {
    std::mt19937_64 rng(seed);
    cave::FreeList fl;
    fl.reset(pool_units * kUnit);
    Model m(pool_units);
    struct Live {
        uint64_t off, bytes;
    };
    std::vector<Live> live;
    for (int i = 0; i < steps; i++) {
        const bool do_alloc = live.empty() || (rng() % 100) < 55;
        if (do_alloc) {
            // sizes from one byte to an eighth of the pool, unaligned on purpose
            const uint64_t bytes = rng() % (pool_units * kUnit / 8) + (rng() % 4 == 0 ? 0 : 1);
            uint64_t a = 0, b = 0;
            const bool ra = fl.alloc(bytes, a), rb = m.alloc(bytes, b);
            if (ra != rb || (ra && a != b)) {
                std::printf("seed %u step %d: alloc(%llu) gave %d@%llu, model %d@%llu\n", seed, i,
                            (unsigned long long)bytes, ra, (unsigned long long)a, rb, (unsigned long long)b);
                return 1;
            }
            if (ra) {
                for (const Live& l : live)
                    if (a < l.off + ((l.bytes ? l.bytes : 1) + kUnit - 1) / kUnit * kUnit &&
                        l.off < a + ((bytes ? bytes : 1) + kUnit - 1) / kUnit * kUnit) {
                        std::printf("seed %u step %d: overlapping ranges\n", seed, i);
                        return 1;
                    }
                live.push_back({a, bytes});
            }
        } else {
            const size_t k = rng() % live.size();
            fl.free(live[k].off, live[k].bytes);
            m.free(live[k].off, live[k].bytes);
            live[k] = live.back();
            live.pop_back();
        }
        if (fl.used() != m.used || fl.peak() != m.peak) {
            std::printf("seed %u step %d: used/peak %llu/%llu, model %llu/%llu\n", seed, i,
                        (unsigned long long)fl.used(), (unsigned long long)fl.peak(), (unsigned long long)m.used,
                        (unsigned long long)m.peak);
            return 1;
        }
    }
    for (const Live& l : live) fl.free(l.off, l.bytes);
    uint64_t off = 1;
    if (fl.used() != 0 || !fl.alloc(pool_units * kUnit, off) || off != 0) {
        std::printf("seed %u: the freed pool did not coalesce into one range\n", seed);
        return 1;
    }
    return 0;
}
}  // namespace

int main() {
    for (uint32_t seed = 1; seed <= 40; seed++)
        if (run(seed, 64 + seed * 37, 4000)) return 1;
    std::printf("ok\n");
    return 0;
}
