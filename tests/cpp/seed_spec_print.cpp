// Prints the spawn box that the library's seeding uses (cave::make_seed_spec, cave_ca.cpp) for
// each input line "X Y Z spawnX spawnY spawnZ spawnSizeIndex": "lo_x lo_y lo_z hi_x hi_y hi_z"
// (the box [lo, hi) per axis). Host code only; tests/test_seed_spec.py compares the boxes with
// the oracle's seeding.
#include <cstdint>
#include <cstdio>

#include "engine.h"

int main() {
    unsigned X, Y, Z, sx, sy, sz, idx;
    while (std::scanf("%u %u %u %u %u %u %u", &X, &Y, &Z, &sx, &sy, &sz, &idx) == 7) {
        const cave::SeedSpec s = cave::make_seed_spec(X, Y, Z, sx, sy, sz, idx, 0, true, 0, 1);
        std::printf("%u %u %u %u %u %u\n", s.lo[0], s.lo[1], s.lo[2], s.hi[0], s.hi[1], s.hi[2]);
    }
    return 0;
}
