// rules.h -- host-side decoding of SimulationParameters into the kernels' DeviceRule.
#pragma once
#include <cstdint>
#include <vector>

#include "cave_internal.h"

namespace cave {

// Fields of SimulationParameters after the K-index lookup (searchSimulationCube.slang:139-157).
struct DecodedRule {
    uint32_t maxcs;   // 1..16
    uint32_t flags;   // low 4 bits of survivalAndNeighborhoodRules >> 60
    uint64_t birth, survival;
};

// Returns false when maxRuleBits > 0 and an index falls outside the table.
bool decode_params(const cave_sim_params& p, const uint64_t* valid, uint32_t nValid, uint32_t maxRuleBits,
                   DecodedRule& out);

// Builds the LUTs / sparse term table the strip kernels consume.
DeviceRule make_device_rule(const DecodedRule& d);

// True when the kernels should use the sparse-term rule evaluation for this rule.
inline bool rule_is_sparse(const DeviceRule& r) { return r.nterms > 0; }

// permutationMath.h:101-128
std::vector<uint64_t> enumerate_valid_bitmasks(uint32_t neighborCount, uint32_t maxBits);

// Neighbour count of a flag set (cube: F 6, E 12, C 8; shape.h:110-127).
inline uint32_t neighbor_count(uint32_t flags) {
    return ((flags & 1u) ? 6u : 0u) + ((flags & 2u) ? 12u : 0u) + ((flags & 4u) ? 8u : 0u);
}

}  // namespace cave
