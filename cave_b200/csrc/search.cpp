// search.cpp -- cave_search_run: the reference's search mode on top of the CUDA paths.
//
// Sweep expansion follows searchMode.cpp:49-218, per-chunk slot set-up searchSystem.cpp:34-200,
// classification searchSystem.cpp:646-713, JSONL lines searchSystem.cpp:959-978, file names
// searchMode.cpp:104-120 and :1030-1038, aggregation ruleAggregator.h:19-141.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <functional>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/cave_ca.h"
#include "context.h"
#include "kernels.h"
#include "rules.h"
#include "trace.h"

namespace cave {

struct GridConfig {          // SearchGridConfig (searchSystem.h:20-26)
    uint32_t maxCellState;
    uint32_t flags;          // neighbourhood bits incl. W
    uint64_t maxPermutation; // 2^n - 1, or the K-index table size when K > 0
    uint32_t neighborCount;
    std::vector<uint64_t> valid;  // K-index table (K > 0)
};

struct Chunk {               // ChunkConfiguration (structs.h:109-128)
    uint32_t X, Y, Z;
    uint32_t spawnX, spawnY, spawnZ;
    uint32_t spawnRegionShapeId;
    uint32_t densityIndex, seed;
    uint32_t partitionIndex, partitionCount;
    uint32_t ordinal;
};

struct SimRef {              // one (chunk, slot, survival, birth) simulation
    uint32_t chunk, slot;
    uint64_t survival, birth;  // 1-based indices (K > 0) or raw masks (K == 0)
};

struct Outcome {
    cave_sim_params params;  // translated rule
    cave_grid_info info;
    uint32_t category;
};

static uint32_t density_index(float p) {  // searchMode.cpp:135-136, :175
    int i = (int)(p * 16.0f) - 1;
    return (uint32_t)std::clamp(i, 0, 15);
}

static uint64_t threshold_from_index(uint32_t idx) {  // searchSystem.cpp:240, :260-262
    const float d = ((float)idx + 1.0f) / 16.0f;
    if (d >= 1.0f) return 1ull << 32;
    return (uint64_t)(uint32_t)(d * 4294967296.0);
}

struct Sweep {
    std::vector<GridConfig> configs;
    std::vector<Chunk> chunks;
    std::string folder, prefixBase;
};

static Sweep expand(const cave_search_config& c) {
    Sweep s;
    // neighbourhood subsets (searchMode.cpp:50-69)
    std::vector<uint32_t> nbs;
    uint32_t sel = (c.faces ? 1u : 0u) | (c.edges ? 2u : 0u) | (c.corners ? 4u : 0u);
    for (uint32_t sub = 1; sub <= sel; sub++) {
        if ((sub & sel) == sub) {
            nbs.push_back(sub);
            if (c.wrap) nbs.push_back(sub | 8u);
        }
    }
    if (nbs.empty()) nbs.push_back(1u);
    // grid configs (searchMode.cpp:81-102) and K-index tables (searchSystem.cpp:38-53)
    for (uint32_t m = c.minMaxCellState; m <= c.maxMaxCellState; m++) {
        for (uint32_t f : nbs) {
            GridConfig g;
            g.maxCellState = m;
            g.flags = f;
            g.neighborCount = neighbor_count(f);
            g.maxPermutation = g.neighborCount < 60 ? ((1ull << g.neighborCount) - 1) : kPermMask;
            if (c.maxRuleBits > 0) {
                g.valid = enumerate_valid_bitmasks(g.neighborCount, c.maxRuleBits);
                g.maxPermutation = g.valid.size();
            }
            s.configs.push_back(std::move(g));
        }
    }
    // file prefix (searchMode.cpp:104-120)
    std::string tag;
    if (c.faces) tag += "F";
    if (c.edges) tag += "E";
    if (c.corners) tag += "C";
    if (c.wrap) tag += "W";
    if (tag.empty()) tag = "F";
    s.prefixBase = "cs" + std::to_string(c.minMaxCellState) + "-" + std::to_string(c.maxMaxCellState) + "_" + tag +
                   "_t" + std::to_string(c.maxTicks);
    if (c.maxRuleBits > 0) s.prefixBase += "_b" + std::to_string(c.maxRuleBits);
    if (c.outputFolder && *c.outputFolder) s.folder = std::string(c.outputFolder) + "cube/";
    // chunk axes (searchMode.cpp:143-218)
    std::vector<uint32_t> grids;
    if (c.gridSweepStep > 0 && c.gridSweepMin > 0 && c.gridSweepMin <= c.gridSweepMax) {
        for (uint32_t g = c.gridSweepMin; g <= c.gridSweepMax; g += c.gridSweepStep) grids.push_back(g);
    } else {
        grids.push_back(c.grid);
    }
    std::vector<uint32_t> dens;
    if (c.densitySweepStep > 0.0f && c.spawnMode == 0 && c.densitySweepMin <= c.densitySweepMax) {
        for (float d = c.densitySweepMin; d <= c.densitySweepMax + 1e-6f; d += c.densitySweepStep)
            dens.push_back(density_index(d));
    } else {
        dens.push_back(density_index(c.spawnDensity));
    }
    const uint32_t seeds = std::max(1u, c.seedRuns);
    const uint32_t parts = std::max(1u, c.chunksPerConfig);
    uint32_t ordinal = 1;
    for (uint32_t g : grids) {
        const uint32_t X = g, Y = g, Z = g;
        for (uint32_t d : dens)
            for (uint32_t sd = 0; sd < seeds; sd++)
                for (uint32_t p = 0; p < parts; p++) {
                    Chunk ch{};
                    ch.X = X;
                    ch.Y = Y;
                    ch.Z = Z;
                    ch.spawnX = std::min(c.spawnX, X);
                    ch.spawnY = std::min(c.spawnY, Y);
                    ch.spawnZ = std::min(c.spawnZ, Z);
                    ch.spawnRegionShapeId = c.spawnMode;
                    ch.densityIndex = d;
                    ch.seed = sd;
                    ch.partitionIndex = p;
                    ch.partitionCount = parts;
                    ch.ordinal = ordinal++;
                    s.chunks.push_back(ch);
                }
    }
    return s;
}

// Survival range of a slot in a chunk (searchSystem.cpp:88-96, :170-188); empty when degenerate.
static void survival_range(const GridConfig& g, const Chunk& ch, uint64_t& lo, uint64_t& hi) {
    hi = g.maxPermutation;
    lo = 1;
    if (ch.partitionCount > 1) {
        hi = (uint64_t)(ch.partitionIndex + 1) * g.maxPermutation / ch.partitionCount;
        lo = 1 + (uint64_t)ch.partitionIndex * g.maxPermutation / ch.partitionCount;
    }
}

static std::string chunk_prefix(const Sweep& s, const Chunk& ch) {  // searchMode.cpp:1030-1038, :1078
    return s.prefixBase + "_c" + std::to_string(ch.ordinal) + "_g" + std::to_string(ch.X) + "x" +
           std::to_string(ch.Y) + "x" + std::to_string(ch.Z) + "_d" + std::to_string(ch.densityIndex) + "_s" +
           std::to_string(ch.seed) + "_gpu0";
}

// nlohmann::json dump() of the entry at searchSystem.cpp:964-976: keys sorted, compact.
static std::string result_line(const Outcome& o) {
    char buf[512];
    std::snprintf(buf, sizeof(buf),
                  "{\"birthAndMaxCellStateRules\":%llu,\"finalAliveCount\":%u,\"maxAliveCount\":%u,"
                  "\"shapeAndGridConfiguration\":%llu,\"survivalAndNeighborhoodRules\":%llu,\"ticksSurvived\":%u,"
                  "\"totalBirths\":%u,\"totalDeaths\":%u}",
                  (unsigned long long)o.params.birthAndMaxCellStateRules, o.info.finalAliveCount,
                  o.info.maxAliveCount, (unsigned long long)o.params.shapeAndGridConfiguration,
                  (unsigned long long)o.params.survivalAndNeighborhoodRules, o.info.numberOfSimulationTicksSurvived,
                  o.info.totalNumberOfCellsThatWereBorn, o.info.totalNumberOfCellsThatDied);
    return buf;
}

struct AggStats {  // RuleStats (ruleAggregator.h:57-66)
    uint32_t total = 0, viable = 0, possible = 0, unviable = 0, maxT = 0, minT = UINT32_MAX;
    uint64_t sumT = 0;
};
using AggKey = std::tuple<uint64_t, uint64_t, uint32_t, uint32_t, uint32_t>;  // birth, survival, maxCS, flags, shape

static void aggregate(std::map<AggKey, AggStats>& agg, const Outcome& o) {  // ruleAggregator.h:69-90
    AggKey k{o.params.birthAndMaxCellStateRules & kPermMask, o.params.survivalAndNeighborhoodRules & kPermMask,
             (uint32_t)((o.params.birthAndMaxCellStateRules >> 60) & 0xF) + 1,
             (uint32_t)(o.params.survivalAndNeighborhoodRules >> 60), 0u};
    AggStats& st = agg[k];
    st.total++;
    if (o.category == 0) st.viable++;
    else if (o.category == 1) st.possible++;
    else st.unviable++;
    const uint32_t t = o.info.numberOfSimulationTicksSurvived;
    st.maxT = std::max(st.maxT, t);
    st.minT = std::min(st.minT, t);
    st.sumT += t;
}

static bool write_aggregate(const std::string& path, const std::map<AggKey, AggStats>& agg) {  // :105-135
    std::ofstream out(path, std::ios::out | std::ios::trunc);
    if (!out.is_open()) return false;
    for (const auto& [k, st] : agg) {
        const float avg = st.total ? (float)st.sumT / (float)st.total : 0.0f;
        const float rate = st.total ? (float)st.viable / (float)st.total : 0.0f;
        out << "{\"birth\":" << std::get<0>(k) << ",\"survival\":" << std::get<1>(k)
            << ",\"maxCellState\":" << std::get<2>(k) << ",\"neighborhoodFlags\":" << std::get<3>(k)
            << ",\"shapeId\":" << std::get<4>(k) << ",\"totalRuns\":" << st.total << ",\"viableRuns\":" << st.viable
            << ",\"possibleRuns\":" << st.possible << ",\"unviableRuns\":" << st.unviable
            << ",\"viabilityRate\":" << rate << ",\"minTicksSurvived\":" << (st.minT == UINT32_MAX ? 0 : st.minT)
            << ",\"maxTicksSurvived\":" << st.maxT << ",\"avgTicksSurvived\":" << avg << "}\n";
    }
    return out.good();
}

// ---------------------------------------------------------------- output
// Per-chunk JSONL output, appended and flushed as results arrive (searchSystem.cpp:959-978:
// one line per finished rule, flushed at once), so that a sweep that is stopped or dies keeps
// every result written so far. A chunk's three files are created (truncated) when its first
// results arrive, and reopened for appending by later waves.
struct ChunkWriter {
    const Sweep& s;
    std::vector<char> started;
    explicit ChunkWriter(const Sweep& sw) : s(sw), started(sw.chunks.size(), 0) {}
    cave_status write(cave_ctx* ctx, size_t ci, const std::vector<Outcome>& outs) {
        if (s.folder.empty()) return CAVE_OK;
        const std::string p = s.folder + chunk_prefix(s, s.chunks[ci]);
        const char* names[3] = {"_viable.jsonl", "_possible.jsonl", "_unviable.jsonl"};
        std::ofstream f[3];
        for (int k = 0; k < 3; k++) {
            f[k].open(p + names[k], std::ios::out | (started[ci] ? std::ios::app : std::ios::trunc));
            if (!f[k].is_open()) return set_error(ctx, CAVE_ERR_IO, "cannot write " + p + names[k]);
        }
        started[ci] = 1;
        for (const Outcome& o : outs) f[o.category] << result_line(o) << '\n';
        for (auto& ff : f) {
            ff.flush();
            if (!ff.good()) return set_error(ctx, CAVE_ERR_IO, "JSONL write failed: " + p);
        }
        return CAVE_OK;
    }
};

// Simulations of chunk ci: every (slot, survival, birth) of the chunk's survival range.
static uint64_t chunk_sim_count(const Sweep& s, size_t ci) {
    uint64_t n = 0;
    for (const GridConfig& g : s.configs) {
        uint64_t lo, hi;
        survival_range(g, s.chunks[ci], lo, hi);
        if (hi >= lo) n += (hi - lo + 1) * g.maxPermutation;
    }
    return n;
}

// Reads a chunk's three JSONL files back (resume). True when they hold exactly the chunk's
// `expected` results, every line exactly as result_line writes it; `outs` then holds them.
static bool read_chunk(const std::string& prefix, uint64_t expected, std::vector<Outcome>& outs) {
    const char* names[3] = {"_viable.jsonl", "_possible.jsonl", "_unviable.jsonl"};
    outs.clear();
    for (uint32_t k = 0; k < 3; k++) {
        std::ifstream f(prefix + names[k]);
        if (!f.is_open()) return false;
        std::string line;
        while (std::getline(f, line)) {
            unsigned long long birth = 0, shape = 0, surv = 0;
            unsigned fin = 0, mx = 0, ticks = 0, births = 0, deaths = 0;
            if (std::sscanf(line.c_str(),
                            "{\"birthAndMaxCellStateRules\":%llu,\"finalAliveCount\":%u,\"maxAliveCount\":%u,"
                            "\"shapeAndGridConfiguration\":%llu,\"survivalAndNeighborhoodRules\":%llu,"
                            "\"ticksSurvived\":%u,\"totalBirths\":%u,\"totalDeaths\":%u}",
                            &birth, &fin, &mx, &shape, &surv, &ticks, &births, &deaths) != 8)
                return false;
            Outcome o{};
            o.params = cave_sim_params{birth, surv, shape};
            o.info.finalAliveCount = fin;
            o.info.maxAliveCount = mx;
            o.info.numberOfSimulationTicksSurvived = ticks;
            o.info.totalNumberOfCellsThatWereBorn = births;
            o.info.totalNumberOfCellsThatDied = deaths;
            o.category = k;
            if (result_line(o) != line || outs.size() >= expected) return false;
            outs.push_back(o);
        }
    }
    return outs.size() == expected;
}

// Results of one chunk as they arrive (the chunk's index and its outcomes in rule order).
using ResultSink = std::function<cave_status(size_t chunk, const std::vector<Outcome>& outs)>;

// Simulations per batched wave: results are written out after each wave, and a stop request
// is honoured between waves. CAVE_SEARCH_WAVE_SIMS overrides the size.
static uint64_t wave_sims() {
    const char* v = std::getenv("CAVE_SEARCH_WAVE_SIMS");
    const long long n = v ? std::atoll(v) : 0;
    return n > 0 ? (uint64_t)n : (1ull << 20);
}

static bool stop_requested(cave_ctx* ctx) { return ctx->search_stop.load(std::memory_order_acquire); }

// ---------------------------------------------------------------- batched execution
// The sweep's simulations in chunk order (birth index fastest within a slot, as the reference
// walks them), run in waves of up to wave_sims() simulations: one batch per wave, holding the
// initial grids and K-index tables of the chunks the wave touches.
static cave_status run_batched(cave_ctx* ctx, const cave_search_config& c, const Sweep& s, const ResultSink& sink,
                               const std::vector<char>& skip, uint64_t limit, double& dev_s, uint64_t& nsims,
                               bool& stopped) {
    struct Piece {
        uint32_t chunk, gi;
        uint64_t sv, bi;  // first simulation of the piece
    };
    dev_s = 0;
    nsims = 0;
    stopped = false;
    const uint64_t per_wave = wave_sims();
    // simulations of chunk ci, slot gi, in order
    auto chunk_sims = [&](uint32_t ci, std::vector<std::pair<uint32_t, std::pair<uint64_t, uint64_t>>>& out) {
        const Chunk& ch = s.chunks[ci];
        for (uint32_t gi = 0; gi < s.configs.size(); gi++) {
            uint64_t lo, hi;
            survival_range(s.configs[gi], ch, lo, hi);
            for (uint64_t sv = lo; sv <= hi; sv++)
                for (uint64_t bi = 1; bi <= s.configs[gi].maxPermutation; bi++) out.push_back({gi, {sv, bi}});
        }
    };
    std::vector<std::pair<uint32_t, std::pair<uint64_t, uint64_t>>> sims_of;  // (slot, (survival, birth))
    uint32_t ci = 0;
    size_t pos = 0;  // next simulation of chunk ci
    bool loaded = false;
    while (ci < s.chunks.size() && !(limit && nsims >= limit)) {
        if (stop_requested(ctx)) {
            stopped = true;
            break;
        }
        // ---- one wave
        TraceRange trace("search_wave");
        cave_batch* b = nullptr;
        cave_status rc = cave_batch_create(ctx, &b);
        if (rc) return rc;
        struct Guard {
            cave_batch* b;
            ~Guard() { cave_batch_destroy(b); }
        } guard{b};
        std::vector<uint32_t> table_ix(s.configs.size(), 0);
        if (c.maxRuleBits > 0)
            for (size_t i = 0; i < s.configs.size(); i++) {
                rc = cave_batch_add_table(b, s.configs[i].valid.data(), (uint32_t)s.configs[i].valid.size(),
                                          &table_ix[i]);
                if (rc) return rc;
            }
        std::vector<cave_sim_desc> descs;
        std::vector<uint32_t> owner;  // chunk of each simulation
        while (ci < s.chunks.size() && descs.size() < per_wave && !(limit && nsims + descs.size() >= limit)) {
            if (!loaded && skip[ci]) {  // its results were read back from its files
                ci++;
                continue;
            }
            if (!loaded) {
                sims_of.clear();
                chunk_sims(ci, sims_of);
                pos = 0;
                loaded = true;
            }
            const Chunk& ch = s.chunks[ci];
            // initial cells per maxCellState (searchSystem.cpp:219-306): one grid per distinct maxCS
            std::map<uint32_t, uint32_t> init_ix;
            const bool random = ch.spawnRegionShapeId == 0;
            const uint64_t thr = random ? threshold_from_index(ch.densityIndex) : (1ull << 32);
            for (; pos < sims_of.size() && descs.size() < per_wave && !(limit && nsims + descs.size() >= limit); pos++) {
                const uint32_t gi = sims_of[pos].first;
                const GridConfig& g = s.configs[gi];
                auto it = init_ix.find(g.maxCellState);
                if (it == init_ix.end()) {
                    uint32_t ix = 0;
                    rc = cave_batch_add_init_seeded(b, ch.X, ch.Y, ch.Z, ch.spawnX, ch.spawnY, ch.spawnZ, thr, ch.seed,
                                                    g.maxCellState, &ix);
                    if (rc) return rc;
                    it = init_ix.emplace(g.maxCellState, ix).first;
                }
                cave_sim_desc d{};
                d.params.birthAndMaxCellStateRules = ((uint64_t)((g.maxCellState - 1) & 0xF) << 60) | sims_of[pos].second.second;
                d.params.survivalAndNeighborhoodRules = ((uint64_t)(g.flags & 0xF) << 60) | sims_of[pos].second.first;
                d.params.shapeAndGridConfiguration = 0;
                d.init = it->second;
                d.maxTicks = c.maxTicks;
                d.validTable = table_ix[gi];
                d.tag = (uint32_t)descs.size();
                owner.push_back(ci);
                descs.push_back(d);
            }
            if (pos >= sims_of.size()) {
                ci++;
                loaded = false;
            }
        }
        if (descs.empty()) break;
        rc = cave_batch_add_sims(b, descs.data(), descs.size(), c.maxRuleBits);
        if (rc) return rc;
        rc = cave_batch_launch(b);
        if (rc) return rc;
        std::vector<cave_sim_result> res(descs.size());
        rc = cave_batch_results(b, res.data(), res.size());
        if (rc) return rc;
        dev_s += ctx->last_timing.tick_ms / 1e3;  // the wave's kernels, resident and tiled
        nsims += descs.size();
        // hand each chunk's results over in order
        size_t i = 0;
        while (i < res.size()) {
            const uint32_t chunk = owner[i];
            std::vector<Outcome> outs;
            for (; i < res.size() && owner[i] == chunk; i++) outs.push_back(Outcome{res[i].params, res[i].info, res[i].category});
            rc = sink(chunk, outs);
            if (rc) return rc;
        }
    }
    return CAVE_OK;
}

// ---------------------------------------------------------------- plain execution
// SearchSystem's loop (searchSystem.cpp:480-713): per tick, reset finished slots from their
// initial cells, launch the step (with the fused manager) once per slot, fence, read the copy
// buffers and record finished rules.
static cave_status run_plain(cave_ctx* ctx, const cave_search_config& c, const Sweep& s, const ResultSink& sink,
                             const std::vector<char>& skip, uint64_t limit, double& dev_s, uint64_t& nsims,
                             bool& stopped) {
    nsims = 0;
    stopped = false;
    double dev_ms = 0;
    cudaEvent_t e0, e1;
    CAVE_CUDA(ctx, cudaEventCreate(&e0));
    CAVE_CUDA(ctx, cudaEventCreate(&e1));
    for (uint32_t ci = 0; ci < s.chunks.size() && !(limit && nsims >= limit); ci++) {
        if (stop_requested(ctx)) {
            stopped = true;
            break;
        }
        if (skip[ci]) continue;  // its results were read back from its files
        const Chunk& ch = s.chunks[ci];
        const uint32_t nslot = (uint32_t)s.configs.size();
        std::vector<Outcome> outs;  // this chunk's results, handed over when it completes
        const uint64_t words = cave_grid_words(ch.X, ch.Y, ch.Z);
        // device buffers: per slot cur/next/initial cells, the slot records, K-index tables
        uint32_t* cells = nullptr;
        PlainSlot* slots = nullptr;
        uint64_t* tables = nullptr;
        std::vector<uint64_t> tab_off(nslot, 0);
        std::vector<uint64_t> host_tab;
        for (uint32_t gi = 0; gi < nslot; gi++) {
            tab_off[gi] = host_tab.size();
            host_tab.insert(host_tab.end(), s.configs[gi].valid.begin(), s.configs[gi].valid.end());
        }
        CAVE_CUDA(ctx, cudaMalloc(&cells, words * 4 * 3 * nslot));
        CAVE_CUDA(ctx, cudaMalloc(&slots, sizeof(PlainSlot) * nslot));
        CAVE_CUDA(ctx, cudaMalloc(&tables, sizeof(uint64_t) * std::max<size_t>(host_tab.size(), 1)));
        if (!host_tab.empty())
            CAVE_CUDA(ctx, cudaMemcpy(tables, host_tab.data(), sizeof(uint64_t) * host_tab.size(), cudaMemcpyHostToDevice));
        std::vector<PlainSlot> hs(nslot);
        std::vector<int> cur(nslot, 0);
        const bool random = ch.spawnRegionShapeId == 0;
        const uint64_t thr = random ? threshold_from_index(ch.densityIndex) : (1ull << 32);
        for (uint32_t gi = 0; gi < nslot; gi++) {
            const GridConfig& g = s.configs[gi];
            uint32_t* base = cells + (uint64_t)gi * 3 * words;
            SeedSpec sp = make_seed_spec(ch.X, ch.Y, ch.Z, ch.spawnX, ch.spawnY, ch.spawnZ, 0, thr, thr == (1ull << 32),
                                         ch.seed, g.maxCellState);
            CAVE_CUDA(ctx, launch_seed_nib(base + 2 * words, sp, ctx->stream));
            CAVE_CUDA(ctx, cudaMemcpyAsync(base, base + 2 * words, words * 4, cudaMemcpyDeviceToDevice, ctx->stream));
            PlainSlot& p = hs[gi];
            std::memset(&p, 0, sizeof(p));
            for (int k = 0; k < 3; k++) p.bmin[k] = 0xFFFFFFFFu;
            uint64_t lo, hi;
            survival_range(g, ch, lo, hi);
            if (lo <= hi) {  // degenerate partitions start exhausted (searchSystem.cpp:175-188)
                p.perms.birthAndMaxCellStateRules = ((uint64_t)((g.maxCellState - 1) & 0xF) << 60) | 1;
                p.perms.survivalAndNeighborhoodRules = ((uint64_t)(g.flags & 0xF) << 60) | lo;
            }
            p.permsCopy = p.perms;
            p.run_manager = 1;
            p.maxPermutation = g.maxPermutation;
            p.survivalEnd = hi;
            p.maxTicks = c.maxTicks;
        }
        CAVE_CUDA(ctx, cudaMemcpyAsync(slots, hs.data(), sizeof(PlainSlot) * nslot, cudaMemcpyHostToDevice, ctx->stream));
        std::vector<cave_sim_params> last_saved(nslot, cave_sim_params{0, 0, 0});
        std::vector<bool> need_reset(nslot, false);
        std::vector<cave_sim_params> read_perms(nslot);
        for (uint32_t gi = 0; gi < nslot; gi++) read_perms[gi] = hs[gi].perms;
        bool running = true;
        while (running && !(limit && nsims >= limit)) {
            cudaEventRecord(e0, ctx->stream);
            for (uint32_t gi = 0; gi < nslot; gi++) {
                const bool exhausted = read_perms[gi].birthAndMaxCellStateRules == 0 &&
                                       read_perms[gi].survivalAndNeighborhoodRules == 0;
                if (exhausted) continue;  // the reference still dispatches; its result is never read
                uint32_t* base = cells + (uint64_t)gi * 3 * words;
                if (need_reset[gi]) {  // Phase 0
                    CAVE_CUDA(ctx, cudaMemcpyAsync(base + (uint64_t)cur[gi] * words, base + 2 * words, words * 4,
                                                   cudaMemcpyDeviceToDevice, ctx->stream));
                    need_reset[gi] = false;
                }
                // Phase 1 + 2 (sim + fused manager) + 3 (ping-pong instead of the copy)
                CAVE_CUDA(ctx, launch_plain_step(base + (uint64_t)cur[gi] * words, base + (uint64_t)(cur[gi] ^ 1) * words,
                                                 ch.X, ch.Y, ch.Z, slots + gi, c.maxRuleBits ? tables + tab_off[gi] : nullptr,
                                                 (uint32_t)s.configs[gi].valid.size(), c.maxRuleBits, ctx->stream));
                cur[gi] ^= 1;
            }
            CAVE_CUDA(ctx, cudaMemcpyAsync(hs.data(), slots, sizeof(PlainSlot) * nslot, cudaMemcpyDeviceToHost, ctx->stream));
            cudaEventRecord(e1, ctx->stream);
            CAVE_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // the tick fence
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            dev_ms += ms;
            // PollCopyBuffers + CacheCompletedResults (searchSystem.cpp:631-713)
            running = false;
            for (uint32_t gi = 0; gi < nslot; gi++) {
                const cave_grid_info& info = hs[gi].infoCopy;
                const cave_sim_params& pm = hs[gi].permsCopy;
                read_perms[gi] = pm;
                if (pm.birthAndMaxCellStateRules != 0 || pm.survivalAndNeighborhoodRules != 0) running = true;
                if (hs[gi].error) {
                    cudaFree(cells);
                    cudaFree(slots);
                    cudaFree(tables);
                    return set_error(ctx, CAVE_ERR_INVALID_ARG, "rule index outside the valid-bitmask table");
                }
                if (info.status == 0) continue;
                if (pm.birthAndMaxCellStateRules == 0 && pm.survivalAndNeighborhoodRules == 0) continue;
                if (pm.birthAndMaxCellStateRules == last_saved[gi].birthAndMaxCellStateRules &&
                    pm.survivalAndNeighborhoodRules == last_saved[gi].survivalAndNeighborhoodRules)
                    continue;
                last_saved[gi] = pm;
                need_reset[gi] = true;
                Outcome o;
                o.params = pm;
                if (c.maxRuleBits > 0) {
                    const auto& v = s.configs[gi].valid;
                    const uint64_t bi = (pm.birthAndMaxCellStateRules & kPermMask) - 1;
                    const uint64_t si = (pm.survivalAndNeighborhoodRules & kPermMask) - 1;
                    if (bi < v.size() && si < v.size()) {
                        o.params.birthAndMaxCellStateRules = (pm.birthAndMaxCellStateRules & ~kPermMask) | v[bi];
                        o.params.survivalAndNeighborhoodRules = (pm.survivalAndNeighborhoodRules & ~kPermMask) | v[si];
                    }
                }
                o.info = info;
                const uint64_t mcs = ((pm.birthAndMaxCellStateRules >> 60) & 0xF) + 1;
                o.category = info.status == 2 ? 0u : ((uint64_t)info.numberOfSimulationTicksSurvived > mcs + 1 ? 1u : 2u);
                outs.push_back(o);
                nsims++;
            }
        }
        cudaFree(cells);
        cudaFree(slots);
        cudaFree(tables);
        if (cave_status rc = sink(ci, outs); rc != CAVE_OK) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return rc;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    dev_s = dev_ms / 1e3;
    return CAVE_OK;
}

}  // namespace cave

using namespace cave;

extern "C" {

cave_status cave_search_run(cave_ctx* ctx, const cave_search_config* config, uint32_t mode, uint64_t simLimit,
                            cave_search_summary* summary) {
    if (!ctx || !config || mode > 1) return CAVE_ERR_INVALID_ARG;
    const cave_search_config& c = *config;
    if (c.minMaxCellState < 1 || c.maxMaxCellState > 16 || c.minMaxCellState > c.maxMaxCellState || c.maxTicks == 0)
        return set_error(ctx, CAVE_ERR_INVALID_ARG, "maxCellState range must lie in 1..16 and ticks must be > 0");
    const auto t0 = std::chrono::steady_clock::now();
    ctx->search_stop.store(false, std::memory_order_release);  // a stop applies to the run in progress
    CAVE_CUDA(ctx, cudaSetDevice(ctx->device));
    Sweep s = expand(c);
    for (const Chunk& ch : s.chunks)
        if (ch.X == 0 || ch.Y == 0 || ch.Z == 0) return set_error(ctx, CAVE_ERR_INVALID_ARG, "grid extents must be > 0");
    if (!s.folder.empty()) {
        std::error_code ec;
        std::filesystem::create_directories(s.folder, ec);
        if (ec) return set_error(ctx, CAVE_ERR_IO, "cannot create " + s.folder + ": " + ec.message());
    }
    cave_search_summary sum{};
    std::map<AggKey, AggStats> agg;
    ChunkWriter writer(s);
    std::vector<char> chunk_done(s.chunks.size(), 0);
    // every chunk's results: into the summary and the aggregate (ruleAggregator.h:69-90), then
    // appended to its files
    const ResultSink sink = [&](size_t ci, const std::vector<Outcome>& outs) -> cave_status {
        const Chunk& ch = s.chunks[ci];
        for (const Outcome& o : outs) {
            sum.sims++;
            (o.category == 0 ? sum.viable : o.category == 1 ? sum.possible : sum.unviable)++;
            sum.ticks += o.info.numberOfSimulationTicksSurvived;
            sum.cellUpdates += (uint64_t)o.info.numberOfSimulationTicksSurvived * ch.X * ch.Y * ch.Z;
            aggregate(agg, o);
        }
        chunk_done[ci] = 1;
        return writer.write(ctx, ci, outs);
    };
    // resume: chunks whose files already hold all their results are read back, not run
    std::vector<char> skip(s.chunks.size(), 0);
    if (c.resume && !s.folder.empty()) {
        std::vector<Outcome> outs;
        for (size_t ci = 0; ci < s.chunks.size(); ci++) {
            if (!read_chunk(s.folder + chunk_prefix(s, s.chunks[ci]), chunk_sim_count(s, ci), outs)) continue;
            skip[ci] = 1;
            const Chunk& ch = s.chunks[ci];
            for (const Outcome& o : outs) {
                sum.sims++;
                sum.resumedSims++;
                (o.category == 0 ? sum.viable : o.category == 1 ? sum.possible : sum.unviable)++;
                sum.ticks += o.info.numberOfSimulationTicksSurvived;
                sum.cellUpdates += (uint64_t)o.info.numberOfSimulationTicksSurvived * ch.X * ch.Y * ch.Z;
                aggregate(agg, o);
            }
            chunk_done[ci] = 1;
        }
    }
    double dev_s = 0;
    uint64_t nsims = 0;
    bool stopped = false;
    cave_status rc = mode == 0 ? run_batched(ctx, c, s, sink, skip, simLimit, dev_s, nsims, stopped)
                               : run_plain(ctx, c, s, sink, skip, simLimit, dev_s, nsims, stopped);
    if (rc) return rc;
    if (!s.folder.empty()) {
        if (!stopped) {
            // chunks without any result (an empty sweep range) still get their three files
            for (size_t ci = 0; ci < s.chunks.size(); ci++)
                if (!chunk_done[ci] && !simLimit) {
                    rc = writer.write(ctx, ci, {});
                    if (rc) return rc;
                }
            if (!write_aggregate(s.folder + s.prefixBase + "_aggregate.jsonl", agg))
                return set_error(ctx, CAVE_ERR_IO, "aggregate JSONL write failed");
        } else if (!agg.empty()) {
            // searchMode.cpp:437-449: a stopped sweep writes what it has as a partial aggregate
            if (!write_aggregate(s.folder + s.prefixBase + "_aggregate_partial.jsonl", agg))
                return set_error(ctx, CAVE_ERR_IO, "partial aggregate JSONL write failed");
        }
    }
    sum.chunks = (uint32_t)s.chunks.size();
    sum.uniqueRules = (uint32_t)agg.size();
    sum.deviceSeconds = dev_s;
    sum.wallSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    sum.stopped = stopped ? 1u : 0u;
    (void)nsims;
    if (summary) *summary = sum;
    return CAVE_OK;
}

cave_status cave_search_stop(cave_ctx* ctx) {
    if (!ctx) return CAVE_ERR_INVALID_ARG;
    ctx->search_stop.store(true, std::memory_order_release);
    return CAVE_OK;
}

// guiSystem.cpp:129-163
uint64_t cave_rule_string_to_bitmask(const char* rule) {
    if (!rule) return 0;
    uint64_t mask = 0;
    std::stringstream ss(rule);
    std::string tok;
    while (std::getline(ss, tok, ',')) {
        tok.erase(std::remove_if(tok.begin(), tok.end(), [](unsigned char ch) { return std::isspace(ch); }), tok.end());
        if (tok.empty()) continue;
        try {
            const size_t dash = tok.find('-');
            if (dash != std::string::npos) {
                const int a = std::stoi(tok.substr(0, dash)), b = std::stoi(tok.substr(dash + 1));
                for (int i = a; i <= b && i <= 60; i++)
                    if (i >= 1) mask |= 1ull << (i - 1);
            } else {
                const int v = std::stoi(tok);
                if (v >= 1 && v <= 60) mask |= 1ull << (v - 1);
            }
        } catch (...) {
            // the reference's std::stoi would throw; a malformed token contributes nothing here
        }
    }
    return mask;
}

// guiSystem.cpp:92-127
uint64_t cave_bitmask_to_rule_string(uint64_t bitmask, char* out, uint64_t cap) {
    std::vector<int> bits;
    for (int b = 0; b < 60; b++)
        if ((bitmask >> b) & 1) bits.push_back(b + 1);
    std::string s;
    if (bits.empty()) {
        s = "-";
    } else {
        size_t i = 0;
        while (i < bits.size()) {
            const size_t start = i;
            while (i + 1 < bits.size() && bits[i + 1] == bits[i] + 1) i++;
            if (!s.empty()) s += ",";
            if (i - start >= 2) {
                s += std::to_string(bits[start]) + "-" + std::to_string(bits[i]);
            } else {
                for (size_t j = start; j <= i; j++) {
                    if (j > start) s += ",";
                    s += std::to_string(bits[j]);
                }
            }
            i++;
        }
    }
    if (out && cap) {
        const size_t n = std::min<size_t>(s.size(), cap - 1);
        std::memcpy(out, s.data(), n);
        out[n] = '\0';
    }
    return s.size();
}

}  // extern "C"
