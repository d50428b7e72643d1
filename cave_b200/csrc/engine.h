// engine.h -- scheduler for many independent simulations of mixed sizes on one GPU.
//
// The reference keeps one SearchSystem per chunk, each recording one dispatch per slot per
// tick and polling a fence per tick (searchSystem.cpp:467-629); chunks are admitted into a
// pool against a VRAM budget (searchMode.cpp:349-404). The engine replaces that machinery:
//
//  * Simulations whose grid fits one CTA's shared memory run on the resident kernel: one
//    persistent launch per admitted group, every tick on chip, until the search manager stops
//    the simulation (kernels_resident.cu).
//  * Larger grids run "tiled": each keeps two bit-plane copies in a device cell pool, and in
//    every round the engine launches `ticks_per_round` tick launches per launch class
//    (kernels_stream.cu), each launch covering every active simulation of the class. A
//    simulation that the manager stops is skipped by later launches; it leaves the launch
//    lists at the next round. Classes run on separate streams so that small classes overlap.
//  * Finished simulations report through a completion ring in host-mapped memory
//    (DoneRing); the host frees their memory and admits waiting simulations in the next
//    round (continuous batching). Admission is first-come first-served against the cell-pool
//    budget and the slot count.
//
// The engine is driven by one host thread at a time (the batch worker or the server loop);
// submit() and take_results() may be called from any thread.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdio>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "context.h"
#include "kernels.h"

namespace cave {

// Largest resident grid: strips * 16 B plus the exchange buffers within the shared memory
// a CTA may use.
bool resident_fits(uint32_t X, uint32_t Y, uint32_t Z);
ResLaunch resident_geometry(uint32_t X, uint32_t Y, uint32_t Z, uint32_t nseg_hint, uint32_t& threads);
// Resident CTAs that fit one SM for a geometry.
uint32_t resident_ctas_per_sm(const ResLaunch& P, uint32_t threads);
// Work items of one tiled simulation for a choice (rows, log2 cells per CTA).
bool plan_tiled(uint32_t sim_index, uint32_t X, uint32_t Y, uint32_t Z, const ExecChoice& c, StreamPlan& plan);

struct EngineSim;
// The execution choice for a simulation's class (grid shape, neighbourhood): the context's
// tuning cache when it has one, else trials when `autotune` is set (adding the time spent to
// *tune_ms), else the defaults (resident when the grid fits, tiled otherwise).
ExecChoice choose_exec(cave_ctx* ctx, cudaStream_t st, const EngineSim& s, bool tiled_only, bool autotune,
                       double* tune_ms);
// Times candidate executions of replicas of `s` for a few ticks and returns the fastest.
cave_status tune_class(cave_ctx* ctx, cudaStream_t st, const EngineSim& s, bool tiled_only, ExecChoice& out);

// One simulation handed to the engine.
struct EngineSim {
    uint64_t key = 0;          // returned with the result
    DeviceRule rule{};         // compiled rule (rules.h)
    uint32_t nb = 0, nt = 0;   // neighbourhood bits; sparse term count (0 = table)
    uint32_t X = 0, Y = 0, Z = 0;
    uint32_t max_ticks = 0;
    const uint4* init = nullptr;  // initial grid in device memory (strip layout), or
    SeedSpec seed{};              // seeded on the device when init is null
};

struct EngineConfig {
    uint64_t pool_bytes = 0;         // cell pool (tiled copies, seeded initial grids)
    uint32_t max_slots = 1u << 14;   // simulations in flight at most (completion-ring size)
    uint32_t ticks_per_round = 8;    // tick launches per class per round
    uint32_t tiled_only = 0;         // 1: never use the resident kernel
    uint32_t autotune = 0;           // 1: time candidate choices for unseen classes
    uint64_t max_active_cells = 0;   // admission stops while admitted grids hold this many
                                     // cells (0: no limit besides memory and slots)
};

struct EngineResult {
    uint64_t key;
    cave_sim_result result;
};

struct EngineStats {
    uint64_t admitted = 0, finished = 0, rounds = 0, tick_launches = 0, resident_launches = 0;
    uint64_t cell_updates = 0;       // ticks run x grid volume, summed over finished simulations
    uint64_t peak_pool_bytes = 0;    // largest cell-pool use
    double tune_ms = 0;              // host time spent in autotuning trials
};

// First-fit free list over [0, size) in 256-byte units (offsets into a device buffer).
class FreeList {
public:
    void reset(uint64_t size);
    bool alloc(uint64_t bytes, uint64_t& off);
    void free(uint64_t off, uint64_t bytes);
    uint64_t used() const { return used_; }
    uint64_t peak() const { return peak_; }

private:
    std::map<uint64_t, uint64_t> free_;  // offset -> bytes
    uint64_t used_ = 0, peak_ = 0;
};

class Engine {
public:
    explicit Engine(cave_ctx* ctx);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    cave_status init(const EngineConfig& cfg);
    // Queues simulations. Rejects (CAVE_ERR_OUT_OF_MEMORY) a simulation that could never fit
    // the cell pool.
    cave_status submit(std::vector<EngineSim>& sims);
    // One scheduling step: reads completions, admits, launches a round when fewer than two are
    // in flight. Sets *idle when nothing is queued or running. Blocks at most briefly.
    cave_status step(bool* idle);
    // Runs until every submitted simulation has finished.
    cave_status run_until_idle();
    // Orders all later engine work after `ev` (e.g. initial grids written on another stream).
    cave_status after(cudaEvent_t ev);
    // Records `ev` after all work the engine has issued.
    cave_status record_end(cudaEvent_t ev);
    // Moves finished results into out (appends).
    void take_results(std::vector<EngineResult>& out);
    // Drops the simulations with keys in [key_lo, key_hi) that are not admitted yet; each is
    // reported by take_results with its result's error set to kErrCancelled. Admitted ones run
    // to completion. Any thread; applied by the driving thread's next step.
    void cancel(uint64_t key_lo, uint64_t key_hi);
    EngineStats stats();
    // Device time from the first set-up to the last completed work (CUDA events), ms.
    float device_ms();
    std::string plan_json();   // the choice used per class, for reports

private:
    struct Slot;
    struct TiledClass;
    struct Round;
    struct ResGroup;
    cave_status admit(std::vector<EngineSim>& admitted_now);
    cave_status launch_round(std::vector<EngineSim>& admitted);
    cave_status consume_ring(bool* any);
    cave_status retire(bool block);
    cave_status finish_timing();
    ExecChoice choose(const EngineSim& s);

    cave_ctx* ctx_;
    EngineConfig cfg_{};
    bool ready_ = false;
    cudaStream_t main_ = nullptr;    // set-up, round joins
    cudaStream_t copy_ = nullptr;    // staging uploads
    std::vector<cudaStream_t> class_streams_, res_streams_;
    // device memory
    uint4* pool_ = nullptr;          // cell pool
    StripSim* recs_ = nullptr;       // one record per slot
    DoneRing* ring_ = nullptr;       // device ring header
    DoneEntry* host_entries_ = nullptr;  // host-mapped entries
    uint32_t consumed_ = 0;          // ring entries read by the host
    // staging (two rounds in flight): pinned host and device mirrors
    unsigned char* stage_h_[2] = {nullptr, nullptr};
    unsigned char* stage_d_[2] = {nullptr, nullptr};
    uint64_t stage_cap_ = 0;
    FreeList cells_;                 // the cell pool
    unsigned char* desc_ = nullptr;  // resident launch descriptors (queue counter, sims, rules)
    FreeList descs_;                 // sized so that it cannot run out (see init)
    std::vector<Slot*> slots_;
    std::vector<uint32_t> free_slots_;
    std::map<std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>, TiledClass*> classes_;
    std::deque<Round*> rounds_;      // in flight, oldest first
    std::vector<ResGroup*> groups_;  // resident launches in flight
    uint64_t round_no_ = 0;
    uint64_t active_cells_ = 0;      // grid volume of the admitted, unfinished simulations
    uint32_t res_rr_ = 0;
    // queues
    std::mutex mu_;
    std::deque<EngineSim> incoming_;
    std::deque<EngineSim> pending_;
    std::vector<EngineResult> results_;
    std::vector<std::pair<uint64_t, uint64_t>> cancels_;  // key ranges to drop from the queues
    EngineStats stats_;
    cudaEvent_t ev_first_ = nullptr, ev_last_ = nullptr;
    bool first_recorded_ = false;
    std::map<TuneKey, ExecChoice> plan_used_;
    // optional scheduling trace (JSON lines): path from the CAVE_ENGINE_TRACE environment variable
    FILE* trace_ = nullptr;
    std::chrono::steady_clock::time_point trace_t0_;
    double trace_us() const;
};

}  // namespace cave
