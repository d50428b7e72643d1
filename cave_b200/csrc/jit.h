// jit.h -- rule-specialised streaming tick kernels, compiled at run time with NVRTC.
//
// The library's own tick kernel reads the rule (state count, survival and birth tables) at run
// time, which costs logic operations on every strip: the alive test compares four planes with
// the maxCellState bits, and the tables are matched term by term. Compiled with the rule as
// compile-time constants (stream_tick.cuh with a Fixed rule), the same source folds those into
// the fewest operations for that rule. Kernels are keyed by (neighbourhood, maxCellState,
// survival table, birth table), kept per process and, as cubins, in an on-disk cache.
//
// Modes (environment variable CAVE_JIT): "off"/"0" never specialise; "async" (the default)
// starts a background compile the first time a large grid meets a rule and keeps using the
// generic kernel until the specialised one is ready; "sync"/"1" compiles before the first
// launch for every grid size. cave_prepare_rule() compiles ahead of time in any mode but off.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "cave_internal.h"

namespace cave {

enum class JitMode { Off, Async, Sync };
JitMode jit_mode();

struct JitKey {
    uint32_t nb;      // neighbourhood bits (F=1 E=2 C=4)
    uint32_t maxcs;   // 1..16
    uint32_t lut_s;   // DeviceRule::lut_s / lut_b (count-indexed tables)
    uint32_t lut_b;
};
inline JitKey jit_key(const DeviceRule& r) { return JitKey{r.flags & 7u, r.maxcs, r.lut_s, r.lut_b}; }

// Grids at least this large (cells) start a background compile in async mode.
constexpr uint64_t kJitMinCells = 1ull << 21;

// The two specialised kernels of one key, both for deferred-fold runs: `counting` (a run's first
// tick) counts the surviving, born and formerly-zero cells but not the population; `derived`
// (every later tick) counts the surviving and born cells and the population and bounding box of
// its input, i.e. of the previous tick, into that tick's slot. The fold derives the zero cells
// from the previous population; a pass over the final grid (launch_strip_stats) supplies the
// last tick's population and bounding box.
// Each comes in two forms, indexed by `dense`: [1] for launches whose rows fill the lanes
// (strips per row a power of two), [0] for any launch.
// The two-tick kernels (stream_tick2.cuh) come in the same forms: pair_first for a run's first
// two ticks, pair for later ones.
struct JitKernels {
    cudaKernel_t counting[2] = {nullptr, nullptr};
    cudaKernel_t derived[2] = {nullptr, nullptr};
    cudaKernel_t pair_first[2] = {nullptr, nullptr};
    cudaKernel_t pair[2] = {nullptr, nullptr};
    explicit operator bool() const { return counting[0] != nullptr; }
    cudaKernel_t pick(bool first_tick, bool dense) const { return first_tick ? counting[dense] : derived[dense]; }
    cudaKernel_t pick2(bool first_pair, bool dense) const { return first_pair ? pair_first[dense] : pair[dense]; }
};

// The specialised kernels for `k` if they are ready (loaded into the runtime), else empty. In
// sync mode a missing key is compiled first; in async mode a compile is queued when `start`
// is set. A key whose compile failed stays on the generic kernel.
JitKernels jit_stream_kernel(const JitKey& k, JitMode mode, bool start);

// Queues `k` for the background compile (no device needed; returns at once).
void jit_compile_async(const JitKey& k);

// Compiles the kernel for `k` into the caches (no device needed). Returns false with the
// compiler's log (or the reason NVRTC is unavailable) in *log.
bool jit_compile(const JitKey& k, std::string* log);

// Launches one tick with a specialised kernel: the arguments of launch_stream_tick without the
// rule (it is compiled in); the kernels take kJitRowsPerThread rows per thread, so `threads`
// comes from a plan made with that many rows per thread (at most kJitMaxThreads).
cudaError_t launch_stream_tick_jit(cudaKernel_t k, const StreamItem* items, uint32_t n_items, StripSim* sims,
                                   uint4* pool, uint32_t SX, uint32_t SXp, uint32_t threads, cudaStream_t st,
                                   bool pdl, int tick_arg);

// Launches two ticks (tick_arg, tick_arg + 1) with a specialised two-tick kernel, reading cell
// copy src_sel and writing the other; `threads` from a plan made with kJit2RowsPerThread rows
// per thread and two halo rows on each side.
cudaError_t launch_stream_tick2_jit(cudaKernel_t k, const StreamItem* items, uint32_t n_items, StripSim* sims,
                                    uint4* pool, uint32_t SX, uint32_t SXp, uint32_t threads, cudaStream_t st,
                                    bool pdl, int tick_arg, int src_sel);

// Dynamic shared memory of a two-tick launch with `rows` rows per CTA (incl. halo rows).
size_t tick2_smem_bytes(uint32_t rows, uint32_t SX, uint32_t SXp);

// Rows per thread, most threads per CTA and CTAs per SM of the two-tick kernels:
// kJit2RowsPerThread, kJit2MaxThreads and kJit2CtasPerSm unless CAVE_TICK2_ROWS (1..3),
// CAVE_TICK2_THREADS (a multiple of 32 up to 1024) or CAVE_TICK2_CTAS (1..4) set them for the
// process (read once; the kernels are compiled with the same values).
struct Tick2Geometry {
    uint32_t rows_per_thread, max_threads, ctas_per_sm;
};
Tick2Geometry tick2_geometry();

// Process-wide counters behind cave_jit_stats.
void jit_count_launch();
void jit_counts(uint32_t* loaded, uint64_t* launches);

}  // namespace cave
