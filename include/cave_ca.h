/*
 * cave_ca.h -- C ABI of the B200 (sm_100a) CA stepping library (libcave_ca.so).
 *
 * Drop-in for the search-mode stepping path of CAVE (Scub3d/CAVE). The reference has no
 * FFI of its own: its hot path sits behind a Vulkan shader-binding contract and the C++
 * class SearchSystem. Each entry point below names the reference interface it replaces.
 *
 * Conventions: every function returns cave_status (0 = CAVE_OK); no C++ exception crosses
 * this boundary; host buffers are caller-owned; device buffers are library-owned and
 * addressed by opaque handles; one CUDA stream per context; a context may be used from one
 * host thread at a time. cave_last_error() returns the context's last error text.
 *
 * Cell layout at this boundary is the reference's padded nibble layout
 * (searchSimulationCube.slang:52-53, :88-93; searchSystem.cpp:140-143, :290-295):
 * 4 bits per cell, 8 cells per uint32 along x (low nibble = lowest x), word index
 * x/8 + y*W + z*W*Y with W = ceil(X/8); padding nibbles are 0.
 */
#ifndef CAVE_CA_H
#define CAVE_CA_H

#ifndef __CUDACC_RTC__ /* NVRTC has no C library headers; the kernel sources declare the types */
#include <stddef.h>
#include <stdint.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int cave_status;
enum {
    CAVE_OK = 0,
    CAVE_ERR_INVALID_ARG = 1,   /* bad size, pointer, rule index, or unsupported geometry */
    CAVE_ERR_CUDA = 2,          /* a CUDA runtime call failed (text in cave_last_error)   */
    CAVE_ERR_OUT_OF_MEMORY = 3, /* device allocation or admission budget exceeded          */
    CAVE_ERR_NOT_READY = 4,     /* non-blocking poll: work still in flight                 */
    CAVE_ERR_TIMEOUT = 5,       /* a bounded device-side wait gave up (kernel error flag) */
    CAVE_ERR_IO = 6,            /* JSONL output could not be written                       */
    CAVE_ERR_INTERNAL = 7
};

/* ---- reference data structures (bit-exact layouts) --------------------------------- */

/* SimulationParameters (src/common/structs.h:89-99; encoding simulation.h:43-59):
 *   birthAndMaxCellStateRules    [63:60] = maxCellState-1, [59:0] birth mask or 1-based K-index
 *   survivalAndNeighborhoodRules [63:60] = flags W=8 C=4 E=2 F=1, [59:0] survival mask or K-index
 *   shapeAndGridConfiguration    [4:0] shape id (0 = cube)                                 */
typedef struct {
    uint64_t birthAndMaxCellStateRules;
    uint64_t survivalAndNeighborhoodRules;
    uint64_t shapeAndGridConfiguration;
} cave_sim_params;

/* GridSnapshot (structs.h:130-136). */
typedef struct {
    uint32_t numberOfDeadCells;
    uint32_t numberOfDyingCells;
    uint32_t numberOfCellsBorn;
    uint32_t numberOfSurvivingCells;
} cave_grid_snapshot;

/* GridInfo (structs.h:79-87). */
typedef struct {
    uint32_t totalNumberOfCellsThatDied;
    uint32_t totalNumberOfCellsThatWereBorn;
    uint32_t numberOfSimulationTicksSurvived;
    uint32_t status; /* 0 running, 1 early death, 2 reached the tick limit (viable) */
    uint32_t maxAliveCount;
    uint32_t finalAliveCount;
} cave_grid_info;

/* ChunkConfiguration (structs.h:109-128). */
typedef struct {
    uint32_t shapeId;
    uint32_t gridDimensionX, gridDimensionY, gridDimensionZ;
    uint32_t spawnAreaDimensionX, spawnAreaDimensionY, spawnAreaDimensionZ;
    uint32_t spawnPlacementId;
    uint32_t spawnRegionShapeId; /* 0 = random fill, otherwise filled box */
    uint32_t spawnSizeIndex;
    uint32_t spawnDensityIndex;  /* density (i+1)/16 */
    uint32_t runSeedIndex;
    uint32_t partitionIndex;
    uint32_t partitionCount;
} cave_chunk_config;

/* Per-tick statistics: the reference GridSnapshot plus fields the reference does not
 * compute. population = non-zero cells after the tick; changed = cells whose state
 * changed (= born + dying); bbox of non-zero cells after the tick (min = 0xFFFFFFFF and
 * max = 0 on every axis when no cell is non-zero). */
typedef struct {
    cave_grid_snapshot snapshot;
    uint32_t population;
    uint32_t changed;
    uint32_t bbox_min[3];
    uint32_t bbox_max[3];
} cave_tick_stats;

/* ---- context ------------------------------------------------------------------------ */
typedef struct cave_ctx cave_ctx;

/* Replaces DeviceContext construction for the search path (src/vulkan/deviceContext.*). */
cave_status cave_ctx_create(int device, cave_ctx** out);
void cave_ctx_destroy(cave_ctx* ctx);
const char* cave_status_string(cave_status s);
const char* cave_last_error(const cave_ctx* ctx);
/* Blocks until all work queued on the context's stream is done. */
cave_status cave_ctx_synchronize(cave_ctx* ctx);

/* Device-side timing of the last cave_step / cave_run / cave_run_host call, or of the last
 * batch whose results were read (tick_ms = its kernels, total_ms = uploads, kernels and
 * read-back), measured with CUDA events on
 * the context's stream (replaces the reference's timestamp queries, queryManager.h:13-97).
 * Recorded only while enabled (off by default; it adds one event pair per phase). */
typedef struct {
    uint32_t ticks;          /* tick launches in the call                               */
    uint32_t launches;       /* kernels this library launched in the call               */
    float tick_ms;           /* from the first tick launch to the end of the last one   */
    float convert_ms;        /* layout conversions (nibble <-> bit-plane), both ways    */
    float total_ms;          /* whole call on the device, copies included               */
} cave_timing;
cave_status cave_ctx_set_timing(cave_ctx* ctx, int enable);
cave_status cave_ctx_last_timing(const cave_ctx* ctx, cave_timing* out);

/* ---- grids --------------------------------------------------------------------------- */
typedef struct cave_grid cave_grid;

/* Replaces the per-slot cellsIn/cellsOut/initialCells buffers of
 * SearchSystem::BuildBuffers (searchSystem.cpp:126-394). The grid holds two device copies of
 * the cells (ping-pong); the "current" one is what upload/download/step see. */
cave_status cave_grid_create(cave_ctx* ctx, uint32_t X, uint32_t Y, uint32_t Z, cave_grid** out);
void cave_grid_destroy(cave_grid* g);
/* Number of uint32 words in the padded nibble layout: ceil(X/8)*Y*Z. */
uint64_t cave_grid_words(uint32_t X, uint32_t Y, uint32_t Z);
cave_status cave_grid_upload(cave_grid* g, const uint32_t* words, uint64_t nwords);
cave_status cave_grid_download(cave_grid* g, uint32_t* words, uint64_t nwords);

/* Initial cells on the device, same cells as searchSystem.cpp:219-306 for `chunk` and
 * `maxCellState` (random fill when spawnRegionShapeId == 0, density from spawnDensityIndex). */
cave_status cave_grid_seed(cave_grid* g, const cave_chunk_config* chunk, uint32_t maxCellState);
/* Same hash and spawn box with an explicit fill threshold: a box cell is alive iff
 * cellHash(x,y,z,seed) < threshold; threshold = 2^32 fills the whole box. This expresses
 * fills such as 0.30 (threshold (uint32)((double)0.30f * 2^32)) that the 1/16-step density
 * index cannot. */
cave_status cave_grid_seed_threshold(cave_grid* g, uint32_t spawnX, uint32_t spawnY, uint32_t spawnZ,
                                     uint64_t threshold, uint32_t runSeedIndex, uint32_t maxCellState);

/* ---- plain path: one launch per tick ------------------------------------------------- */
/* Replaces one Phase-1 + Phase-2 + Phase-3 pass of SearchSystem::SubmitNextTick
 * (searchSystem.cpp:541-616): searchSimulationCube.slang computeMain over the grid, its
 * GridSnapshot reduction, and the cellsOut -> cellsIn copy (here a ping-pong swap).
 * Runs `nticks` launches; per_tick (host array of nticks, may be NULL) receives each
 * tick's statistics. validBitmasks/nValid are the K-index table (binding 4, used when
 * maxRuleBits > 0; EnumerateValidBitmasks order). Rule indices outside the table are
 * rejected with CAVE_ERR_INVALID_ARG. */
cave_status cave_step(cave_grid* g, const cave_sim_params* params, const uint64_t* validBitmasks,
                      uint32_t nValid, uint32_t maxRuleBits, uint32_t nticks, cave_tick_stats* per_tick);

/* ---- streaming path: many ticks in the library's bit-plane layout -------------------- */
/* Same results as cave_step for the same inputs (every cell, every statistic), computed by
 * the z-slab streaming kernel: the grid is converted to a bit-plane layout once, stepped
 * nticks times (one launch per tick, each allowed to start its prologue while the previous
 * tick drains: programmatic dependent launch) and converted back. The
 * GridInfo of the manager shader (searchManager.slang:98-139) for those ticks is returned in
 * *info (may be NULL) with maxTicks as MAX_NUMBER_OF_TICKS_TO_SURVIVE; the run does not stop
 * on status > 0 (raw stepping). */
cave_status cave_run(cave_grid* g, const cave_sim_params* params, const uint64_t* validBitmasks,
                     uint32_t nValid, uint32_t maxRuleBits, uint32_t nticks, uint32_t maxTicks,
                     cave_tick_stats* per_tick, cave_grid_info* info);

/* cave_run with host buffers: copies in_words (nwords, host memory, ideally pinned) to the
 * grid, runs, and copies the result to out_words, all in one stream-ordered call -- the
 * end-to-end form of the reference's upload / tick loop / read-back
 * (searchSystem.cpp:314, :480-629, :631-644). */
cave_status cave_run_host(cave_grid* g, const uint32_t* in_words, uint32_t* out_words, uint64_t nwords,
                          const cave_sim_params* params, const uint64_t* validBitmasks, uint32_t nValid,
                          uint32_t maxRuleBits, uint32_t nticks, uint32_t maxTicks, cave_tick_stats* per_tick,
                          cave_grid_info* info);

/* ---- rule-specialised tick kernels ----------------------------------------------------
 * The reference builds one compute pipeline per shader, with the rule read from a buffer on
 * every cell (searchSystem.cpp:419, computePipeline.cpp:11-29). Here cave_run and
 * cave_render_step may run a tick kernel compiled for the rule itself (NVRTC, sm_100a): the
 * rule's state count and tables become compile-time constants, which removes per-cell logic.
 * Results are identical either way. Environment variable CAVE_JIT selects the policy: "async"
 * (default; the first run of a grid of at least 2^21 cells with a new rule starts a
 * background compile and the following runs use the specialised kernel once it is ready),
 * "sync" (compile before the first launch, any grid size) or "off". Compiled kernels are
 * cached per process and on disk (CAVE_JIT_CACHE, default ~/.cache/cave_b200; "off" disables
 * it).
 *
 * cave_prepare_rule: compiles (or loads from the cache) the specialised kernel for this rule
 * and neighbourhood now, so that every later cave_run / cave_render_step with it uses it.
 * Returns CAVE_OK (a no-op when CAVE_JIT=off), CAVE_ERR_INVALID_ARG for a rule index outside
 * the table, or CAVE_ERR_INTERNAL when the kernel could not be compiled or loaded (reason in
 * cave_last_error; runs then use the generic kernel). */
cave_status cave_prepare_rule(cave_ctx* ctx, const cave_sim_params* params, const uint64_t* validBitmasks,
                              uint32_t nValid, uint32_t maxRuleBits);
/* Compiles the specialised kernel for a rule without any device (fills the caches; e.g. on a
 * build host with the same disk cache). log (may be NULL) receives up to log_size-1 bytes of
 * the compiler's output. Returns CAVE_OK, CAVE_ERR_INVALID_ARG or CAVE_ERR_INTERNAL. */
cave_status cave_jit_compile(const cave_sim_params* params, const uint64_t* validBitmasks, uint32_t nValid,
                             uint32_t maxRuleBits, char* log, size_t log_size);
/* Starts compiling the specialised kernel for a rule in the background and returns at once (no
 * device needed; a no-op when CAVE_JIT=off). Later runs with the rule use it once it is ready;
 * a process may exit while the compile runs (the library waits for it at exit). Returns
 * CAVE_OK or CAVE_ERR_INVALID_ARG. */
cave_status cave_jit_compile_async(const cave_sim_params* params, const uint64_t* validBitmasks, uint32_t nValid,
                                   uint32_t maxRuleBits);
/* Diagnostics: rule-specialised kernels loaded into this process so far, and tick launches
 * made with them. Either pointer may be NULL. */
void cave_jit_stats(uint32_t* loaded, uint64_t* launches);

/* cave_run without any device allocation. No counterpart in the reference (its buffers are
 * always created per slot, searchSystem.cpp:126-394); it exists for callers that must not
 * allocate device memory while they run -- a serving loop whose HBM is held by another
 * allocator, where cudaMalloc can fail, or that cannot take cudaFree's device-wide
 * synchronisation between requests.
 * d_in / d_out: caller-owned DEVICE buffers of cave_grid_words(X, Y, Z) words in the nibble
 * layout (4-byte aligned; d_in == d_out is allowed), in memory of the context's device (or
 * managed memory); another GPU's memory is rejected with CAVE_ERR_INVALID_ARG. d_per_tick:
 * caller-owned device array of nticks entries, or NULL. *info (host, may be NULL) receives
 * the GridInfo as in cave_run. Cells, statistics and GridInfo equal cave_run's for the same
 * inputs. Blocking. The work runs on the context's own stream, which is not ordered after
 * any other stream: the caller's writes of d_in must be complete, and d_out not in use, on
 * every other stream before the call (synchronise those streams, or wait on an event).
 * Scratch: one static device array of CAVE_NOALLOC_SCRATCH_BYTES per GPU, part of the
 * library's device image. Under CUDA's lazy module loading (the default) a GPU takes that
 * memory when the first cave_run_noalloc call on it loads the array's module, and then holds
 * it until exit: make the first call on a device before another allocator reserves that
 * device's memory (if it cannot be had, the call fails with CAVE_ERR_OUT_OF_MEMORY naming the
 * array). A grid needs 32 bytes per 32 x-cells (rounded up) per row and plane plus a few KB;
 * larger grids are rejected with CAVE_ERR_INVALID_ARG (256^3 and 320^3 fit). The first call on
 * a device looks the array up (cudaGetSymbolAddress with that device current); make that
 * first call before any stream capture. Every call on a device shares the array: calls that
 * overlap on the GPU (two contexts, or two host threads, on one device) race and must be
 * serialised by the caller. The simulation record in the array is rewritten by each call. Not
 * timed by cave_ctx_set_timing. */
#define CAVE_NOALLOC_SCRATCH_BYTES (32u << 20)
cave_status cave_run_noalloc(cave_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t X, uint32_t Y,
                             uint32_t Z, const cave_sim_params* params, const uint64_t* validBitmasks,
                             uint32_t nValid, uint32_t maxRuleBits, uint32_t nticks, uint32_t maxTicks,
                             cave_tick_stats* d_per_tick, cave_grid_info* info);

/* ---- batched path: many small simulations ------------------------------------------ */
/* One simulation of a batch: a rule run from an initial grid until the search manager
 * reports status > 0 (early death, or maxTicks reached), exactly the per-rule lifecycle of a
 * SearchSystem slot (searchSystem.cpp:496-526, :608-616; searchManager.slang:98-149). */
typedef struct {
    cave_sim_params params;   /* rule; K-index form when maxRuleBits > 0 */
    uint32_t init;            /* index of the initial grid (cave_batch_add_init)        */
    uint32_t maxTicks;        /* MAX_NUMBER_OF_TICKS_TO_SURVIVE                          */
    uint32_t validTable;      /* index of the K-index table (cave_batch_add_table)      */
    uint32_t tag;             /* caller's id, copied to the result                       */
} cave_sim_desc;

/* Result of one simulation: the final GridInfo plus the derived statistics. */
typedef struct {
    cave_grid_info info;      /* as the manager's copy buffer at the final tick          */
    uint32_t category;        /* 0 viable, 1 possible, 2 unviable (searchSystem.cpp:697-711) */
    uint32_t tag;
    uint32_t population;      /* non-zero cells after the final tick                     */
    uint32_t activeTicks;     /* ticks in which at least one cell changed                */
    uint64_t totalChanged;    /* cells changed, summed over ticks                        */
    uint32_t bbox_min[3];     /* of the non-zero cells after the final tick              */
    uint32_t bbox_max[3];
    cave_sim_params params;   /* rule with K-indices translated to bitmasks (:668-685)   */
    uint32_t error;
    uint32_t pad;
} cave_sim_result;

typedef struct cave_batch cave_batch;

/* A batch owns device copies of initial grids, K-index tables and simulation descriptors.
 * Replaces the chunk-level buffers and the per-slot tick loop of SearchSystem
 * (searchSystem.cpp:126-394, :480-713) by one persistent launch per simulation class. */
cave_status cave_batch_create(cave_ctx* ctx, cave_batch** out);
void cave_batch_destroy(cave_batch* b);
/* Adds an initial grid in the reference nibble layout (host words). Returns its index. */
cave_status cave_batch_add_init(cave_batch* b, uint32_t X, uint32_t Y, uint32_t Z, const uint32_t* words,
                                uint64_t nwords, uint32_t* index);
/* Adds an initial grid seeded on the device (searchSystem.cpp:219-306 with an explicit fill
 * threshold, as cave_grid_seed_threshold). Returns its index. */
cave_status cave_batch_add_init_seeded(cave_batch* b, uint32_t X, uint32_t Y, uint32_t Z, uint32_t spawnX,
                                       uint32_t spawnY, uint32_t spawnZ, uint64_t threshold,
                                       uint32_t runSeedIndex, uint32_t maxCellState, uint32_t* index);
/* Adds a K-index table (EnumerateValidBitmasks order). Returns its index. */
cave_status cave_batch_add_table(cave_batch* b, const uint64_t* validBitmasks, uint32_t nValid, uint32_t* index);
/* Queues simulations (maxRuleBits applies to all of them). */
cave_status cave_batch_add_sims(cave_batch* b, const cave_sim_desc* sims, uint64_t n, uint32_t maxRuleBits);
/* How a batch runs (set before cave_batch_launch; all-zero = defaults). Grids that fit one
 * CTA's shared memory run on the resident kernel (one persistent launch per class, every tick
 * on chip); larger grids run tiled: each keeps two bit-plane copies in HBM and every tick is a
 * multi-CTA launch over all active simulations of its class, in rounds driven by a host
 * worker thread, finished simulations leaving and waiting ones entering between rounds
 * (searchMode.cpp:349-404 admits whole chunks against a VRAM budget instead). */
typedef struct {
    uint32_t autotune;       /* 1: time candidate executions (resident vs tiled, CTA size,
                                CTAs per simulation) of each grid class once per context and
                                keep the fastest; 0: defaults                                */
    uint32_t tiledOnly;      /* 1: run every grid tiled (never resident)                       */
    uint32_t ticksPerRound;  /* tiled: tick launches per class between scheduling steps (0 = 8) */
    uint32_t pad;
    uint64_t memoryBudget;   /* tiled: device bytes for grid copies (0 = half the free memory);
                                a batch larger than this runs in waves                        */
} cave_batch_options;
cave_status cave_batch_set_options(cave_batch* b, const cave_batch_options* options);
/* JSON array describing how each grid class of the last launch runs (path, tile shape);
 * writes up to cap bytes (NUL-terminated) and returns the full length. */
uint64_t cave_batch_plan(const cave_batch* b, char* out, uint64_t cap);

/* Starts every queued simulation on the device (non-blocking). A context with a batch in
 * flight should not be used for other calls until cave_batch_results has returned. */
cave_status cave_batch_launch(cave_batch* b);
/* Non-blocking completion poll (the IsTickComplete of searchSystem.cpp:467-478): CAVE_OK
 * when the launched work has finished, CAVE_ERR_NOT_READY otherwise. */
cave_status cave_batch_poll(cave_batch* b);
/* Waits for the launched work and copies results (in queue order) to out[0..n). Call it once per
 * launch: simulations that ran tiled hand their results over on the first call. `out` may be
 * pageable or pinned host memory; pinned memory (cudaMallocHost) is written at full link speed,
 * which matters for sweeps of millions of simulations (104 B per result). */
cave_status cave_batch_results(cave_batch* b, cave_sim_result* out, uint64_t n);
/* Simulations queued so far. */
uint64_t cave_batch_size(const cave_batch* b);
/* Runs the queued simulations on the plain path instead, the way SearchSystem drives its
 * slots (searchSystem.cpp:480-713): `slots` simulations in flight, each tick one step launch
 * per active slot (searchSimulationCube + fused manager), then one read-back and a host fence;
 * a slot whose rule finished takes the next simulation and restarts from its initial cells.
 * Blocking. Results are identical to cave_batch_launch's; *deviceSeconds (may be NULL)
 * receives the device time of the tick loops. */
cave_status cave_batch_run_plain(cave_batch* b, uint32_t slots, double* deviceSeconds);

/* ---- serving: sweep requests admitted as they arrive -------------------------------------- */
/* A server runs requests -- each a list of simulations, every one with its own grid, rule,
 * tick limit and seeded initial cells -- on one GPU while more requests arrive. Simulations
 * are admitted first-come first-served as slots and grid memory free up (continuous
 * batching: a request that arrives while others run shares the GPU with them), grid state
 * stays on the device between ticks, and a request completes when its last simulation has.
 * Replaces SearchMode's chunk pool (searchMode.cpp:252-459; VRAM admission :349-404), which
 * runs one sweep per process. Results are the same as a batch's for the same simulations. */
typedef struct cave_server cave_server;

/* One simulation of a request. The initial cells are the reference's seeding
 * (searchSystem.cpp:219-306): a centred spawn box, a cell alive (state maxCellState) iff
 * cellHash(x, y, z, runSeedIndex) < threshold (2^32 fills the box). */
typedef struct {
    uint32_t X, Y, Z;
    uint32_t maxTicks;          /* MAX_NUMBER_OF_TICKS_TO_SURVIVE                         */
    cave_sim_params params;     /* rule in bitmask form (no K-index)                      */
    uint32_t spawnX, spawnY, spawnZ;
    uint32_t runSeedIndex;
    uint64_t threshold;
    uint32_t tag;               /* caller's id, not interpreted                           */
    uint32_t pad;
} cave_request_sim;

typedef struct {
    uint64_t hbmBudget;         /* device bytes for grid state (0 = half the free memory)  */
    uint32_t maxInFlight;       /* simulations on the device at once at most (0 = 16384)  */
    uint32_t ticksPerRound;     /* tiled grids: tick launches per scheduling step (0 = 8)  */
    uint32_t autotune;          /* as cave_batch_options                                   */
    uint32_t tiledOnly;
    uint64_t maxActiveCells;    /* admission pauses while the admitted grids hold this many
                                   cells (0 = 2^31, several ticks of work for the GPU): the
                                   oldest requests run first instead of every request
                                   sharing the GPU; ~0 = limited by memory only            */
    double requestDeadlineSeconds; /* a request not complete this long after its submission
                                   expires (0 = never): its queued simulations leave the
                                   queue, running ones finish unreported, and wait / fetch
                                   return CAVE_ERR_TIMEOUT (fetch releases it)              */
} cave_server_options;

typedef struct {
    uint64_t submitted, completed;      /* requests                                          */
    uint64_t simsCompleted;
    uint64_t cellUpdates;               /* ticks run x grid volume, finished simulations    */
    double p50LatencySeconds;           /* submit -> last result, over completed requests   */
    double p99LatencySeconds;
    double busySeconds;                 /* wall time with at least one request outstanding  */
    uint64_t peakBytes;                 /* largest grid memory in use                       */
    uint64_t rounds, tickLaunches, residentLaunches;
    double tuneMs;                      /* host time spent autotuning                       */
    uint64_t expired;                   /* requests that passed requestDeadlineSeconds      */
} cave_server_stats;

cave_status cave_server_create(cave_ctx* ctx, const cave_server_options* options, cave_server** out);
/* Stops the scheduler and waits for device work in flight; unfetched results are dropped. */
void cave_server_destroy(cave_server* s);
/* Queues a request of n simulations (non-blocking) and returns its id. Fails with
 * CAVE_ERR_OUT_OF_MEMORY when one simulation alone needs more than the budget. */
cave_status cave_server_submit(cave_server* s, const cave_request_sim* sims, uint64_t n, uint64_t* requestId);
/* Ids of requests that completed or expired since the last poll (up to cap). Non-blocking. */
cave_status cave_server_poll(cave_server* s, uint64_t* requestIds, uint64_t cap, uint64_t* n);
/* Blocks until the request has completed (timeoutSeconds <= 0: no limit; CAVE_ERR_TIMEOUT
 * when the time ran out, or when the request passed requestDeadlineSeconds). When the
 * scheduler thread has failed, submit, poll and stats return its error, and so do wait and
 * fetch for a request that had not completed (completed results can still be fetched). */
cave_status cave_server_wait(cave_server* s, uint64_t requestId, double timeoutSeconds);
/* Cancels a request (the reference's stop request, searchMode.cpp:437-449, for one request):
 * its simulations not yet admitted leave the queue at once, those already on the device run to
 * completion and their results are dropped; a completed request's results are discarded. After
 * the call the id is unknown to wait / fetch (CAVE_ERR_INVALID_ARG), and requests submitted
 * before or after it are unaffected. CAVE_ERR_INVALID_ARG for an unknown id. */
cave_status cave_server_cancel(cave_server* s, uint64_t requestId);
/* Copies a completed request's results (n = its simulation count, submission order, params in
 * the submitted form) and releases it; *latencySeconds = submit to completion. An expired
 * request returns CAVE_ERR_TIMEOUT and is released (the id becomes unknown). */
cave_status cave_server_fetch(cave_server* s, uint64_t requestId, cave_sim_result* out, uint64_t n,
                              double* latencySeconds);
cave_status cave_server_get_stats(cave_server* s, cave_server_stats* out);

/* Progress of one request (the reference's SearchProgress, searchSystem.h:29-38, per request):
 * its simulations, how many have reported, and their categories so far. */
typedef struct {
    uint64_t total, done;
    uint64_t viable, possible, unviable;
    uint32_t complete;       /* all simulations reported                                  */
    uint32_t expired;        /* passed requestDeadlineSeconds                             */
} cave_request_progress;
/* Non-blocking. CAVE_ERR_INVALID_ARG for an unknown (fetched, cancelled) request. */
cave_status cave_server_progress(cave_server* s, uint64_t requestId, cave_request_progress* out);

/* ---- render-mode cell buffers ---------------------------------------------------------- */
/* Render mode keeps its cells in a different layout (cellStateUtils.slang:18-54, buffer mode):
 * two cells per texel along x (low nibble = even x), one texel per uint32 element, texels in
 * 8x8x8 blocks (block-major x, then y, then z) with Morton order inside a block; texel width
 * ceil(X/2) (simulationRenderer.cpp:58-68). Elements of such a buffer: */
uint64_t cave_render_buffer_elements(uint32_t X, uint32_t Y, uint32_t Z);
/* Elements of the skip grid: 8-cell chunks per axis, tiled the same way (simulationRenderer.cpp:86-95). */
uint64_t cave_render_skip_elements(uint32_t X, uint32_t Y, uint32_t Z);
/* nticks of the render mode's tick (rayMarchCompute.slang:211-280 computeMain with compute skip
 * off) on caller-owned DEVICE buffers in that layout: d_in -> d_out (may be the same buffer).
 * The rule is `params` in bitmask form; the W neighbourhood flag selects wrap-around on every
 * axis (WRAP_AT_BOUNDARY, simulationRenderer.cpp:595, :623), otherwise out-of-grid cells are
 * dead. Block-padding elements of d_out are written as 0. d_skip (device, may be NULL)
 * receives the skip grid the shader scatter-writes for the next frame after the last tick
 * (:182-205): 1 for every 8-cell chunk within one cell (clamped to the grid, not wrapped) of a
 * non-zero cell, else 0. X <= 1022. */
cave_status cave_render_step(cave_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t X, uint32_t Y, uint32_t Z,
                             const cave_sim_params* params, uint32_t nticks, uint32_t* d_skip);

/* ---- search sweeps (SearchMode + SearchSystem + RuleAggregator) ------------------------ */
/* The search flags of the reference CLI (src/main.cpp:27-44, startupConfig.h) that shape a
 * sweep. A zero step disables a sweep axis. */
typedef struct {
    uint32_t grid;                                /* --grid: chunks are grid^3 (searchMode.cpp:160, :218) */
    uint32_t gridSweepMin, gridSweepMax, gridSweepStep; /* --grid-sweep min:max:step       */
    uint32_t spawnX, spawnY, spawnZ;              /* --spawn                              */
    uint32_t spawnMode;                           /* --spawn-mode: 0 random, 1 filled     */
    float spawnDensity;                           /* --spawn-density                      */
    float densitySweepMin, densitySweepMax, densitySweepStep; /* --density-sweep           */
    uint32_t seedRuns;                            /* --seed-runs                          */
    uint32_t faces, edges, corners, wrap;         /* --neighborhood F/E/C/W               */
    uint32_t minMaxCellState, maxMaxCellState;    /* --min-cs, --max-cs-range             */
    uint32_t maxTicks;                            /* --ticks                              */
    uint32_t maxRuleBits;                         /* --max-rule-bits                      */
    uint32_t chunksPerConfig;                     /* --chunks-per-config                  */
    const char* outputFolder;                     /* --output (NULL or "" = no files)     */
    uint32_t resume;   /* 1: a chunk whose three JSONL files already hold all its results (a
                          sweep run before into the same folder, stopped or cut short) is not
                          run again: its lines go into the aggregate and the summary as read;
                          incomplete chunks are rewritten (the reference resumes at script
                          level, bench_grand_resume.ps1)                                   */
    uint32_t pad;
} cave_search_config;

typedef struct {
    uint64_t sims;           /* (rule, chunk) simulations run                          */
    uint64_t viable, possible, unviable;
    uint64_t ticks;          /* ticks run, summed over simulations                    */
    uint64_t cellUpdates;    /* ticks x grid volume, summed                           */
    uint32_t chunks;
    uint32_t uniqueRules;    /* entries of the aggregate                              */
    double deviceSeconds;    /* device time of the simulation work (CUDA events)      */
    double wallSeconds;      /* whole call                                            */
    uint32_t stopped;        /* 1: cave_search_stop ended the sweep early             */
    uint32_t pad;
    uint64_t resumedSims;    /* of sims: read from complete chunk files (resume), not run;
                                the other totals cover them too                         */
} cave_search_summary;

/* Runs a whole sweep as SearchMode::OnFrame does (searchMode.cpp:49-218 expansion,
 * :252-459 run, :1030-1054 files and aggregation) and writes, when outputFolder is set,
 * <out>cube/<prefix>_c<n>_g<X>x<Y>x<Z>_d<d>_s<s>_gpu0_{viable,possible,unviable}.jsonl per chunk
 * (searchSystem.cpp:959-978 line format, keys sorted) and <out>cube/<prefix>_aggregate.jsonl
 * (ruleAggregator.h:105-134). mode 0 runs the simulations on the device in persistent batched
 * launches, in waves of up to 2^20 simulations (CAVE_SEARCH_WAVE_SIMS overrides); mode 1 is the
 * plain path, SearchSystem's own loop -- one launch per slot per tick and a host fence per tick
 * (searchSystem.cpp:480-713), a chunk at a time. Results are appended to their chunk's files and
 * flushed after every wave (mode 0) or chunk (mode 1), as the reference appends and flushes each
 * line (searchSystem.cpp:974-977), so a sweep that is stopped or dies keeps what it wrote.
 * simLimit > 0 stops after that many simulations (for sampling the plain path). Lines within
 * a file are in rule order (slot, survival, birth); the reference writes them in completion
 * order, which depends on scheduling. A folder that cannot be created or a file that cannot be
 * written gives CAVE_ERR_IO. */
cave_status cave_search_run(cave_ctx* ctx, const cave_search_config* config, uint32_t mode, uint64_t simLimit,
                            cave_search_summary* summary);
/* Asks the cave_search_run in progress on ctx to stop (the reference's stop request,
 * searchMode.cpp:437-449): it finishes the wave or chunk on the device, writes its results, then
 * writes <out>cube/<prefix>_aggregate_partial.jsonl (when any rule finished) instead of the
 * aggregate and returns CAVE_OK with summary->stopped = 1. Safe to call from any host thread while
 * the run is in progress (the one exception to one thread per context); a request made when no
 * run is in progress is dropped by the next run's start. */
cave_status cave_search_stop(cave_ctx* ctx);

/* Reference rule-string helpers (guiSystem.cpp:92-163): "3,5-7" <-> bitmask (bit n-1 = n). */
uint64_t cave_rule_string_to_bitmask(const char* rule);
/* Writes the string form of a bitmask into out (capacity cap incl. NUL); returns its length. */
uint64_t cave_bitmask_to_rule_string(uint64_t bitmask, char* out, uint64_t cap);

/* ---- manager (host restatement) ------------------------------------------------------ */
/* One dispatch of searchManager.slang computeMain (:98-149) including NextPermutation
 * (:56-96), for callers that drive the plain path themselves. */
void cave_manager_update(const cave_grid_snapshot* snapshot, cave_grid_info* info, cave_sim_params* perms,
                         uint64_t maxPermutation, uint64_t survivalEndPermutation, uint32_t maxTicks,
                         cave_grid_info* infoCopy, cave_sim_params* permsCopy);

/* ---- valid bitmasks (permutationMath.h:101-128) ---------------------------------------- */
/* Returns the number of masks with 1..maxBits bits set among the low neighborCount bits and
 * writes up to cap of them, sorted ascending. */
uint64_t cave_enumerate_valid_bitmasks(uint32_t neighborCount, uint32_t maxBits, uint64_t* out, uint64_t cap);

#ifdef __cplusplus
}
#endif
#endif /* CAVE_CA_H */
