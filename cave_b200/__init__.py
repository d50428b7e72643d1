"""cave_b200 -- B200 (sm_100a) CA stepping for CAVE's search path, Python binding.

Thin ctypes binding over ``libcave_ca.so`` (the C ABI declared in ``include/cave_ca.h``).
All computation happens in the library's CUDA kernels; this module only marshals arguments.
If the shared library is missing the import of any entry point raises -- there is no CPU
fallback in the product.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# CAVE_LIB selects another build of the library, e.g. cave_b200/libcave_ca_checked.so
LIB_PATH = os.environ.get("CAVE_LIB") or os.path.join(_HERE, "libcave_ca.so")
HEADER_PATH = os.path.join(_HERE, "..", "include", "cave_ca.h")

PERM_MASK = (1 << 60) - 1

OK, ERR_INVALID_ARG, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_NOT_READY, ERR_TIMEOUT, ERR_IO, ERR_INTERNAL = range(8)

u8, u32, u64, i32, sz = ctypes.c_uint8, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_size_t
P = ctypes.POINTER


class SimParams(ctypes.Structure):
    _fields_ = [("birthAndMaxCellStateRules", u64), ("survivalAndNeighborhoodRules", u64),
                ("shapeAndGridConfiguration", u64)]


class GridSnapshot(ctypes.Structure):
    _fields_ = [("numberOfDeadCells", u32), ("numberOfDyingCells", u32), ("numberOfCellsBorn", u32),
                ("numberOfSurvivingCells", u32)]

    def as_tuple(self):
        return (self.numberOfDeadCells, self.numberOfDyingCells, self.numberOfCellsBorn, self.numberOfSurvivingCells)


class GridInfo(ctypes.Structure):
    _fields_ = [("totalNumberOfCellsThatDied", u32), ("totalNumberOfCellsThatWereBorn", u32),
                ("numberOfSimulationTicksSurvived", u32), ("status", u32), ("maxAliveCount", u32),
                ("finalAliveCount", u32)]

    def as_tuple(self):
        return (self.totalNumberOfCellsThatDied, self.totalNumberOfCellsThatWereBorn,
                self.numberOfSimulationTicksSurvived, self.status, self.maxAliveCount, self.finalAliveCount)


class ChunkConfig(ctypes.Structure):
    _fields_ = [(n, u32) for n in (
        "shapeId", "gridDimensionX", "gridDimensionY", "gridDimensionZ", "spawnAreaDimensionX",
        "spawnAreaDimensionY", "spawnAreaDimensionZ", "spawnPlacementId", "spawnRegionShapeId", "spawnSizeIndex",
        "spawnDensityIndex", "runSeedIndex", "partitionIndex", "partitionCount")]


class TickStats(ctypes.Structure):
    _fields_ = [("snapshot", GridSnapshot), ("population", u32), ("changed", u32), ("bbox_min", u32 * 3),
                ("bbox_max", u32 * 3)]

    def as_tuple(self):
        return self.snapshot.as_tuple() + (self.population, self.changed, tuple(self.bbox_min),
                                           tuple(self.bbox_max))


class SimDesc(ctypes.Structure):
    _fields_ = [("params", SimParams), ("init", u32), ("maxTicks", u32), ("validTable", u32), ("tag", u32)]


class SimResult(ctypes.Structure):
    _fields_ = [("info", GridInfo), ("category", u32), ("tag", u32), ("population", u32), ("activeTicks", u32),
                ("totalChanged", u64), ("bbox_min", u32 * 3), ("bbox_max", u32 * 3), ("params", SimParams),
                ("error", u32), ("pad", u32)]


class SearchConfig(ctypes.Structure):
    _fields_ = [("grid", u32), ("gridSweepMin", u32), ("gridSweepMax", u32), ("gridSweepStep", u32),
                ("spawnX", u32), ("spawnY", u32), ("spawnZ", u32), ("spawnMode", u32),
                ("spawnDensity", ctypes.c_float), ("densitySweepMin", ctypes.c_float),
                ("densitySweepMax", ctypes.c_float), ("densitySweepStep", ctypes.c_float), ("seedRuns", u32),
                ("faces", u32), ("edges", u32), ("corners", u32), ("wrap", u32), ("minMaxCellState", u32),
                ("maxMaxCellState", u32), ("maxTicks", u32), ("maxRuleBits", u32), ("chunksPerConfig", u32),
                ("outputFolder", ctypes.c_char_p), ("resume", u32), ("pad", u32)]


class SearchSummary(ctypes.Structure):
    _fields_ = [("sims", u64), ("viable", u64), ("possible", u64), ("unviable", u64), ("ticks", u64),
                ("cellUpdates", u64), ("chunks", u32), ("uniqueRules", u32), ("deviceSeconds", ctypes.c_double),
                ("wallSeconds", ctypes.c_double), ("stopped", u32), ("pad", u32), ("resumedSims", u64)]


def search_config(grid=49, spawn=11, spawn_mode="filled", density=0.5, neighborhood="F", min_cs=3, max_cs=10,
                  ticks=50, max_rule_bits=0, chunks_per_config=1, seed_runs=1, grid_sweep=None, density_sweep=None,
                  output=None, resume=False) -> SearchConfig:
    """SearchConfig from the reference CLI's search flags (defaults as src/main.cpp:29-44, except
    --chunks-per-config, whose partitions only change scheduling)."""
    c = SearchConfig()
    c.grid = grid
    if grid_sweep:
        c.gridSweepMin, c.gridSweepMax, c.gridSweepStep = grid_sweep
    c.spawnX = c.spawnY = c.spawnZ = spawn
    c.spawnMode = 0 if spawn_mode == "random" else 1
    c.spawnDensity = density
    if density_sweep:
        c.densitySweepMin, c.densitySweepMax, c.densitySweepStep = density_sweep
    c.seedRuns = seed_runs
    c.faces, c.edges, c.corners, c.wrap = [int(ch in neighborhood) for ch in "FECW"]
    c.minMaxCellState, c.maxMaxCellState = min_cs, max_cs
    c.maxTicks = ticks
    c.maxRuleBits = max_rule_bits
    c.chunksPerConfig = chunks_per_config
    c.outputFolder = (output.encode() if output else None)
    c.resume = 1 if resume else 0
    return c


def rule_string_to_bitmask(s: str) -> int:
    return int(lib().cave_rule_string_to_bitmask(s.encode()))


def bitmask_to_rule_string(mask: int) -> str:
    buf = ctypes.create_string_buffer(512)
    lib().cave_bitmask_to_rule_string(mask, buf, 512)
    return buf.value.decode()


SIM_DESC_DTYPE = np.dtype([("birth", "<u8"), ("survival", "<u8"), ("shape", "<u8"), ("init", "<u4"),
                           ("maxTicks", "<u4"), ("validTable", "<u4"), ("tag", "<u4")])
SIM_RESULT_DTYPE = np.dtype([("info", "<u4", (6,)), ("category", "<u4"), ("tag", "<u4"), ("population", "<u4"),
                             ("activeTicks", "<u4"), ("totalChanged", "<u8"), ("bbox_min", "<u4", (3,)),
                             ("bbox_max", "<u4", (3,)), ("birth", "<u8"), ("survival", "<u8"), ("shape", "<u8"),
                             ("error", "<u4"), ("pad", "<u4")])
assert SIM_DESC_DTYPE.itemsize == ctypes.sizeof(SimDesc)
assert SIM_RESULT_DTYPE.itemsize == ctypes.sizeof(SimResult)


class BatchOptions(ctypes.Structure):
    _fields_ = [("autotune", u32), ("tiledOnly", u32), ("ticksPerRound", u32), ("pad", u32), ("memoryBudget", u64)]


class ServerOptions(ctypes.Structure):
    _fields_ = [("hbmBudget", u64), ("maxInFlight", u32), ("ticksPerRound", u32), ("autotune", u32),
                ("tiledOnly", u32), ("maxActiveCells", u64), ("requestDeadlineSeconds", ctypes.c_double)]


class RequestProgress(ctypes.Structure):
    _fields_ = [("total", u64), ("done", u64), ("viable", u64), ("possible", u64), ("unviable", u64),
                ("complete", u32), ("expired", u32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", u64), ("completed", u64), ("simsCompleted", u64), ("cellUpdates", u64),
                ("p50LatencySeconds", ctypes.c_double), ("p99LatencySeconds", ctypes.c_double),
                ("busySeconds", ctypes.c_double), ("peakBytes", u64), ("rounds", u64), ("tickLaunches", u64),
                ("residentLaunches", u64), ("tuneMs", ctypes.c_double), ("expired", u64)]


REQUEST_SIM_DTYPE = np.dtype([("X", "<u4"), ("Y", "<u4"), ("Z", "<u4"), ("maxTicks", "<u4"), ("birth", "<u8"),
                              ("survival", "<u8"), ("shape", "<u8"), ("spawnX", "<u4"), ("spawnY", "<u4"),
                              ("spawnZ", "<u4"), ("runSeedIndex", "<u4"), ("threshold", "<u8"), ("tag", "<u4"),
                              ("pad", "<u4")])


class Timing(ctypes.Structure):
    _fields_ = [("ticks", u32), ("launches", u32), ("tick_ms", ctypes.c_float), ("convert_ms", ctypes.c_float),
                ("total_ms", ctypes.c_float)]


class CaveError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{msg} (status {code})")
        self.code = code


_lib = None

# name -> (restype, argtypes); every entry point of include/cave_ca.h
_SIGS = {
    "cave_ctx_create": (i32, [i32, P(ctypes.c_void_p)]),
    "cave_ctx_destroy": (None, [ctypes.c_void_p]),
    "cave_status_string": (ctypes.c_char_p, [i32]),
    "cave_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "cave_ctx_synchronize": (i32, [ctypes.c_void_p]),
    "cave_ctx_set_timing": (i32, [ctypes.c_void_p, i32]),
    "cave_ctx_last_timing": (i32, [ctypes.c_void_p, P(Timing)]),
    "cave_run_host": (i32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, u64, P(SimParams), P(u64), u32, u32,
                            u32, u32, P(TickStats), P(GridInfo)]),
    "cave_run_noalloc": (i32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, u32, u32, u32, P(SimParams),
                               P(u64), u32, u32, u32, u32, ctypes.c_void_p, P(GridInfo)]),
    "cave_grid_create": (i32, [ctypes.c_void_p, u32, u32, u32, P(ctypes.c_void_p)]),
    "cave_grid_destroy": (None, [ctypes.c_void_p]),
    "cave_grid_words": (u64, [u32, u32, u32]),
    "cave_grid_upload": (i32, [ctypes.c_void_p, P(u32), u64]),
    "cave_grid_download": (i32, [ctypes.c_void_p, P(u32), u64]),
    "cave_grid_seed": (i32, [ctypes.c_void_p, P(ChunkConfig), u32]),
    "cave_grid_seed_threshold": (i32, [ctypes.c_void_p, u32, u32, u32, u64, u32, u32]),
    "cave_step": (i32, [ctypes.c_void_p, P(SimParams), P(u64), u32, u32, u32, P(TickStats)]),
    "cave_run": (i32, [ctypes.c_void_p, P(SimParams), P(u64), u32, u32, u32, u32, P(TickStats), P(GridInfo)]),
    "cave_prepare_rule": (i32, [ctypes.c_void_p, P(SimParams), P(u64), u32, u32]),
    "cave_jit_compile": (i32, [P(SimParams), P(u64), u32, u32, ctypes.c_char_p, ctypes.c_size_t]),
    "cave_jit_stats": (None, [P(u32), P(u64)]),
    "cave_jit_compile_async": (i32, [P(SimParams), P(u64), u32, u32]),
    "cave_manager_update": (None, [P(GridSnapshot), P(GridInfo), P(SimParams), u64, u64, u32, P(GridInfo),
                                   P(SimParams)]),
    "cave_enumerate_valid_bitmasks": (u64, [u32, u32, P(u64), u64]),
    "cave_batch_create": (i32, [ctypes.c_void_p, P(ctypes.c_void_p)]),
    "cave_batch_destroy": (None, [ctypes.c_void_p]),
    "cave_batch_add_init": (i32, [ctypes.c_void_p, u32, u32, u32, P(u32), u64, P(u32)]),
    "cave_batch_add_init_seeded": (i32, [ctypes.c_void_p, u32, u32, u32, u32, u32, u32, u64, u32, u32, P(u32)]),
    "cave_batch_add_table": (i32, [ctypes.c_void_p, P(u64), u32, P(u32)]),
    "cave_batch_add_sims": (i32, [ctypes.c_void_p, P(SimDesc), u64, u32]),
    "cave_batch_launch": (i32, [ctypes.c_void_p]),
    "cave_batch_poll": (i32, [ctypes.c_void_p]),
    "cave_batch_results": (i32, [ctypes.c_void_p, P(SimResult), u64]),
    "cave_batch_size": (u64, [ctypes.c_void_p]),
    "cave_batch_run_plain": (i32, [ctypes.c_void_p, u32, P(ctypes.c_double)]),
    "cave_batch_set_options": (i32, [ctypes.c_void_p, P(BatchOptions)]),
    "cave_batch_plan": (u64, [ctypes.c_void_p, ctypes.c_char_p, u64]),
    "cave_server_create": (i32, [ctypes.c_void_p, P(ServerOptions), P(ctypes.c_void_p)]),
    "cave_server_destroy": (None, [ctypes.c_void_p]),
    "cave_server_submit": (i32, [ctypes.c_void_p, ctypes.c_void_p, u64, P(u64)]),
    "cave_server_poll": (i32, [ctypes.c_void_p, P(u64), u64, P(u64)]),
    "cave_server_wait": (i32, [ctypes.c_void_p, u64, ctypes.c_double]),
    "cave_server_cancel": (i32, [ctypes.c_void_p, u64]),
    "cave_server_progress": (i32, [ctypes.c_void_p, u64, ctypes.c_void_p]),
    "cave_server_fetch": (i32, [ctypes.c_void_p, u64, ctypes.c_void_p, u64, P(ctypes.c_double)]),
    "cave_server_get_stats": (i32, [ctypes.c_void_p, P(ServerStats)]),
    "cave_render_buffer_elements": (u64, [u32, u32, u32]),
    "cave_render_skip_elements": (u64, [u32, u32, u32]),
    "cave_render_step": (i32, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, u32, u32, u32, P(SimParams), u32,
                               ctypes.c_void_p]),
    "cave_search_run": (i32, [ctypes.c_void_p, P(SearchConfig), u32, u64, P(SearchSummary)]),
    "cave_search_stop": (i32, [ctypes.c_void_p]),
    "cave_rule_string_to_bitmask": (u64, [ctypes.c_char_p]),
    "cave_bitmask_to_rule_string": (u64, [u64, ctypes.c_char_p, u64]),
}


def jit_compile(params: "SimParams", valid=None, max_rule_bits=0):
    """Compiles the rule-specialised tick kernel without a device. Returns (ok, compiler log)."""
    v = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint64)
    buf = ctypes.create_string_buffer(1 << 16)
    rc = lib().cave_jit_compile(ctypes.byref(params), _u64p(v), 0 if v is None else v.size, max_rule_bits, buf,
                                len(buf))
    return rc == 0, buf.value.decode(errors="replace")


def jit_compile_async(params: "SimParams", valid=None, max_rule_bits=0):
    """Starts compiling the rule-specialised tick kernel in the background (no device)."""
    v = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint64)
    rc = lib().cave_jit_compile_async(ctypes.byref(params), _u64p(v), 0 if v is None else v.size, max_rule_bits)
    if rc != 0:
        raise CaveError(rc, "cave_jit_compile_async")


def jit_stats():
    """(specialised kernels loaded in this process, tick launches made with them)."""
    a, b = u32(), u64()
    lib().cave_jit_stats(ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def lib():
    """Loads libcave_ca.so (raises OSError if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: run `python -m cave_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _u32p(a):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(P(u32))


def _u64p(a):
    if a is None:
        return None
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(P(u64))


def make_params(max_cell_state, flags, birth, survival, shape_id=0) -> SimParams:
    """SimulationParameters with the simulation.h:58 maxCellState encoding."""
    return SimParams((((max_cell_state - 1) & 0xF) << 60) | (birth & PERM_MASK),
                     ((flags & 0xF) << 60) | (survival & PERM_MASK), shape_id & 0x1F)


def threshold_from_fill(p: float) -> int:
    """Fill threshold of the reference's raw-density seeding (searchSystem.cpp:260-262):
    (uint32)((double)(float)p * 2^32); 2^32 (every cell of the box) for p >= 1."""
    if p >= 1.0:
        return 1 << 32
    return int(float(np.float32(p)) * 4294967296.0) & 0xFFFFFFFF


def grid_words(X, Y, Z) -> int:
    return int(lib().cave_grid_words(X, Y, Z))


def valid_bitmasks(neighbor_count, max_bits) -> np.ndarray:
    n = lib().cave_enumerate_valid_bitmasks(neighbor_count, max_bits, None, 0)
    out = np.zeros(max(n, 1), dtype=np.uint64)
    lib().cave_enumerate_valid_bitmasks(neighbor_count, max_bits, _u64p(out), n)
    return out[:n].copy()


class Context:
    """One device + stream (cave_ctx)."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        rc = lib().cave_ctx_create(device, ctypes.byref(h))
        if rc != OK:
            raise CaveError(rc, f"cave_ctx_create({device}) failed: {lib().cave_status_string(rc).decode()}")
        self.h = h

    def check(self, rc, what):
        if rc != OK:
            raise CaveError(rc, f"{what}: {lib().cave_status_string(rc).decode()}: "
                                f"{lib().cave_last_error(self.h).decode()}")

    def synchronize(self):
        self.check(lib().cave_ctx_synchronize(self.h), "cave_ctx_synchronize")

    def prepare_rule(self, params: SimParams, valid=None, max_rule_bits=0):
        """Compiles (or loads from the cache) the rule-specialised tick kernel for this rule
        now, so later streaming runs with it use it (no-op when CAVE_JIT=off)."""
        v = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint64)
        self.check(lib().cave_prepare_rule(self.h, ctypes.byref(params), _u64p(v), 0 if v is None else v.size,
                                           max_rule_bits), "cave_prepare_rule")

    def set_timing(self, enable=True):
        self.check(lib().cave_ctx_set_timing(self.h, 1 if enable else 0), "cave_ctx_set_timing")

    def last_timing(self) -> Timing:
        t = Timing()
        self.check(lib().cave_ctx_last_timing(self.h, ctypes.byref(t)), "cave_ctx_last_timing")
        return t

    def close(self):
        if self.h:
            lib().cave_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Grid:
    """A device grid in the reference's padded nibble layout (cave_grid)."""

    def __init__(self, ctx: Context, X, Y, Z):
        self.ctx, self.X, self.Y, self.Z = ctx, X, Y, Z
        h = ctypes.c_void_p()
        ctx.check(lib().cave_grid_create(ctx.h, X, Y, Z, ctypes.byref(h)), "cave_grid_create")
        self.h = h
        self.words = grid_words(X, Y, Z)

    def close(self):
        if self.h:
            lib().cave_grid_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, words):
        w = np.ascontiguousarray(words, dtype=np.uint32)
        self.ctx.check(lib().cave_grid_upload(self.h, _u32p(w), w.size), "cave_grid_upload")

    def download(self) -> np.ndarray:
        out = np.zeros(self.words, dtype=np.uint32)
        self.ctx.check(lib().cave_grid_download(self.h, _u32p(out), out.size), "cave_grid_download")
        return out

    def seed(self, chunk: ChunkConfig, max_cell_state):
        self.ctx.check(lib().cave_grid_seed(self.h, ctypes.byref(chunk), max_cell_state), "cave_grid_seed")

    def seed_threshold(self, spawn, threshold, run_seed, max_cell_state):
        self.ctx.check(lib().cave_grid_seed_threshold(self.h, spawn[0], spawn[1], spawn[2], threshold, run_seed,
                                                      max_cell_state), "cave_grid_seed_threshold")

    def step(self, params: SimParams, nticks=1, valid=None, max_rule_bits=0, stats=True):
        """Plain path (one launch per tick). Returns the list of per-tick TickStats."""
        v = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint64)
        pt = (TickStats * max(nticks, 1))() if stats else None
        self.ctx.check(lib().cave_step(self.h, ctypes.byref(params), _u64p(v), 0 if v is None else v.size,
                                       max_rule_bits, nticks, pt), "cave_step")
        return [pt[i] for i in range(nticks)] if stats else None

    def run(self, params: SimParams, nticks, max_ticks=None, valid=None, max_rule_bits=0, stats=True):
        """Streaming path. Returns (per-tick TickStats list, GridInfo)."""
        v = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint64)
        pt = (TickStats * max(nticks, 1))() if stats else None
        info = GridInfo()
        self.ctx.check(lib().cave_run(self.h, ctypes.byref(params), _u64p(v), 0 if v is None else v.size,
                                      max_rule_bits, nticks, nticks if max_ticks is None else max_ticks, pt,
                                      ctypes.byref(info)), "cave_run")
        return ([pt[i] for i in range(nticks)] if stats else None), info

    def run_host(self, in_ptr, out_ptr, params: SimParams, nticks, max_ticks=None, valid=None, max_rule_bits=0,
                 stats=True):
        """Streaming path with host buffers (raw pointers to `words` uint32 each, ideally pinned)."""
        v = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint64)
        pt = (TickStats * max(nticks, 1))() if stats else None
        info = GridInfo()
        self.ctx.check(lib().cave_run_host(self.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr), self.words,
                                           ctypes.byref(params), _u64p(v), 0 if v is None else v.size, max_rule_bits,
                                           nticks, nticks if max_ticks is None else max_ticks, pt,
                                           ctypes.byref(info)), "cave_run_host")
        return ([pt[i] for i in range(nticks)] if stats else None), info


NOALLOC_SCRATCH_BYTES = 32 << 20


def result_records(res: np.ndarray, index) -> np.ndarray:
    """Simulation results (SIM_RESULT_DTYPE) packed as 18 little-endian uint32 each, the form
    the golden fixtures hash: index, GridInfo (6), category, population, activeTicks,
    totalChanged (low, high word), bbox_min (3), bbox_max (3)."""
    n = res.size
    out = np.zeros((n, 18), dtype="<u4")
    out[:, 0] = np.asarray(index, dtype=np.uint64) & 0xFFFFFFFF
    out[:, 1:7] = res["info"]
    out[:, 7] = res["category"]
    out[:, 8] = res["population"]
    out[:, 9] = res["activeTicks"]
    out[:, 10] = res["totalChanged"] & 0xFFFFFFFF
    out[:, 11] = res["totalChanged"] >> 32
    out[:, 12:15] = res["bbox_min"]
    out[:, 15:18] = res["bbox_max"]
    return out


def tick_records(ticks) -> np.ndarray:
    """Per-tick statistics (TickStats list) as a (ticks, 12) little-endian uint32 array: the
    GridSnapshot (dead, dying, born, surviving), population, changed, bbox_min, bbox_max."""
    return np.frombuffer(b"".join(bytes(t) for t in ticks), dtype="<u4").reshape(-1, 12)


def run_noalloc(ctx: Context, in_ptr, out_ptr, X, Y, Z, params: SimParams, nticks, max_ticks=None, valid=None,
                max_rule_bits=0, per_tick_ptr=None) -> GridInfo:
    """cave_run_noalloc: the streaming run on caller-owned device buffers (device addresses as
    ints; per_tick_ptr: device array of nticks TickStats, or None). Allocates no device memory;
    its scratch is one static array of NOALLOC_SCRATCH_BYTES per GPU. Returns the GridInfo."""
    v = None if valid is None else np.ascontiguousarray(valid, dtype=np.uint64)
    info = GridInfo()
    ctx.check(lib().cave_run_noalloc(ctx.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr), X, Y, Z,
                                     ctypes.byref(params), _u64p(v), 0 if v is None else v.size, max_rule_bits,
                                     nticks, nticks if max_ticks is None else max_ticks,
                                     ctypes.c_void_p(per_tick_ptr or 0), ctypes.byref(info)), "cave_run_noalloc")
    return info


def render_buffer_elements(X, Y, Z) -> int:
    return int(lib().cave_render_buffer_elements(X, Y, Z))


def render_skip_elements(X, Y, Z) -> int:
    return int(lib().cave_render_skip_elements(X, Y, Z))


def render_step(ctx: Context, in_ptr, out_ptr, X, Y, Z, params: SimParams, nticks=1, skip_ptr=None):
    """cave_render_step on device buffers (addresses as ints) in the render mode's layout."""
    ctx.check(lib().cave_render_step(ctx.h, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr), X, Y, Z,
                                     ctypes.byref(params), nticks, ctypes.c_void_p(skip_ptr or 0)), "cave_render_step")


def search_run(ctx: Context, config: SearchConfig, plain=False, sim_limit=0) -> SearchSummary:
    """A whole search sweep (cave_search_run); mode plain = the per-slot per-tick path."""
    s = SearchSummary()
    ctx.check(lib().cave_search_run(ctx.h, ctypes.byref(config), 1 if plain else 0, sim_limit, ctypes.byref(s)),
              "cave_search_run")
    return s


def search_stop(ctx: Context):
    """Asks the search_run in progress on ctx (in another thread) to stop after its current wave."""
    ctx.check(lib().cave_search_stop(ctx.h), "cave_search_stop")


def manager_update(snapshot: GridSnapshot, info: GridInfo, perms: SimParams, max_permutation, survival_end,
                   max_ticks):
    ic, pc = GridInfo(), SimParams()
    lib().cave_manager_update(ctypes.byref(snapshot), ctypes.byref(info), ctypes.byref(perms), max_permutation,
                              survival_end, max_ticks, ctypes.byref(ic), ctypes.byref(pc))
    return ic, pc


class Batch:
    """Many independent simulations run to completion on the device (cave_batch)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        h = ctypes.c_void_p()
        ctx.check(lib().cave_batch_create(ctx.h, ctypes.byref(h)), "cave_batch_create")
        self.h = h

    def close(self):
        if self.h:
            lib().cave_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add_init(self, X, Y, Z, words) -> int:
        w = np.ascontiguousarray(words, dtype=np.uint32)
        ix = u32()
        self.ctx.check(lib().cave_batch_add_init(self.h, X, Y, Z, _u32p(w), w.size, ctypes.byref(ix)),
                       "cave_batch_add_init")
        return ix.value

    def add_init_seeded(self, X, Y, Z, spawn, threshold, run_seed, max_cell_state) -> int:
        ix = u32()
        self.ctx.check(lib().cave_batch_add_init_seeded(self.h, X, Y, Z, spawn[0], spawn[1], spawn[2], threshold,
                                                        run_seed, max_cell_state, ctypes.byref(ix)),
                       "cave_batch_add_init_seeded")
        return ix.value

    def add_table(self, valid) -> int:
        v = np.ascontiguousarray(valid, dtype=np.uint64)
        ix = u32()
        self.ctx.check(lib().cave_batch_add_table(self.h, _u64p(v), v.size, ctypes.byref(ix)), "cave_batch_add_table")
        return ix.value

    def add_sims(self, descs, max_rule_bits=0):
        arr = (SimDesc * len(descs))(*descs)
        self.ctx.check(lib().cave_batch_add_sims(self.h, arr, len(descs), max_rule_bits), "cave_batch_add_sims")

    def add_sims_array(self, arr: np.ndarray, max_rule_bits=0):
        """Simulations from a numpy array of dtype SIM_DESC_DTYPE (same layout as cave_sim_desc)."""
        assert arr.dtype == SIM_DESC_DTYPE and arr.flags["C_CONTIGUOUS"]
        self.ctx.check(lib().cave_batch_add_sims(self.h, arr.ctypes.data_as(P(SimDesc)), arr.size, max_rule_bits),
                       "cave_batch_add_sims")

    def results_array(self, out: np.ndarray = None) -> np.ndarray:
        """All results as a numpy array of dtype SIM_RESULT_DTYPE, written into `out` when given
        (e.g. a view of pinned host memory, which the device writes at full link speed). Read the
        results once per launch: simulations that ran tiled hand theirs over on the first read."""
        n = lib().cave_batch_size(self.h)
        if out is None:
            out = np.zeros(max(n, 1), dtype=SIM_RESULT_DTYPE)
        elif not (isinstance(out, np.ndarray) and out.dtype == SIM_RESULT_DTYPE and out.flags["C_CONTIGUOUS"]
                  and out.flags["WRITEABLE"] and out.size >= n):
            raise ValueError(f"results_array: out must be a writeable C-contiguous array of SIM_RESULT_DTYPE "
                             f"with at least {n} elements")
        self.ctx.check(lib().cave_batch_results(self.h, out.ctypes.data_as(P(SimResult)), n), "cave_batch_results")
        return out[:n]

    def set_options(self, autotune=False, tiled_only=False, ticks_per_round=0, memory_budget=0):
        o = BatchOptions(1 if autotune else 0, 1 if tiled_only else 0, ticks_per_round, 0, memory_budget)
        self.ctx.check(lib().cave_batch_set_options(self.h, ctypes.byref(o)), "cave_batch_set_options")

    def plan(self):
        """How each grid class of the last launch ran (list of dicts)."""
        import json

        n = lib().cave_batch_plan(self.h, None, 0)
        buf = ctypes.create_string_buffer(n + 1)
        lib().cave_batch_plan(self.h, buf, n + 1)
        return json.loads(buf.value.decode() or "[]")

    def launch(self):
        self.ctx.check(lib().cave_batch_launch(self.h), "cave_batch_launch")

    def run_plain(self, slots) -> float:
        """Plain path (one launch per slot per tick); returns device seconds."""
        s = ctypes.c_double()
        self.ctx.check(lib().cave_batch_run_plain(self.h, slots, ctypes.byref(s)), "cave_batch_run_plain")
        return s.value

    def poll(self) -> bool:
        rc = lib().cave_batch_poll(self.h)
        if rc == ERR_NOT_READY:
            return False
        self.ctx.check(rc, "cave_batch_poll")
        return True

    def results(self):
        n = lib().cave_batch_size(self.h)
        out = (SimResult * max(n, 1))()
        self.ctx.check(lib().cave_batch_results(self.h, out, n), "cave_batch_results")
        return [out[i] for i in range(n)]


def request_sims(n) -> np.ndarray:
    """An empty request (numpy array of cave_request_sim)."""
    return np.zeros(n, dtype=REQUEST_SIM_DTYPE)


class Server:
    """Sweep requests served as they arrive (cave_server): continuous batching on one GPU."""

    def __init__(self, ctx: Context, hbm_budget=0, max_in_flight=0, ticks_per_round=0, autotune=False,
                 tiled_only=False, max_active_cells=0, request_deadline=0.0):
        self.ctx = ctx
        o = ServerOptions(hbm_budget, max_in_flight, ticks_per_round, 1 if autotune else 0, 1 if tiled_only else 0,
                          max_active_cells, request_deadline)
        h = ctypes.c_void_p()
        ctx.check(lib().cave_server_create(ctx.h, ctypes.byref(o), ctypes.byref(h)), "cave_server_create")
        self.h = h
        self.sizes = {}

    def close(self):
        if self.h:
            lib().cave_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, sims: np.ndarray) -> int:
        assert sims.dtype == REQUEST_SIM_DTYPE and sims.flags["C_CONTIGUOUS"]
        rid = u64()
        self.ctx.check(lib().cave_server_submit(self.h, sims.ctypes.data, sims.size, ctypes.byref(rid)),
                       "cave_server_submit")
        self.sizes[rid.value] = sims.size
        return rid.value

    def poll(self, cap=4096):
        ids = (u64 * cap)()
        n = u64()
        self.ctx.check(lib().cave_server_poll(self.h, ids, cap, ctypes.byref(n)), "cave_server_poll")
        return [ids[i] for i in range(n.value)]

    def wait(self, rid, timeout=0.0):
        rc = lib().cave_server_wait(self.h, rid, timeout)
        if rc == ERR_TIMEOUT:
            return False
        self.ctx.check(rc, "cave_server_wait")
        return True

    def progress(self, rid) -> RequestProgress:
        """Simulations of the request that have reported, and their categories so far."""
        p = RequestProgress()
        self.ctx.check(lib().cave_server_progress(self.h, rid, ctypes.byref(p)), "cave_server_progress")
        return p

    def cancel(self, rid):
        """Cancels a request: queued simulations leave the queue, running ones finish unreported."""
        self.ctx.check(lib().cave_server_cancel(self.h, rid), "cave_server_cancel")
        self.sizes.pop(rid, None)

    def fetch(self, rid):
        """(results as SIM_RESULT_DTYPE array, latency seconds) of a completed request."""
        n = self.sizes.pop(rid)
        out = np.zeros(n, dtype=SIM_RESULT_DTYPE)
        lat = ctypes.c_double()
        self.ctx.check(lib().cave_server_fetch(self.h, rid, out.ctypes.data, n, ctypes.byref(lat)),
                       "cave_server_fetch")
        return out, lat.value

    def stats(self) -> ServerStats:
        st = ServerStats()
        self.ctx.check(lib().cave_server_get_stats(self.h, ctypes.byref(st)), "cave_server_get_stats")
        return st
