"""CPU oracle for CAVE's search-mode CA step -- TEST INFRASTRUCTURE ONLY.

ctypes bindings over ``oracle/cave_oracle.c`` (a plain-C restatement of the reference's
shader and host arithmetic; see the header of that file for the reference lines it
follows). Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this package, and only to check results or as the timed CPU baseline -- the product
(``cave_b200``) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libcave_oracle.so")
_lib = None

PERM_MASK = (1 << 60) - 1


class TickStats(ctypes.Structure):
    """Per-tick counters: the reference GridSnapshot (structs.h:130-136) + derived fields."""

    _fields_ = [
        ("dead", ctypes.c_uint32),
        ("dying", ctypes.c_uint32),
        ("born", ctypes.c_uint32),
        ("surviving", ctypes.c_uint32),
        ("population", ctypes.c_uint32),
        ("changed", ctypes.c_uint32),
        ("bbox_min", ctypes.c_uint32 * 3),
        ("bbox_max", ctypes.c_uint32 * 3),
    ]

    def as_tuple(self):
        return (self.dead, self.dying, self.born, self.surviving, self.population, self.changed,
                tuple(self.bbox_min), tuple(self.bbox_max))


class GridInfo(ctypes.Structure):
    """GridInfo (structs.h:79-87)."""

    _fields_ = [
        ("totalDied", ctypes.c_uint32),
        ("totalBorn", ctypes.c_uint32),
        ("ticks", ctypes.c_uint32),
        ("status", ctypes.c_uint32),
        ("maxAlive", ctypes.c_uint32),
        ("finalAlive", ctypes.c_uint32),
    ]

    def as_tuple(self):
        return (self.totalDied, self.totalBorn, self.ticks, self.status, self.maxAlive, self.finalAlive)


class Perms(ctypes.Structure):
    _fields_ = [("birthAndMaxCellStateRules", ctypes.c_uint64),
                ("survivalAndNeighborhoodRules", ctypes.c_uint64)]


class SlotResult(ctypes.Structure):
    _fields_ = [
        ("birthAndMaxCellStateRules", ctypes.c_uint64),
        ("survivalAndNeighborhoodRules", ctypes.c_uint64),
        ("info", GridInfo),
        ("category", ctypes.c_int32),
        ("pad", ctypes.c_uint32),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(_HERE, "cave_oracle.c")
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        u32, u64, i32, i64, sz = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_int64, ctypes.c_size_t
        P = ctypes.POINTER
        L.oracle_words_per_row.argtypes = [u32]
        L.oracle_words_per_row.restype = u32
        L.oracle_grid_words.argtypes = [u32, u32, u32]
        L.oracle_grid_words.restype = u64
        L.oracle_enumerate_valid_bitmasks.argtypes = [u32, u32, P(u64), sz]
        L.oracle_enumerate_valid_bitmasks.restype = sz
        L.oracle_cell_hash.argtypes = [u32, u32, u32, u32]
        L.oracle_cell_hash.restype = u32
        L.oracle_density_threshold_from_index.argtypes = [u32]
        L.oracle_density_threshold_from_index.restype = u64
        L.oracle_density_threshold_from_float.argtypes = [ctypes.c_float]
        L.oracle_density_threshold_from_float.restype = u64
        L.oracle_seed.argtypes = [u32, u32, u32, u32, u32, u32, u32, i32, u64, u32, u32, P(u32)]
        L.oracle_seed.restype = None
        L.oracle_step.argtypes = [u32, u32, u32, P(u64), P(u64), u32, u32, P(u32), P(u32), P(TickStats)]
        L.oracle_step.restype = i32
        L.oracle_step_fast.argtypes = [u32, u32, u32, P(u64), P(u64), u32, u32, P(u32), P(u32), P(u32), i32]
        L.oracle_step_fast.restype = i32
        L.oracle_derived_stats_fast.argtypes = [u32, u32, u32, P(u32), P(u32), P(TickStats), i32]
        L.oracle_derived_stats_fast.restype = None
        L.oracle_manager.argtypes = [P(u32), P(GridInfo), P(Perms), u64, u64, u32, P(GridInfo), P(Perms)]
        L.oracle_manager.restype = None
        L.oracle_run_sim.argtypes = [u32, u32, u32, P(u64), P(u64), u32, u32, P(u32), u32, i32,
                                     P(GridInfo), P(TickStats), P(u32)]
        L.oracle_run_sim.restype = i32
        L.oracle_classify.argtypes = [P(GridInfo), u32]
        L.oracle_classify.restype = i32
        L.oracle_run_slot.argtypes = [u32, u32, u32, u64, u64, u64, u64, P(u64), u32, u32, P(u32), u32, i32,
                                      P(SlotResult), sz]
        L.oracle_run_slot.restype = i64
        L.oracle_render_index.argtypes = [u32, u32, u32, u32, u32, u32]
        L.oracle_render_index.restype = u64
        L.oracle_render_elements.argtypes = [u32, u32, u32]
        L.oracle_render_elements.restype = u64
        L.oracle_render_skip_elements.argtypes = [u32, u32, u32]
        L.oracle_render_skip_elements.restype = u64
        L.oracle_render_step.argtypes = [u32, u32, u32, P(u64), i32, P(u32), P(u32), P(u32)]
        L.oracle_render_step.restype = None
        _lib = L
    return _lib


def _u32p(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def _u64p(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def words_per_row(X: int) -> int:
    return (X + 7) // 8


def grid_words(X: int, Y: int, Z: int) -> int:
    return words_per_row(X) * Y * Z


def valid_bitmasks(neighbor_count: int, max_bits: int) -> np.ndarray:
    L = lib()
    n = L.oracle_enumerate_valid_bitmasks(neighbor_count, max_bits, None, 0)
    out = np.zeros(max(n, 1), dtype=np.uint64)
    L.oracle_enumerate_valid_bitmasks(neighbor_count, max_bits, _u64p(out), n)
    return out[:n].copy()


def cell_hash(x: int, y: int, z: int, seed: int) -> int:
    return lib().oracle_cell_hash(x, y, z, seed)


def threshold_from_index(density_index: int) -> int:
    return lib().oracle_density_threshold_from_index(density_index)


def threshold_from_float(p: float) -> int:
    return lib().oracle_density_threshold_from_float(p)


def seed(X, Y, Z, spawn=(None, None, None), spawn_size_index=0, random=True, threshold=1 << 32,
         run_seed=0, max_cell_state=1) -> np.ndarray:
    sx, sy, sz = [(d if s is None else min(s, d)) for s, d in zip(spawn, (X, Y, Z))]
    out = np.zeros(grid_words(X, Y, Z), dtype=np.uint32)
    lib().oracle_seed(X, Y, Z, sx, sy, sz, spawn_size_index, 1 if random else 0, threshold, run_seed,
                      max_cell_state, _u32p(out))
    return out


def make_params(max_cell_state: int, flags: int, birth: int, survival: int, shape_id: int = 0) -> np.ndarray:
    """SimulationParameters (structs.h:89-99) with simulation.h:58 encoding of maxCellState."""
    return np.array([(((max_cell_state - 1) & 0xF) << 60) | (birth & PERM_MASK),
                     ((flags & 0xF) << 60) | (survival & PERM_MASK),
                     shape_id & 0x1F], dtype=np.uint64)


def _vb(valid):
    if valid is None:
        valid = np.zeros(1, dtype=np.uint64)
        return valid, 0
    valid = np.ascontiguousarray(valid, dtype=np.uint64)
    return valid, len(valid)


def step(X, Y, Z, params, cells, valid=None, max_rule_bits=0):
    """Literal one-tick step. Returns (new_cells, TickStats)."""
    params = np.ascontiguousarray(params, dtype=np.uint64)
    cells = np.ascontiguousarray(cells, dtype=np.uint32)
    v, nv = _vb(valid)
    out = np.zeros_like(cells)
    st = TickStats()
    rc = lib().oracle_step(X, Y, Z, _u64p(params), _u64p(v), nv, max_rule_bits, _u32p(cells), _u32p(out),
                           ctypes.byref(st))
    if rc != 0:
        raise ValueError("oracle_step: rule index outside the valid-bitmask table")
    return out, st


def step_fast(X, Y, Z, params, cells, valid=None, max_rule_bits=0, nthreads=0):
    params = np.ascontiguousarray(params, dtype=np.uint64)
    cells = np.ascontiguousarray(cells, dtype=np.uint32)
    v, nv = _vb(valid)
    out = np.zeros_like(cells)
    snap = np.zeros(4, dtype=np.uint32)
    rc = lib().oracle_step_fast(X, Y, Z, _u64p(params), _u64p(v), nv, max_rule_bits, _u32p(cells), _u32p(out),
                                _u32p(snap), nthreads)
    if rc != 0:
        raise ValueError(f"oracle_step_fast failed ({rc})")
    return out, snap


def step_stats_fast(X, Y, Z, params, cells, valid=None, max_rule_bits=0, nthreads=0):
    """One tick by the OpenMP step with every per-tick statistic (snapshot and derived), both
    computed in parallel. Returns (new_cells, TickStats); bit-identical to step()."""
    out, snap = step_fast(X, Y, Z, params, cells, valid, max_rule_bits, nthreads)
    st = TickStats()
    st.dead, st.dying, st.born, st.surviving = (int(v) for v in snap)
    lib().oracle_derived_stats_fast(X, Y, Z, _u32p(np.ascontiguousarray(cells, dtype=np.uint32)), _u32p(out),
                                    ctypes.byref(st), nthreads)
    return out, st


def manager(snapshot, info: GridInfo, perms: Perms, max_permutation, survival_end, max_ticks):
    snap = np.ascontiguousarray(snapshot, dtype=np.uint32)
    ic, pc = GridInfo(), Perms()
    lib().oracle_manager(_u32p(snap), ctypes.byref(info), ctypes.byref(perms), max_permutation, survival_end,
                         max_ticks, ctypes.byref(ic), ctypes.byref(pc))
    return ic, pc


def run_sim(X, Y, Z, params, initial, max_ticks, valid=None, max_rule_bits=0, fast=False, per_tick=False,
            final_cells=False):
    """One rule from the initial cells until status > 0. Returns (GridInfo, [TickStats], cells)."""
    params = np.ascontiguousarray(params, dtype=np.uint64)
    initial = np.ascontiguousarray(initial, dtype=np.uint32)
    v, nv = _vb(valid)
    info = GridInfo()
    pt = (TickStats * max(max_ticks, 1))() if per_tick else None
    fc = np.zeros_like(initial) if final_cells else None
    t = lib().oracle_run_sim(X, Y, Z, _u64p(params), _u64p(v), nv, max_rule_bits, _u32p(initial), max_ticks,
                             1 if fast else 0, ctypes.byref(info), pt,
                             _u32p(fc) if fc is not None else None)
    if t < 0:
        raise ValueError("oracle_run_sim failed")
    ticks = [pt[i] for i in range(t)] if per_tick else None
    return info, ticks, fc


def classify(info: GridInfo, max_cell_state: int) -> int:
    return lib().oracle_classify(ctypes.byref(info), max_cell_state)


def aggregate_lines(results, shape_id=0):
    """RuleAggregator restated (src/common/ruleAggregator.h:69-90 Record, :105-135 WriteJsonl):
    results = iterable of (birth field, survival field, ticks survived, category 0/1/2) with the
    rule fields in bitmask form. Rule identity = (birth mask, survival mask, maxCellState,
    neighbourhood flags, shape id); per rule: runs per category, min / max / average ticks and the
    viable fraction, the two averages computed in float32 and printed like a C++ ostream float
    (six significant digits, %g). Returns {rule key: JSONL line} in the reference's key order."""
    import numpy as _np

    stats = {}
    for birth, survival, ticks, cat in results:
        birth, survival = int(birth), int(survival)
        key = (birth & PERM_MASK, survival & PERM_MASK, ((birth >> 60) & 0xF) + 1, survival >> 60, shape_id)
        st = stats.setdefault(key, [0, 0, 0, 0, 0, 0xFFFFFFFF, 0])
        st[0] += 1
        st[1 + int(cat)] += 1
        st[4] = max(st[4], int(ticks))
        st[5] = min(st[5], int(ticks))
        st[6] += int(ticks)
    out = {}
    for key, (total, viable, possible, unviable, mx, mn, sm) in stats.items():
        avg = _np.float32(sm) / _np.float32(total) if total else _np.float32(0)
        rate = _np.float32(viable) / _np.float32(total) if total else _np.float32(0)
        out[key] = ("{\"birth\":%d,\"survival\":%d,\"maxCellState\":%d,\"neighborhoodFlags\":%d,\"shapeId\":%d,"
                    "\"totalRuns\":%d,\"viableRuns\":%d,\"possibleRuns\":%d,\"unviableRuns\":%d,"
                    "\"viabilityRate\":%s,\"minTicksSurvived\":%d,\"maxTicksSurvived\":%d,\"avgTicksSurvived\":%s}"
                    % (key + (total, viable, possible, unviable, "%g" % float(rate), 0 if mn == 0xFFFFFFFF else mn, mx,
                              "%g" % float(avg))))
    return out


def run_slot(X, Y, Z, start_birth_field, start_survival_field, max_permutation, survival_end, initial,
             max_ticks, valid=None, max_rule_bits=0, fast=True, cap=1 << 16):
    initial = np.ascontiguousarray(initial, dtype=np.uint32)
    v, nv = _vb(valid)
    out = (SlotResult * cap)()
    n = lib().oracle_run_slot(X, Y, Z, start_birth_field, start_survival_field, max_permutation, survival_end,
                              _u64p(v), nv, max_rule_bits, _u32p(initial), max_ticks, 1 if fast else 0, out, cap)
    if n < 0:
        raise ValueError("oracle_run_slot failed")
    return [out[i] for i in range(min(n, cap))]


# ---- cell-level helpers for tests ------------------------------------------------------
def unpack(cells: np.ndarray, X: int, Y: int, Z: int) -> np.ndarray:
    """Packed words -> uint8 [Z, Y, X] states (padding nibbles dropped)."""
    wpr = words_per_row(X)
    w = np.asarray(cells, dtype=np.uint32).reshape(Z, Y, wpr)
    nib = np.stack([(w >> np.uint32(4 * k)) & np.uint32(0xF) for k in range(8)], axis=-1)
    return nib.reshape(Z, Y, wpr * 8)[:, :, :X].astype(np.uint8)


def pack(states: np.ndarray) -> np.ndarray:
    """uint8 [Z, Y, X] states -> packed words with zero padding."""
    Z, Y, X = states.shape
    wpr = words_per_row(X)
    full = np.zeros((Z, Y, wpr * 8), dtype=np.uint32)
    full[:, :, :X] = states & 0xF
    full = full.reshape(Z, Y, wpr, 8)
    out = np.zeros((Z, Y, wpr), dtype=np.uint32)
    for k in range(8):
        out |= full[:, :, :, k] << np.uint32(4 * k)
    return out.reshape(-1)


# ---- render-mode layout (cellStateUtils.slang:18-54) -----------------------------------
def _expand3(v):
    v = v & 7
    v = (v | (v << 8)) & 0x100F
    v = (v | (v << 4)) & 0x10C30C3
    v = (v | (v << 2)) & 0x1249249
    return v


def render_elements(X, Y, Z) -> int:
    return int(lib().oracle_render_elements(X, Y, Z))


def render_skip_elements(X, Y, Z) -> int:
    return int(lib().oracle_render_skip_elements(X, Y, Z))


def render_indices(X, Y, Z) -> np.ndarray:
    """Element index of every texel, as an array [Z, Y, ceil(X/2)] (vectorised restatement of
    cellStateUtils.slang:37-45)."""
    W = (X + 1) // 2
    nbx, nby = (W + 7) // 8, (Y + 7) // 8
    tz, ty, tx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(W), indexing="ij")
    block = (tz // 8) * nbx * nby + (ty // 8) * nbx + (tx // 8)
    m = _expand3(tx % 8) | (_expand3(ty % 8) << 1) | (_expand3(tz % 8) << 2)
    return (block * 512 + m).astype(np.int64)


def render_pack(states: np.ndarray) -> np.ndarray:
    """uint8 [Z, Y, X] states -> the render mode's tiled buffer (uint32 per texel, 2 cells per
    texel along x, block padding 0)."""
    Z, Y, X = states.shape
    W = (X + 1) // 2
    full = np.zeros((Z, Y, 2 * W), dtype=np.uint32)
    full[:, :, :X] = states & 0xF
    texel = full[:, :, 0::2] | (full[:, :, 1::2] << np.uint32(4))
    out = np.zeros(render_elements(X, Y, Z), dtype=np.uint32)
    out[render_indices(X, Y, Z).reshape(-1)] = texel.reshape(-1)
    return out


def render_unpack(buf: np.ndarray, X, Y, Z) -> np.ndarray:
    W = (X + 1) // 2
    texel = np.asarray(buf, dtype=np.uint32)[render_indices(X, Y, Z)]
    full = np.zeros((Z, Y, 2 * W), dtype=np.uint8)
    full[:, :, 0::2] = texel & 0xF
    full[:, :, 1::2] = (texel >> 4) & 0xF
    return full[:, :, :X]


def render_step(X, Y, Z, params, buf, wrap, nticks=1, skip=False):
    """nticks of rayMarchCompute computeMain (compute skip off) on a render-layout buffer.
    Returns (buffer, skip grid after the last tick or None)."""
    params = np.ascontiguousarray(params, dtype=np.uint64)
    cur = np.ascontiguousarray(buf, dtype=np.uint32).copy()
    sk = None
    for t in range(nticks):
        out = np.zeros_like(cur)
        last = t == nticks - 1
        sk = np.zeros(render_skip_elements(X, Y, Z), dtype=np.uint32) if (skip and last) else None
        lib().oracle_render_step(X, Y, Z, _u64p(params), 1 if wrap else 0, _u32p(cur), _u32p(out),
                                 _u32p(sk) if sk is not None else None)
        cur = out
    return cur, sk
