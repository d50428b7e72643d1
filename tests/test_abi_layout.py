"""The Python binding's structure layouts against the C header: every ctypes Structure and numpy
record dtype that crosses the C ABI has the size and field offsets that a C compiler gives the
struct it stands for in include/cave_ca.h (a probe program compiled with gcc prints them). A
field missing from the header fails the probe's compile; a shifted field or a size mismatch
would corrupt every call that passes the struct."""
import os
import shutil
import subprocess

import pytest

import cave_b200 as cb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# C struct -> its ctypes Structure
CTYPES = {
    "cave_sim_params": cb.SimParams,
    "cave_grid_snapshot": cb.GridSnapshot,
    "cave_grid_info": cb.GridInfo,
    "cave_chunk_config": cb.ChunkConfig,
    "cave_tick_stats": cb.TickStats,
    "cave_timing": cb.Timing,
    "cave_sim_desc": cb.SimDesc,
    "cave_sim_result": cb.SimResult,
    "cave_batch_options": cb.BatchOptions,
    "cave_server_options": cb.ServerOptions,
    "cave_server_stats": cb.ServerStats,
    "cave_request_progress": cb.RequestProgress,
    "cave_search_config": cb.SearchConfig,
    "cave_search_summary": cb.SearchSummary,
}

_PARAMS = {"birth": "params.birthAndMaxCellStateRules", "survival": "params.survivalAndNeighborhoodRules",
           "shape": "params.shapeAndGridConfiguration"}
# C struct -> (numpy record dtype, dtype field -> C member designator)
DTYPES = {
    "cave_sim_desc": (cb.SIM_DESC_DTYPE, _PARAMS),
    "cave_sim_result": (cb.SIM_RESULT_DTYPE, _PARAMS),
    "cave_request_sim": (cb.REQUEST_SIM_DTYPE, _PARAMS),
}


def _probe(tmp_path):
    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("no C compiler")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "cave_ca.h"', "int main(void) {"]
    for s, cls in CTYPES.items():
        lines.append(f'  printf("{s} sizeof %zu\\n", sizeof({s}));')
        for name, _ in cls._fields_:
            lines.append(f'  printf("{s} {name} %zu\\n", offsetof({s}, {name}));')
    for s, (dt, alias) in DTYPES.items():
        lines.append(f'  printf("{s} sizeof %zu\\n", sizeof({s}));')
        for name in dt.names:
            lines.append(f'  printf("{s} dtype:{name} %zu\\n", offsetof({s}, {alias.get(name, name)}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    r = subprocess.run([gcc, "-std=c11", "-Wall", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    return {(a, b): int(c) for a, b, c in (l.split() for l in out.splitlines())}


def test_ctypes_structures_match_the_header(tmp_path):
    c = _probe(tmp_path)
    for s, cls in CTYPES.items():
        assert c[(s, "sizeof")] == __import__("ctypes").sizeof(cls), s
        for name, _ in cls._fields_:
            assert c[(s, name)] == getattr(cls, name).offset, f"{s}.{name}"


def test_record_dtypes_match_the_header(tmp_path):
    c = _probe(tmp_path)
    for s, (dt, _) in DTYPES.items():
        assert c[(s, "sizeof")] == dt.itemsize, s
        for name in dt.names:
            assert c[(s, f"dtype:{name}")] == dt.fields[name][1], f"{s} dtype field {name}"
