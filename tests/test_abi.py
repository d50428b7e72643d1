"""The C ABI library: it loads without a GPU, exports every entry point declared in
include/*.h, and its host-only functions agree with the oracle."""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

import cave_b200 as cb
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"\b(cave_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_builds_and_loads():
    assert os.path.exists(cb.LIB_PATH), "run python -m cave_b200.build"
    cb.lib()


CHECKED_LIB = os.path.join(ROOT, "cave_b200", "libcave_ca_checked.so")


@pytest.mark.parametrize("path", [cb.LIB_PATH, CHECKED_LIB], ids=["library", "checked-library"])
def test_every_declared_symbol_is_exported(path):
    assert os.path.exists(path), "run python -m cave_b200.build (--checked for the checked library)"
    decl = declared_functions()
    assert len(decl) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = decl - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    L = ctypes.CDLL(path)
    for n in decl:
        getattr(L, n)


def test_python_binding_covers_header():
    assert declared_functions() <= set(cb._SIGS), sorted(declared_functions() - set(cb._SIGS))


@pytest.mark.parametrize("n,k", [(6, 1), (6, 2), (12, 2), (18, 2), (26, 2), (26, 3), (14, 4)])
def test_enumerate_matches_oracle(n, k):
    assert np.array_equal(cb.valid_bitmasks(n, k), O.valid_bitmasks(n, k))


def test_manager_update_matches_oracle():
    rng = np.random.default_rng(1)
    for _ in range(300):
        snap = rng.integers(0, 5, size=4).astype(np.uint32)
        info_vals = rng.integers(0, 4, size=6).tolist()
        b = int(rng.integers(0, 6)) | (int(rng.integers(0, 16)) << 60)
        s = int(rng.integers(0, 6)) | (int(rng.integers(0, 16)) << 60)
        maxp, send, T = int(rng.integers(1, 6)), int(rng.integers(1, 6)), int(rng.integers(1, 5))
        oi, op = O.GridInfo(*info_vals), O.Perms(b, s)
        oic, opc = O.manager(snap, oi, op, maxp, send, T)
        ci = cb.GridInfo(*info_vals)
        cp = cb.SimParams(b, s, 0)
        cs = cb.GridSnapshot(*[int(v) for v in snap])
        cic, cpc = cb.manager_update(cs, ci, cp, maxp, send, T)
        assert cic.as_tuple() == oic.as_tuple() and ci.as_tuple() == oi.as_tuple()
        assert (cp.birthAndMaxCellStateRules, cp.survivalAndNeighborhoodRules) == (
            op.birthAndMaxCellStateRules, op.survivalAndNeighborhoodRules)
        assert (cpc.birthAndMaxCellStateRules, cpc.survivalAndNeighborhoodRules) == (
            opc.birthAndMaxCellStateRules, opc.survivalAndNeighborhoodRules)


def test_grid_words():
    assert cb.grid_words(49, 49, 49) == 7 * 49 * 49 == O.grid_words(49, 49, 49)
    assert cb.grid_words(512, 512, 512) == 64 * 512 * 512


def test_status_strings():
    for code in range(8):
        assert cb.lib().cave_status_string(code)
