"""The library's spawn box (cave::make_seed_spec: spawn size clamped to the grid, scaled by the
spawn-size index and centred, searchSystem.cpp:226-232 and :270-273) against the oracle's seeding
on the host: tests/cpp/seed_spec_print.cpp prints the box the device seeding kernels fill for
3,000 random grids, spawn sizes and size indices, and each must equal the bounding box of the
cells the oracle seeds with a filled spawn. No GPU needed."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import cave_b200 as cb
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def test_spawn_box_equals_the_oracle_seeding(tmp_path):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no C++ compiler")
    lib_dir = os.path.dirname(cb.LIB_PATH)
    exe = tmp_path / "seed_spec_print"
    r = subprocess.run([gxx, "-std=c++20", "-O1", f"-I{CUDA_HOME}/include", "-I", os.path.join(ROOT, "cave_b200", "csrc"),
                        "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "seed_spec_print.cpp"),
                        "-o", str(exe), "-L", lib_dir, "-l:" + os.path.basename(cb.LIB_PATH),
                        "-Wl,-rpath," + lib_dir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    rng = np.random.default_rng(7)
    cases = [(int(rng.integers(1, 41)), int(rng.integers(1, 41)), int(rng.integers(1, 41)),
              int(rng.integers(1, 46)), int(rng.integers(1, 46)), int(rng.integers(1, 46)), int(rng.integers(0, 16)))
             for _ in range(3000)]
    cases += [(49, 49, 49, 11, 11, 11, 0), (25, 25, 25, 11, 11, 11, 0), (49, 49, 49, 16, 16, 16, 0),
              (512, 512, 512, 512, 512, 512, 0), (1, 1, 1, 1, 1, 1, 15)]
    inp = "".join(" ".join(map(str, c)) + "\n" for c in cases)
    r = subprocess.run([str(exe)], input=inp, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    boxes = [tuple(map(int, l.split())) for l in r.stdout.splitlines()]
    assert len(boxes) == len(cases)
    for (X, Y, Z, sx, sy, sz, idx), box in zip(cases, boxes):
        if X * Y * Z > 64 ** 3:  # too large to seed in the test: the full-grid spawn fills the grid
            assert box == (0, 0, 0, X, Y, Z)
            continue
        cells = O.unpack(O.seed(X, Y, Z, spawn=(sx, sy, sz), spawn_size_index=idx, random=False, max_cell_state=1),
                         X, Y, Z)
        nz = np.argwhere(cells != 0)  # (z, y, x)
        lo = tuple(int(v) for v in nz.min(axis=0)[::-1])
        hi = tuple(int(v) + 1 for v in nz.max(axis=0)[::-1])
        assert box == lo + hi, ((X, Y, Z, sx, sy, sz, idx), box, lo + hi)
        assert int((cells != 0).sum()) == int(np.prod(np.subtract(hi, lo)))  # the box is filled
