"""The engine's device-pool allocator (cave::FreeList, engine.cpp: first fit over 256-byte units,
coalescing on free) against a model, on the host: tests/cpp/freelist_check.cpp is compiled with
g++ against the library's headers, linked with libcave_ca.so and run (no GPU needed)."""
import os
import shutil
import subprocess

import pytest

import cave_b200 as cb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def test_freelist_matches_first_fit_model(tmp_path):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no C++ compiler")
    lib_dir = os.path.dirname(cb.LIB_PATH)
    exe = tmp_path / "freelist_check"
    r = subprocess.run([gxx, "-std=c++20", "-O1", f"-I{CUDA_HOME}/include", "-I", os.path.join(ROOT, "cave_b200", "csrc"),
                        "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "freelist_check.cpp"),
                        "-o", str(exe), "-L", lib_dir, "-l:" + os.path.basename(cb.LIB_PATH),
                        "-Wl,-rpath," + lib_dir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:] + r.stderr[-2000:]
