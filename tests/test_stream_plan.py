"""The tiling of the streaming tick kernels (cave::plan_stream) over 20,000 random grid shapes,
CTA targets, row hints, rows per thread and halo widths, plus the benchmarked shapes, on the host:
tests/cpp/plan_check.cpp is compiled with nvcc (host code; the kernels' shared-memory size
functions come from their headers), linked with libcave_ca.so and run. No GPU needed. Checked:
strips per row, whole warps within the kernel's thread limit, tiles within the CTA's rows,
every (y, z) of the grid covered by exactly one work item, and the tile's shared memory within
one CTA's 227 KB. The same program checks the resident kernel's geometry (z-segments, threads,
shared memory, CTAs per SM) for every grid that fits shared memory in a 23,000-shape sweep."""
import os
import shutil
import subprocess

import pytest

import cave_b200 as cb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def test_stream_plans_and_resident_geometry_within_the_kernel_limits(tmp_path):
    nvcc = os.path.join(CUDA_HOME, "bin", "nvcc")
    if not os.path.exists(nvcc):
        nvcc = shutil.which("nvcc")
    if not nvcc:
        pytest.skip("no nvcc")
    lib_dir = os.path.dirname(cb.LIB_PATH)
    exe = tmp_path / "plan_check"
    r = subprocess.run([nvcc, "-std=c++20", "-O1", "-x", "cu", "-gencode", "arch=compute_100a,code=sm_100a",
                        "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "cave_b200", "csrc"),
                        "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "plan_check.cpp"),
                        "-o", str(exe), "-L", lib_dir, "-l:" + os.path.basename(cb.LIB_PATH),
                        "-Xlinker", "-rpath", "-Xlinker", lib_dir], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    env = {k: v for k, v in os.environ.items() if k != "CAVE_RESIDENT_NSEG"}  # the default geometry rule
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0 and r.stdout.strip().startswith("ok"), r.stdout[-2000:] + r.stderr[-2000:]
