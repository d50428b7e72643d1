"""The rule compiler (cave::make_device_rule, rules.cpp) on the host: tests/cpp/rule_check.cpp is
compiled with g++, linked with libcave_ca.so and run over about 119,000 rules -- every
neighbourhood flag set (the wrap bit included), every state count 1..16, edge masks (empty, full,
single and highest counts) and random sparse and dense masks. For every neighbour count a cell
can see, the tables or sparse terms the kernels evaluate must give the reference's survive / birth
decision (searchSimulationCube.slang:163-216), with the kernels' count convention (a face
neighbourhood's row sums include an alive cell itself). No GPU needed."""
import os
import shutil
import subprocess

import pytest

import cave_b200 as cb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def test_device_rules_give_the_reference_decisions(tmp_path):
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no C++ compiler")
    lib_dir = os.path.dirname(cb.LIB_PATH)
    exe = tmp_path / "rule_check"
    r = subprocess.run([gxx, "-std=c++20", "-O1", f"-I{CUDA_HOME}/include", "-I", os.path.join(ROOT, "cave_b200", "csrc"),
                        "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "rule_check.cpp"),
                        "-o", str(exe), "-L", lib_dir, "-l:" + os.path.basename(cb.LIB_PATH),
                        "-Wl,-rpath," + lib_dir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().startswith("ok"), r.stdout[-2000:] + r.stderr[-2000:]
