"""Builds cave_b200/libcave_ca.so in-tree (nvcc for .cu at sm_100a, g++ -std=c++20 for .cpp).

With --checked it builds the checked library instead, cave_b200/libcave_ca_checked.so: every source
(and the kernels it compiles at run time) with -DCAVE_CHECKED, so that the hot kernels test their
shared- and global-memory indices and report a failed test as an error flag. Load it in place of the
normal library with CAVE_LIB=<path>.

Usage: python -m cave_b200.build [--force] [--verbose] [--checked]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcave_ca.so")
OBJ_CHECKED = os.path.join(HERE, "_build_checked")
LIB_CHECKED = os.path.join(HERE, "libcave_ca_checked.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++20", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                     "-Xptxas", "-warn-spills"]
CXX = shutil.which("g++") or "g++"
CXX_FLAGS = ["-O2", "-std=c++20", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter",
             f"-I{CUDA_HOME}/include"]


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + \
        [os.path.join(HERE, "..", "include", "cave_ca.h")]


# Device headers NVRTC compiles the rule-specialised tick kernel from (csrc/jit.cpp), by the
# name each is included under.
JIT_SOURCES = [(n, os.path.join(CSRC, n)) for n in (
    "cave_stdint.h", "ca_types.h", "ca_core.cuh", "cave_internal.h", "ptx.cuh", "ring.cuh",
    "stream_common.cuh", "stream_tick.cuh", "stream_tick2.cuh")] + [("../../include/cave_ca.h", os.path.join(HERE, "..", "include", "cave_ca.h"))]
_DELIM = "cave_jit_src"


def _gen_jit_sources(obj_dir, force=False):
    """Writes <obj_dir>/jit_sources.cpp: the JIT headers as string literals (kJitSource*)."""
    out = os.path.join(obj_dir, "jit_sources.cpp")
    paths = [p for _, p in JIT_SOURCES] + [os.path.abspath(__file__)]
    if not force and not _stale(out, paths):
        return out
    lines = ["// Generated by cave_b200/build.py from the device headers; do not edit.",
             "namespace cave {",
             f"extern const int kJitSourceCount = {len(JIT_SOURCES)};",
             "extern const char* const kJitSourceNames[] = {" + ", ".join(f'"{n}"' for n, _ in JIT_SOURCES) + "};",
             "extern const char* const kJitSourceTexts[] = {"]
    for _, p in JIT_SOURCES:
        text = open(p).read()
        if f"){_DELIM}\"" in text:
            raise RuntimeError(f"{p} contains the raw-string delimiter")
        lines.append(f'R"{_DELIM}({text}){_DELIM}",')
    lines += ["};", "}  // namespace cave", ""]
    tmp = out + ".tmp"
    with open(tmp, "w") as f:
        f.write("\n".join(lines))
    os.replace(tmp, out)
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src, obj_dir, defines, verbose):
    obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + defines + ["-c", src, "-o", obj]
    else:
        cmd = [CXX] + CXX_FLAGS + defines + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> str:
    obj_dir, lib = (OBJ_CHECKED, LIB_CHECKED) if checked else (OBJ, LIB)
    defines = ["-DCAVE_CHECKED"] if checked else []
    os.makedirs(obj_dir, exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))
    srcs.append(_gen_jit_sources(obj_dir, force))
    hdrs = _headers()
    todo = [s for s in srcs if force or _stale(os.path.join(obj_dir, os.path.basename(s) + ".o"), [s] + hdrs)]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            for obj, err in ex.map(lambda s: _compile(s, obj_dir, defines, verbose), todo):
                if err.strip() and verbose:
                    print(err, file=sys.stderr)
    objs = [os.path.join(obj_dir, os.path.basename(s) + ".o") for s in srcs]
    if force or todo or _stale(lib, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart_static", "-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv, checked="--checked" in sys.argv))
