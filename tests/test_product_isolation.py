"""The product (cave_b200/ and include/) stands alone: no source of it names the oracle, the built
library needs no library besides the C/C++ runtime (CUDA's runtime is linked in statically; NVRTC
is opened only when a rule-specialised kernel is compiled), and the Python binding raises when the
library is missing instead of falling back to anything."""
import os
import re
import shutil
import subprocess
import sys

import pytest

import cave_b200 as cb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _product_sources():
    for base in ("cave_b200", "include"):
        for d, _, files in os.walk(os.path.join(ROOT, base)):
            if "_build" in d or "__pycache__" in d:
                continue
            for f in files:
                if f.endswith((".py", ".cpp", ".cu", ".cuh", ".h")):
                    yield os.path.join(d, f)


def test_no_product_source_names_the_oracle():
    hits = []
    for p in _product_sources():
        for i, line in enumerate(open(p, encoding="utf-8"), 1):
            if re.search(r"\boracle\b|cave_oracle", line):
                hits.append(f"{os.path.relpath(p, ROOT)}:{i}: {line.strip()}")
    assert not hits, "\n".join(hits)


def test_library_needs_only_the_c_runtime():
    readelf = shutil.which("readelf")
    if not readelf or not os.path.exists(cb.LIB_PATH):
        pytest.skip("readelf or the library missing")
    out = subprocess.run([readelf, "-d", cb.LIB_PATH], capture_output=True, text=True, check=True).stdout
    needed = set(re.findall(r"\(NEEDED\)\s+Shared library: \[([^\]]+)\]", out))
    allowed = {"libstdc++.so.6", "libgcc_s.so.1", "libc.so.6", "libm.so.6", "ld-linux-x86-64.so.2",
               "libpthread.so.0", "libdl.so.2", "librt.so.1"}
    assert needed and needed <= allowed, needed - allowed


def test_binding_raises_without_the_library(tmp_path):
    code = ("import cave_b200 as cb\n"
            "try:\n    cb.lib()\nexcept OSError as e:\n    print('raised', e)\n")
    env = dict(os.environ, CAVE_LIB=str(tmp_path / "missing" / "libcave_ca.so"))
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("raised") and "missing" in r.stdout, r.stdout + r.stderr
