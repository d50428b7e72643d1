"""The rule-specialised tick kernel compiles with NVRTC for every neighbourhood, state count and
table shape, without a device, and lands in the on-disk cache (CPU only)."""
import os
import subprocess
import sys
import time

import pytest

import cave_b200 as cb
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def params(maxcs, flags, birth, survival):
    return cb.SimParams(*[int(v) for v in O.make_params(maxcs, flags, birth, survival)])


# (maxCellState, neighbourhood flags, birth mask, survival mask): every neighbourhood, the
# extremes of the state count (1 and 15; 16 never has an alive cell), empty and dense tables.
CASES = [
    (15, 0x7, 0x10, 0x18),
    (1, 0x0, 0x1, 0x1),
    (2, 0x1, 0x3F, 0x0),
    (3, 0x2, 0x0, 0xFFF),
    (4, 0x3, 0x60, 0x70),
    (7, 0x4, 0x81, 0x42),
    (9, 0x5, 0x5555, 0x2AAA),
    (16, 0x6, 0x1, 0x3),
    (12, 0xB, 0x3FFFFFF, 0x1555555),
]


@pytest.fixture(scope="module")
def cache_dir(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("jit_cache"))
    old = os.environ.get("CAVE_JIT_CACHE")
    os.environ["CAVE_JIT_CACHE"] = d
    yield d
    if old is None:
        os.environ.pop("CAVE_JIT_CACHE", None)
    else:
        os.environ["CAVE_JIT_CACHE"] = old


@pytest.mark.parametrize("case", CASES)
def test_compiles_without_device(cache_dir, case):
    ok, log = cb.jit_compile(params(*case))
    assert ok, log


def test_cubins_cached_on_disk(cache_dir):
    p = params(13, 0x7, 0x1F0, 0x0F0)
    before = set(os.listdir(cache_dir))
    ok, log = cb.jit_compile(p)
    assert ok, log
    new = set(os.listdir(cache_dir)) - before
    assert len(new) == 1 and next(iter(new)).endswith(".cubin")
    # a fresh process finds the cubin instead of compiling again
    code = ("import time, cave_b200 as cb, oracle as O\n"
            "p = cb.SimParams(*[int(v) for v in O.make_params(13, 0x7, 0x1F0, 0x0F0)])\n"
            "t = time.time(); ok, log = cb.jit_compile(p); print(ok, time.time() - t)\n")
    env = dict(os.environ, CAVE_JIT_CACHE=cache_dir)
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    ok_s, secs = out.stdout.split()
    assert ok_s == "True" and float(secs) < 0.3, out.stdout + out.stderr
    assert set(os.listdir(cache_dir)) - before == new


def test_disk_cache_off(cache_dir):
    before = set(os.listdir(cache_dir))
    os.environ["CAVE_JIT_CACHE"] = "off"
    try:
        ok, log = cb.jit_compile(params(11, 0x3, 0x4, 0x8))
        assert ok, log
    finally:
        os.environ["CAVE_JIT_CACHE"] = cache_dir
    assert set(os.listdir(cache_dir)) == before


def test_bad_rule_index_rejected():
    p = cb.SimParams((3 << 60) | 10 ** 6, (0x3 << 60) | 1, 0)  # K-index 10^6 of a 3-entry table
    ok, _ = cb.jit_compile(p, [1, 2, 3], max_rule_bits=2)
    assert not ok


def test_in_process_cache_is_immediate(cache_dir):
    p = params(*CASES[0])
    ok, _ = cb.jit_compile(p)
    t = time.time()
    ok2, _ = cb.jit_compile(p)
    assert ok and ok2 and time.time() - t < 0.05


@pytest.mark.parametrize("wait_s", [0.0, 0.3])
def test_exit_while_compiling(tmp_path, wait_s):
    """A process may exit while a background compile runs: the library joins the compile thread
    before NVRTC's own exit-time teardown, so the process still exits cleanly."""
    code = ("import time, cave_b200 as cb, oracle as O\n"
            "p = cb.SimParams(*[int(v) for v in O.make_params(14, 0x7, 0x3C, 0x1E0)])\n"
            f"cb.jit_compile_async(p); time.sleep({wait_s})\n")
    env = dict(os.environ, CAVE_JIT_CACHE=str(tmp_path))
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    # the compile ran to completion before the exit: its cubin is in the cache
    assert any(f.endswith(".cubin") for f in os.listdir(tmp_path))


def test_checked_library_compiles_its_kernels_under_their_own_key(tmp_path):
    """The checked library compiles its rule-specialised kernels with -DCAVE_CHECKED (the bounds
    checks of the streaming kernels) and caches them under a key of their own: the normal library
    sharing the cache folder compiles its own cubin instead of loading the checked one."""
    checked = os.path.join(ROOT, "cave_b200", "libcave_ca_checked.so")
    if not os.path.exists(checked):
        pytest.skip("build it with python -m cave_b200.build --checked")
    cache = tmp_path / "jit"
    code = ("import sys, cave_b200 as cb, oracle as O; "
            "p = cb.SimParams(*[int(v) for v in O.make_params(15, 0x7, 0x10, 0x18)]); "
            "ok, log = cb.jit_compile(p); print(log[-2000:]); sys.exit(0 if ok else 1)")
    for lib in (checked, cb.LIB_PATH):
        env = dict(os.environ, CAVE_LIB=lib, CAVE_JIT_CACHE=str(cache))
        r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
    assert len([f for f in os.listdir(cache) if f.endswith(".cubin")]) == 2
