"""The checked library (cave_b200/libcave_ca_checked.so, every source and every kernel compiled at
run time built with -DCAVE_CHECKED): the hot kernels -- streaming (generic and rule-specialised,
one and two ticks per launch) and resident -- test each shared- and global-memory index against
the extent it must stay in, and a failed test skips the access and raises an error flag that the
call returns as CAVE_ERR_INTERNAL. The engine's tiled tick kernels (one and two rows per thread)
run under the same checks through the engine suite. The parity suites of those kernels run in a child process on
the checked library: every result must equal the oracle's, so no check fired."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "cave_b200", "libcave_ca_checked.so")
SUITES = ["tests/test_gpu_parity.py", "tests/test_gpu_batch.py", "tests/test_gpu_jit.py", "tests/test_gpu_engine.py"]


def test_parity_suites_pass_on_the_checked_library(tmp_path):
    assert os.path.exists(CHECKED), "build it with python -m cave_b200.build --checked"
    env = dict(os.environ, CAVE_LIB=CHECKED, CAVE_JIT_CACHE=str(tmp_path / "jit"))
    probe = ("import cave_b200 as cb; cb.lib(); "
             "print(any('libcave_ca_checked.so' in l for l in open('/proc/self/maps')))")
    r = subprocess.run([sys.executable, "-c", probe], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.stdout.strip().splitlines()[-1:] == ["True"], r.stdout + r.stderr
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-p", "no:cacheprovider", "-m", "gpu"] + SUITES,
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=2400)
    assert r.returncode == 0, r.stdout[-4000:] + r.stderr[-2000:]
