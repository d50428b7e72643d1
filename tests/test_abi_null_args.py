"""The C ABI under null handles and pointers, on the host: every entry point is called with every
pointer NULL and every number 0, in a child process (a crash would show as its exit status and
the last entry point it printed). Every status-returning call must answer CAVE_ERR_INVALID_ARG
before touching a device; destroy calls, size queries and the diagnostics accept NULL; no call
crashes."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r'''
import ctypes
import cave_b200 as cb
L = cb.lib()
for name, (res, args) in cb._SIGS.items():
    vals = [0.0 if a is ctypes.c_double else 0 if a in (cb.i32, cb.u32, cb.u64, ctypes.c_size_t) else None
            for a in args]
    print(name, end=" ", flush=True)
    r = getattr(L, name)(*vals)
    print(repr(r), flush=True)
print("done", flush=True)
'''


def test_every_entry_point_rejects_null_arguments():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=300)
    out = r.stdout.strip().splitlines()
    assert r.returncode == 0 and out and out[-1] == "done", r.stdout[-2000:] + r.stderr[-2000:]
    import cave_b200 as cb

    got = dict(l.split(" ", 1) for l in out[:-1])
    assert set(got) == set(cb._SIGS)
    for name, (res, _) in cb._SIGS.items():
        if res is cb.i32:
            assert got[name] == str(cb.ERR_INVALID_ARG), (name, got[name])
    assert got["cave_last_error"] == repr(b"no context")
    assert got["cave_status_string"] == repr(b"ok")
    for name in ("cave_batch_size", "cave_batch_plan", "cave_grid_words", "cave_enumerate_valid_bitmasks"):
        assert got[name] == "0", (name, got[name])
