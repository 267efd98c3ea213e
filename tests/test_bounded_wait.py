"""Bounded waits end in an error status, never in a hang.

Device side: the stage kernels wait for every plane tile on an mbarrier with an iteration limit.
The wait-test build (libfz_waittest.so, compiled with -DFZ_WAIT_TEST, loaded when FZ_WAIT_TEST=1)
shortens that limit to about a millisecond and has a test hook, fz_test_skip_plane, that makes
the stage kernels never issue the tile of one plane: nothing ever completes that plane's
mbarrier (a flag that nothing sets), so the wait for it runs out. The block then leaves through
its one exit after waiting for the copies it still has in flight (the next plane's tile, issued
normally), so no copy is left behind. The test checks, in a child process on that build, that the
step returns, that fz_sync reports FZ_ETIMEOUT with the kernel's message, and that the context
and the handle stay usable: a new initial state clears the error and the same solve then runs
clean and gives the traces of a solver that never skipped a tile, bit for bit.

Host side: fz_sync with a 1 ms limit on a long queued run returns FZ_ETIMEOUT while the work is
still running; a later fz_sync with a long limit returns FZ_OK.
"""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
WAIT_TEST = os.path.join(ROOT, "fases_b200", "libfz_waittest.so")

SCRIPT = r'''
import ctypes, json, sys, time
import numpy as np
sys.path.insert(0, sys.argv[1])
from fases_b200 import _abi
from tests.helpers import small_room, run_gpu
L = _abi.lib()
assert _abi.LIB_PATH.endswith("libfz_waittest.so"), _abi.LIB_PATH
L.fz_test_skip_plane.argtypes = [ctypes.c_void_p, ctypes.c_int32]
L.fz_test_skip_plane.restype = ctypes.c_int
out = {}
cfg = small_room(seed=3, room=(40, 36, 30), steps=12, source="none")  # a pulse, no source: results do
s = run_gpu(cfg, "fp32", steps=cfg["steps"] + 1, run=False)           # not depend on the step counter
assert L.fz_test_skip_plane(s._h, 2) == 0
t0 = time.perf_counter()
out["run_rc"] = L.fz_run(s._h, 1)
out["sync_rc"] = L.fz_sync(s._h, 60000)
out["sync_s"] = time.perf_counter() - t0
out["message"] = _abi.last_error(s._h)
# the handle stays usable: no skipped tile, a new initial state, the same solve again
assert L.fz_test_skip_plane(s._h, -1) == 0
s.set_fields(p=cfg["p0"])
s.run(cfg["steps"])
out["after_rc"] = L.fz_sync(s._h, 60000)
ir_after = s.ir()[:, 1:]  # sample 0 is the failed step's
s.close()
t = run_gpu(cfg, "fp32")
out["same_as_clean"] = bool(np.array_equal(ir_after, t.ir()))
out["finite"] = bool(np.isfinite(ir_after).all())
t.close()
print(json.dumps(out))
'''


def test_wait_test_library_exports_the_hook_and_the_abi():
    if not os.path.exists(WAIT_TEST):
        pytest.skip("libfz_waittest.so not built")
    from fases_b200 import _abi
    L = ctypes.CDLL(WAIT_TEST)
    assert hasattr(L, "fz_test_skip_plane")
    missing = [n for n in _abi.SIGNATURES if not hasattr(L, n)]
    assert not missing, missing
    # the product library has no test hook
    assert not hasattr(ctypes.CDLL(_abi.LIB_PATH), "fz_test_skip_plane")


@pytest.mark.gpu
def test_device_wait_that_runs_out_reports_timeout_and_recovers():
    if not os.path.exists(WAIT_TEST):
        pytest.skip("libfz_waittest.so not built")
    env = dict(os.environ, FZ_WAIT_TEST="1")
    env.pop("FZ_BOUNDS_CHECK", None)
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT], env=env, capture_output=True, text=True, timeout=300,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    from fases_b200 import _abi
    assert out["run_rc"] == _abi.FZ_OK
    assert out["sync_rc"] == _abi.FZ_ETIMEOUT, out
    assert "bounded wait" in out["message"], out["message"]
    assert out["sync_s"] < 30.0
    assert out["after_rc"] == _abi.FZ_OK
    assert out["finite"] and out["same_as_clean"], out


@pytest.mark.gpu
def test_host_wait_with_a_short_limit_times_out_then_completes():
    from fases_b200 import _abi
    from tests.helpers import run_gpu, small_room
    cfg = small_room(seed=4, room=(96, 96, 96), steps=400)
    s = run_gpu(cfg, "fp32", run=False)
    s.run(2)  # set-up and graphs done before the queued run
    L = _abi.lib()
    assert L.fz_run(s._h, 400) == _abi.FZ_OK
    rc = L.fz_sync(s._h, 1)
    assert rc == _abi.FZ_ETIMEOUT, rc
    assert "did not finish in time" in _abi.last_error(s._h)
    assert L.fz_sync(s._h, 600000) == _abi.FZ_OK
    assert s.steps_done() == 402
    assert np.isfinite(s.ir()).all()
    s.close()
