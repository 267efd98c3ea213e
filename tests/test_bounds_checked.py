"""The bounds-checked build (libfz_checked.so, compiled with -DFZ_BOUNDS_CHECK; loaded when
FZ_BOUNDS_CHECK=1): every computed global index of the stepping kernels (stage, band, receivers)
and of the adjoint kernels is checked against its array, and an out-of-range one would set an
error bit (FZ_EBOUNDS at the next sync) instead of being accessed. compute-sanitizer is not
available for this purpose, so this build stands in for its memcheck. The same solves -- cPML on
every face, an obstacle band, PCS source, receivers; a batch of three; ragged tiles; FP32 and
FP64 -- and a gradient with every output (materials, sources, cPML, initial fields) run in a child
process on the checked build must finish without an error and reproduce the normal build's traces
bit for bit (the gradient to 1e-5: its atomics sum in a varying order)."""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CHECKED = os.path.join(ROOT, "fases_b200", "libfz_checked.so")

SCRIPT = r'''
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from tests.helpers import small_room, run_gpu
from tests import test_batch as tb
out = {}
for name, kw, prec in [("box_all_pml", dict(seed=6, room=(30, 30, 30), pml=(1, 1, 1, 1, 1, 1), pml_cells=5, steps=25), "fp32"),
                       ("box_fp64", dict(seed=7, steps=25), "fp64"),
                       ("ragged", dict(seed=8, room=(37, 21, 19), pml=(0, 1, 0, 1, 0, 1), pml_cells=4, steps=22), "fp32")]:
    cfg = small_room(**kw)
    s = run_gpu(cfg, prec)
    s.sync()
    out[name] = s.ir().tolist()
    s.close()
cfg = small_room(seed=11, pml=(1, 0, 1, 0, 0, 1), steps=21, pulse=False)
b = tb._solver(cfg, "fp32", batch=3, members=np.arange(3))
b.run(21)
out["batch"] = b.ir().tolist()
b.close()
from tests import test_adjoint_params as ap
cfg = ap._cfg()
tgt = ap._target(cfg)
s = ap._solver(cfg, precision="fp32")
g = s.misfit_gradient(tgt, segment_steps=16, sources=True, pml=True, initial=True)
s.close()
out["grad"] = [g["raw"].ravel().tolist(), g["sval"].tolist(), [g["pml"][k] for k in ("R0", "kappa_max", "alpha_max")],
               g["initial"][0].ravel().tolist()]
print(json.dumps(out))
'''


def test_checked_library_exports_the_same_symbols():
    if not os.path.exists(CHECKED):
        pytest.skip("libfz_checked.so not built")
    from fases_b200 import _abi
    L = ctypes.CDLL(CHECKED)
    missing = [n for n in _abi.SIGNATURES if not hasattr(L, n)]
    assert not missing, missing


def _run(checked):
    env = dict(os.environ)
    env["FZ_BOUNDS_CHECK"] = "1" if checked else "0"
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT], env=env, capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.gpu
def test_checked_build_runs_clean_and_matches():
    if not os.path.exists(CHECKED):
        pytest.skip("libfz_checked.so not built")
    a = _run(True)
    b = _run(False)
    assert a.keys() == b.keys()
    for k in a:
        if k == "grad":  # the adjoint's atomics sum in an order that varies from run to run
            for x, y in zip(a[k], b[k]):
                x, y = np.asarray(x), np.asarray(y)
                assert np.linalg.norm(x - y) <= 1e-5 * np.linalg.norm(y), k
        else:
            assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
