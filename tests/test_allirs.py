"""The reference's own post-processing runs unchanged on this library's outputs.

common/allIRs.py:172-264 (`broadband_ir`) builds the broadband impulse response of a
source-receiver pair from the solver's output/IR<r>_<s>.bin, output/header.txt (dt) and
config/p_ref.bin (the radiated pulse it deconvolves), reading config/config.txt for the crossover.
For each golden project, this test runs it on the outputs this library wrote
(tests/golden/<case>/fz_output/, made on a GPU by tests/golden/make_fz_outputs.py through
fz_load_project and fz_write_outputs) and on the reference solver's own outputs of the same
project, and requires the same broadband IR from both, to the tolerance of the receiver traces
themselves (the FP32 traces agree to 2e-5 rel-L2; resampling, deconvolution and filtering are
linear, with a regularised inverse whose gain is bounded).

The reference module is imported from the reference checkout ($FZ_REFERENCE_ROOT, else a
directory named "reference" beside this repository's directory) with a stand-in for matplotlib,
which it imports at the top for its plotting functions only; that test is skipped where the
checkout is absent.
"""
import importlib.util
import os
import shutil
import sys
import types

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CASES = ["box_pcs", "box_ricker", "box_sine", "box_poles"]
TOL = 2e-5  # measured: at most 3.4e-6


def _reference_root():
    env = os.environ.get("FZ_REFERENCE_ROOT")
    return env if env else os.path.join(os.path.dirname(os.path.realpath(ROOT)), "reference")


def _stub_matplotlib():
    """A minimal matplotlib: allIRs calls matplotlib.use, plt.rcParams.update and plt.cycler at
    import time; broadband_ir never plots."""
    if "matplotlib" in sys.modules and not getattr(sys.modules["matplotlib"], "_fz_stub", False):
        return
    mpl = types.ModuleType("matplotlib")
    mpl._fz_stub = True
    mpl.use = lambda *a, **k: None
    plt = types.ModuleType("matplotlib.pyplot")
    plt.rcParams = {}
    plt.cycler = lambda *a, **k: None
    mpl.pyplot = plt
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt


def _load_allirs():
    path = os.path.join(_reference_root(), "common", "allIRs.py")
    if not os.path.exists(path):
        pytest.skip("reference checkout not present (common/allIRs.py)")
    _stub_matplotlib()
    spec = importlib.util.spec_from_file_location("fz_ref_allIRs", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)  # a fresh module per project: it caches the project's config
    return mod


def _project(tmp, name, case, outputs_from):
    """A project directory laid out as allIRs expects (cwd = <proj>/output): the golden
    project's config.txt, and the IR files, header.txt and p_ref.bin of `outputs_from`."""
    proj = os.path.join(tmp, name)
    os.makedirs(os.path.join(proj, "config"))
    os.makedirs(os.path.join(proj, "output"))
    shutil.copyfile(os.path.join(HERE, "golden", case, "config", "config.txt"),
                    os.path.join(proj, "config", "config.txt"))
    src_out = os.path.join(outputs_from, "output")
    for f in os.listdir(src_out):
        if (f.startswith("IR") and f.endswith(".bin")) or f == "header.txt":
            shutil.copyfile(os.path.join(src_out, f), os.path.join(proj, "output", f))
    pr = os.path.join(outputs_from, "config", "p_ref.bin")
    if os.path.exists(pr):
        shutil.copyfile(pr, os.path.join(proj, "config", "p_ref.bin"))
    return proj


def _broadband(proj, n_rec):
    mod = _load_allirs()
    cwd = os.getcwd()
    os.chdir(os.path.join(proj, "output"))
    try:
        return [mod.broadband_ir(r, 0) for r in range(n_rec)]
    finally:
        os.chdir(cwd)


def _n_rec(case):
    return len([f for f in os.listdir(os.path.join(HERE, "golden", case, "output")) if f.startswith("IR")])


@pytest.mark.parametrize("case", CASES)
def test_fz_outputs_are_the_reference_formats(case):
    """The committed outputs are what fz_write_outputs writes for the golden project: one IR and
    one VEL file per receiver with the reference's sample count, a 13-field header whose grid, step
    count, dt, h and tol/h are the reference's, and (not for sinusoidal sources) p_ref.bin equal
    to the reference's to 1e-12."""
    fz = os.path.join(HERE, "golden", case, "fz_output")
    ref = os.path.join(HERE, "golden", case)
    n_rec = _n_rec(case)
    assert n_rec > 0
    for r in range(n_rec):
        a = np.fromfile(os.path.join(fz, "output", f"IR{r}_0.bin"), np.float32)
        b = np.fromfile(os.path.join(ref, "output", f"IR{r}_0.bin"), np.float32)
        assert a.shape == b.shape
        assert np.linalg.norm(a - b) <= 2e-5 * np.linalg.norm(b)
        va = np.fromfile(os.path.join(fz, "output", f"VEL{r}_0.bin"), np.float32)
        assert va.size == 3 * a.size
    hdr = open(os.path.join(fz, "output", "header.txt")).read().split()
    ref_hdr = open(os.path.join(ref, "output", "header.txt")).read().split()
    assert len(hdr) == len(ref_hdr) == 13
    assert hdr[:4] == ref_hdr[:4] and hdr[9] == ref_hdr[9] and hdr[11:] == ref_hdr[11:]
    ref_pr = os.path.join(ref, "config", "p_ref.bin")
    fz_pr = os.path.join(fz, "config", "p_ref.bin")
    assert os.path.exists(ref_pr) == os.path.exists(fz_pr)
    if os.path.exists(ref_pr):
        a, b = np.fromfile(fz_pr, np.float64), np.fromfile(ref_pr, np.float64)
        assert a.shape == b.shape and np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))


@pytest.mark.parametrize("case", CASES)
def test_reference_broadband_ir_on_fz_outputs(case, tmp_path):
    ref = os.path.join(HERE, "golden", case)
    n_rec = _n_rec(case)
    mine = _broadband(_project(str(tmp_path), "fz", case, os.path.join(ref, "fz_output")), n_rec)
    theirs = _broadband(_project(str(tmp_path), "ref", case, ref), n_rec)
    for r in range(n_rec):
        assert mine[r] is not None and theirs[r] is not None
        bb, low, high = mine[r]
        bb_ref, low_ref, high_ref = theirs[r]
        assert bb.shape == bb_ref.shape and bb.size > 0
        assert np.all(np.isfinite(bb))
        assert not high.any() and not high_ref.any()  # FVM only: no geometric-acoustics bands
        err = np.linalg.norm(bb - bb_ref) / np.linalg.norm(bb_ref)
        assert err <= TOL, (case, r, err)
