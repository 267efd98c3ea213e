"""Same project, same B200: the reference solver `fases3D` (built from its own sources for sm_100a
by oracle/build_ref.sh) against this stepper driven through fz_load_project on the reference's own
scene cache. Checks that the receiver traces agree and that this stepper is faster, and writes both
timings to $FZ_RESULTS_DIR/reference_speed.json when that variable names a folder.

Room (default 5 x 4 x 2 m at h = 0.02 m = 250 x 200 x 100 cells, 5 obstacles, one cPML face,
PCS source, 8 receivers) can be scaled with FZ_REFSPEED_ROOM="Lx Ly Lz" (metres)."""
import json
import os
import re
import time

import numpy as np
import pytest

from tests.golden import fixture
from tests.golden import make_golden as mg

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _spec():
    L = [float(x) for x in os.environ.get("FZ_REFSPEED_ROOM", "5.0 4.0 2.0").split()]
    h = 0.02
    cc = 343.2
    dt = 0.5 * h / cc
    steps = int(os.environ.get("FZ_REFSPEED_STEPS", "1500"))
    rng = np.random.default_rng(7)
    obstacles = []
    for _ in range(5):
        lo = [float(rng.uniform(0.2 * x, 0.7 * x)) for x in L]
        hi = [lo[a] + float(rng.uniform(0.05, 0.12)) * L[a] for a in range(3)]
        obstacles.append((tuple(lo), tuple(hi)))
    src = [(0.3 * L[0], 0.4 * L[1], 0.5 * L[2], 90.0)]
    rec = [tuple(float(rng.uniform(0.15, 0.85)) * x for x in L) for _ in range(8)]
    return dict(room=tuple(L), h=h, t_max=(steps - 0.5) * dt, f_in=250.0, temp=20.0, cfl=0.5,
                pml=(0, 0, 1, 0, 0, 0), obstacles=obstacles, src_opt=0, glob_f=100.0, src=src, rec=rec, seed=3,
                open_wall=1, frames=60)


def test_this_stepper_beats_the_reference_on_the_same_project(tmp_path):
    if not os.path.exists(mg.REF_EXE):
        pytest.skip("reference solver not built (oracle/build_ref.sh)")
    from fases_b200 import Solver
    proj = str(tmp_path / "proj")
    mg.make_project("speed", proj, spec=_spec())
    t0 = time.perf_counter()
    rc, stamped = mg.run_reference_timed(proj, timeout=1800)
    t_ref_wall = time.perf_counter() - t0
    out = "".join(line for _, line in stamped)
    assert rc == 0, out[-2000:]
    t_start = next(t for t, line in stamped if "Will now start" in line)
    t_stop = next(t for t, line in stamped if "Simulation time" in line)
    t_ref_loop = t_stop - t_start  # wall clock of its time loop (its own figure is CPU time)
    nt_ref = int(re.search(r"Will now start (\d+) iterations", out).group(1))
    ref = fixture.load(proj)
    s, nt = Solver.from_project(os.path.join(proj, "scene.obj"), os.path.join(proj, "config", "config.txt"),
                                os.path.join(proj, "src.txt"), os.path.join(proj, "rec.txt"))
    assert nt == nt_ref
    t1 = time.perf_counter()
    s.run(nt)
    ir = s.ir()
    t_fz_wall = time.perf_counter() - t1
    info = s.info()
    s.close()
    s2, _ = Solver.from_project(os.path.join(proj, "scene.obj"), os.path.join(proj, "config", "config.txt"),
                                os.path.join(proj, "src.txt"), os.path.join(proj, "rec.txt"))
    s2.run(20)
    t_fz_dev = s2.run_timed(nt - 20) * 1e-3 * nt / (nt - 20)
    s2.close()
    # relative L2 per receiver; a receiver the wave has not reached yet reads exactly zero in both
    scale = max(float(np.linalg.norm(ref["ir"][r])) for r in range(ir.shape[0]))
    errs = []
    for r in range(ir.shape[0]):
        nr = float(np.linalg.norm(ref["ir"][r]))
        d = float(np.linalg.norm(ir[r] - ref["ir"][r]))
        errs.append(d / nr if nr > 0 else (0.0 if d <= 1e-12 * scale else float("inf")))
    nx, ny, nz = info["dims"]
    room_cells = (nx - 6) * (ny - 6) * (nz - 6)
    result = {
        "room_cells": room_cells, "steps": nt,
        "reference_loop_s": t_ref_loop, "reference_process_s": t_ref_wall,
        "reference_gcell_s": room_cells * nt / t_ref_loop / 1e9,
        "fz_run_s": t_fz_wall, "fz_gcell_s": room_cells * nt / t_fz_wall / 1e9,
        "fz_device_s": t_fz_dev, "fz_device_gcell_s": room_cells * nt / t_fz_dev / 1e9,
        "speedup_loop": t_ref_loop / t_fz_wall, "speedup_device": t_ref_loop / t_fz_dev, "ir_rel_l2_vs_reference": errs,
    }
    print(json.dumps(result))
    outdir = os.environ.get("FZ_RESULTS_DIR", "")
    if outdir and os.path.isdir(outdir):
        with open(os.path.join(outdir, "reference_speed.json"), "w") as f:
            json.dump(result, f, indent=1)
    assert max(errs) < 5e-5, errs
    assert t_fz_wall < t_ref_loop
