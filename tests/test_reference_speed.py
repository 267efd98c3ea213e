"""Same project, same B200: the reference solver `fases3D` (built from its own sources for sm_100a
by oracle/build_ref.sh) against this stepper driven through fz_load_project on the reference's own
scene cache; and the reference's 2D solver `phases2D` against the 2D legacy scheme. Checks that the receiver traces agree and that this stepper is faster, and writes both
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


def test_legacy2d_beats_the_reference_2d_solver_on_the_same_project(tmp_path):
    """The reference's 2D solver `phases2D` and the 2D legacy scheme here on one project the size
    of the reference's shipped 2D scene (4.0 x 4.06 m at h = 5 mm: 801 x 813 nodes), with solid
    rows along the bottom and top so that the reference's run is deterministic (see
    include/fz_legacy2d.h). The reference's time loop includes what it always does per step (a
    device-to-host copy of the pressure field for its receiver and its animation frames)."""
    from tests.golden import make_golden_legacy2d as mg2
    from tests.golden.fixture import load_legacy2d
    from fases_b200.legacy2d import Legacy2D
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "phases2D")):
        pytest.skip("reference 2D solver not built (oracle/build_ref.sh)")
    Lx, Ly = 4.0, 4.06
    steps = int(os.environ.get("FZ_REFSPEED2D_STEPS", "1500"))
    dt = 0.2 * 0.005 / 344.4
    spec = dict(L=(Lx, Ly), h=0.005, t_max=(steps - 0.5) * dt, temp=22.0, cfl=0.2, pml=(0, 0, 1, 0),
                polys=[("floor", [(0.0, 0.0), (Lx, 0.0), (Lx, 0.03), (0.0, 0.03)]),
                       ("barrier", [(1.6, 0.8), (1.7, 0.8), (2.2, 3.0), (2.1, 3.0)]),
                       ("ceiling", [(0.0, Ly - 0.03), (Lx, Ly - 0.03), (Lx, Ly), (0.0, Ly)])],
                fits={"floor": (0.95, [(40.0, 2500.0)], []),
                      "barrier": (0.8, [(171.9, 317.2), (-343.5, 3796.2)], [(-21.96, -42.35, 39.14, 348.0)]),
                      "ceiling": (0.9, [], [(5.0, 8.0, 900.0, 2600.0)])},
                poles=(2, 1), src=(1.0, 2.0, 9.0), rec=(1.4, 2.2))
    proj = str(tmp_path / "proj2d")
    mg2.write_project("speed2d", proj, spec=spec)
    rc, stamped = mg2.run_reference_timed(proj)
    out = "".join(line for _, line in stamped)
    assert rc == 0, out[-2000:]
    t_start = next(t for t, line in stamped if "Simulation start" in line)
    t_stop = next(t for t, line in stamped if "Simulation time" in line)
    t_ref_loop = t_stop - t_start
    fx = load_legacy2d(proj)
    Ny, Nx = fx["S"].shape
    s = Legacy2D(Nx, Ny, h=fx["h"], dt=fx["dt"], c=fx["c"], rho=fx["rho"], eps=fx["eps"], tol=fx["tol"],
                 pml_n=fx["pml"][0], pml_s=fx["pml"][1], pml_e=fx["pml"][2], pml_w=fx["pml"][3])
    t0 = time.perf_counter()
    s.load_geometry(fx["S"], fx["oid"])
    m = fx["materials"]
    s.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["C"], m["alpha"], m["beta"])
    s.set_fields(fx["p0"], fx["u0"])
    s.set_receiver(fx["rec"][0], fx["rec"][1], fx["Nt"])
    t1 = time.perf_counter()
    s.run(fx["Nt"])
    ir = s.ir()
    t_fz = time.perf_counter() - t1
    t_fz_setup = t1 - t0
    s.close()
    nodes = (Nx - 6) * (Ny - 6)
    err = float(np.linalg.norm(ir - fx["ir"]) / np.linalg.norm(fx["ir"]))
    result = {"nodes": nodes, "steps": fx["Nt"], "reference_loop_s": t_ref_loop,
              "reference_gnode_s": nodes * fx["Nt"] / t_ref_loop / 1e9, "fz_run_s": t_fz, "fz_setup_s": t_fz_setup,
              "fz_gnode_s": nodes * fx["Nt"] / t_fz / 1e9, "speedup_loop": t_ref_loop / t_fz,
              "ir_rel_l2_vs_reference": err}
    print(json.dumps(result))
    outdir = os.environ.get("FZ_RESULTS_DIR", "")
    if outdir and os.path.isdir(outdir):
        with open(os.path.join(outdir, "reference_speed_2d.json"), "w") as f:
            json.dump(result, f, indent=1)
    assert np.abs(fx["ir"]).max() > 1e-4
    assert err < 1e-5, err
    assert t_fz < t_ref_loop
