"""Material refinement against a target impulse response (fases_b200.fit): L-BFGS-B on the
adjoint gradient recovers perturbed wall coefficients of a small room, keeps them passive, and the
.fit / poles.txt writers produce the files the project loader reads back."""
import os

import numpy as np
import pytest

from fases_b200 import fit
from fases_b200 import materials as mats
from tests.helpers import small_room

STEPS = 60


def test_fit_files_round_trip(tmp_path):
    m = mats.Material(0.7, np.array([120.0]), np.array([900.0]), np.array([3.0, -2.0]), np.array([1.5, 0.5]),
                      np.array([400.0, 800.0]), np.array([2000.0, 4000.0]))
    fit.write_fits(str(tmp_path / "fit"), ["wall"], [m])
    txt = open(tmp_path / "fit" / "wall.fit").read().split("\n")
    assert txt[0] == "# R_inf" and txt[2] == "# K L" and txt[3] == "1 2"
    p = str(tmp_path / "config" / "poles.txt")
    assert fit.write_poles(p, [m, mats.rigid()]) == (1, 2)
    open(p, "w").write("3 1\n")
    assert fit.write_poles(p, [m]) == (3, 2)  # running maximum
    assert fit.passivity_penalty(mats.rigid(0.99), 1e-5) == 0.0
    assert fit.passivity_penalty(mats.Material(1.2), 1e-5) > 0.0


@pytest.mark.gpu
def test_refine_recovers_perturbed_walls():
    from fases_b200 import Solver, params
    cfg = small_room(seed=61, pml=(1, 0, 0, 0, 0, 0), steps=STEPS)
    sc = cfg["scene"]
    p0 = cfg["p0"].copy()
    p0[sc.S < cfg["h"]] = 0.0
    rng = np.random.default_rng(5)
    f_cutoff = cfg["f_cutoff"]
    truth = [mats.random_passive(rng, cfg["dt"], f_cutoff, K=1, L=1) for _ in range(6)] + [mats.rigid(0.99)]
    truth[5] = mats.matched()  # z-hi face under the cPML

    def make(packed):
        s = Solver(params(h=cfg["h"], c=cfg["c"], rho=cfg["rho"], dt=cfg["dt"], pml=cfg["pml"],
                          pml_cells=cfg["pml_cells"], precision="fp64"))
        s.load_geometry(sc.S, sc.oid)
        s.set_materials(packed["Rinf"], packed["A"], packed["zeta"], packed["B"], packed["Cc"], packed["alpha"],
                        packed["beta"])
        s.set_sources(cfg["src"], cfg["sval"], cfg["src_opt"], u_s=cfg["u_s"])
        s.set_receivers(cfg["recs"], STEPS)
        s.set_fields(p=p0)
        return s

    s = make(mats.pack(truth))
    s.run(STEPS)
    target = s.ir()
    s.close()
    start = [m for m in (mats.Material(t.Rinf, t.A.copy(), t.zeta.copy(), t.B.copy(), t.C.copy(), t.alpha.copy(),
                                       t.beta.copy()) for t in truth)]
    for m in (0, 1):  # x-lo and x-hi walls: residues and R_inf off by 20 %
        start[m].Rinf *= 0.8
        start[m].A = start[m].A * 1.2
        start[m].B = start[m].B * 0.8
    free = [(m, key, 0) for m in (0, 1) for key in ("Rinf", "A", "B")]
    out = fit.refine(make, target, start, free, cfg["dt"], f_cutoff, nsteps=STEPS, segment_steps=20, maxiter=25)
    assert out["J"] < 1e-3 * out["J0"], (out["J0"], out["J"])
    for m in (0, 1):
        assert abs(out["materials"][m].Rinf - truth[m].Rinf) < 0.05 * abs(truth[m].Rinf)
        assert out["passive"][m]
