"""Planar (two_d) solves: the 3D scheme restricted to one z-plane (config 1 semantics), CUDA vs the
FP64 oracle run with the same restriction."""
import numpy as np
import pytest

from fases_b200 import materials as mats
from fases_b200 import scenes
from tests.helpers import rel_l2


def _room(seed=0, steps=80):
    rng = np.random.default_rng(seed)
    h, c, rho = 0.05, 343.0, 1.2
    dt = 0.5 * h / c
    sc = scenes.box_room_2d((60, 48), h, [((25, 18), (33, 26))])
    walls = [mats.random_passive(rng, dt, c / (4 * h), K=2, L=1) for _ in range(4)]
    walls[1] = mats.matched()  # x-hi under the cPML
    packed = mats.pack(walls + [mats.rigid(0.99)])
    p0 = scenes.gaussian_pulse(sc.shape, h, (18, 20, 3), 3.0)
    p0[:3] = 0.0
    p0[4:] = 0.0
    recs = np.array([[40, 30, 3], [10, 44, 3], [55, 8, 3]], np.int32)
    return dict(scene=sc, materials=packed, h=h, c=c, rho=rho, dt=dt, pml=(0, 0, 1, 0, 0, 0), pml_cells=8, p0=p0,
                recs=recs, steps=steps)


def _oracle(cfg):
    from oracle.oracle import Oracle
    sc = cfg["scene"]
    o = Oracle(sc.S, sc.oid, cfg["h"], cfg["c"], cfg["rho"], cfg["dt"], pml=cfg["pml"], pml_cells=cfg["pml_cells"],
               materials=cfg["materials"], rec_cells=cfg["recs"], max_steps=cfg["steps"], two_d=True)
    o.set_fields(p=cfg["p0"])
    o.run(cfg["steps"])
    return o


def test_planar_oracle_keeps_w_zero_and_absorbs():
    cfg = _room(steps=60)
    o = _oracle(cfg)
    p, u, v, w = o.fields()
    assert np.all(w == 0.0)
    assert np.all(p[:3] == 0.0) and np.all(p[4:] == 0.0)
    assert np.isfinite(p).all()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 1e-5)])
def test_planar_gpu_matches_oracle(precision, tol):
    from fases_b200 import Solver, params
    cfg = _room(seed=3, steps=120)
    s = Solver(params(h=cfg["h"], c=cfg["c"], rho=cfg["rho"], dt=cfg["dt"], pml=cfg["pml"],
                      pml_cells=cfg["pml_cells"], precision=precision, two_d=True))
    s.load_geometry(cfg["scene"].S, cfg["scene"].oid)
    m = cfg["materials"]
    s.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    s.set_receivers(cfg["recs"], cfg["steps"])
    s.set_fields(p=cfg["p0"])
    s.run(cfg["steps"])
    o = _oracle(cfg)
    ir_o, _ = o.ir()
    ir = s.ir()
    for r in range(ir.shape[0]):
        assert rel_l2(ir[r], ir_o[r]) < tol, (precision, r, rel_l2(ir[r], ir_o[r]))
    if precision == "fp64":
        for a, b in zip(s.fields(), o.fields()):
            assert rel_l2(a, b) < tol or np.linalg.norm(b) == 0.0
    s.close()


def test_planar_grid_rules():
    import ctypes

    from fases_b200 import FzError, Solver, params
    p = params(two_d=True, pml=(1, 0, 0, 0, 0, 0))
    h = ctypes.c_void_p()
    from fases_b200 import _abi
    rc = _abi.lib().fz_create(ctypes.byref(p), ctypes.byref(h))
    assert rc in (_abi.FZ_EINVAL,)  # z faces have no cPML in a planar solve (checked before the device)
