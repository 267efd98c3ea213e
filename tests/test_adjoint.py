"""Discrete adjoint (fz_misfit_gradient): the gradient of the receiver misfit with respect to the
ADE coefficients against central finite differences of the forward solver (FP64, agreement within
1e-3), independence of the checkpoint segment length, and the FP32 gradient against the FP64 one.

The finite differences use a relative step of 1e-5: WENO-Z's weights switch where the smoothness
indicators cross (|beta0 - beta2|), so J is only piecewise smooth, and a step of 1e-4 crossed such
switches for some coefficients of this room (differences of up to 2 % there, shrinking to 1e-5 at
the smaller step), while the adjoint is the derivative of the piece the forward run is on."""
import numpy as np
import pytest

from fases_b200 import materials as mats
from tests.helpers import small_room

STEPS = 48


def _cfg(seed=41):
    cfg = small_room(seed=seed, pml=(1, 0, 1, 0, 0, 0), steps=STEPS)
    sc = cfg["scene"]
    p0 = cfg["p0"].copy()
    p0[sc.S < cfg["h"]] = 0.0  # cells the stage kernels skip start at zero
    cfg["p0"] = p0
    return cfg


def _packed_with(cfg, key, m, idx, value):
    pk = {k: np.array(v, dtype=np.float64, copy=True) for k, v in cfg["materials"].items()}
    if pk[key].ndim == 1:
        pk[key][m] = value
    else:
        pk[key][m, idx] = value
    return pk


def _solver(cfg, precision, packed=None):
    from fases_b200 import Solver, params
    s = Solver(params(h=cfg["h"], c=cfg["c"], rho=cfg["rho"], dt=cfg["dt"], pml=cfg["pml"],
                      pml_cells=cfg["pml_cells"], precision=precision))
    s.load_geometry(cfg["scene"].S, cfg["scene"].oid)
    m = cfg["materials"] if packed is None else packed
    s.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    s.set_sources(cfg["src"], cfg["sval"], cfg["src_opt"], u_s=cfg["u_s"])
    s.set_receivers(cfg["recs"], STEPS)
    s.set_fields(p=cfg["p0"])
    return s


def _J(cfg, packed, target):
    s = _solver(cfg, "fp64", packed)
    s.run(STEPS)
    ir = s.ir()
    s.close()
    return float(np.sum((ir - target[:, :STEPS]) ** 2))


def _target(cfg):
    rng = np.random.default_rng(5)
    pk = {k: np.array(v, dtype=np.float64, copy=True) for k, v in cfg["materials"].items()}
    for k in ("A", "B", "Cc"):
        pk[k] = pk[k] * (1.0 + 0.2 * rng.standard_normal(pk[k].shape))
    pk["Rinf"] = np.clip(pk["Rinf"] * 0.9, -0.99, 0.99)
    s = _solver(cfg, "fp64", pk)
    s.run(STEPS)
    ir = s.ir()
    s.close()
    return ir


KEYS = {"Rinf": "Rinf", "A": "A", "zeta": "zeta", "B": "B", "C": "Cc", "alpha": "alpha", "beta": "beta"}


def test_gradient_entry_point_checks_arguments():
    import ctypes

    from fases_b200 import _abi
    L = _abi.lib()
    assert L.fz_misfit_gradient(None, 10, 5, None, 10, None, None, 0, None) == _abi.FZ_EINVAL


@pytest.mark.gpu
def test_adjoint_gradient_matches_central_differences():
    cfg = _cfg()
    target = _target(cfg)
    s = _solver(cfg, "fp64")
    g = s.misfit_gradient(target, segment_steps=16)
    s.close()
    assert g["J"] > 0
    assert abs(g["J"] - _J(cfg, None, target)) <= 1e-12 * g["J"]
    nm = g["raw"].shape[0]
    # every wall material (obstacles are rigid K = L = 0 fits): one coefficient of each kind
    checked = 0
    for m in range(nm):
        for name in ("Rinf", "A", "zeta", "B", "C", "alpha", "beta"):
            key = KEYS[name]
            arr = np.asarray(cfg["materials"][key], dtype=np.float64)
            if arr.ndim == 1:
                theta = arr[m]
                gval = g[name][m]
                idx = None
            else:
                if arr.shape[1] == 0:
                    continue
                idx = 0
                theta = arr[m, 0]
                gval = g[name][m, 0]
            if theta == 0.0 or abs(gval) < 1e-6 * abs(g["J"]) / max(abs(theta), 1e-30):
                continue
            hstep = 1e-5 * abs(theta)
            jp = _J(cfg, _packed_with(cfg, key, m, idx, theta + hstep), target)
            jm = _J(cfg, _packed_with(cfg, key, m, idx, theta - hstep), target)
            fd = (jp - jm) / (2 * hstep)
            assert abs(fd - gval) <= 1e-3 * abs(fd), (m, name, gval, fd)
            checked += 1
            if checked >= 14:
                break
        if checked >= 14:
            break
    assert checked >= 7


@pytest.mark.gpu
def test_adjoint_gradient_independent_of_segment_and_fp32_close():
    cfg = _cfg(seed=42)
    target = _target(cfg)
    grads = []
    for seg in (16, 48, 7):
        s = _solver(cfg, "fp64")
        grads.append(s.misfit_gradient(target, segment_steps=seg))
        # the handle ends at the forward's final state with its traces
        assert s.steps_done() == STEPS
        s.close()
    for g in grads[1:]:
        assert np.allclose(g["raw"], grads[0]["raw"], rtol=1e-10, atol=1e-14 * np.abs(grads[0]["raw"]).max())
    s = _solver(cfg, "fp32")
    g32 = s.misfit_gradient(target, segment_steps=16)
    s.close()
    ref = grads[0]["raw"]
    assert np.linalg.norm(g32["raw"] - ref) <= 2e-3 * np.linalg.norm(ref)


@pytest.mark.gpu
@pytest.mark.parametrize("K,L", [(0, 2), (2, 0), (3, 1)])
def test_adjoint_other_pole_counts(K, L):
    """Materials with complex pairs only, real poles only, and more real poles than the band
    kernels' fixed-size forms hold: the ADE sets of a segment (written straight into the segment
    storage by the recompute, their adjoints assigned by the first write of each step) give the
    same gradient for any segment length, and one coefficient of each kind present matches central
    differences."""
    cfg = small_room(seed=50 + 3 * K + L, pml=(1, 0, 1, 0, 0, 0), K=K, L=L, steps=STEPS)
    sc = cfg["scene"]
    p0 = cfg["p0"].copy()
    p0[sc.S < cfg["h"]] = 0.0
    cfg["p0"] = p0
    target = _target(cfg)
    grads = []
    for seg in (48, 7):
        s = _solver(cfg, "fp64")
        grads.append(s.misfit_gradient(target, segment_steps=seg))
        s.close()
    ref = grads[0]["raw"]
    assert np.allclose(grads[1]["raw"], ref, rtol=1e-10, atol=1e-14 * np.abs(ref).max())
    g = grads[0]
    names = ["Rinf"] + (["A", "zeta"] if K else []) + (["B", "C", "alpha", "beta"] if L else [])
    checked = 0
    for name in names:
        key = KEYS[name]
        arr = np.asarray(cfg["materials"][key], dtype=np.float64)
        # the wall material whose coefficient J depends on most (obstacles are rigid fits)
        gk = np.abs(g[name] if arr.ndim == 1 else g[name][:, 0])
        m = int(np.argmax(gk))
        idx = None if arr.ndim == 1 else 0
        theta = arr[m] if idx is None else arr[m, 0]
        gval = g[name][m] if idx is None else g[name][m, 0]
        if theta == 0.0:
            continue
        hstep = 1e-5 * abs(theta)
        fd = (_J(cfg, _packed_with(cfg, key, m, idx, theta + hstep), target) -
              _J(cfg, _packed_with(cfg, key, m, idx, theta - hstep), target)) / (2 * hstep)
        assert abs(fd - gval) <= 1e-3 * abs(fd), (K, L, name, gval, fd)
        checked += 1
    assert checked >= 2
