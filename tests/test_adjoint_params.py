"""Gradients beyond the ADE coefficients (fz_misfit_gradient_ex) and the torch.autograd front end.

FP64 solves of the small cPML room of test_adjoint (cPML on the z-hi and x-hi faces, PCS source,
Gaussian pulse), checked against central differences of the forward solver:
- source strengths and waveform samples: J would be quadratic in both but for WENO-Z's nonlinear
  weights (the pulse and the source field do not superpose exactly): the strength agrees to about
  1e-6 (checked at 1e-5), a smooth waveform direction within 1e-3, and the waveform gradient
  reproduces the strength gradient exactly (sum_nn dJ/du_s u_s = sval dJ/dsval);
- cPML profile parameters (R0, kappa_max, alpha_max) and the initial pressure field: relative step
  1e-5 (WENO-Z's weights make J piecewise smooth), agreement within 1e-3 as the adjoint tests ask;
- the cotangent (vector-Jacobian) mode against the misfit mode, and torch.autograd through
  impulse_responses / misfit against Solver.misfit_gradient_ex (same numbers, 1e-9)."""
import ctypes

import numpy as np
import pytest

from tests.helpers import small_room

STEPS = 48


def _cfg():
    cfg = small_room(seed=41, pml=(1, 0, 1, 0, 0, 0), steps=STEPS)
    p0 = cfg["p0"].copy()
    p0[cfg["scene"].S < cfg["h"]] = 0.0
    cfg["p0"] = p0
    return cfg


def _solver(cfg, sval=None, u_s=None, p0=None, pml=None, precision="fp64"):
    from fases_b200 import Solver, params
    kw = {}
    if pml is not None:
        kw = dict(pml_R0=pml[0], pml_kappa_max=pml[1], pml_alpha_max=pml[2])
    s = Solver(params(h=cfg["h"], c=cfg["c"], rho=cfg["rho"], dt=cfg["dt"], pml=cfg["pml"],
                      pml_cells=cfg["pml_cells"], precision=precision, **kw))
    s.load_geometry(cfg["scene"].S, cfg["scene"].oid)
    m = cfg["materials"]
    s.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    s.set_sources(cfg["src"], cfg["sval"] if sval is None else sval, cfg["src_opt"],
                  u_s=cfg["u_s"] if u_s is None else u_s)
    s.set_receivers(cfg["recs"], STEPS)
    s.set_fields(p=cfg["p0"] if p0 is None else p0)
    return s


def _J(cfg, target, **kw):
    s = _solver(cfg, **kw)
    s.run(STEPS)
    ir = s.ir()
    s.close()
    return float(np.sum((ir - target) ** 2))


def _target(cfg):
    s = _solver(cfg, sval=cfg["sval"] * 0.8, pml=(1e-5, 3.0, 40.0))
    s.run(STEPS)
    ir = s.ir()
    s.close()
    return ir


def test_gradient_struct_matches_header():
    from fases_b200 import _abi
    # int32 cotangent (+4 padding) and five (double*, int64) pairs
    assert ctypes.sizeof(_abi.FzGradients) == 88
    assert ctypes.sizeof(_abi.FzParams) == 4 * 10 + 8 * 5 + 4 * 2 + 8 * 4
    p = _abi.FzParams()
    assert _abi.lib().fz_params_init(ctypes.byref(p)) == 0
    assert p.pml_R0 == 1e-7 and p.pml_kappa_max == 5.0 and abs(p.pml_alpha_max - 20 * np.pi) < 1e-12
    assert p.pml_order == 2.0
    g = _abi.FzGradients()
    assert _abi.lib().fz_misfit_gradient_ex(None, 10, 5, None, 10, None, ctypes.byref(g), None) == _abi.FZ_EINVAL


def test_material_rows_round_trip():
    from fases_b200.autograd import pack_materials, unpack_materials
    rng = np.random.default_rng(0)
    rows = rng.standard_normal((3, 1 + 2 * 2 + 4 * 3))
    assert np.array_equal(pack_materials(*unpack_materials(rows, 2, 3)), rows)


@pytest.mark.gpu
def test_source_gradients_match_central_differences():
    cfg = _cfg()
    target = _target(cfg)
    s = _solver(cfg)
    g = s.misfit_gradient(target, segment_steps=16, sources=True)
    s.close()
    sval = np.asarray(cfg["sval"], dtype=np.float64)
    e = 1e-3 * abs(sval[0])
    fd = (_J(cfg, target, sval=sval + e) - _J(cfg, target, sval=sval - e)) / (2 * e)
    assert abs(g["sval"][0] - fd) <= 1e-5 * abs(fd), (g["sval"][0], fd)
    # waveform: the waveform modulated by a slow cosine over the samples the run reads
    # (nn < 2 * STEPS + 1), so the perturbation stays small against the field it changes (a
    # perturbation that dominates the early, near-zero samples makes WENO-Z's weights move inside
    # the difference step)
    us = np.asarray(cfg["u_s"], dtype=np.float64)
    nn = np.arange(us.size, dtype=np.float64)
    dirn = us * np.cos(2.0 * np.pi * nn / 50.0)
    dirn[2 * STEPS + 1:] = 0.0
    e = 1e-5
    fd = (_J(cfg, target, u_s=us + e * dirn) - _J(cfg, target, u_s=us - e * dirn)) / (2 * e)
    ad = float(np.sum(g["wave"].sum(axis=0) * dirn))
    assert abs(ad - fd) <= 1e-3 * abs(fd), (ad, fd)
    # dJ/dsval = sum over the samples of dJ/du_s * u_s / sval
    assert abs(float(np.sum(g["wave"][0] * us)) / sval[0] - g["sval"][0]) <= 1e-9 * abs(g["sval"][0])


@pytest.mark.gpu
def test_pml_gradient_matches_central_differences():
    cfg = _cfg()
    target = _target(cfg)
    s = _solver(cfg)
    g = s.misfit_gradient(target, segment_steps=16, pml=True)
    s.close()
    base = (1e-7, 5.0, 20 * np.pi)
    for q, name in enumerate(("R0", "kappa_max", "alpha_max")):
        e = 1e-5 * base[q]
        up = list(base)
        dn = list(base)
        up[q] += e
        dn[q] -= e
        fd = (_J(cfg, target, pml=up) - _J(cfg, target, pml=dn)) / (2 * e)
        assert abs(g["pml"][name] - fd) <= 1e-3 * abs(fd), (name, g["pml"][name], fd)


@pytest.mark.gpu
def test_initial_field_gradient_matches_central_differences():
    from fases_b200 import scenes
    cfg = _cfg()
    target = _target(cfg)
    s = _solver(cfg)
    g = s.misfit_gradient(target, segment_steps=16, initial=True)
    s.close()
    dp = g["initial"][0]
    assert dp.shape == cfg["scene"].S.shape
    dirn = scenes.gaussian_pulse(cfg["scene"].shape, cfg["h"], (10, 12, 9), 2.5, amplitude=1.0)
    dirn[cfg["scene"].S < cfg["h"]] = 0.0
    e = 1e-5 * np.abs(cfg["p0"]).max()
    fd = (_J(cfg, target, p0=cfg["p0"] + e * dirn) - _J(cfg, target, p0=cfg["p0"] - e * dirn)) / (2 * e)
    ad = float(np.sum(dp * dirn))
    assert abs(ad - fd) <= 1e-3 * abs(fd), (ad, fd)
    # ghost cells are written by no kernel: zero there
    assert np.all(dp[:3] == 0.0) and np.all(dp[:, :, :3] == 0.0)


@pytest.mark.gpu
def test_cotangent_mode_equals_misfit_mode():
    cfg = _cfg()
    target = _target(cfg)
    s = _solver(cfg)
    g = s.misfit_gradient(target, segment_steps=16, sources=True, pml=True, initial=True)
    ir = s.ir()
    s.close()
    s = _solver(cfg)
    gv = s.misfit_gradient(2.0 * (ir - target), segment_steps=16, sources=True, pml=True, initial=True,
                           cotangent=True)
    s.close()
    assert abs(gv["J"] - float(np.sum(2.0 * (ir - target) * ir))) <= 1e-12 * abs(gv["J"])
    for key in ("raw", "sval", "wave"):
        assert np.allclose(gv[key], g[key], rtol=1e-9, atol=1e-12 * np.abs(g[key]).max()), key
    for name in ("R0", "kappa_max", "alpha_max"):
        assert abs(gv["pml"][name] - g["pml"][name]) <= 1e-9 * abs(g["pml"][name]), name
    assert np.allclose(gv["initial"][0], g["initial"][0], rtol=1e-9, atol=1e-12 * np.abs(g["initial"][0]).max())


@pytest.mark.gpu
def test_torch_autograd_matches_adjoint():
    import torch

    from fases_b200 import autograd as fa
    cfg = _cfg()
    target = _target(cfg)
    m = cfg["materials"]
    K, L = np.asarray(m["A"]).shape[1], np.asarray(m["B"]).shape[1]
    rows = fa.pack_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    room = fa.Room(cfg["scene"].S, cfg["scene"].oid,
                   dict(h=cfg["h"], c=cfg["c"], rho=cfg["rho"], dt=cfg["dt"], pml=cfg["pml"],
                        pml_cells=cfg["pml_cells"], precision="fp64"),
                   cfg["recs"], STEPS, rows, src_cells=cfg["src"], sval0=cfg["sval"], src_opt=cfg["src_opt"],
                   u_s=cfg["u_s"], p0=cfg["p0"], K=K, L=L, segment_steps=16)
    theta = torch.tensor(rows, requires_grad=True)
    sval = torch.tensor(np.asarray(cfg["sval"], dtype=np.float64), requires_grad=True)
    pml = torch.tensor([1e-7, 5.0, 20 * np.pi], dtype=torch.float64, requires_grad=True)
    p0 = torch.tensor(cfg["p0"], requires_grad=True)
    tgt = torch.tensor(target)
    ir = fa.impulse_responses(room, theta, sval, pml, p0)
    assert ir.shape == (cfg["recs"].shape[0], STEPS) and ir.dtype == torch.float64
    loss = ((ir - tgt) ** 2).sum()
    loss.backward()
    s = _solver(cfg)
    g = s.misfit_gradient(target, segment_steps=16, sources=True, pml=True, initial=True)
    s.close()
    assert abs(loss.item() - g["J"]) <= 1e-12 * g["J"]
    assert np.allclose(theta.grad.numpy(), g["raw"], rtol=1e-9, atol=1e-12 * np.abs(g["raw"]).max())
    assert np.allclose(sval.grad.numpy(), g["sval"], rtol=1e-9)
    assert np.allclose(pml.grad.numpy(), [g["pml"]["R0"], g["pml"]["kappa_max"], g["pml"]["alpha_max"]], rtol=1e-9)
    assert np.allclose(p0.grad.numpy(), g["initial"][0], rtol=1e-9, atol=1e-12 * np.abs(g["initial"][0]).max())
    # misfit(): J and the same gradient from one call
    theta2 = torch.tensor(rows, requires_grad=True)
    J = fa.misfit(room, tgt, theta2)
    (2.0 * J).backward()
    assert abs(J.item() - g["J"]) <= 1e-12 * g["J"]
    assert np.allclose(theta2.grad.numpy(), 2.0 * g["raw"], rtol=1e-9, atol=1e-12 * np.abs(g["raw"]).max())
