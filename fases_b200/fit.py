"""Wall materials fitted to receiver traces with the solver's discrete adjoint.

The reference fits each material's ADE coefficients to an octave absorption spectrum in the
frequency domain (common/fminconFIT.py:239-348: bounded BFGS in sigmoid pole coordinates with a
passivity penalty; common/vectFIT.py:335-459) and never differentiates the time-domain solver.
`refine` fits chosen coefficients to a target impulse response instead: it minimises
J = sum_r sum_n (IR_r[n] - target_r[n])^2 with L-BFGS-B, the gradient of J coming from
fz_misfit_gradient, under the same pole bounds and the same passivity penalty (continuous |R| up to
Nyquist and the gain of the discrete SSP-RK3 recursion must stay below 1 - margin). `write_fits` and
`write_poles` write the files the solver reads (the .fit format of common/vectFIT.py:443-458 and
common/filterABC.h:31-90; poles.txt as the running maximum of common/vectFIT.py:484-507).
"""
import copy
import os

import numpy as np

from . import materials as mats

KEYS = ("Rinf", "A", "zeta", "B", "C", "alpha", "beta")
_ATTR = {"Rinf": "Rinf", "A": "A", "zeta": "zeta", "B": "B", "C": "C", "alpha": "alpha", "beta": "beta"}
_RK3_BOX = 0.76  # stability margin the reference's fitter applies to the poles (fminconFIT.py:280-291)


def _get(m, key, idx):
    v = getattr(m, _ATTR[key])
    return float(v) if key == "Rinf" else float(v[idx])


def _set(m, key, idx, value):
    if key == "Rinf":
        m.Rinf = float(value)
    else:
        arr = np.array(getattr(m, _ATTR[key]), dtype=float, copy=True)
        arr[idx] = value
        setattr(m, _ATTR[key], arr)


def pole_bounds(key, dt, f_cutoff):
    """Bounds of one coefficient: |R_inf| <= 1, real and complex pole rates in (0, 2.5127 * 0.76 /
    dt], pair frequencies in (0, min(1.732 * 0.76 / dt, 2 pi f_cutoff)] (fminconFIT.py:287-290)."""
    if key == "Rinf":
        return (-1.0, 1.0)
    if key in ("zeta", "alpha"):
        return (1e-6, 2.5127 * _RK3_BOX / dt)
    if key == "beta":
        return (1e-6, min(1.732 * _RK3_BOX / dt, 2 * np.pi * f_cutoff))
    return (None, None)


def passivity_penalty(m, dt, margin=1e-3):
    """Sum of squared excesses of |R(j w)| (1 Hz .. Nyquist) and of the discrete recursion's gain
    (5 Hz .. Nyquist) over 1 - margin: zero for a passive material."""
    f_nyq = 0.5 / dt
    w = 2 * np.pi * np.logspace(0.0, np.log10(f_nyq), 1024)
    ov = np.maximum(np.abs(mats.R_continuous(m, w)) - (1.0 - margin), 0.0)
    fd = np.logspace(np.log10(5.0), np.log10(0.999 * f_nyq), 256)
    ovd = np.maximum(np.abs(mats.R_discrete(m, dt, fd)) - (1.0 - margin), 0.0)
    return float(np.sum(ov ** 2) + np.sum(ovd ** 2))


def refine(make_solver, target, materials, free, dt, f_cutoff, nsteps=None, segment_steps=250, maxiter=30,
           passivity_weight=1e3, margin=1e-3):
    """Fits the coefficients `free` = [(material index, key, pole index), ...] (key in KEYS, pole
    index ignored for Rinf) of `materials` to `target` [n_rec, n_steps].

    make_solver(packed) must return a Solver at step 0 (geometry, sources, receivers with capacity
    >= nsteps, initial fields) using the material arrays `packed` (materials.pack layout). Returns
    a dict: the fitted materials, J at the start and end, the J of every evaluation, whether each
    fitted material is passive, and the scipy result."""
    from scipy.optimize import minimize

    cur = [copy.deepcopy(m) for m in materials]
    K = max([len(m.A) for m in cur] + [1])
    L = max([len(m.B) for m in cur] + [1])
    theta0 = np.array([_get(cur[m], key, idx) for m, key, idx in free])
    scale = np.where(theta0 != 0.0, np.abs(theta0), 1.0)
    bounds = []
    for (m, key, idx), sc in zip(free, scale):
        lo, hi = pole_bounds(key, dt, f_cutoff)
        bounds.append((None if lo is None else lo / sc, None if hi is None else hi / sc))
    touched = sorted({m for m, _, _ in free})
    history = []
    state = {"J0": None}

    def setup(u):
        for (m, key, idx), v in zip(free, u * scale):
            _set(cur[m], key, idx, v)

    def penalty(u):
        setup(u)
        return sum(passivity_penalty(cur[m], dt, margin) for m in touched)

    def fun(u):
        setup(u)
        s = make_solver(mats.pack(cur, K, L))
        try:
            g = s.misfit_gradient(target, nsteps=nsteps, segment_steps=segment_steps)
        finally:
            s.close()
        J = g["J"]
        if state["J0"] is None:
            state["J0"] = J if J > 0 else 1.0
        history.append(J)
        grad = np.array([g["Rinf"][m] if key == "Rinf" else g[key][m, idx] for m, key, idx in free])
        f = J / state["J0"]
        df = grad * scale / state["J0"]
        p0 = penalty(u)
        if p0 > 0.0 or passivity_weight > 0.0:
            # the penalty is cheap (closed forms): central differences per coefficient
            dp = np.zeros_like(u)
            if p0 > 0.0:
                for q in range(u.size):
                    e = np.zeros_like(u)
                    e[q] = 1e-6 * max(abs(u[q]), 1.0)
                    dp[q] = (penalty(u + e) - penalty(u - e)) / (2 * e[q])
            setup(u)
            f += passivity_weight * p0
            df = df + passivity_weight * dp
        return f, df

    u0 = theta0 / scale
    res = minimize(fun, u0, jac=True, method="L-BFGS-B", bounds=bounds, options={"maxiter": int(maxiter)})
    setup(res.x)
    return {"materials": cur, "J0": state["J0"], "J": history[-1] if history else None, "history": history,
            "passive": {m: mats.is_passive(cur[m], dt, margin=0.0) for m in touched}, "result": res}


def write_fits(fit_dir, names, materials):
    """One <name>.fit per material (input/fit/ of a project, read per OBJ layer)."""
    os.makedirs(fit_dir, exist_ok=True)
    for name, m in zip(names, materials):
        m.write_fit(os.path.join(fit_dir, name + ".fit"))


def write_poles(path, materials):
    """poles.txt = "K_m L_m", the running maximum of the pole counts over the materials and the file's
    previous content (the solver zero-pads every material to K_m, L_m)."""
    K = max([len(m.A) for m in materials] + [0])
    L = max([len(m.B) for m in materials] + [0])
    if os.path.exists(path):
        try:
            prev = open(path).read().split()
            K, L = max(K, int(float(prev[0]))), max(L, int(float(prev[1])))
        except (ValueError, IndexError):
            pass
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        f.write("%d %d\n" % (K, L))
    return K, L
