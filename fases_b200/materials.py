"""ADE pole-residue materials: the continuous reflection model, the closed-form response of the
solver's discrete ADE recursion, and seeded passive random materials for the synthetic rooms.

R(s) = R_inf + sum_k A_k/(s + zeta_k) + sum_l (B_l s + C_l beta_l + alpha_l B_l)/((s + alpha_l)^2 + beta_l^2)
(3D-solver/tests/ADE_benchmark/ADE_TST_3D.py:14-26, the model the .fit files hold).
"""
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Material:
    Rinf: float
    A: np.ndarray = field(default_factory=lambda: np.zeros(0))
    zeta: np.ndarray = field(default_factory=lambda: np.zeros(0))
    B: np.ndarray = field(default_factory=lambda: np.zeros(0))
    C: np.ndarray = field(default_factory=lambda: np.zeros(0))
    alpha: np.ndarray = field(default_factory=lambda: np.zeros(0))
    beta: np.ndarray = field(default_factory=lambda: np.zeros(0))

    def write_fit(self, path):
        """Writes the .fit text format read by common/filterABC.h:31-90."""
        with open(path, "w") as f:
            f.write("# R_inf\n%.17g\n# K L\n%d %d\n# A_k zeta_k\n" % (self.Rinf, len(self.A), len(self.B)))
            for a, z in zip(self.A, self.zeta):
                f.write("%.17g %.17g\n" % (a, z))
            f.write("# B_l C_l alpha_l beta_l\n")
            for b, c, al, be in zip(self.B, self.C, self.alpha, self.beta):
                f.write("%.17g %.17g %.17g %.17g\n" % (b, c, al, be))


def R_continuous(m: Material, w):
    s = 1j * np.asarray(w, float)
    R = np.full(s.shape, m.Rinf + 0j)
    for a, z in zip(m.A, m.zeta):
        R += a / (z + s)
    for b, c, al, be in zip(m.B, m.C, m.alpha, m.beta):
        R += (b * s + c * be + al * b) / ((al + s) ** 2 + be ** 2)
    return R


def R_discrete(m: Material, dt, freqs):
    """Steady-state complex response of the SSP-RK3 ADE recursion the solver runs per band cell
    (functions3D.cuh:426-459 with stages (0,1,1), (3,1,4), (1,2,3), inputs at t, t+dt, t+dt/2),
    read after the last stage. Derived here from the stage algebra: for one step with state x,
    input e^{j w t}, and the linear per-stage operator M (x' = M x + e1 w) with Am = I + dt M:
        stage 0: x1 = Am x + dt e1 w(t)
        stage 1: x2 = (3x + x1 + dt (M x1 + e1 w(t+dt)))/4
        stage 2: x3 = (x + 2 (x2 + dt (M x2 + e1 w(t+dt/2))))/3
    so x3 = G x + u(z) e1 with G = I/3 + Am/2 + Am^3/6 and
    u(z) = dt (Am^2/6 + Am z/6 + 2 z^{1/2}/3) e1,  z = e^{j w dt}.  Steady state x = z u/(z I - G);
    output y = R_inf w(t+dt/2) + c^T x3."""
    th = 2 * np.pi * np.asarray(freqs, float) * dt
    z = np.exp(1j * th)
    zh = np.exp(0.5j * th)
    y = m.Rinf * zh
    for a, ze in zip(m.A, m.zeta):
        g = 1.0 - ze * dt
        G = 1.0 / 3.0 + g / 2.0 + g ** 3 / 6.0
        u = dt * (g * g / 6.0 + g * z / 6.0 + 2.0 * zh / 3.0)
        y = y + a * z * u / (z - G)
    for b, c, al, be in zip(m.B, m.C, m.alpha, m.beta):
        Am = np.array([[1.0 - al * dt, -be * dt], [be * dt, 1.0 - al * dt]])
        A2 = Am @ Am
        G = np.eye(2) / 3.0 + Am / 2.0 + (A2 @ Am) / 6.0
        u0 = dt * (A2[0, 0] / 6.0 + Am[0, 0] * z / 6.0 + 2.0 * zh / 3.0)
        u1 = dt * (A2[1, 0] / 6.0 + Am[1, 0] * z / 6.0)
        a11, a12, a21, a22 = z - G[0, 0], -G[0, 1], -G[1, 0], z - G[1, 1]
        det = a11 * a22 - a12 * a21
        x1 = (a22 * u0 - a12 * u1) / det
        x2 = (-a21 * u0 + a11 * u1) / det
        y = y + z * (b * x1 + c * x2)
    return y


def is_passive(m: Material, dt, margin=0.0):
    """|R| <= 1 on a dense grid up to Nyquist and discrete gain <= 1: the accept test of the
    material fitter (common/fminconFIT.py:303-327)."""
    f_nyq = 0.5 / dt
    w = 2 * np.pi * np.logspace(0.0, np.log10(f_nyq), 2048)
    if np.max(np.abs(R_continuous(m, w))) > 1.0 - margin:
        return False
    fd = np.logspace(np.log10(5.0), np.log10(0.999 * f_nyq), 512)
    return bool(np.max(np.abs(R_discrete(m, dt, fd))) <= 1.0 - margin)


def random_passive(rng, dt, f_cutoff, K=2, L=2, zeta_range=(1e2, 1e4), alpha_range=(1e2, 1e4),
                   beta_lo=2 * np.pi * 50.0, max_tries=10000):
    """Seeded passive material with K real poles and L complex-conjugate pairs: poles drawn
    log-uniform, residues drawn and accepted only if passive (continuous and discrete)."""
    beta_hi = 2 * np.pi * 0.9 * f_cutoff
    for _ in range(max_tries):
        zeta = np.exp(rng.uniform(np.log(zeta_range[0]), np.log(zeta_range[1]), K))
        alpha = np.exp(rng.uniform(np.log(alpha_range[0]), np.log(alpha_range[1]), L))
        beta = rng.uniform(beta_lo, beta_hi, L)
        Rinf = rng.uniform(0.2, 0.9)
        A = zeta * rng.uniform(-0.3, 0.3, K)
        B = alpha * rng.uniform(-0.3, 0.3, L)
        Cc = alpha * rng.uniform(-0.3, 0.3, L)
        m = Material(Rinf, A, zeta, B, Cc, alpha, beta)
        if is_passive(m, dt, margin=1e-3):
            return m
    raise RuntimeError("no passive material found")


def rigid(Rinf=0.99):
    """Frequency-independent reflector (K = L = 0), like 3D-solver/input/fit/Material0.fit."""
    return Material(Rinf)


def matched():
    """All-zero coefficients: the R = 0 wall a BoundingBox layer gets (main3D.cu:625-631)."""
    return Material(0.0)


def pack(materials, K=None, L=None):
    """Stacks materials into the arrays of Solver.set_materials (zero-padded to K, L)."""
    K = max([len(m.A) for m in materials] + [0]) if K is None else K
    L = max([len(m.B) for m in materials] + [0]) if L is None else L
    n = len(materials)
    out = {k: np.zeros((n, K)) for k in ("A", "zeta")}
    out.update({k: np.zeros((n, L)) for k in ("B", "Cc", "alpha", "beta")})
    out["Rinf"] = np.array([m.Rinf for m in materials], float)
    for i, m in enumerate(materials):
        out["A"][i, :len(m.A)] = m.A
        out["zeta"][i, :len(m.zeta)] = m.zeta
        out["B"][i, :len(m.B)] = m.B
        out["Cc"][i, :len(m.C)] = m.C
        out["alpha"][i, :len(m.alpha)] = m.alpha
        out["beta"][i, :len(m.beta)] = m.beta
    return out
