"""Known-answer checks of the CPU oracle (no GPU): the ADE stage recursion against the closed-form
discrete response, the source waveform against the product's host code, physical sanity of the
stepping (energy decay in a rigid box, reciprocity)."""
import numpy as np
import pytest

from fases_b200 import materials as mats
from fases_b200 import scenes
from fases_b200.solver import source_waveform
from oracle import oracle as orc


def _sample_fit():
    # 3D-solver/tests/ADE_benchmark/sample.fit (K = 2, L = 3)
    return mats.Material(
        0.5021750604967876,
        np.array([328.5183890078403, -0.46803927460631534]), np.array([1071.6694737064222, 145.55896191182228]),
        np.array([-31.7133539445234, 51.27216735785404, -19.005306676212616]),
        np.array([123.06056772771578, 58.37901412199519, 74.64689114204187]),
        np.array([730.4911674793447, 456.76397711838615, 209.20766378183606]),
        np.array([2293.0412990105087, 1738.5911565662373, 529.8926564688727]))


@pytest.mark.parametrize("f", [50.0, 300.0, 1500.0, 4000.0])
def test_ade_recursion_matches_closed_form(f):
    """Drive the oracle's ADE_solver recursion (functions3D.cuh:426-459, stage inputs at t, t+dt,
    t+dt/2) with a complex exponential and compare the steady state after stage 2 with
    R_discrete."""
    m = _sample_fit()
    dt = 0.5 * 0.034 / 343.2
    n = 40000
    t = np.arange(n) * dt
    w = 2 * np.pi * f
    tin = np.stack([t, t + dt, t + 0.5 * dt], axis=1)
    yr = orc.ade_drive(m, dt, np.cos(w * tin))
    yi = orc.ade_drive(m, dt, np.sin(w * tin))
    y = yr[:, 2] + 1j * yi[:, 2]
    Rd = mats.R_discrete(m, dt, [f])[0]
    tail = slice(n - 2000, n)
    pred = Rd * np.exp(1j * w * t[tail])
    assert np.max(np.abs(y[tail] - pred)) < 1e-9 * max(1.0, abs(Rd))


def test_discrete_response_tends_to_continuous_at_low_frequency():
    m = _sample_fit()
    dt = 1e-6
    f = np.array([100.0, 500.0, 1000.0])
    Rc = mats.R_continuous(m, 2 * np.pi * f)
    Rd = mats.R_discrete(m, dt, f) * np.exp(-0.5j * 2 * np.pi * f * dt)
    assert np.max(np.abs(Rd - Rc)) < 1e-3


@pytest.mark.parametrize("src_opt", [0, 1])
def test_waveform_host_code_matches_oracle(src_opt):
    args = (src_opt, 25.0 if src_opt == 0 else 300.0, 707.1, 4.9529e-5, 3029, 0.034, float(np.float32(1.225)))
    us, pr, pk = source_waveform(*args)
    uo, po, pko = orc.waveform(*args)
    assert np.max(np.abs(us - uo)) <= 1e-12 * np.max(np.abs(uo))
    assert np.max(np.abs(pr - po)) <= 1e-12 * np.max(np.abs(po))
    assert abs(pk - pko) <= 1e-12 * pko


def test_interior_scheme_does_not_create_energy():
    """Free propagation (the pulse does not reach the walls): WENO-Z + Godunov + SSP-RK3 only
    dissipates, and only a little for a well-resolved pulse."""
    sc = scenes.box_room((40, 40, 40), 0.05)
    m = mats.pack([mats.rigid(0.99)] * 6)
    dt = 0.5 * 0.05 / 343.0
    o = orc.Oracle(sc.S, sc.oid, 0.05, 343.0, 1.2, dt, materials=m, max_steps=0)
    o.set_fields(p=scenes.gaussian_pulse(sc.shape, 0.05, (23, 23, 23), 2.5))
    E = [o.energy()]
    for _ in range(4):
        o.run(5)
        E.append(o.energy())
    assert all(np.diff(E) <= 1e-12 * E[0])
    assert E[-1] > 0.9 * E[0]


def test_matched_walls_absorb():
    """All walls matched (R = 0, the BoundingBox layer): the energy leaves the box."""
    sc = scenes.box_room((20, 18, 16), 0.05)
    m = mats.pack([mats.matched()] * 6)
    dt = 0.5 * 0.05 / 343.0
    o = orc.Oracle(sc.S, sc.oid, 0.05, 343.0, 1.2, dt, materials=m, max_steps=0)
    o.set_fields(p=scenes.gaussian_pulse(sc.shape, 0.05, (12, 11, 10), 2.0))
    E0 = o.energy()
    o.run(120)
    assert o.energy() < 1e-4 * E0


def test_linear_below_weno_eps_and_nonlinear_above():
    """WENO-Z weights (functions3D.cuh:839-844) are data dependent, so the solver is not linear in
    the source: doubling a 1 Pa pulse does not double the trace. For amplitudes whose smoothness
    indicators sit far below eps = 1e-10 the weights freeze at the linear ones and it is."""
    sc = scenes.box_room((22, 20, 18), 0.05)
    m = mats.pack([mats.rigid(0.95)] * 6)
    dt = 0.5 * 0.05 / 343.0
    def trace(amp):
        o = orc.Oracle(sc.S, sc.oid, 0.05, 343.0, 1.2, dt, materials=m, rec_cells=np.array([(16, 14, 13)]),
                       max_steps=60)
        o.set_fields(p=scenes.gaussian_pulse(sc.shape, 0.05, (9, 9, 9), 1.5, amplitude=amp))
        o.run(60)
        return o.ir()[0][0]
    lo1, lo2 = trace(1e-9), trace(2e-9)
    assert np.max(np.abs(lo2 - 2 * lo1)) < 1e-5 * np.max(np.abs(lo2))
    hi1, hi2 = trace(1.0), trace(2.0)
    assert np.max(np.abs(hi2 - 2 * hi1)) > 1e-4 * np.max(np.abs(hi2))
