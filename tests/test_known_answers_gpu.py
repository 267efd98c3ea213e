"""The reference's own validation procedures, run through the GPU stepper.

ADE wall reflection (3D-solver/tests/ADE_benchmark/ADE_TST_3D.py:166-221, configuration in
About.txt and config.txt there): a 2 x 8 x 2 m box at h = 0.034 m, source at (1, 1, 1) m, receiver
at (1, 7, 1) m, cPML on every face but the north wall (y = 8 m); three runs -- cPML on all faces
(the direct sound alone), a rigid north wall (R = 0.999 at every frequency) and the north wall
made of the benchmark's fitted material (sample.fit, 2 real poles and 3 complex pairs). The direct
sound is subtracted from both wall runs, and the ratio of their spectra is the numerical
reflection coefficient, compared with the analytical rational R(w) of the fit below the
benchmark's f_cutoff (1000 Hz). The reference's own run of this procedure stays within 0.26 dB
(its impedance_error.png).

Room modes (3D-solver/tests/Room_Modes_benchmark/validate_modes.py:161-176, README.txt there): a
5.5 x 4.0 x 2.8 m shoebox, absorption 0.05 on every surface, source (1, 1, 1) m, 1.9 s; the
spectrum of the receiver trace has its peaks at the room's modal frequencies
f_lmn = c/2 sqrt((l/Lx)^2 + (m/Ly)^2 + (n/Lz)^2), of the effective room -- the reference's
script shrinks each edge by 6h (3h per face: the immersed wall sits inside its blending band).
"""
import itertools

import numpy as np
import pytest

from tests.test_oracle_known_answers import _sample_fit

H = 0.034


def _run(room, walls, pml, src, recs, nt, pml_cells=20):
    from fases_b200 import Solver, materials as mats, params, scenes
    from fases_b200.solver import source_waveform
    prm = params(h=H, pml=pml, pml_cells=pml_cells)
    sc = scenes.box_room(room, H)
    m = mats.pack(walls)
    s = Solver(prm)
    s.load_geometry(sc.S, sc.oid)
    s.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    us, _, pk = source_waveform(0, 25.0, 2000.0, prm.dt, nt + 2, H, prm.rho)
    s.set_sources(np.array([src], np.int32), np.array([1.0 / pk]), 0, u_s=us)
    s.set_receivers(np.array(recs, np.int32), nt)
    s.run(nt)
    ir = s.ir()
    s.close()
    return ir, prm.dt, prm.c


def _cell(x):
    return int(x / H) + 3  # main3D.cu:874-876, 938-940


def R_model(w, m):
    s = 1j * np.asarray(w, float)
    R = np.full(s.shape, m.Rinf + 0j)
    for A, z in zip(m.A, m.zeta):
        R += A / (z + s)
    for B, C, a, b in zip(m.B, m.C, m.alpha, m.beta):
        R += (B * s + C * b + a * B) / ((a + s) ** 2 + b ** 2)
    return R


@pytest.mark.gpu
def test_ade_wall_reflection_matches_the_fitted_model():
    from fases_b200 import materials as mats
    room = (round(2.0 / H), round(8.0 / H), round(2.0 / H))
    M = mats.matched
    src, rec = (_cell(1.0), _cell(1.0), _cell(1.0)), [(_cell(1.0), _cell(7.0), _cell(1.0))]
    probe = (1, 1, 1, 1, 0, 1)  # cPML faces U D R L F B: every face but the north wall (F)
    nt = int(0.15 / (0.5 * H / 343.2)) + 1
    sample = _sample_fit()
    p_d, dt, _ = _run(room, [M()] * 6, (1,) * 6, src, rec, nt)
    p0, _, _ = _run(room, [M(), M(), M(), mats.rigid(0.999), M(), M()], probe, src, rec, nt)
    p1, _, _ = _run(room, [M(), M(), M(), sample, M(), M()], probe, src, rec, nt)
    p_f, p_r = p0[0] - p_d[0], p1[0] - p_d[0]
    Pf, Pr = np.fft.rfft(p_f), np.fft.rfft(p_r)
    f = np.fft.rfftfreq(p_r.size, d=dt)
    mask = (f >= 20.0) & (f <= 1000.0) & (np.abs(Pr) > 1e-6 * np.abs(Pr).max())
    assert mask.sum() > 100
    R_num = Pr[mask] / Pf[mask]
    R_ana = R_model(2 * np.pi * f[mask], sample) / 0.999  # the reference wall reflects 0.999
    err_db = 20 * np.log10(np.abs(R_ana) / np.abs(R_num))
    assert np.max(np.abs(err_db)) <= ERR_DB_MAX, float(np.max(np.abs(err_db)))
    # the phase follows the model as well
    dphi = np.angle(R_num / R_ana)
    assert np.max(np.abs(dphi)) <= PHASE_MAX, float(np.max(np.abs(dphi)))


@pytest.mark.gpu
def test_room_mode_peaks_sit_at_the_modal_frequencies():
    from fases_b200 import materials as mats
    room = (round(5.5 / H), round(4.0 / H), round(2.8 / H))
    R = float(np.sqrt(1.0 - 0.05))
    nt = int(1.9 / (0.5 * H / 343.2)) + 1
    src = (_cell(1.0), _cell(1.0), _cell(1.0))
    recs = [(_cell(2.0), _cell(3.0), _cell(1.5)), (_cell(3.3), _cell(2.3), _cell(0.92))]
    ir, dt, c = _run(room, [mats.rigid(R)] * 6, (0,) * 6, src, recs, nt)
    L = [n * H - 6 * H for n in room]  # the effective room: each wall 3h inside its face
    modes = sorted({(0.5 * c * np.sqrt(sum((q / Lq) ** 2 for q, Lq in zip(lmn, L))), lmn)
                    for lmn in itertools.product(range(4), repeat=3) if any(lmn)})
    modes = [m for m in modes if m[0] <= 100.0]
    checked = 0
    for r, rec in enumerate(recs):
        x = ir[r] - ir[r].mean()
        spec = np.abs(np.fft.rfft(x * np.hanning(x.size)))
        f = np.fft.rfftfreq(x.size, d=dt)
        # cell-centre positions in the effective room
        pos = [[(q - 3) * H + 0.5 * H - 3 * H for q in p] for p in (src, rec)]
        for fm, lmn in modes:
            # modes another mode crowds (within 4 %), and modes the source or the receiver sits
            # near a node of, give no clean peak
            if any(abs(f2 - fm) < 0.04 * fm for f2, l2 in modes if l2 != lmn):
                continue
            coupling = abs(np.prod([np.cos(q * np.pi * x_ / Lq) for q, x_, Lq in zip(lmn, pos[0], L)]) *
                           np.prod([np.cos(q * np.pi * x_ / Lq) for q, x_, Lq in zip(lmn, pos[1], L)]))
            if coupling < 0.15:
                continue
            band = (f > 0.97 * fm) & (f < 1.03 * fm)
            fpk = f[band][np.argmax(spec[band])]
            assert abs(fpk - fm) <= max(MODE_TOL * fm, f[1]), (r, lmn, fm, fpk)
            # the room without the inset would put this mode more than 2 % lower
            f_raw = 0.5 * c * np.sqrt(sum((q / (Lq + 6 * H)) ** 2 for q, Lq in zip(lmn, L)))
            assert abs(fpk - f_raw) > 2 * abs(fpk - fm)
            checked += 1
    assert checked >= 4


# |R_num / R_model| in dB and the phase of the ratio, 20 Hz to f_cutoff: the reference's own run
# of the procedure stays within 0.26 dB; this stepper measured 0.27 dB and 0.037 rad
ERR_DB_MAX = 0.35
PHASE_MAX = 0.06
# peak frequency against the effective room's modal frequency (measured: within 0.8 %)
MODE_TOL = 0.01
