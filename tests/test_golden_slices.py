"""Animation slices pinned to the reference solver's own files.

tests/golden/box_slices is a reference project whose config asks for animation frames on the
planes through (0.5, 0.45, 0.35) m (config lines 19-22); its output/ holds the reference's
pressure{X,Y,Z}.bin and the in-plane energy-flow directions I{y,z}_X.bin, I{x,z}_Y.bin,
I{x,y}_Z.bin (3D-solver/core/main3D.cu:1326-1394), written by the reference solver built from its
own sources (tests/golden/make_golden.py). The stepper, driven through the project loader on the
same files, must write the same frames: the pressure planes to the receiver-trace tolerance, and
the unit directions sign(p) u/|u| where they are defined robustly (|u| and |p| well above their
rounding noise; elsewhere sign(p) and the direction flip with the noise).
"""
import os
import shutil

import numpy as np
import pytest


HERE = os.path.dirname(os.path.abspath(__file__))
CASE = os.path.join(HERE, "golden", "box_slices")
TOL_P = 2e-5


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.gpu
def test_slice_files_match_the_reference(tmp_path):
    if not os.path.isdir(CASE):
        pytest.skip("box_slices fixture not present")
    from fases_b200 import Solver
    proj = str(tmp_path / "box_slices")
    shutil.copytree(CASE, proj)
    args = (os.path.join(proj, "scene.obj"), os.path.join(proj, "config", "config.txt"),
            os.path.join(proj, "src.txt"), os.path.join(proj, "rec.txt"))
    Solver.from_project(*args)[0].close()  # restamps the scene cache, then the reference geometry goes back
    for f in ("S.bin", "oid.bin"):
        shutil.copyfile(os.path.join(CASE, "output", f), os.path.join(proj, "output", f))
    s, nt = Solver.from_project(*args)
    s.run(nt)
    out = os.path.join(proj, "fz_out")
    s.write_outputs(out, 0, "./scene.obj")
    Nz, Ny, Nx = s.shape
    s.close()
    hdr = open(os.path.join(out, "header.txt")).read().split()
    ref_hdr = open(os.path.join(CASE, "output", "header.txt")).read().split()
    assert hdr[7:9] == ref_hdr[7:9]  # frame count and anim_step
    nf = int(hdr[7])
    assert nf > 10
    planes = {"X": Ny * Nz, "Y": Nx * Nz, "Z": Nx * Ny}
    for ax, n in planes.items():
        a = np.fromfile(os.path.join(out, f"pressure{ax}.bin"), np.float32)
        b = np.fromfile(os.path.join(CASE, "output", f"pressure{ax}.bin"), np.float32)
        assert a.size == b.size == nf * n, (ax, a.size, b.size)
        assert _rel(a, b) < TOL_P, (ax, _rel(a, b))
        pa = np.abs(b).reshape(nf, n)
        for comp in {"X": "yz", "Y": "xz", "Z": "xy"}[ax]:
            ia = np.fromfile(os.path.join(out, f"I{comp}_{ax}.bin"), np.float32).reshape(nf, n)
            ib = np.fromfile(os.path.join(CASE, "output", f"I{comp}_{ax}.bin"), np.float32).reshape(nf, n)
            # well-defined directions: pressure above 1e-3 of the frame's peak
            ok = pa > 1e-3 * pa.max(axis=1, keepdims=True)
            assert ok.sum() > 100
            assert np.max(np.abs(ia[ok] - ib[ok])) < 1e-3, (ax, comp)
