"""Animation slices (fz_set_slices / fz_get_slices / fz_write_outputs): the frames taken every
anim_step steps inside the CUDA graphs equal the planes of the fields read back after the same
step, with the unit energy-flow components sign(p) u / |u| (main3D.cu:1326-1394)."""
import os

import numpy as np
import pytest

from tests.helpers import run_gpu, small_room


def test_slice_entry_points_check_arguments():
    from fases_b200 import _abi
    L = _abi.lib()
    assert L.fz_set_slices(None, 1, 1, 1, 2, 4) == _abi.FZ_EINVAL
    assert L.fz_get_slices(None, None, 0, None) == _abi.FZ_EINVAL


@pytest.mark.gpu
def test_slice_frames_equal_fields(tmp_path):
    cfg = small_room(seed=51, steps=25)
    i0, j0, k0, step = 10, 7, 12, 4
    s = run_gpu(cfg, "fp32", run=False)
    s.set_slices(i0, j0, k0, step, 10)
    s.run(25)
    fr = s.slices()
    assert fr["pX"].shape[0] == 7  # after steps 1, 5, ..., 25
    ref = run_gpu(cfg, "fp32", run=False)
    done = 0
    for q in range(7):
        n = q * step + 1
        ref.run(n - done)
        done = n
        p, u, v, w = [a.astype(np.float32) for a in ref.fields()]
        np.testing.assert_array_equal(fr["pX"][q], p[:, :, i0])
        np.testing.assert_array_equal(fr["pY"][q], p[:, j0, :])
        np.testing.assert_array_equal(fr["pZ"][q], p[k0, :, :])
        sp = np.where(p >= 0, np.float32(1), np.float32(-1))
        inv = sp / (np.sqrt(u * u + v * v + w * w) + np.float32(1e-20))
        np.testing.assert_allclose(fr["IyX"][q], (v * inv)[:, :, i0], rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(fr["IzY"][q], (w * inv)[:, j0, :], rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(fr["IxZ"][q], (u * inv)[k0, :, :], rtol=1e-6, atol=1e-7)
    out = str(tmp_path / "out")
    s.write_outputs(out, 0, "scene.obj")
    Nz, Ny, Nx = s.shape
    assert os.path.getsize(os.path.join(out, "pressureX.bin")) == 7 * Ny * Nz * 4
    assert os.path.getsize(os.path.join(out, "Iy_Z.bin")) == 7 * Nx * Ny * 4
    hdr = open(os.path.join(out, "header.txt")).read().split()
    assert hdr[7] == "7" and hdr[8] == str(step)
    s.close()
    ref.close()
