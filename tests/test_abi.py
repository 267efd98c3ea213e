"""The C ABI library loads and exports every function include/fz.h and include/fz_legacy2d.h declare
(no GPU needed)."""
import ctypes
import os
import re

import numpy as np

from fases_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for hdr in ("fz.h", "fz_legacy2d.h"):
        src = open(os.path.join(ROOT, "include", hdr)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(fz_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    L = ctypes.CDLL(_abi.LIB_PATH)
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_table_covers_header():
    assert set(_declared()) == set(_abi.SIGNATURES)


def test_params_struct_layout_matches_header():
    p = _abi.FzParams()
    assert _abi.lib().fz_params_init(ctypes.byref(p)) == 0
    assert p.abi_version == 2 and p.pml_cells == 20 and abs(p.tol_cells - 3.0) < 1e-15
    # c at 20 degC in the reference's float arithmetic (main3D.cu:450-456)
    T = np.float32(20.0) + np.float32(273.15)
    c = np.sqrt(np.float32(1.4) * np.float32(287.05) * T, dtype=np.float32)
    assert p.c == float(c)
    assert p.rho == float(np.float32(1.225))


def test_create_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        return
    p = _abi.FzParams()
    _abi.lib().fz_params_init(ctypes.byref(p))
    h = ctypes.c_void_p()
    rc = _abi.lib().fz_create(ctypes.byref(p), ctypes.byref(h))
    assert rc == _abi.FZ_ENODEV
    assert not h.value
    assert "CUDA" in _abi.last_error() or "device" in _abi.last_error()


def test_invalid_params_rejected():
    p = _abi.FzParams()
    _abi.lib().fz_params_init(ctypes.byref(p))
    p.h = -1.0
    h = ctypes.c_void_p()
    assert _abi.lib().fz_create(ctypes.byref(p), ctypes.byref(h)) == _abi.FZ_EINVAL
    p.h = 0.02
    p.abi_version = 99
    assert _abi.lib().fz_create(ctypes.byref(p), ctypes.byref(h)) == _abi.FZ_EINVAL


def test_null_handle_calls_are_errors():
    L = _abi.lib()
    assert L.fz_run(None, 1) == _abi.FZ_EINVAL
    assert L.fz_sync(None, 1) == _abi.FZ_EINVAL
    assert L.fz_energy(None, None) == _abi.FZ_EINVAL
    L.fz_destroy(None)


def test_legacy2d_params_and_errors_without_gpu():
    import torch
    L = _abi.lib()
    p = _abi.FzL2dParams()
    L.fz_l2d_params_init(ctypes.byref(p))
    # the reference's float set-up at 22 degC, C_CFL 0.2 (2D-solver/core/main.cu:82, 378-392, 591)
    f32 = np.float32
    c = np.sqrt(f32(1.4) * f32(287.05) * (f32(22.0) + f32(273.15)), dtype=f32)
    assert p.c == float(c) and p.h == float(f32(0.005)) and p.dt == float(f32(0.2) * f32(0.005) / c)
    assert p.tol == float(f32(3.0) * f32(0.005)) and p.eps == float(f32(1e-7))
    assert (p.pml_n, p.pml_s, p.pml_e, p.pml_w) == (1, 1, 0, 0) and p.Nx == 0
    h = ctypes.c_void_p()
    assert L.fz_l2d_create(ctypes.byref(p), ctypes.byref(h)) == _abi.FZ_EINVAL  # grid not set
    p.Nx, p.Ny = 40, 30
    if not torch.cuda.is_available():
        assert L.fz_l2d_create(ctypes.byref(p), ctypes.byref(h)) == _abi.FZ_ENODEV
        assert not h.value
    assert L.fz_l2d_run(None, 1) == _abi.FZ_EINVAL
    assert L.fz_l2d_destroy(None) == _abi.FZ_EINVAL
    assert L.fz_l2d_step_count(None) == -1
