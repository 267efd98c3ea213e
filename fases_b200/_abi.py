"""ctypes binding of libfz.so (include/fz.h).

The library is loaded from this package directory. There is no fallback: if libfz.so is missing
or does not load, importing the solver raises, so a machine without the CUDA build fails loudly
instead of silently running something else.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# FZ_BOUNDS_CHECK=1 loads the bounds-checked build (every computed index of the stepping kernels
# checked against its array; an out-of-range one sets an error bit and is skipped)
LIB_PATH = os.path.join(HERE, "libfz_checked.so" if os.environ.get("FZ_BOUNDS_CHECK") == "1" else "libfz.so")
# FZ_WAIT_TEST=1 loads the wait-test build (bounded waits of about a millisecond and the test hook
# fz_test_skip_plane); only the bounded-wait tests use it
if os.environ.get("FZ_WAIT_TEST") == "1":
    LIB_PATH = os.path.join(HERE, "libfz_waittest.so")
# FZ_LIB=<path> loads another build of the same sources (a kernel variant being measured)
if os.environ.get("FZ_LIB"):
    LIB_PATH = os.path.abspath(os.environ["FZ_LIB"])

FZ_OK = 0
FZ_EINVAL = -1
FZ_ENOMEM = -2
FZ_ECUDA = -3
FZ_EIO = -4
FZ_EPARSE = -5
FZ_ESTATE = -6
FZ_ETIMEOUT = -7
FZ_ENONFINITE = -8
FZ_ENODEV = -9
FZ_EBOUNDS = -10
FZ_FP32 = 0
FZ_FP64 = 1
FZ_SRC_PCS = 0
FZ_SRC_RICKER = 1
FZ_SRC_SINE = 2
FZ_NOALLOC_MAX_BLOCKS = 4096
FZ_NOALLOC_MAX_CELLS = 4096 * 16384

ERROR_NAMES = {
    FZ_EINVAL: "FZ_EINVAL", FZ_ENOMEM: "FZ_ENOMEM", FZ_ECUDA: "FZ_ECUDA", FZ_EIO: "FZ_EIO",
    FZ_EPARSE: "FZ_EPARSE", FZ_ESTATE: "FZ_ESTATE", FZ_ETIMEOUT: "FZ_ETIMEOUT",
    FZ_ENONFINITE: "FZ_ENONFINITE", FZ_ENODEV: "FZ_ENODEV", FZ_EBOUNDS: "FZ_EBOUNDS",
}


class FzParams(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32),
        ("precision", C.c_int32),
        ("device", C.c_int32),
        ("pml_cells", C.c_int32),
        ("pml", C.c_int32 * 6),
        ("h", C.c_double),
        ("c", C.c_double),
        ("rho", C.c_double),
        ("dt", C.c_double),
        ("tol_cells", C.c_double),
        ("two_d", C.c_int32),
        ("batch", C.c_int32),
        ("pml_R0", C.c_double),
        ("pml_kappa_max", C.c_double),
        ("pml_alpha_max", C.c_double),
        ("pml_order", C.c_double),
    ]


class FzGradients(C.Structure):
    _fields_ = [
        ("cotangent", C.c_int32),
        ("materials", C.POINTER(C.c_double)),
        ("materials_cap", C.c_int64),
        ("source_sval", C.POINTER(C.c_double)),
        ("source_sval_cap", C.c_int64),
        ("source_wave", C.POINTER(C.c_double)),
        ("source_wave_cap", C.c_int64),
        ("pml", C.POINTER(C.c_double)),
        ("pml_cap", C.c_int64),
        ("initial", C.POINTER(C.c_double)),
        ("initial_cap", C.c_int64),
    ]


# int (*fz_progress_fn)(int64_t done, int64_t total, void* user)
PROGRESS_FN = C.CFUNCTYPE(C.c_int, C.c_int64, C.c_int64, C.c_void_p)


class FzL2dParams(C.Structure):
    """fz_l2d_params of include/fz_legacy2d.h."""
    _fields_ = [
        ("Nx", C.c_int32), ("Ny", C.c_int32),
        ("h", C.c_double), ("dt", C.c_double), ("rho", C.c_double), ("c", C.c_double),
        ("eps", C.c_double), ("tol", C.c_double),
        ("pml_n", C.c_int32), ("pml_s", C.c_int32), ("pml_e", C.c_int32), ("pml_w", C.c_int32),
        ("precision", C.c_int32), ("device", C.c_int32),
    ]


class FzError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


_P = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_i64p = C.POINTER(C.c_int64)
_u8p = C.POINTER(C.c_uint8)

# name -> (restype, argtypes); the exported surface of include/fz.h and include/fz_legacy2d.h
SIGNATURES = {
    "fz_params_init": (C.c_int, [C.POINTER(FzParams)]),
    "fz_create": (C.c_int, [C.POINTER(FzParams), C.POINTER(_P)]),
    "fz_destroy": (None, [_P]),
    "fz_load_geometry_raw": (C.c_int, [_P, _fp, _u8p, _i32, _i32, _i32]),
    "fz_device_memory": (C.c_int, [_i32, _i64p, _i64p]),
    "fz_scene_dims": (C.c_int, [C.c_char_p, C.c_double, _ip, _dp]),
    "fz_build_scene": (C.c_int, [C.c_char_p, C.c_double, C.c_double, _i32, _fp, _u8p, _i64]),
    "fz_set_materials": (C.c_int, [_P, _i32, _i32, _i32, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    "fz_set_sources": (C.c_int, [_P, _i32, _ip, _dp, _i32, _dp, _dp, _i64]),
    "fz_set_source_members": (C.c_int, [_P, _i32, _ip]),
    "fz_set_receivers": (C.c_int, [_P, _i32, _ip, _i64]),
    "fz_set_slices": (C.c_int, [_P, _i32, _i32, _i32, _i64, _i64]),
    "fz_get_slices": (C.c_int, [_P, _fp, _i64, _i64p]),
    "fz_set_fields": (C.c_int, [_P, _dp, _dp, _dp, _dp]),
    "fz_run": (C.c_int, [_P, _i64]),
    "fz_run_timed": (C.c_int, [_P, _i64, _dp]),
    "fz_prepare": (C.c_int, [_P]),
    "fz_run_progress": (C.c_int, [_P, _i64, _i32, C.c_void_p, C.c_void_p]),
    "fz_sync": (C.c_int, [_P, _i64]),
    "fz_steps_done": (C.c_int, [_P, _i64p]),
    "fz_check_health": (C.c_int, [_P, _i64p]),
    "fz_state_bytes": (C.c_int, [_P, _i64p]),
    "fz_state_save": (C.c_int, [_P, _P, _i64]),
    "fz_state_load": (C.c_int, [_P, _P, _i64]),
    "fz_misfit_gradient": (C.c_int, [_P, _i64, _i32, _dp, _i64, _dp, _dp, _i64, _dp]),
    "fz_misfit_gradient_ex": (C.c_int, [_P, _i64, _i32, _dp, _i64, _dp, C.POINTER(FzGradients), _dp]),
    "fz_autotune": (C.c_int, [_P, _i32, _ip, _dp]),
    "fz_group_autotune": (C.c_int, [_P, _i32, _ip, _dp]),
    "fz_set_kz_chunk": (C.c_int, [_P, _i32]),
    "fz_get_kz_chunk": (C.c_int, [_P, _ip, _ip]),
    "fz_get_z_schedule": (C.c_int, [_P, _ip, _i32, _ip]),
    "fz_set_z_schedule": (C.c_int, [_P, _ip, _i32]),
    "fz_material_layout": (C.c_int, [_P, _ip, _ip, _ip]),
    "fz_group_create": (C.c_int, [C.POINTER(_P), _i32, C.POINTER(_P)]),
    "fz_group_run": (C.c_int, [_P, _i64]),
    "fz_group_run_timed": (C.c_int, [_P, _i64, _dp]),
    "fz_group_sync": (C.c_int, [_P, _i64]),
    "fz_group_destroy": (None, [_P]),
    "fz_group_info": (C.c_int, [_P, _ip, _ip]),
    "fz_group_set_branches": (C.c_int, [_P, _i32]),
    "fz_get_ir": (C.c_int, [_P, _fp, _i64]),
    "fz_get_ir64": (C.c_int, [_P, _dp, _i64]),
    "fz_get_vel": (C.c_int, [_P, _fp, _i64]),
    "fz_get_fields": (C.c_int, [_P, _dp, _dp, _dp, _dp]),
    "fz_energy": (C.c_int, [_P, _dp]),
    "fz_write_outputs": (C.c_int, [_P, C.c_char_p, _i32, C.c_char_p]),
    "fz_info": (C.c_int, [_P, _ip, _i64p, _i64p]),
    "fz_profile_enable": (C.c_int, [_P, _i32]),
    "fz_profile_read": (C.c_int, [_P, _dp, _i64p, _i32]),
    "fz_load_project": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, _i32, _i32,
                                  C.POINTER(_P), _i64p]),
    "fz_source_waveform": (C.c_int, [_i32, C.c_double, C.c_double, C.c_double, _i64, C.c_double,
                                     C.c_double, _dp, _dp, _dp]),
    "fz_energy_noalloc": (C.c_int, [_P, _P, _P, _P, _i64, C.c_double, C.c_double, _P, _P]),
    "fz_last_error": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "fz_global_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    # include/fz_legacy2d.h
    "fz_l2d_params_init": (None, [C.POINTER(FzL2dParams)]),
    "fz_l2d_create": (C.c_int, [C.POINTER(FzL2dParams), C.POINTER(_P)]),
    "fz_l2d_destroy": (C.c_int, [_P]),
    "fz_l2d_load_geometry": (C.c_int, [_P, _fp, _u8p]),
    "fz_l2d_set_materials": (C.c_int, [_P, _i32, _i32, _i32, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    "fz_l2d_set_fields": (C.c_int, [_P, _dp, _dp, _dp]),
    "fz_l2d_set_receiver": (C.c_int, [_P, _i32, _i32, _i64]),
    "fz_l2d_run": (C.c_int, [_P, _i64]),
    "fz_l2d_run_timed": (C.c_int, [_P, _i64, _dp]),
    "fz_l2d_step_count": (C.c_int64, [_P]),
    "fz_l2d_samples": (C.c_int64, [_P]),
    "fz_l2d_get_ir": (C.c_int, [_P, _dp, _i64]),
    "fz_l2d_get_fields": (C.c_int, [_P, _dp, _dp, _dp]),
    "fz_l2d_band_cells": (C.c_int64, [_P]),
    "fz_l2d_last_error": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
}

_lib = None


def lib():
    """The loaded libfz.so (raises OSError if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"libfz.so not built at {LIB_PATH}: run fases_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error(handle=None) -> str:
    buf = C.create_string_buffer(4096)
    if handle:
        lib().fz_last_error(handle, buf, len(buf))
    else:
        lib().fz_global_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc, handle=None):
    if rc != FZ_OK:
        raise FzError(rc, last_error(handle))
    return rc
