"""Python mirror of the fases3D solver interface, on top of libfz.so.

`Solver` is the library form of one `fases3D` FVM run (3D-solver/core/main3D.cu:26-1449):
geometry (S, oid) -> materials -> sources -> receivers -> `run(nsteps)` -> receiver traces and the
reference output files. `Solver.from_project` takes the same four paths as the `fases3D` command
line and reads the reference's project files.
"""
import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import FzParams, check, lib


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def params(h=0.02, c=None, rho=None, dt=None, cfl=0.5, pml=(0, 0, 0, 0, 0, 0), pml_cells=20,
           precision="fp32", device=0, tol_cells=3.0, two_d=False, batch=1, pml_R0=None, pml_kappa_max=None,
           pml_alpha_max=None, pml_order=None):
    """Solver parameters. c/rho default to the reference's 20 degC air (main3D.cu:450-456);
    dt = cfl*h/c (main3D.cu:729-730). pml = (U, D, R, L, F, B) face keys (main3D.cu:155-160).
    batch > 1 steps that many independent field sets (one per source position) over the same
    room in the same launches. pml_R0 / pml_kappa_max / pml_alpha_max / pml_order override the
    reference's cPML profile constants (1e-7, 5, 20 pi, 2; functions3D.cuh:689-723)."""
    p = FzParams()
    check(lib().fz_params_init(C.byref(p)))
    p.precision = _abi.FZ_FP64 if precision == "fp64" else _abi.FZ_FP32
    p.device = int(device)
    p.pml_cells = int(pml_cells)
    for f in range(6):
        p.pml[f] = int(bool(pml[f]))
    p.h = float(h)
    if c is not None:
        p.c = float(c)
    if rho is not None:
        p.rho = float(rho)
    p.dt = float(dt) if dt is not None else float(cfl) * p.h / p.c
    p.tol_cells = float(tol_cells)
    p.two_d = 1 if two_d else 0
    p.batch = int(batch)
    for name, v in (("pml_R0", pml_R0), ("pml_kappa_max", pml_kappa_max), ("pml_alpha_max", pml_alpha_max),
                    ("pml_order", pml_order)):
        if v is not None:
            setattr(p, name, float(v))
    return p


class Solver:
    """One GPU solver instance (a libfz handle). Not thread-safe; one CUDA stream."""

    def __init__(self, prm: FzParams = None, _handle=None, **kw):
        self._h = None
        if _handle is not None:
            self._h = _handle
        else:
            prm = prm if prm is not None else params(**kw)
            h = C.c_void_p()
            check(lib().fz_create(C.byref(prm), C.byref(h)))
            self._h = h
        self.batch = max(1, int(prm.batch)) if prm is not None else 1
        self._nrec = 0
        self._cap = 0
        self._nsrc = 0
        self._n_us = 0
        self._src_opt = 0

    # -- lifetime --------------------------------------------------------------------------
    def close(self):
        if self._h:
            lib().fz_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _chk(self, rc):
        return check(rc, self._h)

    # -- setup -----------------------------------------------------------------------------
    def load_geometry(self, S, oid):
        """S: float32 [Nz,Ny,Nx] signed distance (air > 0); oid: uint8 [Nz,Ny,Nx] material id + 1
        (0xFF none) -- the reference's output/S.bin and output/oid.bin as 3-D arrays."""
        S = np.ascontiguousarray(S, dtype=np.float32)
        oid = np.ascontiguousarray(oid, dtype=np.uint8)
        if S.shape != oid.shape or S.ndim != 3:
            raise ValueError("S and oid must be 3-D arrays of the same shape [Nz, Ny, Nx]")
        Nz, Ny, Nx = S.shape
        self._chk(lib().fz_load_geometry_raw(
            self._h, S.ctypes.data_as(C.POINTER(C.c_float)), oid.ctypes.data_as(C.POINTER(C.c_uint8)),
            Nx, Ny, Nz))
        self.shape = (Nz, Ny, Nx)

    def set_materials(self, Rinf, A=None, zeta=None, B=None, Cc=None, alpha=None, beta=None):
        """Per material m: Rinf[m], real poles A/zeta[m, K], complex pairs B/C/alpha/beta[m, L]."""
        Rinf = np.ascontiguousarray(Rinf, dtype=np.float64).reshape(-1)
        n = Rinf.size
        def arr(x):
            if x is None:
                return np.zeros((n, 0))
            return np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(n, -1))
        A, zeta, B, Cc, alpha, beta = map(arr, (A, zeta, B, Cc, alpha, beta))
        K, L = A.shape[1], B.shape[1]
        self._chk(lib().fz_set_materials(self._h, n, K, L, _dptr(Rinf), _dptr(A), _dptr(zeta), _dptr(B),
                                         _dptr(Cc), _dptr(alpha), _dptr(beta)))

    def set_sources(self, cells, sval, src_opt=0, u_s=None, freq=None):
        cells = np.ascontiguousarray(cells, dtype=np.int32).reshape(-1, 3)
        sval = np.ascontiguousarray(sval, dtype=np.float64).reshape(-1)
        us = None if u_s is None else np.ascontiguousarray(u_s, dtype=np.float64)
        fr = None if freq is None else np.ascontiguousarray(freq, dtype=np.float64)
        self._chk(lib().fz_set_sources(self._h, cells.shape[0], cells.ctypes.data_as(C.POINTER(C.c_int32)),
                                       _dptr(sval), int(src_opt), _dptr(fr), _dptr(us),
                                       0 if us is None else us.size))
        self._nsrc = cells.shape[0]
        self._n_us = 0 if us is None else us.size
        self._src_opt = int(src_opt)

    def set_source_members(self, member):
        """Batched solves: the batch member (0 .. batch-1, or -1 for all) of each source of the last
        set_sources call."""
        member = np.ascontiguousarray(member, dtype=np.int32).reshape(-1)
        self._chk(lib().fz_set_source_members(self._h, member.size, member.ctypes.data_as(C.POINTER(C.c_int32))))

    def set_receivers(self, cells, capacity_steps):
        cells = np.ascontiguousarray(cells, dtype=np.int32).reshape(-1, 3)
        self._chk(lib().fz_set_receivers(self._h, cells.shape[0], cells.ctypes.data_as(C.POINTER(C.c_int32)),
                                         int(capacity_steps)))
        self._nrec = cells.shape[0]
        self._cap = int(capacity_steps)

    def set_slices(self, i0, j0, k0, anim_step, max_frames):
        """Animation slices on the planes x = i0, y = j0, z = k0 (cell indices) every anim_step steps."""
        self._chk(lib().fz_set_slices(self._h, int(i0), int(j0), int(k0), int(anim_step), int(max_frames)))

    def slices(self):
        """Frames taken so far: dict of pX [F, Nz, Ny], pY [F, Nz, Nx], pZ [F, Ny, Nx] and the in-plane
        unit energy-flow components IyX, IzX, IxY, IzY, IxZ, IyZ of the same shapes."""
        n = C.c_int64()
        self._chk(lib().fz_get_slices(self._h, None, 0, C.byref(n)))
        Nz, Ny, Nx = self.shape
        sizes = [Ny * Nz, Nx * Nz, Nx * Ny]
        per = 3 * sum(sizes)
        buf = np.zeros(n.value * per, np.float32)
        if n.value:
            self._chk(lib().fz_get_slices(self._h, buf.ctypes.data_as(C.POINTER(C.c_float)), buf.size, C.byref(n)))
        fr = buf.reshape(n.value, per)
        shapes = [(Nz, Ny), (Nz, Nx), (Ny, Nx)]
        out, o = {}, 0
        for name, q in (("pX", 0), ("pY", 1), ("pZ", 2)):
            out[name] = fr[:, o:o + sizes[q]].reshape((n.value,) + shapes[q])
            o += sizes[q]
        for name, q in (("IyX", 0), ("IzX", 0), ("IxY", 1), ("IzY", 1), ("IxZ", 2), ("IyZ", 2)):
            out[name] = fr[:, o:o + sizes[q]].reshape((n.value,) + shapes[q])
            o += sizes[q]
        return out

    def set_fields(self, p=None, u=None, v=None, w=None):
        """Arrays of shape [Nz, Ny, Nx] (or [batch, Nz, Ny, Nx] for batched solves)."""
        if self.batch > 1:
            n = self.batch * int(np.prod(self.shape))
            for a in (p, u, v, w):
                if a is not None and np.size(a) != n:
                    raise ValueError("batched set_fields needs arrays of shape [batch, Nz, Ny, Nx]")
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (p, u, v, w)]
        self._chk(lib().fz_set_fields(self._h, *[_dptr(a) for a in arrs]))

    # -- stepping --------------------------------------------------------------------------
    def run(self, nsteps, sync=True, timeout_ms=0):
        self._chk(lib().fz_run(self._h, int(nsteps)))
        if sync:
            self.sync(timeout_ms)

    def run_progress(self, nsteps, callback, every_percent=5):
        """Runs nsteps in slices of every_percent %, calling callback(done, total) after each slice
        (the reference's "NN%" protocol); a truthy return value stops the run."""
        def _cb(done, total, _user):
            return 1 if callback(done, total) else 0
        fn = _abi.PROGRESS_FN(_cb)
        self._chk(lib().fz_run_progress(self._h, int(nsteps), int(every_percent), C.cast(fn, C.c_void_p), None))

    def prepare(self):
        """Finalises the set-up and instantiates the step graphs, so the next run launches
        without capturing (call after autotune / set_z_schedule, which discard the graphs)."""
        self._chk(lib().fz_prepare(self._h))

    def run_timed(self, nsteps):
        """Runs nsteps and returns their device time in ms (CUDA events on the solver's stream)."""
        ms = C.c_double()
        self._chk(lib().fz_run_timed(self._h, int(nsteps), C.byref(ms)))
        return ms.value

    def sync(self, timeout_ms=0):
        self._chk(lib().fz_sync(self._h, int(timeout_ms)))

    def autotune(self, reps=3):
        """Times the stage kernels for the heuristic tile depth (z planes per CTA) and the
        alternatives worth trying, keeps the fastest and returns (depth, stage ms per step); the
        solve does not advance and its results do not depend on the depth."""
        k, ms = C.c_int32(), C.c_double()
        self._chk(lib().fz_autotune(self._h, int(reps), C.byref(k), C.byref(ms)))
        return k.value, ms.value

    def set_kz_chunk(self, depth):
        """Tile depth of the stage kernels (0 = the wave-filling heuristic), e.g. from a cache."""
        self._chk(lib().fz_set_kz_chunk(self._h, int(depth)))

    def z_schedule(self):
        """Lengths (planes) of the stage kernels' z chunks, longest first."""
        n = C.c_int32()
        self._chk(lib().fz_get_z_schedule(self._h, None, 0, C.byref(n)))
        out = (C.c_int32 * max(1, n.value))()
        self._chk(lib().fz_get_z_schedule(self._h, out, n.value, C.byref(n)))
        return [out[q] for q in range(n.value)]

    def set_z_schedule(self, sizes):
        """Sets the z chunk lengths directly (summing to the interior planes), e.g. from z_schedule."""
        arr = (C.c_int32 * len(sizes))(*[int(x) for x in sizes])
        self._chk(lib().fz_set_z_schedule(self._h, arr, len(sizes)))

    def kz_chunk(self):
        """(current tile depth, heuristic tile depth)."""
        k, hk = C.c_int32(), C.c_int32()
        self._chk(lib().fz_get_kz_chunk(self._h, C.byref(k), C.byref(hk)))
        return k.value, hk.value

    def save_state(self, path=None):
        """The solver's complete state (checkpoint) as a uint8 array, also written to `path` if given."""
        n = C.c_int64()
        self._chk(lib().fz_state_bytes(self._h, C.byref(n)))
        buf = np.empty(n.value, np.uint8)
        self._chk(lib().fz_state_save(self._h, buf.ctypes.data_as(C.c_void_p), buf.size))
        if path is not None:
            buf.tofile(path)
        return buf

    def load_state(self, state):
        """Resumes from a checkpoint of save_state (an array or a file path) taken by a solver set up
        the same way."""
        buf = np.fromfile(state, np.uint8) if isinstance(state, (str, os.PathLike)) else np.ascontiguousarray(state, np.uint8)
        self._chk(lib().fz_state_load(self._h, buf.ctypes.data_as(C.c_void_p), buf.size))

    def check_health(self):
        """Number of NaN/Inf values in the current state (raises FzError FZ_ENONFINITE if any)."""
        n = C.c_int64()
        self._chk(lib().fz_check_health(self._h, C.byref(n)))
        return n.value

    def steps_done(self):
        n = C.c_int64()
        self._chk(lib().fz_steps_done(self._h, C.byref(n)))
        return n.value

    # -- results ---------------------------------------------------------------------------
    def _nsamples(self):
        return min(self.steps_done(), self._cap)

    def _lead(self):
        return (self.batch,) if self.batch > 1 else ()

    def ir(self, fp64=True):
        """Receiver traces [n_rec, n_steps] ([batch, n_rec, n_steps] for batched solves)."""
        n = self._nsamples()
        shape = self._lead() + (self._nrec, n)
        if fp64:
            out = np.zeros(shape, np.float64)
            self._chk(lib().fz_get_ir64(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), out.size))
        else:
            out = np.zeros(shape, np.float32)
            self._chk(lib().fz_get_ir(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        return out

    def vel(self):
        n = self._nsamples()
        out = np.zeros(self._lead() + (self._nrec, n, 3), np.float32)
        self._chk(lib().fz_get_vel(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), out.size))
        return out

    def fields(self):
        """(p, u, v, w), each [Nz, Ny, Nx] ([batch, Nz, Ny, Nx] for batched solves)."""
        out = [np.zeros(self._lead() + tuple(self.shape), np.float64) for _ in range(4)]
        self._chk(lib().fz_get_fields(self._h, *[_dptr(a) for a in out]))
        return out

    def material_layout(self):
        """(nMat, K, L) of the material table after setup (K, L >= 1, zero-padded)."""
        n, k, l = C.c_int32(), C.c_int32(), C.c_int32()
        self._chk(lib().fz_material_layout(self._h, C.byref(n), C.byref(k), C.byref(l)))
        return n.value, k.value, l.value

    def misfit_gradient(self, target, nsteps=None, segment_steps=250, sources=False, pml=False, initial=False,
                        cotangent=False):
        """J = sum (IR - target)^2 over nsteps steps from the current (step-0) state and its gradient
        by the discrete adjoint; with cotangent=True, `target` is a cotangent g of the traces, J =
        sum g IR and the gradients are the vector-Jacobian products sum g dIR/dtheta. target:
        [n_rec, >= nsteps]. Returns a dict with J, the ADE-coefficient gradient split per coefficient
        (arrays [nMat], [nMat, K] or [nMat, L]) and as the raw [nMat, 1 + 2K + 4L] array, the
        forward / backward device times in ms, and on request: sources -> "sval" [nsrc] (dJ/dsval)
        and "wave" [nsrc, n_us] (dJ/du_s per source, PCS / Ricker waveforms); pml -> "pml" {R0,
        kappa_max, alpha_max}; initial -> "initial" (p, u, v, w) gradients, each [Nz, Ny, Nx]."""
        target = np.ascontiguousarray(target, dtype=np.float64)
        if target.ndim != 2 or target.shape[0] != self._nrec:
            raise ValueError("target must be [n_rec, n_steps]")
        nsteps = target.shape[1] if nsteps is None else int(nsteps)
        nm, K, L = self.material_layout()
        P = 1 + 2 * K + 4 * L
        grad = np.zeros((nm, P), np.float64)
        J = C.c_double()
        ms = (C.c_double * 2)()
        g = _abi.FzGradients()
        g.cotangent = 1 if cotangent else 0
        g.materials, g.materials_cap = _dptr(grad), grad.size
        keep = {}
        if sources:
            n_us = 0 if self._src_opt == 2 else self._n_us
            keep["sval"] = np.zeros(self._nsrc, np.float64)
            keep["wave"] = np.zeros((self._nsrc, n_us), np.float64)
            g.source_sval, g.source_sval_cap = _dptr(keep["sval"]), keep["sval"].size
            g.source_wave, g.source_wave_cap = _dptr(keep["wave"]), keep["wave"].size
        if pml:
            keep["pml"] = np.zeros(4, np.float64)
            g.pml, g.pml_cap = _dptr(keep["pml"]), 4
        if initial:
            keep["initial"] = np.zeros((4,) + tuple(self.shape), np.float64)
            g.initial, g.initial_cap = _dptr(keep["initial"]), keep["initial"].size
        self._chk(lib().fz_misfit_gradient_ex(self._h, nsteps, int(segment_steps), _dptr(target), target.shape[1],
                                              C.byref(J), C.byref(g), ms))
        o = 1 + 2 * K
        out = {"J": J.value, "raw": grad, "Rinf": grad[:, 0], "A": grad[:, 1:1 + K], "zeta": grad[:, 1 + K:o],
               "B": grad[:, o:o + L], "C": grad[:, o + L:o + 2 * L], "alpha": grad[:, o + 2 * L:o + 3 * L],
               "beta": grad[:, o + 3 * L:o + 4 * L], "forward_ms": ms[0], "backward_ms": ms[1]}
        if sources:
            out["sval"], out["wave"] = keep["sval"], keep["wave"]
        if pml:
            out["pml"] = {"R0": keep["pml"][0], "kappa_max": keep["pml"][1], "alpha_max": keep["pml"][2]}
        if initial:
            out["initial"] = tuple(keep["initial"][f] for f in range(4))
        return out

    def energy(self):
        e = C.c_double()
        self._chk(lib().fz_energy(self._h, C.byref(e)))
        return e.value

    def info(self):
        dims = (C.c_int32 * 3)()
        nb, nu = C.c_int64(), C.c_int64()
        self._chk(lib().fz_info(self._h, dims, C.byref(nb), C.byref(nu)))
        return {"dims": tuple(dims), "n_band": nb.value, "n_update": nu.value}

    def profile(self, on=True):
        self._chk(lib().fz_profile_enable(self._h, 1 if on else 0))

    def profile_read(self):
        ms = (C.c_double * 8)()
        n = (C.c_int64 * 8)()
        self._chk(lib().fz_profile_read(self._h, ms, n, 8))
        kinds = ["stage0", "stage1", "stage2", "band", "receivers"]
        return {k: (ms[i], n[i]) for i, k in enumerate(kinds)}

    def write_outputs(self, output_dir, src_idx=0, scene_name="scene"):
        os.makedirs(output_dir, exist_ok=True)
        self._chk(lib().fz_write_outputs(self._h, output_dir.encode(), int(src_idx), scene_name.encode()))

    # -- whole reference project -----------------------------------------------------------
    @classmethod
    def from_project(cls, scene, config, src, rec, precision="fp32", device=0):
        """Same four inputs as `fases3D <scene.obj> <config.txt> <src.txt> <rec.txt>`; returns
        (solver, Nt)."""
        h = C.c_void_p()
        nt = C.c_int64()
        rc = lib().fz_load_project(os.fsencode(scene), os.fsencode(config), os.fsencode(src), os.fsencode(rec),
                                   _abi.FZ_FP64 if precision == "fp64" else _abi.FZ_FP32, int(device),
                                   C.byref(h), C.byref(nt))
        check(rc)
        s = cls(_handle=h)
        # receivers were set by the loader with capacity Nt
        s._cap = nt.value
        info = s.info()
        s.shape = tuple(reversed(info["dims"]))
        s._nrec = _count_rec(rec)
        return s, nt.value


class Group:
    """Several solvers (rooms) on one device advanced together. 3D rooms of one precision without
    animation slices (up to 64) share their launches (per stage one band launch for all and one
    stage launch per 28 rooms); other groups run each member's launches as parallel graph branches. Runs of 10 steps are CUDA
    graphs. The members stay usable alone and must outlive the group."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s._h.value if isinstance(s._h, C.c_void_p) else s._h
                                                 for s in self.solvers])
        g = C.c_void_p()
        check(lib().fz_group_create(arr, len(self.solvers), C.byref(g)))
        self._g = g

    def shared_launches(self):
        """True when the members share their launches."""
        v, b = C.c_int32(), C.c_int32()
        check(lib().fz_group_info(self._g, C.byref(v), C.byref(b)))
        return bool(v.value)

    def branches(self):
        """Concurrent branches the group's launches run as."""
        v, b = C.c_int32(), C.c_int32()
        check(lib().fz_group_info(self._g, C.byref(v), C.byref(b)))
        return b.value

    def set_branches(self, n):
        """Launch arrangement: n >= 1 shared launches in n concurrent branches, -1 each member's own
        launches as graph branches, 0 the default."""
        check(lib().fz_group_set_branches(self._g, int(n)))

    def run(self, nsteps, sync=True, timeout_ms=0):
        check(lib().fz_group_run(self._g, int(nsteps)))
        if sync:
            self.sync(timeout_ms)

    def run_timed(self, nsteps):
        ms = C.c_double()
        check(lib().fz_group_run_timed(self._g, int(nsteps), C.byref(ms)))
        return ms.value

    def autotune(self, reps=3):
        """One tile depth for every member and the launch arrangement (shared launches in 1, 2, 4
        or 8 branches, or each member's own launches), timed on the stage kernels; keeps the
        fastest and returns (depth, stage ms per step of the group)."""
        k, ms = C.c_int32(), C.c_double()
        check(lib().fz_group_autotune(self._g, int(reps), C.byref(k), C.byref(ms)))
        return k.value, ms.value

    def sync(self, timeout_ms=0):
        check(lib().fz_group_sync(self._g, int(timeout_ms)))

    def close(self):
        if self._g:
            lib().fz_group_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def _count_rec(path):
    n = 0
    with open(path) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            parts = line.split()
            try:
                [float(x) for x in parts[:3]]
            except ValueError:
                continue
            if len(parts) >= 3:
                n += 1
    return n


def source_waveform(src_opt, glob_f, f_cutoff, dt, Nt, h, rho):
    """(u_s, p_ref, p_peak) of main3D.cu:963-1110, 2*Nt+1 samples at dt/2."""
    n = 2 * int(Nt) + 1
    us = np.zeros(n)
    pr = np.zeros(n)
    pk = C.c_double()
    check(lib().fz_source_waveform(int(src_opt), float(glob_f), float(f_cutoff), float(dt), int(Nt), float(h),
                                   float(rho), _dptr(us), _dptr(pr), C.byref(pk)))
    return us, pr, pk.value
