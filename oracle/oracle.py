"""ctypes front end of the CPU oracle (oracle/fz_oracle.cpp) -- TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, always as the
checker or the timed CPU baseline, never as a product path.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


class OrcSetup(C.Structure):
    _fields_ = [
        ("Nx", C.c_int32), ("Ny", C.c_int32), ("Nz", C.c_int32),
        ("h", C.c_double), ("c", C.c_double), ("rho", C.c_double), ("dt", C.c_double),
        ("pml", C.c_int32 * 6), ("pml_cells", C.c_int32), ("tol", C.c_double),
        ("S", C.POINTER(C.c_float)), ("oid", C.POINTER(C.c_uint8)),
        ("nMat", C.c_int32), ("K", C.c_int32), ("L", C.c_int32),
        ("Rinf", C.POINTER(C.c_double)), ("A", C.POINTER(C.c_double)), ("zeta", C.POINTER(C.c_double)),
        ("B", C.POINTER(C.c_double)), ("C", C.POINTER(C.c_double)), ("alpha", C.POINTER(C.c_double)),
        ("beta", C.POINTER(C.c_double)),
        ("nsrc", C.c_int32), ("src_cell", C.POINTER(C.c_int64)), ("sval", C.POINTER(C.c_double)),
        ("src_opt", C.c_int32), ("src_freq", C.POINTER(C.c_double)), ("u_s", C.POINTER(C.c_double)),
        ("n_us", C.c_int64),
        ("nrec", C.c_int32), ("rec_cell", C.POINTER(C.c_int64)),
        ("max_steps", C.c_int64),
        ("two_d", C.c_int32),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _load():
    import importlib.util
    spec = importlib.util.spec_from_file_location("oracle_build", os.path.join(HERE, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    path = mod.build()
    L = C.CDLL(path)
    L.orc_create.restype = C.c_void_p
    L.orc_create.argtypes = [C.POINTER(OrcSetup)]
    L.orc_set_fields.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 4
    L.orc_run.argtypes = [C.c_void_p, C.c_int64, C.c_int32]
    L.orc_get_ir.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.orc_get_fields.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 4
    L.orc_energy.restype = C.c_double
    L.orc_energy.argtypes = [C.c_void_p]
    L.orc_n_band.restype = C.c_int64
    L.orc_n_band.argtypes = [C.c_void_p]
    L.orc_destroy.argtypes = [C.c_void_p]
    L.orc_ade_drive.argtypes = [C.c_int32, C.c_int32, C.c_double] + [C.POINTER(C.c_double)] * 6 + \
        [C.c_double, C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.orc_waveform.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_int64, C.c_double,
                               C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.orc_l2d_run.argtypes = [C.c_int32, C.c_int32, C.c_int32] + [C.c_double] * 6 + \
        [C.POINTER(C.c_int32), C.POINTER(C.c_float), C.POINTER(C.c_uint8), C.c_int32, C.c_int32, C.c_int32] + \
        [C.POINTER(C.c_double)] * 10 + [C.c_int32, C.c_int32, C.c_int64] + [C.POINTER(C.c_double)] * 4
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


class Oracle:
    """FP64 CPU restatement of the reference solver on one scene (reference array layout)."""

    def __init__(self, S, oid, h, c, rho, dt, pml=(0,) * 6, pml_cells=20, tol_cells=3.0, materials=None,
                 src_cells=None, sval=None, src_opt=0, src_freq=None, u_s=None, rec_cells=None, max_steps=0,
                 two_d=False):
        L = lib()
        self._keep = []
        S = np.ascontiguousarray(S, np.float32)
        oid = np.ascontiguousarray(oid, np.uint8)
        Nz, Ny, Nx = S.shape
        self.shape = S.shape
        st = OrcSetup()
        st.Nx, st.Ny, st.Nz = Nx, Ny, Nz
        st.h, st.c, st.rho, st.dt = h, c, rho, dt
        for f in range(6):
            st.pml[f] = int(bool(pml[f]))
        st.pml_cells = pml_cells
        st.tol = tol_cells * h
        st.S = S.ctypes.data_as(C.POINTER(C.c_float))
        st.oid = oid.ctypes.data_as(C.POINTER(C.c_uint8))
        self._keep += [S, oid]
        if materials is not None:
            arrs = {k: np.ascontiguousarray(materials[k], np.float64) for k in
                    ("Rinf", "A", "zeta", "B", "Cc", "alpha", "beta")}
            self._keep += list(arrs.values())
            st.nMat = arrs["Rinf"].size
            st.K = arrs["A"].shape[1] if arrs["A"].ndim == 2 else 0
            st.L = arrs["B"].shape[1] if arrs["B"].ndim == 2 else 0
            st.Rinf, st.A, st.zeta = _dp(arrs["Rinf"]), _dp(arrs["A"]), _dp(arrs["zeta"])
            st.B, st.C, st.alpha, st.beta = _dp(arrs["B"]), _dp(arrs["Cc"]), _dp(arrs["alpha"]), _dp(arrs["beta"])
        def flat(cells):
            cells = np.asarray(cells, np.int64).reshape(-1, 3)
            return np.ascontiguousarray(cells[:, 0] + Nx * (cells[:, 1] + Ny * cells[:, 2]), np.int64)
        if src_cells is not None and len(src_cells):
            sc = flat(src_cells)
            sv = np.ascontiguousarray(sval, np.float64)
            self._keep += [sc, sv]
            st.nsrc = sc.size
            st.src_cell = sc.ctypes.data_as(C.POINTER(C.c_int64))
            st.sval = _dp(sv)
            st.src_opt = src_opt
            if src_freq is not None:
                sf = np.ascontiguousarray(src_freq, np.float64)
                self._keep.append(sf)
                st.src_freq = _dp(sf)
            if u_s is not None:
                us = np.ascontiguousarray(u_s, np.float64)
                self._keep.append(us)
                st.u_s = _dp(us)
                st.n_us = us.size
        if rec_cells is not None and len(rec_cells):
            rc = flat(rec_cells)
            self._keep.append(rc)
            st.nrec = rc.size
            st.rec_cell = rc.ctypes.data_as(C.POINTER(C.c_int64))
        self.nrec = st.nrec
        st.max_steps = max_steps
        st.two_d = 1 if two_d else 0
        self.max_steps = max_steps
        self._h = L.orc_create(C.byref(st))
        if not self._h:
            raise ValueError("orc_create rejected the setup")
        self.steps = 0

    def set_fields(self, p=None, u=None, v=None, w=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (p, u, v, w)]
        lib().orc_set_fields(self._h, *[_dp(a) for a in arrs])

    def run(self, nsteps, threads=0):
        lib().orc_run(self._h, int(nsteps), int(threads))
        self.steps += int(nsteps)

    def ir(self):
        ir = np.zeros((self.nrec, max(self.max_steps, 1)))
        vel = np.zeros((self.nrec, max(self.max_steps, 1), 3))
        lib().orc_get_ir(self._h, _dp(ir), _dp(vel))
        n = min(self.steps, self.max_steps)
        return ir[:, :n], vel[:, :n]

    def fields(self):
        out = [np.zeros(self.shape) for _ in range(4)]
        lib().orc_get_fields(self._h, *[_dp(a) for a in out])
        return out

    def energy(self):
        return lib().orc_energy(self._h)

    def n_band(self):
        return lib().orc_n_band(self._h)

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ade_drive(m, dt, w_in):
    """Runs the ADE stage recursion for one material on inputs w_in[n, 3] (stage inputs)."""
    w = np.ascontiguousarray(w_in, np.float64).reshape(-1, 3)
    out = np.zeros_like(w)
    arr = [np.ascontiguousarray(x, np.float64) for x in (m.A, m.zeta, m.B, m.C, m.alpha, m.beta)]
    lib().orc_ade_drive(len(m.A), len(m.B), float(m.Rinf), *[_dp(a) for a in arr], float(dt), w.shape[0],
                        _dp(w), _dp(out))
    return out


def waveform(src_opt, glob_f, f_cutoff, dt, Nt, h, rho):
    n = 2 * int(Nt) + 1
    us = np.zeros(n)
    pr = np.zeros(n)
    pk = C.c_double()
    lib().orc_waveform(int(src_opt), float(glob_f), float(f_cutoff), float(dt), int(Nt), float(h), float(rho),
                       _dp(us), _dp(pr), C.byref(pk))
    return us, pr, pk.value


def legacy2d_run(S, oid, h, dt, rho, c, eps, tol, pml, mats, p0, u0, v0, rec, nsteps, use_float=False):
    """The reference 2D legacy solver restated (oracle/fz_legacy2d_oracle.cpp): nsteps steps from
    the fields p0, u0, v0 (Ny x Nx arrays, None = zeros) on the node grid of S / oid; pml = the
    sPML keys (N, S, E, W). mats holds Rinf (nmat), A, zeta (nmat x K), B, C, alpha, beta
    (nmat x L). Returns the receiver trace at rec = (i, j) and the final p, u, v."""
    S = np.ascontiguousarray(S, np.float32)
    oid = np.ascontiguousarray(oid, np.uint8)
    Ny, Nx = S.shape
    pml4 = (C.c_int32 * 4)(*[int(x) for x in pml])
    Rinf = np.ascontiguousarray(mats["Rinf"], np.float64)
    nmat = len(Rinf)
    A = np.ascontiguousarray(mats["A"], np.float64).reshape(nmat, -1)
    B = np.ascontiguousarray(mats["B"], np.float64).reshape(nmat, -1)
    K, L = A.shape[1], B.shape[1]
    arr = [Rinf, A, np.ascontiguousarray(mats["zeta"], np.float64).reshape(nmat, K), B,
           np.ascontiguousarray(mats["C"], np.float64).reshape(nmat, L),
           np.ascontiguousarray(mats["alpha"], np.float64).reshape(nmat, L),
           np.ascontiguousarray(mats["beta"], np.float64).reshape(nmat, L)]
    f0 = [None if f is None else np.ascontiguousarray(f, np.float64).reshape(Ny, Nx) for f in (p0, u0, v0)]
    ir = np.zeros(max(nsteps, 1))
    out = [np.zeros((Ny, Nx)) for _ in range(3)]
    rc = lib().orc_l2d_run(int(use_float), Nx, Ny, h, dt, rho, c, eps, tol, pml4,
                           S.ctypes.data_as(C.POINTER(C.c_float)), oid.ctypes.data_as(C.POINTER(C.c_uint8)),
                           nmat, K, L, *[_dp(a) for a in arr], *[_dp(f) for f in f0], int(rec[0]), int(rec[1]),
                           nsteps, _dp(ir), *[_dp(o) for o in out])
    if rc != 0:
        raise ValueError("orc_l2d_run: bad arguments")
    return ir[:nsteps], out
