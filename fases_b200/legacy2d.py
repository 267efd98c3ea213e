"""Host mirror of the 2D legacy solver of the reference (`2D-solver/`, executable `phases2D`) over
the C ABI of include/fz_legacy2d.h.

The reference's 2D solver is an interactive program (2D-solver/core/main.cu): it parses a 2D OBJ
scene into a node-based signed distance S and object ids oid (written to output/S.bin and
output/oid.bin), reads config.txt, poles.txt and one .fit file per layer, starts a raised-cosine
plane wave at the source's x, and appends the pressure at one receiver node to output/IR.bin
after every step. This module takes the same inputs as arrays:

    p = reference_setup("config/config.txt")            # h, dt, c, rho, sPML keys, Nt
    s = Legacy2D(Nx, Ny, **p["params"])
    s.load_geometry(S, oid)                             # output/S.bin, output/oid.bin
    s.set_materials(Rinf, A, zeta, B, C, alpha, beta)   # input/fit/<layer>.fit, zero-padded
    s.set_fields(*plane_wave_fields(Nx, Ny, h, src_x, rho, c))
    s.set_receiver(i_rec, j_rec, Nt)
    s.run(Nt)
    ir = s.ir()

Every call fails loudly (FzError) when the CUDA library or a GPU is missing; there is no CPU path.
"""
import ctypes as C

import numpy as np

from . import _abi
from ._abi import FzError

f32 = np.float32


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def reference_setup(config_path):
    """The scalar set-up of the reference 2D solver from its config.txt (2D-solver/core/main.cu:
    38-82, 378-404): grid spacing, time step, speed of sound, density, sPML keys and the number of
    steps, in the reference's float arithmetic."""
    vals = []
    for line in open(config_path):
        line = line.split("#", 1)[0].strip()
        try:
            vals.append(f32(float(line.split()[0])) if line else f32(0))
        except ValueError:
            vals.append(f32(0))
    h, t_max, temp, cfl = vals[0], vals[1], vals[3], vals[4]
    T = f32(temp + f32(273.15))
    c = np.sqrt(f32(1.4) * f32(287.05) * T, dtype=f32)
    dt = f32(cfl * h / c)
    nt = int(np.floor(f32(t_max / dt))) + 1
    return {"params": dict(h=float(h), dt=float(dt), c=float(c), rho=float(f32(1.225)), eps=float(f32(1e-7)),
                           tol=float(f32(3.0) * h), pml_n=int(vals[6]), pml_s=int(vals[7]), pml_e=int(vals[8]),
                           pml_w=int(vals[9])),
            "steps": nt, "f_cutoff": float(vals[2])}


def plane_wave_fields(Nx, Ny, h, src_x, rho, c, width=0.04, amp=0.1):
    """The reference's initial condition (2D-solver/core/main.cu:455-473, raised_cosine of
    functions.cuh:555-559): a right-going raised-cosine plane wave of full width `width` centred
    at x = src_x, p = amp g(x) and u = p / (rho c) at every node (x = (i + 1/2) h), v = 0; in
    float arithmetic as there. Returns (p, u, v) as (Ny, Nx) float64 arrays."""
    h, src_x, rho, c = f32(h), f32(src_x), f32(rho), f32(c)
    ww = f32(0.5) * f32(width)
    xx = (np.arange(Nx, dtype=f32) + f32(0.5)) * h
    xi = (xx - src_x) / ww
    g = np.where(np.abs(xi) > f32(1.0), f32(0.0), f32(0.5) * (f32(1.0) + np.cos(f32(np.pi) * xi, dtype=f32)))
    pI = (f32(amp) * g).astype(f32)
    uI = (pI / (rho * c)).astype(f32)
    p = np.broadcast_to(pI.astype(np.float64), (Ny, Nx)).copy()
    u = np.broadcast_to(uI.astype(np.float64), (Ny, Nx)).copy()
    return p, u, np.zeros((Ny, Nx))


def rect_scene(Nx, Ny, h, rects, tol_cells=3.0):
    """S and oid of rectangular obstacles on the node grid, by the conventions of the reference's
    2D scene builder (2D-solver/include/parsing.h:248-299, 418-466): nodes at (i h, j h), S > 0 in
    the fluid (the outer boundary polygon adds no distance; FLT_MAX with no obstacle), oid = the
    nearest obstacle's layer (1-based) at nodes 1..N-2 with 0 <= S <= tol and a nonzero
    central-difference gradient, 255 elsewhere. rects: [((x0, y0), (x1, y1), layer), ...]."""
    x = np.arange(Nx) * float(h)
    y = np.arange(Ny) * float(h)
    X, Y = np.meshgrid(x, y)
    S = np.full((Ny, Nx), float(np.finfo(np.float32).max))
    lay = np.zeros((Ny, Nx), np.int64)
    for (x0, y0), (x1, y1), layer in rects:
        cx, cy, hx, hy = (x0 + x1) / 2, (y0 + y1) / 2, (x1 - x0) / 2, (y1 - y0) / 2
        dx, dy = np.abs(X - cx) - hx, np.abs(Y - cy) - hy
        d = np.hypot(np.maximum(dx, 0), np.maximum(dy, 0)) + np.minimum(np.maximum(dx, dy), 0)
        lay = np.where(d < S, layer, lay)
        S = np.minimum(S, d)
    S = S.astype(np.float32)
    hf = f32(h)
    tol = f32(tol_cells) * hf
    oid = np.full((Ny, Nx), 255, np.uint8)
    core = S[1:-1, 1:-1]
    gx = f32(0.5) * (S[1:-1, 2:] - S[1:-1, :-2]) / hf
    gy = f32(0.5) * (S[2:, 1:-1] - S[:-2, 1:-1]) / hf
    band = (core >= 0) & (np.abs(core) <= tol) & (gx * gx + gy * gy > 1e-24)
    oid[1:-1, 1:-1] = np.where(band, lay[1:-1, 1:-1], 255).astype(np.uint8)
    return S, oid


def _parse_obj2d(path):
    """2D OBJ reader of 2D-solver/include/parsing.h:142-237: one polygon per `o`/`g` group (all
    its `f` lines appended to one vertex loop), vertices (x, y) as float, shifted so the minimum
    corner is at the origin; the boundary polygon is the first whose name contains "boundary"
    (any case). Returns (vertices [n, 2] float32, polygons [(name, [indices])], Lx, Ly, boundary)."""
    verts, polys = [], []
    cur, have, cur_name = None, False, "unnamed"

    def flush():
        if have and len(cur[1]) >= 3:
            polys.append(cur)

    for raw in open(path):
        line = raw.strip()
        if not line or line[0] == "#":
            continue
        tok = line.split()
        if tok[0] in ("o", "g"):
            flush()
            cur_name = tok[1] if len(tok) >= 2 else "unnamed"
            cur, have = (cur_name, []), True
        elif tok[0] == "v":
            if len(tok) < 3:
                continue
            verts.append((f32(float(tok[1])), f32(float(tok[2]))))
        elif tok[0] == "f":
            if len(tok) < 4:
                continue
            if not have:
                cur, have = (cur_name, []), True
            for t in tok[1:]:
                t = t.split("/", 1)[0]
                try:
                    idx = int(t)
                except ValueError:
                    idx = 0
                cur[1].append(idx - 1 if idx > 0 else idx)
    flush()
    V = np.array(verts, np.float32).reshape(-1, 2)
    Lx = Ly = f32(0)
    if len(V):
        lo, hi = V.min(axis=0), V.max(axis=0)
        V = (V - lo).astype(np.float32)
        Lx, Ly = f32(hi[0] - lo[0]), f32(hi[1] - lo[1])
    boundary = next((k for k, (nm, _) in enumerate(polys) if "boundary" in nm.lower()), -1)
    return V, polys, Lx, Ly, boundary


def _dist_to_poly(px, py, V, face):
    """dist_to_poly_edges of parsing.h:104-113 (dist_point_seg 76-86) in float, for arrays of
    points."""
    d = np.full(px.shape, np.finfo(np.float32).max, np.float32)
    m = len(face)
    for e in range(m):
        A, B = V[face[e]], V[face[(e + 1) % m]]
        abx, aby = f32(B[0] - A[0]), f32(B[1] - A[1])
        apx, apy = px - A[0], py - A[1]
        den = f32(abx * abx + aby * aby)
        t = (apx * abx + apy * aby) / den if den > 0 else np.zeros_like(px)
        t = np.clip(t, f32(0), f32(1)).astype(np.float32)
        cx, cy = A[0] + t * abx, A[1] + t * aby
        dx, dy = px - cx, py - cy
        d = np.minimum(d, np.sqrt(dx * dx + dy * dy))
    return d


def _inside_poly(px, py, V, face):
    """point_in_poly of parsing.h:88-102 (crossing number) in float, for arrays of points."""
    inside = np.zeros(px.shape, bool)
    m = len(face)
    j = m - 1
    for i in range(m):
        A, B = V[face[i]], V[face[j]]
        cond = (A[1] > py) != (B[1] > py)
        xint = (B[0] - A[0]) * (py - A[1]) / (f32(B[1] - A[1]) + f32(1e-30)) + A[0]
        inside ^= cond & (px < xint)
        j = i
    return inside


def scene_from_obj(path, h, tol_cells=3.0):
    """The reference 2D solver's scene set-up (2D-solver/include/parsing.h: parse_obj2d,
    build_sdf, build_oid_dense_cpu; main.cu:82, 104-144) restated in float arithmetic: the node
    grid Nx = ceil(Lx / h) + 1 by Ny = ceil(Ly / h) + 1, the node-based signed distance S to the
    non-boundary polygons (negative inside any), and oid = the layer id (boundary 0, other names
    1.. in first-appearance order) of the polygon nearest to the wall foot point of each node
    1..N-2 with 0 <= S <= tol and a nonzero gradient, 255 elsewhere. Returns a dict with S, oid,
    Nx, Ny, Lx, Ly and the layer names (the .fit file of layer m >= 1 is input/fit/<name>.fit)."""
    V, polys, Lx, Ly, bnd = _parse_obj2d(path)
    h = f32(h)
    Nx = int(np.ceil(f32(Lx / h))) + 1
    Ny = int(np.ceil(f32(Ly / h))) + 1
    X = np.broadcast_to((np.arange(Nx, dtype=np.float32) * h)[None, :], (Ny, Nx))
    Y = np.broadcast_to((np.arange(Ny, dtype=np.float32) * h)[:, None], (Ny, Nx))
    dmin = np.full((Ny, Nx), np.finfo(np.float32).max, np.float32)
    inside = np.zeros((Ny, Nx), bool)
    for k, (_, face) in enumerate(polys):
        if k == bnd:
            continue
        dmin = np.minimum(dmin, _dist_to_poly(X, Y, V, face))
        inside |= _inside_poly(X, Y, V, face)
    S = np.where(inside, -dmin, dmin).astype(np.float32)
    # layers (parsing.h:316-379)
    names = [polys[bnd][0]] if bnd >= 0 else []
    for k, (nm, _) in enumerate(polys):
        if k != bnd and nm not in names:
            names.append(nm)
    layer = [0 if k == bnd else names.index(nm) for k, (nm, _) in enumerate(polys)]
    # oid (parsing.h:418-466)
    tol = f32(tol_cells) * h
    oid = np.full((Ny, Nx), 255, np.uint8)
    core = S[1:-1, 1:-1]
    gx = f32(0.5) * (S[1:-1, 2:] - S[1:-1, :-2]) / h
    gy = f32(0.5) * (S[2:, 1:-1] - S[:-2, 1:-1]) / h
    gn2 = gx * gx + gy * gy
    sel = (core >= 0) & (np.abs(core) <= tol) & ~(gn2 <= f32(1e-24))
    jj, ii = np.nonzero(sel)
    if len(jj):
        s = core[jj, ii]
        inv = f32(1.0) / np.sqrt(gn2[jj, ii])
        nx, ny = gx[jj, ii] * inv, gy[jj, ii] * inv
        Wx = (ii + 1).astype(np.float32) * h - s * nx
        Wy = (jj + 1).astype(np.float32) * h - s * ny
        best = np.full(len(jj), np.finfo(np.float32).max, np.float32)
        pid = np.full(len(jj), -1)
        for k, (_, face) in enumerate(polys):
            if k == bnd:
                continue
            d = _dist_to_poly(Wx, Wy, V, face)
            closer = d < best
            best = np.where(closer, d, best)
            pid = np.where(closer, k, pid)
        lid = np.array([layer[k] if k >= 0 else -1 for k in pid])
        ok = (pid >= 0) & (lid >= 0) & (lid <= 254)
        oid[jj[ok] + 1, ii[ok] + 1] = lid[ok].astype(np.uint8)
    return {"S": S, "oid": oid, "Nx": Nx, "Ny": Ny, "Lx": float(Lx), "Ly": float(Ly), "layers": names}


class Legacy2D:
    """One 2D legacy solve (include/fz_legacy2d.h) on the given CUDA device."""

    def __init__(self, Nx, Ny, h=None, dt=None, c=None, rho=None, eps=None, tol=None, pml_n=None, pml_s=None,
                 pml_e=None, pml_w=None, precision="fp32", device=0):
        L = _abi.lib()
        p = _abi.FzL2dParams()
        L.fz_l2d_params_init(C.byref(p))
        p.Nx, p.Ny = int(Nx), int(Ny)
        for k, v in dict(h=h, dt=dt, c=c, rho=rho, eps=eps, tol=tol).items():
            if v is not None:
                setattr(p, k, float(v))
        for k, v in dict(pml_n=pml_n, pml_s=pml_s, pml_e=pml_e, pml_w=pml_w).items():
            if v is not None:
                setattr(p, k, int(v))
        p.precision = {"fp32": _abi.FZ_FP32, "fp64": _abi.FZ_FP64}[precision]
        p.device = int(device)
        self.params = p
        self.shape = (int(Ny), int(Nx))
        self._h = C.c_void_p()
        rc = L.fz_l2d_create(C.byref(p), C.byref(self._h))
        if rc != _abi.FZ_OK:
            raise FzError(rc, "fz_l2d_create failed (grid of at least 10 x 10 nodes, positive h/dt/rho/c/eps, "
                              "tol > h, a CUDA device)")

    def _check(self, rc):
        if rc != _abi.FZ_OK:
            buf = C.create_string_buffer(4096)
            _abi.lib().fz_l2d_last_error(self._h, buf, len(buf))
            raise FzError(rc, buf.value.decode(errors="replace"))

    def load_geometry(self, S, oid):
        S = np.ascontiguousarray(S, np.float32).reshape(self.shape)
        oid = np.ascontiguousarray(oid, np.uint8).reshape(self.shape)
        self._check(_abi.lib().fz_l2d_load_geometry(self._h, S.ctypes.data_as(C.POINTER(C.c_float)),
                                                    oid.ctypes.data_as(C.POINTER(C.c_uint8))))

    def set_materials(self, Rinf, A, zeta, B, Cc, alpha, beta):
        Rinf = np.ascontiguousarray(Rinf, np.float64).ravel()
        nmat = len(Rinf)
        A = np.ascontiguousarray(A, np.float64).reshape(nmat, -1)
        B = np.ascontiguousarray(B, np.float64).reshape(nmat, -1)
        K, L = A.shape[1], B.shape[1]
        arr = [np.ascontiguousarray(zeta, np.float64).reshape(nmat, K),
               np.ascontiguousarray(Cc, np.float64).reshape(nmat, L),
               np.ascontiguousarray(alpha, np.float64).reshape(nmat, L),
               np.ascontiguousarray(beta, np.float64).reshape(nmat, L)]
        self._check(_abi.lib().fz_l2d_set_materials(self._h, nmat, K, L, _dp(Rinf), _dp(A), _dp(arr[0]), _dp(B),
                                                    _dp(arr[1]), _dp(arr[2]), _dp(arr[3])))

    def set_fields(self, p=None, u=None, v=None):
        f = [None if a is None else np.ascontiguousarray(a, np.float64).reshape(self.shape) for a in (p, u, v)]
        self._check(_abi.lib().fz_l2d_set_fields(self._h, *[_dp(a) for a in f]))

    def set_receiver(self, i, j, nsamples):
        self._check(_abi.lib().fz_l2d_set_receiver(self._h, int(i), int(j), int(nsamples)))

    def run(self, nsteps):
        self._check(_abi.lib().fz_l2d_run(self._h, int(nsteps)))

    def run_timed(self, nsteps):
        """Runs nsteps steps; returns their device time in ms (CUDA events on the solve's stream)."""
        ms = C.c_double()
        self._check(_abi.lib().fz_l2d_run_timed(self._h, int(nsteps), C.byref(ms)))
        return ms.value

    @property
    def steps(self):
        return int(_abi.lib().fz_l2d_step_count(self._h))

    @property
    def band_cells(self):
        return int(_abi.lib().fz_l2d_band_cells(self._h))

    def ir(self):
        n = int(_abi.lib().fz_l2d_samples(self._h))
        out = np.zeros(max(n, 0))
        if n > 0:
            self._check(_abi.lib().fz_l2d_get_ir(self._h, _dp(out), n))
        return out

    def fields(self):
        out = [np.zeros(self.shape) for _ in range(3)]
        self._check(_abi.lib().fz_l2d_get_fields(self._h, *[_dp(a) for a in out]))
        return out

    def close(self):
        if self._h:
            _abi.lib().fz_l2d_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["Legacy2D", "plane_wave_fields", "rect_scene", "reference_setup", "scene_from_obj"]
