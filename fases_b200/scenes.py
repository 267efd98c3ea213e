"""Synthetic rooms for tests and benchmarks: shoebox rooms with axis-aligned box obstacles, given
as the geometry the reference builds from an OBJ (a signed distance field S, positive in air,
and a material map oid), plus seeded materials, sources, receivers and initial pulses.

Layout follows the reference: the room's bounding box is shifted so its minimum corner sits at
3h (3D-solver/include/parsing3D.h:690-712), the grid adds 3 ghost cells per side
(parsing3D.h:128), cell centres are at (i + 1/2) h, and |S| is clamped at the 8h narrow band of
the reference's SDF builder (parsing3D.h:900). oid = layer + 1 for cells with 0 <= S <= tol
(parsing3D.h:983-1011), 0xFF elsewhere. Layers: 0..5 = the six walls x-lo, x-hi, y-lo, y-hi,
z-lo, z-hi; 6.. = obstacles.
"""
from dataclasses import dataclass, field

import os

import numpy as np

from . import materials as mats

GHOST = 3
WALL_LAYERS = ("x_lo", "x_hi", "y_lo", "y_hi", "z_lo", "z_hi")


@dataclass
class Scene:
    S: np.ndarray            # float32 [Nz, Ny, Nx]
    oid: np.ndarray          # uint8 [Nz, Ny, Nx]
    h: float
    room_cells: tuple        # (nx, ny, nz) interior cells
    layers: list             # layer names, layer m -> oid m + 1
    obstacles: list = field(default_factory=list)  # [(lo_xyz, hi_xyz)] in metres (shifted frame)

    @property
    def shape(self):
        return self.S.shape


def box_room(room_cells, h, obstacles_cells=(), tol_cells=3.0, band_cells=8.0, merge_walls=None):
    """Analytic SDF/OID of a shoebox of room_cells = (nx, ny, nz) cells with solid box obstacles
    given in cell units [((i0, j0, k0), (i1, j1, k1)), ...] relative to the room's min corner.
    merge_walls optionally maps wall index -> layer index (to give several walls one layer).
    Ties between equidistant surfaces go to the lower layer index."""
    nx, ny, nz = room_cells
    Nx, Ny, Nz = nx + 2 * GHOST, ny + 2 * GHOST, nz + 2 * GHOST
    f32 = np.float32
    X = ((np.arange(Nx) + 0.5) * h).astype(f32)[None, None, :]
    Y = ((np.arange(Ny) + 0.5) * h).astype(f32)[None, :, None]
    Z = ((np.arange(Nz) + 0.5) * h).astype(f32)[:, None, None]
    lo = np.array([GHOST * h] * 3, f32)
    hi = (lo + np.array([nx, ny, nz]) * h).astype(f32)
    # distance from the inside to each wall plane (positive inside the room); nearest wall wins
    walls = [X - lo[0], hi[0] - X, Y - lo[1], hi[1] - Y, Z - lo[2], hi[2] - Z]
    shape = (Nz, Ny, Nx)
    S = np.full(shape, np.inf, f32)
    nearest = np.zeros(shape, np.int16)
    for wi, d in enumerate(walls):
        d = np.broadcast_to(d, shape)
        m = d < S
        S = np.where(m, d, S)
        nearest = np.where(m, np.int16(wi), nearest)
    # outside the room: Euclidean distance to the box, negative
    ox = np.maximum(np.maximum(lo[0] - X, X - hi[0]), 0)
    oy = np.maximum(np.maximum(lo[1] - Y, Y - hi[1]), 0)
    oz = np.maximum(np.maximum(lo[2] - Z, Z - hi[2]), 0)
    d_out = np.sqrt(ox * ox + oy * oy + oz * oz)
    S = np.where(S > 0, S, -d_out).astype(f32)
    wall_layer = np.arange(6) if merge_walls is None else np.asarray(merge_walls)
    layer = wall_layer.astype(np.int16)[nearest]
    n_wall_layers = int(wall_layer.max()) + 1
    obs_m = []
    for q, (c0, c1) in enumerate(obstacles_cells):
        b0 = (lo + np.array(c0, float) * h).astype(f32)
        b1 = (lo + np.array(c1, float) * h).astype(f32)
        obs_m.append((b0, b1))
        # signed distance to the obstacle box, positive outside
        qx = np.maximum(b0[0] - X, X - b1[0])
        qy = np.maximum(b0[1] - Y, Y - b1[1])
        qz = np.maximum(b0[2] - Z, Z - b1[2])
        ext = np.sqrt(np.maximum(qx, 0) ** 2 + np.maximum(qy, 0) ** 2 + np.maximum(qz, 0) ** 2)
        intr = np.minimum(np.maximum(qx, np.maximum(qy, qz)), 0)
        d = (ext + intr).astype(f32)
        closer = d < S
        layer = np.where(closer, np.int16(n_wall_layers + q), layer)
        S = np.minimum(S, d)
    band = f32(band_cells * h)
    S = np.clip(S, -band, band).astype(f32)
    tol = f32(tol_cells * h)
    oid = np.full(shape, 0xFF, np.uint8)
    sel = (S >= 0) & (S <= tol)
    # the reference's OID builder skips the outermost cells (parsing3D.h:985-987)
    sel[0, :, :] = sel[-1, :, :] = False
    sel[:, 0, :] = sel[:, -1, :] = False
    sel[:, :, 0] = sel[:, :, -1] = False
    oid[sel] = (layer[sel] + 1).astype(np.uint8)
    names = [WALL_LAYERS[i] for i in range(6)] if merge_walls is None else [f"wall{i}" for i in range(n_wall_layers)]
    names += [f"obstacle{q}" for q in range(len(obstacles_cells))]
    return Scene(np.ascontiguousarray(S), oid, h, (nx, ny, nz), names, obs_m)


def seeded_obstacles(rng, room_cells, n, size_frac=(0.05, 0.15), margin_cells=24):
    """n axis-aligned boxes inside the room, away from the walls by margin_cells."""
    out = []
    nx, ny, nz = room_cells
    for _ in range(n):
        c0, c1 = [], []
        for L in (nx, ny, nz):
            s = max(4, int(rng.uniform(*size_frac) * L))
            a = int(rng.integers(margin_cells, max(margin_cells + 1, L - margin_cells - s)))
            c0.append(a)
            c1.append(a + s)
        out.append((tuple(c0), tuple(c1)))
    return out


def gaussian_pulse(shape, h, center_cells, sigma_cells, amplitude=1.0, cutoff_sigmas=12.0):
    """Pressure initial condition p = A exp(-r^2 / (2 sigma^2)) about a cell centre (zero beyond
    cutoff_sigmas, where it is below 1e-31 A)."""
    Nz, Ny, Nx = shape
    ci, cj, ck = [int(x) for x in center_cells]
    r = int(np.ceil(cutoff_sigmas * sigma_cells))
    p = np.zeros(shape, np.float64)
    k0, k1 = max(0, ck - r), min(Nz, ck + r + 1)
    j0, j1 = max(0, cj - r), min(Ny, cj + r + 1)
    i0, i1 = max(0, ci - r), min(Nx, ci + r + 1)
    k = np.arange(k0, k1)[:, None, None]
    j = np.arange(j0, j1)[None, :, None]
    i = np.arange(i0, i1)[None, None, :]
    r2 = (i - ci) ** 2 + (j - cj) ** 2 + (k - ck) ** 2
    p[k0:k1, j0:j1, i0:i1] = amplitude * np.exp(-r2 / (2.0 * sigma_cells ** 2))
    return p


def seeded_cells(rng, room_cells, n, margin_cells=8):
    """n grid cells (i, j, k) inside the room, margin_cells from the walls."""
    nx, ny, nz = room_cells
    pts = []
    for _ in range(n):
        pts.append([int(rng.integers(min(margin_cells, L // 3), L - min(margin_cells, L // 3))) + GHOST
                    for L in (nx, ny, nz)])
    return np.array(pts, np.int32)


def free_cells(scene, cells, min_s_cells=4.0):
    """Keeps only cells at least min_s_cells from any surface."""
    keep = [c for c in cells if scene.S[c[2], c[1], c[0]] >= min_s_cells * scene.h]
    return np.array(keep, np.int32).reshape(-1, 3)


def benchmark_room(room_cells=(500, 400, 200), h=0.02, seed=0, n_obstacles=5, open_face=1, K=2, L=2,
                   c=343.0, rho=1.2, cfl=0.5, n_receivers=16, pulse_sigma_cells=2.0, clearance_cells=6.0):
    """The plain 3D benchmark room: a shoebox (default 10 x 8 x 4 m at h = 0.02 m), seeded rigid box
    obstacles, six seeded passive ADE wall materials (K real poles, L complex pairs), one open
    face (wall replaced by a matched layer plus a cPML), a Gaussian pressure pulse and seeded
    receivers. open_face is the wall index (0 x-lo, 1 x-hi, ...)."""
    rng = np.random.default_rng(seed)
    obst = seeded_obstacles(rng, room_cells, n_obstacles)
    scene = box_room(room_cells, h, obst)
    dt = cfl * h / c
    f_cutoff = c / (2 * h) / 2  # half the grid Nyquist
    wall_mats = [mats.random_passive(rng, dt, f_cutoff, K=K, L=L) for _ in range(6)]
    wall_mats[open_face] = mats.matched()
    obst_mats = [mats.rigid(0.99) for _ in obst]
    # face keys U D R L F B: z-hi z-lo x-hi x-lo y-hi y-lo
    face_key = {0: 3, 1: 2, 2: 5, 3: 4, 4: 1, 5: 0}
    pml = [0] * 6
    pml[face_key[open_face]] = 1
    cand = seeded_cells(rng, room_cells, 4 * n_receivers + 8, margin_cells=30)
    cand = free_cells(scene, cand, min(clearance_cells, min(room_cells) / 3.0))
    src = cand[0]
    recs = cand[1:1 + n_receivers]
    p0 = gaussian_pulse(scene.shape, h, src, pulse_sigma_cells)
    return {
        "scene": scene, "materials": wall_mats + obst_mats, "pml": tuple(pml), "c": c, "rho": rho, "dt": dt,
        "h": h, "source_cell": src, "receivers": recs, "p0": p0, "seed": seed, "f_cutoff": f_cutoff,
    }


def box_room_2d(room_cells, h, obstacles_cells=(), tol_cells=3.0, band_cells=8.0):
    """Planar room for the two_d solve: the 2D signed distance of an (nx, ny) rectangle with box
    obstacles [((i0, j0), (i1, j1)), ...], replicated over the 7 planes of a planar grid (one
    updated plane between 3 ghost planes on each side). Layers: x_lo, x_hi, y_lo, y_hi, then
    obstacles."""
    nx, ny = room_cells
    Nx, Ny, Nz = nx + 2 * GHOST, ny + 2 * GHOST, 2 * GHOST + 1
    f32 = np.float32
    X = ((np.arange(Nx) + 0.5) * h).astype(f32)[None, :]
    Y = ((np.arange(Ny) + 0.5) * h).astype(f32)[:, None]
    lo = np.array([GHOST * h] * 2, f32)
    hi = (lo + np.array([nx, ny]) * h).astype(f32)
    walls = [X - lo[0], hi[0] - X, Y - lo[1], hi[1] - Y]
    shape = (Ny, Nx)
    S = np.full(shape, np.inf, f32)
    layer = np.zeros(shape, np.int16)
    for wi, d in enumerate(walls):
        d = np.broadcast_to(d, shape)
        m = d < S
        S = np.where(m, d, S)
        layer = np.where(m, np.int16(wi), layer)
    ox = np.maximum(np.maximum(lo[0] - X, X - hi[0]), 0)
    oy = np.maximum(np.maximum(lo[1] - Y, Y - hi[1]), 0)
    S = np.where(S > 0, S, -np.sqrt(ox * ox + oy * oy)).astype(f32)
    for q, (c0, c1) in enumerate(obstacles_cells):
        b0 = (lo + np.array(c0, float) * h).astype(f32)
        b1 = (lo + np.array(c1, float) * h).astype(f32)
        qx = np.maximum(b0[0] - X, X - b1[0])
        qy = np.maximum(b0[1] - Y, Y - b1[1])
        d = (np.sqrt(np.maximum(qx, 0) ** 2 + np.maximum(qy, 0) ** 2) + np.minimum(np.maximum(qx, qy), 0)).astype(f32)
        layer = np.where(d < S, np.int16(4 + q), layer)
        S = np.minimum(S, d)
    S = np.clip(S, -f32(band_cells * h), f32(band_cells * h)).astype(f32)
    oid2 = np.full(shape, 0xFF, np.uint8)
    sel = (S >= 0) & (S <= f32(tol_cells * h))
    sel[0, :] = sel[-1, :] = False
    sel[:, 0] = sel[:, -1] = False
    oid2[sel] = (layer[sel] + 1).astype(np.uint8)
    S3 = np.ascontiguousarray(np.broadcast_to(S, (Nz,) + shape))
    oid3 = np.ascontiguousarray(np.broadcast_to(oid2, (Nz,) + shape)).copy()
    oid3[0] = oid3[-1] = 0xFF  # outermost planes carry no material (parsing3D.h:985-987)
    names = ["x_lo", "x_hi", "y_lo", "y_hi"] + [f"obstacle{q}" for q in range(len(obstacles_cells))]
    return Scene(S3, oid3, h, (nx, ny, 1), names, [])


def benchmark_2d(room_cells=(256, 256), h=0.02, seed=0, c=343.0, rho=1.2, cfl=0.5, pml_cells=16, n_receivers=4,
                 pulse_sigma_cells=3.0):
    """The plain 2D benchmark (FP64): 256 x 256 cells at h = 0.02 m, a 16-cell cPML on the x-hi
    side (whose wall is a matched layer), rigid walls (R = 0.99) on x-lo and y-hi, one ADE wall on
    y-lo with 2 seeded real poles in [1e2, 1e4] 1/s and passive residues, a Gaussian pressure
    pulse (sigma = 3 cells) at a seeded interior point, and seeded receivers."""
    rng = np.random.default_rng(seed)
    scene = box_room_2d(room_cells, h)
    dt = cfl * h / c
    f_cutoff = c / (4 * h)
    ade = mats.random_passive(rng, dt, f_cutoff, K=2, L=0)
    wall_mats = [mats.rigid(0.99), mats.matched(), ade, mats.rigid(0.99)]
    pml = (0, 0, 1, 0, 0, 0)  # R = x-hi
    nx, ny = room_cells
    pts = []
    while len(pts) < n_receivers + 1:
        i = int(rng.integers(pml_cells + 12, nx - pml_cells - 12)) + GHOST
        j = int(rng.integers(12, ny - 12)) + GHOST
        pts.append((i, j, GHOST))
    src = np.array(pts[0], np.int32)
    recs = np.array(pts[1:], np.int32)
    p0 = gaussian_pulse(scene.shape, h, src, pulse_sigma_cells)
    p0[:GHOST] = 0.0
    p0[GHOST + 1:] = 0.0
    return {"scene": scene, "materials": wall_mats, "pml": pml, "pml_cells": pml_cells, "c": c, "rho": rho,
            "dt": dt, "h": h, "source_cell": src, "receivers": recs, "p0": p0, "seed": seed}


def obj_layers(path):
    """Group (layer) names of an OBJ in material order: a group is created at its first face, named
    by the second token of its o/g line when there are two or more (3D-solver/include/parsing3D.h:
    167-288); material m of the scene is layer m (oid m + 1)."""
    names, seen, cur, named, pending = [], set(), "unnamed", False, True
    with open(path) as f:
        for line in f:
            line = line.strip(" \t\r\n")
            if not line or line[0] == "#":
                continue
            if line.startswith("o ") or line.startswith("g "):
                parts = line.split()[1:]
                nm = parts[1] if len(parts) >= 2 else (parts[0] if parts else "unnamed")
                if not named or nm != cur:
                    cur, named, pending = nm, True, True
            elif line.startswith("f ") and len(line.split()) >= 4 and pending:
                nm = cur if named else "unnamed"
                if nm not in seen:
                    seen.add(nm)
                    names.append(nm)
                pending = False
    return names


def from_obj(path, h, tol_cells=3.0, device=0):
    """Scene of an OBJ file built on the GPU by the library (fz_build_scene): the signed distance
    and material ids the reference solver caches in output/S.bin and output/oid.bin."""
    import ctypes as C

    from ._abi import check, lib
    dims = (C.c_int32 * 3)()
    L = (C.c_double * 3)()
    check(lib().fz_scene_dims(os.fsencode(path), float(h), dims, L))
    Nx, Ny, Nz = dims
    S = np.zeros((Nz, Ny, Nx), np.float32)
    oid = np.zeros((Nz, Ny, Nx), np.uint8)
    check(lib().fz_build_scene(os.fsencode(path), float(h), float(tol_cells), int(device),
                               S.ctypes.data_as(C.POINTER(C.c_float)), oid.ctypes.data_as(C.POINTER(C.c_uint8)),
                               S.size))
    return Scene(S=S, oid=oid, h=float(h), room_cells=(Nx - 2 * GHOST, Ny - 2 * GHOST, Nz - 2 * GHOST),
                 layers=obj_layers(path))

