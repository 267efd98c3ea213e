"""Shared scene builders for the parity tests (seeded, small enough for the CPU oracle)."""
import numpy as np

from fases_b200 import materials as mats
from fases_b200 import scenes


def small_room(seed=0, room=(26, 22, 18), pml=(0, 0, 1, 0, 0, 0), pml_cells=6, obstacle=True, K=2, L=2,
               h=0.05, c=343.0, rho=1.2, cfl=0.5, n_rec=4, source="pcs", pulse=True, steps=64):
    """A shoebox with one obstacle, six seeded passive ADE walls (the PML face matched), a PCS point
    source and/or a Gaussian pulse, and seeded receivers."""
    rng = np.random.default_rng(seed)
    obst = [((9, 7, 5), (14, 12, 9))] if obstacle else []
    sc = scenes.box_room(room, h, obst)
    dt = cfl * h / c
    f_cutoff = c / (4 * h)
    walls = [mats.random_passive(rng, dt, f_cutoff, K=K, L=L) for _ in range(6)]
    # the open (cPML) face's wall is a matched layer; face keys U D R L F B -> wall index
    key_to_wall = {0: 5, 1: 4, 2: 1, 3: 0, 4: 3, 5: 2}
    for f in range(6):
        if pml[f]:
            walls[key_to_wall[f]] = mats.matched()
    ms = walls + [mats.rigid(0.99) for _ in obst]
    packed = mats.pack(ms)
    src = np.array([[6, 6, 12]], np.int32)
    recs = np.array([[20, 15, 10], [8, 18, 6], [22, 6, 14], [15, 20, 17]][:n_rec], np.int32)
    out = dict(scene=sc, materials=packed, dt=dt, c=c, rho=rho, h=h, pml=pml, pml_cells=pml_cells,
               recs=recs, steps=steps, f_cutoff=f_cutoff)
    if source == "pcs":
        from fases_b200.solver import source_waveform
        us, _, pk = source_waveform(0, 0.25 * f_cutoff, f_cutoff, dt, steps + 2, h, rho)
        out.update(src=src, sval=np.array([0.5 / pk]), src_opt=0, u_s=us)
    else:
        out.update(src=None)
    if pulse:
        p0 = scenes.gaussian_pulse(sc.shape, h, (13, 9, 14), 2.0, amplitude=0.7)
        out["p0"] = p0
    else:
        out["p0"] = None
    return out


def run_gpu(cfg, precision, steps=None, graph=True, run=True):
    from fases_b200 import Solver, params
    steps = cfg["steps"] if steps is None else steps
    prm = params(h=cfg["h"], c=cfg["c"], rho=cfg["rho"], dt=cfg["dt"], pml=cfg["pml"],
                 pml_cells=cfg["pml_cells"], precision=precision)
    s = Solver(prm)
    s.load_geometry(cfg["scene"].S, cfg["scene"].oid)
    m = cfg["materials"]
    s.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    if cfg.get("src") is not None:
        s.set_sources(cfg["src"], cfg["sval"], cfg["src_opt"], u_s=cfg["u_s"])
    s.set_receivers(cfg["recs"], steps)
    if cfg.get("p0") is not None:
        s.set_fields(p=cfg["p0"])
    if not graph:
        s.profile(True)
    if run:
        s.run(steps)
    return s


def run_oracle(cfg, steps=None):
    from oracle.oracle import Oracle
    steps = cfg["steps"] if steps is None else steps
    sc = cfg["scene"]
    kw = {}
    if cfg.get("src") is not None:
        kw = dict(src_cells=cfg["src"], sval=cfg["sval"], src_opt=cfg["src_opt"], u_s=cfg["u_s"])
    o = Oracle(sc.S, sc.oid, cfg["h"], cfg["c"], cfg["rho"], cfg["dt"], pml=cfg["pml"],
               pml_cells=cfg["pml_cells"], materials=cfg["materials"], rec_cells=cfg["recs"],
               max_steps=steps, **kw)
    if cfg.get("p0") is not None:
        o.set_fields(p=cfg["p0"])
    o.run(steps)
    return o


def rel_l2(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def legacy2d_scene(Nx, Ny, h, rects, tol_cells=3.0):
    """Node-based signed distance S and object ids oid of rectangular obstacles for the 2D legacy
    scheme, by the conventions of 2D-solver/include/parsing.h:248-299, 404-466: nodes at
    (i h, j h), S > 0 in the fluid, the outer boundary polygon contributes no distance (FLT_MAX
    with no obstacle), oid = the nearest obstacle's layer (1-based) at interior nodes with
    0 <= S <= tol and a nonzero central-difference gradient, 255 elsewhere.
    rects: [((x0, y0), (x1, y1), layer), ...]."""
    x = np.arange(Nx) * h
    y = np.arange(Ny) * h
    X, Y = np.meshgrid(x, y)
    S = np.full((Ny, Nx), float(np.finfo(np.float32).max))
    lay = np.zeros((Ny, Nx), np.int32)
    for (x0, y0), (x1, y1), layer in rects:
        cx, cy, hx, hy = (x0 + x1) / 2, (y0 + y1) / 2, (x1 - x0) / 2, (y1 - y0) / 2
        dx, dy = np.abs(X - cx) - hx, np.abs(Y - cy) - hy
        d = np.hypot(np.maximum(dx, 0), np.maximum(dy, 0)) + np.minimum(np.maximum(dx, dy), 0)
        closer = d < S
        S = np.where(closer, d, S)
        lay = np.where(closer, layer, lay)
    S = S.astype(np.float32)
    hf = np.float32(h)
    tol = np.float32(tol_cells) * hf
    oid = np.full((Ny, Nx), 255, np.uint8)
    for j in range(1, Ny - 1):
        for i in range(1, Nx - 1):
            s = S[j, i]
            if not (s >= 0 and abs(s) <= tol):
                continue
            gx = np.float32(0.5) * (S[j, i + 1] - S[j, i - 1]) / hf
            gy = np.float32(0.5) * (S[j + 1, i] - S[j - 1, i]) / hf
            if gx * gx + gy * gy <= 1e-24:
                continue
            oid[j, i] = lay[j, i]
    return S, oid


def legacy2d_materials(nmat, K, L, seed=0):
    """Passive-looking ADE coefficients (Rinf, A, zeta, B, C, alpha, beta) for nmat materials."""
    rng = np.random.default_rng(seed)
    Rinf = rng.uniform(0.5, 0.9, nmat)
    zeta = rng.uniform(300.0, 4000.0, (nmat, K))
    A = rng.uniform(-0.2, 0.2, (nmat, K)) * zeta
    alpha = rng.uniform(200.0, 2000.0, (nmat, L))
    beta = rng.uniform(300.0, 3000.0, (nmat, L))
    B = rng.uniform(-0.1, 0.1, (nmat, L)) * alpha
    Cc = rng.uniform(-0.1, 0.1, (nmat, L)) * beta
    return dict(Rinf=Rinf, A=A, zeta=zeta, B=B, C=Cc, alpha=alpha, beta=beta)
