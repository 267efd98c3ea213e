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
