"""Reads a golden reference project (written by make_golden.py, run through the reference solver)
into the inputs of the CPU oracle, with the reference's float32 conventions (main3D.cu:115-160,
454-456, 729-752, 861-959, 963-1124; common/filterABC.h:31-90). Test infrastructure only; it is
independent of the product's C++ project parser, which the GPU tests exercise on the same files.
"""
import os
import re

import numpy as np

f32 = np.float32


def read_config(path):
    vals = []
    for line in open(path):
        line = line.split("#", 1)[0]
        m = re.match(r"\s*([-+0-9.eE]+)", line)
        if m:
            try:
                vals.append(f32(float(m.group(1))))
            except ValueError:
                pass
    return vals


def read_fit(path):
    toks = []
    for line in open(path):
        s = line.strip()
        if not s or s.startswith("#"):
            continue
        toks += s.split()
    Rinf = f32(toks[0])
    K, L = int(toks[1]), int(toks[2])
    pos = 3
    A, zeta = [], []
    for _ in range(K):
        A.append(f32(toks[pos])); zeta.append(f32(toks[pos + 1])); pos += 2
    B, C, al, be = [], [], [], []
    for _ in range(L):
        B.append(f32(toks[pos])); C.append(f32(toks[pos + 1])); al.append(f32(toks[pos + 2])); be.append(f32(toks[pos + 3]))
        pos += 4
    return Rinf, A, zeta, B, C, al, be


def obj_layers(path):
    names, seen, cur, have, pending = [], set(), "unnamed", False, True
    for raw in open(path):
        line = raw.strip()
        if not line or line.startswith("#"):
            continue
        if line.startswith("o ") or line.startswith("g "):
            parts = line.split()[1:]
            nm = parts[1] if len(parts) >= 2 else (parts[0] if parts else "unnamed")
            if not have or nm != cur:
                cur, have, pending = nm, True, True
        elif line.startswith("f ") and len(line.split()) >= 4 and pending:
            nm = cur if have else "unnamed"
            if nm not in seen:
                seen.add(nm)
                names.append(nm)
            pending = False
    return names


def load(case_dir):
    """Returns a dict with the oracle inputs plus the reference's IR/VEL traces."""
    cfg = read_config(os.path.join(case_dir, "config", "config.txt"))
    h = cfg[0]
    t_max = cfg[1]
    f_in = cfg[2]
    f_x = f_in
    for oc in (63.0, 125.0, 250.0, 500.0, 1000.0, 2000.0, 4000.0, 8000.0):
        hi = f32(oc) * f32(1.41421356)
        if f_in <= hi:
            f_x = hi
            break
    f_cutoff = f32(2.0) * f_x
    rho = f32(1.225)
    Temp = cfg[3] + f32(273.15)
    c = np.sqrt(f32(1.4) * f32(287.05) * Temp, dtype=f32)
    dt = f32(cfg[4] * h / c)
    Nt = int(t_max / dt) + 1
    pml = tuple(int(cfg[6 + i] != 0) for i in range(6))
    src_opt = int(cfg[15]) if len(cfg) > 15 else 0
    glob_f = cfg[16] if len(cfg) > 16 else (f32(25.0) if src_opt == 0 else f32(0.5) * f_cutoff)
    lines = open(os.path.join(case_dir, "output", "scene_cache.txt")).read().split("\n")
    Nx, Ny, Nz = [int(x) for x in lines[1].split()[:3]]
    N = Nx * Ny * Nz
    S = np.fromfile(os.path.join(case_dir, "output", "S.bin"), np.float32, N).reshape(Nz, Ny, Nx)
    oid = np.fromfile(os.path.join(case_dir, "output", "oid.bin"), np.uint8, N).reshape(Nz, Ny, Nx)
    Km, Lm = [int(x) for x in open(os.path.join(case_dir, "config", "poles.txt")).read().split()[:2]]
    Km, Lm = max(1, Km), max(1, Lm)
    layers = obj_layers(os.path.join(case_dir, "scene.obj"))
    nm = len(layers)
    mat = {"Rinf": np.zeros(nm), "A": np.zeros((nm, Km)), "zeta": np.zeros((nm, Km)), "B": np.zeros((nm, Lm)),
           "Cc": np.zeros((nm, Lm)), "alpha": np.zeros((nm, Lm)), "beta": np.zeros((nm, Lm))}
    for m, name in enumerate(layers):
        if "ounding" in name or "oundary" in name:
            continue
        Rinf, A, zeta, B, C_, al, be = read_fit(os.path.join(case_dir, "input", "fit", name + ".fit"))
        mat["Rinf"][m] = Rinf
        mat["A"][m, :len(A)] = A
        mat["zeta"][m, :len(zeta)] = zeta
        mat["B"][m, :len(B)] = B
        mat["Cc"][m, :len(C_)] = C_
        mat["alpha"][m, :len(al)] = al
        mat["beta"][m, :len(be)] = be
    src, spress, sfreq = [], [], []
    for line in open(os.path.join(case_dir, "src.txt")):
        if not line.strip() or line.startswith("#"):
            continue
        v = [f32(x) for x in line.split()]
        if len(v) < 4:
            continue
        ijk = [int(v[a] / h) + 3 for a in range(3)]
        if all(0 <= ijk[a] < n for a, n in enumerate((Nx, Ny, Nz))):
            src.append(ijk)
            spress.append(f32(2e-5 * float(np.power(f32(10.0), f32(v[3] / 20.0), dtype=f32))))
            sfreq.append(v[4] if len(v) > 4 else f32(0.5) * f_cutoff)
    rec = []
    for line in open(os.path.join(case_dir, "rec.txt")):
        if not line.strip() or line.startswith("#"):
            continue
        v = [f32(x) for x in line.split()]
        rec.append([int(v[a] / h) + 3 for a in range(3)])
    from oracle.oracle import waveform
    if src_opt == 2:
        # sinusoids: each source scaled by its own rho A_s f / 2 (main3D.cu:1071-1075), no waveform
        As = 6.0 * float(h) * float(h)
        sval = np.array([f32(s / f32(float(rho) * As * float(f) / 2.0)) for s, f in zip(spress, sfreq)], np.float64)
        us32 = np.zeros(2 * Nt + 1)
        pref, pk = None, None
    else:
        us, pref, pk = waveform(src_opt, float(glob_f), float(f_cutoff), float(dt), Nt, float(h), float(rho))
        sval = np.array([f32(s / f32(pk)) for s in spress], np.float64)
        us32 = us.astype(np.float32).astype(np.float64)
    nrec = len(rec)
    ir = np.stack([np.fromfile(os.path.join(case_dir, "output", f"IR{r}_0.bin"), np.float32) for r in range(nrec)])
    vel = np.stack([np.fromfile(os.path.join(case_dir, "output", f"VEL{r}_0.bin"), np.float32).reshape(-1, 3)
                    for r in range(nrec)])
    return {"S": S, "oid": oid, "h": float(h), "c": float(c), "rho": float(rho), "dt": float(dt), "Nt": Nt,
            "pml": pml, "materials": mat, "src": np.array(src, np.int32), "sval": sval, "src_opt": src_opt,
            "src_freq": np.array(sfreq, np.float64), "u_s": us32, "rec": np.array(rec, np.int32), "ir": ir,
            "vel": vel, "p_ref_scaled": pref * float(f32(spress[0] / f32(pk))) if spress and pref is not None else None,
            "case_dir": case_dir}


def run_oracle(fx, steps=None):
    from oracle.oracle import Oracle
    steps = fx["Nt"] if steps is None else steps
    o = Oracle(fx["S"], fx["oid"], fx["h"], fx["c"], fx["rho"], fx["dt"], pml=fx["pml"], materials=fx["materials"],
               src_cells=fx["src"], sval=fx["sval"], src_opt=fx["src_opt"], src_freq=fx["src_freq"], u_s=fx["u_s"],
               rec_cells=fx["rec"], max_steps=steps)
    o.run(steps)
    return o


def load_legacy2d(case_dir):
    """Oracle inputs of a 2D legacy golden project (make_golden_legacy2d.py) plus the reference's
    receiver trace, in the reference's float conventions (2D-solver/core/main.cu:38-82, 231-295,
    378-404, 430-499; common/filterABC.h:31-90)."""
    cfg = read_config(os.path.join(case_dir, "config", "config.txt"))
    h, t_max = cfg[0], cfg[1]
    c = np.sqrt(f32(1.4) * f32(287.05) * f32(cfg[3] + f32(273.15)), dtype=f32)
    rho = f32(1.225)
    dt = f32(cfg[4] * h / c)
    Nt = int(t_max / dt) + 1
    pml = tuple(int(cfg[6 + q]) for q in range(4))  # N, S, E, W
    hdr = open(os.path.join(case_dir, "output", "pre_header.txt")).read().split()
    Nx, Ny = int(hdr[0]), int(hdr[1])
    S = np.fromfile(os.path.join(case_dir, "output", "S.bin"), np.float32, Nx * Ny).reshape(Ny, Nx)
    oid = np.fromfile(os.path.join(case_dir, "output", "oid.bin"), np.uint8, Nx * Ny).reshape(Ny, Nx)
    Km, Lm = [int(x) for x in open(os.path.join(case_dir, "config", "poles.txt")).read().split()[:2]]
    Km, Lm = max(1, Km), max(1, Lm)
    layers = [n for n in obj_layers(os.path.join(case_dir, "scene.obj")) if "boundary" not in n.lower()]
    nm = len(layers)
    mat = {"Rinf": np.zeros(nm), "A": np.zeros((nm, Km)), "zeta": np.zeros((nm, Km)), "B": np.zeros((nm, Lm)),
           "C": np.zeros((nm, Lm)), "alpha": np.zeros((nm, Lm)), "beta": np.zeros((nm, Lm))}
    for m, name in enumerate(layers):
        Rinf, A, zeta, B, C_, al, be = read_fit(os.path.join(case_dir, "input", "fit", name + ".fit"))
        mat["Rinf"][m] = Rinf
        for key, vals in (("A", A), ("zeta", zeta), ("B", B), ("C", C_), ("alpha", al), ("beta", be)):
            mat[key][m, :len(vals)] = vals
    src_x = None
    for line in open(os.path.join(case_dir, "input", "src", "src.txt")):
        if line.strip() and not line.startswith("#"):
            v = [f32(x) for x in line.split()]
            if 0 <= int(v[0] / h) < Nx and 0 <= int(v[1] / h) < Ny:
                src_x = v[0]
    rec = (Nx // 2, Ny // 2)
    for line in open(os.path.join(case_dir, "input", "rec", "rec.txt")):
        if line.strip() and not line.startswith("#"):
            v = [f32(x) for x in line.split()]
            ij = (int(v[0] / h), int(v[1] / h))
            if 0 <= ij[0] < Nx and 0 <= ij[1] < Ny:
                rec = ij
    # raised-cosine plane wave (main.cu:455-473; functions.cuh:555-559)
    ww = f32(0.5) * f32(0.04)
    xx = (np.arange(Nx, dtype=f32) + f32(0.5)) * h
    xi = (xx - src_x) / ww
    g = np.where(np.abs(xi) > f32(1), f32(0), f32(0.5) * (f32(1) + np.cos(f32(np.pi) * xi, dtype=f32))).astype(f32)
    pI = (f32(0.1) * g).astype(f32)
    uI = (pI / (rho * c)).astype(f32)
    p0 = np.tile(pI.astype(np.float64), (Ny, 1))
    u0 = np.tile(uI.astype(np.float64), (Ny, 1))
    ir = np.fromfile(os.path.join(case_dir, "output", "IR.bin"), np.float32).astype(np.float64)
    return {"S": S, "oid": oid, "h": float(h), "dt": float(dt), "c": float(c), "rho": float(rho),
            "eps": float(f32(1e-7)), "tol": float(f32(3.0) * h), "pml": pml, "materials": mat, "Nt": Nt,
            "p0": p0, "u0": u0, "rec": rec, "src_x": float(src_x), "ir": ir,
            "config": os.path.join(case_dir, "config", "config.txt")}


def run_legacy2d_oracle(fx, steps=None, use_float=False):
    from oracle.oracle import legacy2d_run
    steps = fx["Nt"] if steps is None else steps
    return legacy2d_run(fx["S"], fx["oid"], fx["h"], fx["dt"], fx["rho"], fx["c"], fx["eps"], fx["tol"], fx["pml"],
                        fx["materials"], fx["p0"], fx["u0"], None, fx["rec"], steps, use_float=use_float)
