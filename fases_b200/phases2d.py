"""Command-line drop-in for the reference's 2D legacy solver `phases2D` (2D-solver/core/main.cu):

    python -m fases_b200.phases2d scene.obj config/config.txt input/src/src.txt input/rec/rec.txt [--fp64]

It takes the reference's arguments and project layout -- config/poles.txt and input/fit/<layer>.fit
relative to the working folder, as the reference reads them (main.cu:244-281) -- and writes the
reference's outputs: output/S.bin, output/oid.bin, output/pre_header.txt, output/IR.bin (the
pressure at the receiver node after every step, appended to what the file holds, as the reference
appends), output/pressure.bin (the pressure field after every anim_step-th step) and
output/header.txt. It runs the WENO + SSP-RK3 scheme the reference's menu option 2 selects, without
the prompts. Exit status 0 on success, 1 on a bad project (the reference's "[!]" aborts), 2 on a
solver error.
"""
import argparse
import os
import sys

import numpy as np

from . import legacy2d as L2

f32 = np.float32


def read_fit(path, Km, Lm):
    """read_fit_file (common/filterABC.h:31-90): R_inf, K, L, K x (A, zeta), L x (B, C, alpha,
    beta), '#' comment lines skipped; K <= Km and L <= Lm as the reference demands."""
    toks = []
    for line in open(path):
        s = line.strip()
        if s and not s.startswith("#"):
            toks += s.split()
    Rinf, K, Lc = f32(toks[0]), int(toks[1]), int(toks[2])
    if not (0 <= K <= Km and 0 <= Lc <= Lm):
        raise ValueError(f"{path}: K={K}, L={Lc} exceed poles.txt's {Km}, {Lm}")
    vals = [f32(t) for t in toks[3:3 + 2 * K + 4 * Lc]]
    if len(vals) < 2 * K + 4 * Lc:
        raise ValueError(f"{path}: too few coefficients")
    A, zeta = vals[0:2 * K:2], vals[1:2 * K:2]
    q = vals[2 * K:]
    return Rinf, A, zeta, q[0::4], q[1::4], q[2::4], q[3::4]


def _points(path, n):
    """Lines of n floats (src.txt: x y value; rec.txt: x y), '#' lines skipped."""
    out = []
    for line in open(path):
        if not line.strip() or line.startswith("#"):
            continue
        try:
            v = [f32(float(x)) for x in line.split()[:n]]
        except ValueError:
            continue
        if len(v) == n:
            out.append(v)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="phases2d", description=__doc__.split("\n\n")[0])
    ap.add_argument("scene")
    ap.add_argument("config")
    ap.add_argument("src")
    ap.add_argument("rec")
    ap.add_argument("--fp64", action="store_true", help="every array in FP64 (the reference is FP32)")
    a = ap.parse_args(argv)
    os.makedirs("output", exist_ok=True)
    for f in ("pressure.bin", "oid.bin", "S.bin", "header.txt"):  # main.cu:88
        if os.path.exists(os.path.join("output", f)):
            os.remove(os.path.join("output", f))
    setup = L2.reference_setup(a.config)
    P = setup["params"]
    h = f32(P["h"])
    sc = L2.scene_from_obj(a.scene, P["h"])
    Nx, Ny = sc["Nx"], sc["Ny"]
    sc["S"].tofile(os.path.join("output", "S.bin"))
    sc["oid"].tofile(os.path.join("output", "oid.bin"))
    tol_cells = int(f32(P["tol"]) / h)
    with open(os.path.join("output", "pre_header.txt"), "w") as f:
        f.write("%d %d %f %d\n" % (Nx, Ny, P["h"], tol_cells))
    print(f"\n[OK] Scene processing\n\nDomain info:\n\nLx = {sc['Lx']:.6f} m Ly = {sc['Ly']:.6f} m\n"
          f"Nx = {Nx} Ny = {Ny}")
    # materials (main.cu:231-295)
    Km, Lm = [int(x) for x in open(os.path.join("config", "poles.txt")).read().split()[:2]]
    Km, Lm = max(1, Km), max(1, Lm)
    names = sc["layers"][1:]
    nmat = max(len(names), 1)
    mats = {k: np.zeros((nmat, Km)) for k in ("A", "zeta")}
    mats.update({k: np.zeros((nmat, Lm)) for k in ("B", "C", "alpha", "beta")})
    mats["Rinf"] = np.zeros(nmat)
    try:
        for m, name in enumerate(names):
            Rinf, A, zeta, B, C, al, be = read_fit(os.path.join("input", "fit", name + ".fit"), Km, Lm)
            mats["Rinf"][m] = Rinf
            for key, v in (("A", A), ("zeta", zeta), ("B", B), ("C", C), ("alpha", al), ("beta", be)):
                mats[key][m, :len(v)] = v
    except (OSError, ValueError, IndexError) as e:
        print(f"[!] {e}", file=sys.stderr)
        return 1
    # resolution and Nyquist checks (main.cu:394-404)
    c, dt = f32(P["c"]), f32(P["dt"])
    f_cut = f32(setup["f_cutoff"])
    if f32(c / f_cut) / h < f32(12.0):
        print("[!] Resolution too low, aborting...", file=sys.stderr)
        return 1
    if not min(f32(0.5) * (f32(1.0) / dt), f32(0.5) * c / h) >= f_cut:
        print("[!] Sampling frequency too low, aborting...", file=sys.stderr)
        return 1
    Nt = setup["steps"]
    src = [v for v in _points(a.src, 3) if 0 <= int(v[0] / h) < Nx and 0 <= int(v[1] / h) < Ny]
    if not src:
        print("[!] no source inside the domain", file=sys.stderr)
        return 1
    rec = (Nx // 2, Ny // 2)
    for v in _points(a.rec, 2):
        ij = (int(v[0] / h), int(v[1] / h))
        if 0 <= ij[0] < Nx and 0 <= ij[1] < Ny:
            rec = ij
    anim_step = max(int(0.008 * Nt), 1)
    try:
        s = L2.Legacy2D(Nx, Ny, precision="fp64" if a.fp64 else "fp32", **P)
        s.load_geometry(sc["S"], sc["oid"])
        if names:
            s.set_materials(mats["Rinf"], mats["A"], mats["zeta"], mats["B"], mats["C"], mats["alpha"],
                            mats["beta"])
        s.set_fields(*L2.plane_wave_fields(Nx, Ny, P["h"], float(src[-1][0]), P["rho"], P["c"]))
        s.set_receiver(rec[0], rec[1], Nt)
        print(f"\n[OK] Will now start {Nt} iterations.\n\n[OK] Simulation start\n", flush=True)
        frames = 0
        last = -1
        with open(os.path.join("output", "pressure.bin"), "wb") as fp:
            done = 0
            while done < Nt:
                if 10 * done // Nt > last:
                    # the progress bar of print_progress (functions.cuh:1475-1488), every 10 %
                    last = 10 * done // Nt
                    filled = 50 * done // Nt
                    print("\r[%-50s] %3d%%" % ("=" * filled, int(100.0 * done / Nt + 0.5)), end="", flush=True)
                # a frame after step n (0-based) whenever n % anim_step == 0 (main.cu:838-845)
                n_next = ((done + anim_step - 1) // anim_step) * anim_step if done else 0
                chunk = min(n_next - done + 1, Nt - done)
                s.run(chunk)
                done += chunk
                if (done - 1) % anim_step == 0:
                    s.fields()[0].astype(np.float32).tofile(fp)
                    frames += 1
        print("\r[%-50s] %3d%%" % ("=" * 50, 100), flush=True)
        ir = s.ir().astype(np.float32)
        s.close()
    except L2.FzError as e:
        print(f"[!] {e}", file=sys.stderr)
        return 2
    with open(os.path.join("output", "IR.bin"), "ab") as f:
        ir.tofile(f)
    with open(os.path.join("output", "header.txt"), "w") as f:
        f.write("%d %d %d %f %f %d %d %f %s %f %d\n" % (Nx, Ny, Nt, sc["Lx"], sc["Ly"], frames, anim_step, dt,
                                                        a.scene, P["h"], tol_cells))
    print("\n[OK] Wrote to file for single receiver\n\n[OK] Finished.")
    return 0


if __name__ == "__main__":
    sys.exit(main())
