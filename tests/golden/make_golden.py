"""Generates the golden fixtures that pin the CPU oracle (and the CUDA stepper) to the reference.

For each case it writes a small reference project (OBJ room with named layers, config.txt,
poles.txt, input/fit/*.fit, src.txt, rec.txt), runs the reference solver itself -- built from
its own sources by oracle/build_ref.sh into oracle/_ref/fases3D -- on it, and keeps the inputs
plus the reference's outputs: output/S.bin, output/oid.bin, output/scene_cache.txt,
output/header.txt, output/pre_header.txt, config/p_ref.bin and output/IR*/VEL* traces.

    python tests/golden/make_golden.py OUT_DIR [CASE ...]   # on a machine with a GPU; then copy
                                                            # OUT_DIR/<case> into tests/golden/<case>

The reference needs a CUDA GPU; the committed fixtures let the CPU tests check the oracle
without one.
"""
import json
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from fases_b200 import materials as mats  # noqa: E402


def box_faces(lo, hi):
    """Six quads of an axis-aligned box as vertex index lists into the 8 corners."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = [(x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0),
         (x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)]
    faces = {"x_lo": (0, 3, 7, 4), "x_hi": (1, 5, 6, 2), "y_lo": (0, 4, 5, 1),
             "y_hi": (3, 2, 6, 7), "z_lo": (0, 1, 2, 3), "z_hi": (4, 5, 6, 7)}
    return v, faces


def write_obj(path, room, obstacles, wall_names):
    """OBJ of a shoebox room (one group per wall) plus closed box obstacles (one group each)."""
    lines = ["# synthetic shoebox room"]
    nv = 0
    v, faces = box_faces((0.0, 0.0, 0.0), room)
    for p in v:
        lines.append("v %.6f %.6f %.6f" % p)
    for key, name in zip(("x_lo", "x_hi", "y_lo", "y_hi", "z_lo", "z_hi"), wall_names):
        lines.append("g %s" % name)
        lines.append("f " + " ".join(str(nv + i + 1) for i in faces[key]))
    nv += 8
    for q, (lo, hi) in enumerate(obstacles):
        v, faces = box_faces(lo, hi)
        for p in v:
            lines.append("v %.6f %.6f %.6f" % p)
        lines.append("g obstacle%d" % q)
        for key in ("x_lo", "x_hi", "y_lo", "y_hi", "z_lo", "z_hi"):
            lines.append("f " + " ".join(str(nv + i + 1) for i in faces[key]))
        nv += 8
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


CASES = {
    # PCS source, one open face (x-hi wall is a BoundingBox layer under a cPML), one obstacle
    "box_pcs": dict(room=(1.2, 1.0, 0.8), h=0.04, t_max=0.012, f_in=250.0, temp=20.0, cfl=0.5,
                    pml=(0, 0, 1, 0, 0, 0), obstacles=[((0.5, 0.4, 0.3), (0.7, 0.6, 0.5))],
                    src_opt=0, glob_f=100.0, src=[(0.3, 0.3, 0.4, 85.0)],
                    rec=[(0.9, 0.7, 0.5), (0.2, 0.8, 0.2), (1.0, 0.2, 0.6)], seed=1, open_wall=1),
    # Ricker source, closed room (all six walls ADE), no cPML
    "box_ricker": dict(room=(1.0, 0.9, 0.7), h=0.04, t_max=0.012, f_in=250.0, temp=15.0, cfl=0.45,
                       pml=(0, 0, 0, 0, 0, 0), obstacles=[], src_opt=1, glob_f=300.0,
                       src=[(0.4, 0.35, 0.3, 80.0)], rec=[(0.7, 0.6, 0.45), (0.2, 0.2, 0.5)], seed=2,
                       open_wall=None),
    # two sinusoidal sources of their own frequencies (src.txt's fifth column), one open face
    "box_sine": dict(room=(1.1, 0.9, 0.8), h=0.04, t_max=0.012, f_in=250.0, temp=18.0, cfl=0.5,
                     pml=(0, 0, 1, 0, 0, 0), obstacles=[((0.6, 0.3, 0.2), (0.8, 0.5, 0.45))], src_opt=2,
                     glob_f=200.0, src=[(0.3, 0.3, 0.4, 80.0, 180.0), (0.5, 0.6, 0.5, 75.0, 260.0)],
                     rec=[(0.9, 0.7, 0.5), (0.25, 0.75, 0.3), (0.8, 0.2, 0.6)], seed=3, open_wall=1),
    # walls with 5 real poles and 3 complex pairs (the general-order band path), cPML on the x-hi and
    # y-lo faces, two obstacles
    "box_poles": dict(room=(1.2, 1.0, 0.8), h=0.04, t_max=0.012, f_in=250.0, temp=22.0, cfl=0.5,
                      pml=(0, 0, 1, 0, 1, 0), obstacles=[((0.5, 0.4, 0.3), (0.7, 0.6, 0.5)),
                                                         ((0.85, 0.15, 0.1), (1.0, 0.3, 0.35))],
                      src_opt=0, glob_f=100.0, src=[(0.3, 0.5, 0.4, 85.0)],
                      rec=[(0.9, 0.7, 0.5), (0.2, 0.8, 0.2), (0.6, 0.2, 0.6)], seed=4, open_wall=1, K=5, L=3),
    # animation slices kept (pressure{X,Y,Z}.bin and the energy-flow planes I*_*.bin): 60 frames asked on
    # the planes through (0.5, 0.45, 0.35) m, cPML on one face, one obstacle
    "box_slices": dict(room=(1.2, 1.0, 0.8), h=0.04, t_max=0.012, f_in=250.0, temp=20.0, cfl=0.5,
                       pml=(0, 0, 1, 0, 0, 0), obstacles=[((0.7, 0.5, 0.3), (0.9, 0.7, 0.5))],
                       src_opt=0, glob_f=100.0, src=[(0.3, 0.3, 0.4, 85.0)],
                       rec=[(0.9, 0.3, 0.5), (0.2, 0.8, 0.2)], seed=5, open_wall=1,
                       slice=(0.5, 0.45, 0.35), frames=60, keep_slices=True),
}


def make_project(case, dest, spec=None):
    """Writes the reference project of CASES[case] (or of the given spec) into dest."""
    c = spec if spec is not None else CASES[case]
    os.makedirs(os.path.join(dest, "config"), exist_ok=True)
    os.makedirs(os.path.join(dest, "input", "fit"), exist_ok=True)
    os.makedirs(os.path.join(dest, "output"), exist_ok=True)
    rng = np.random.default_rng(c["seed"])
    Temp = np.float32(c["temp"]) + np.float32(273.15)
    cc = float(np.sqrt(np.float32(1.4) * np.float32(287.05) * Temp, dtype=np.float32))
    dt = c["cfl"] * c["h"] / cc
    f_cut = 707.0
    wall_names = ["x_lo", "x_hi", "y_lo", "y_hi", "z_lo", "z_hi"]
    if c["open_wall"] is not None:
        wall_names[c["open_wall"]] = "BoundingBox"
    write_obj(os.path.join(dest, "scene.obj"), c["room"], c["obstacles"], wall_names)
    materials = {}
    for nm in wall_names:
        if nm == "BoundingBox":
            continue
        m = mats.random_passive(rng, dt, f_cut, K=c.get("K", 2), L=c.get("L", 2))
        m.write_fit(os.path.join(dest, "input", "fit", nm + ".fit"))
        materials[nm] = m
    for q in range(len(c["obstacles"])):
        m = mats.rigid(0.99)
        m.write_fit(os.path.join(dest, "input", "fit", "obstacle%d.fit" % q))
        materials["obstacle%d" % q] = m
    with open(os.path.join(dest, "config", "poles.txt"), "w") as f:
        f.write("%d %d\n" % (c.get("K", 2), c.get("L", 2)))
    x0, y0, z0 = c.get("slice", [0.5 * L for L in c["room"]])
    cfg = [c["h"], c["t_max"], c["f_in"], c["temp"], c["cfl"], 8, *c["pml"], 0, 0, 0, c["src_opt"], c["glob_f"], 0,
           x0, y0, z0, c.get("frames", 60)]
    names = ["h", "t_max", "wave band", "temperature", "CFL", "ADE poles", "U_PML", "D_PML", "R_PML", "L_PML",
             "F_PML", "B_PML", "ISM order", "altitude", "rays", "source type", "source frequency", "source index",
             "slice x0", "slice y0", "slice z0", "frames"]
    with open(os.path.join(dest, "config", "config.txt"), "w") as f:
        for v, n in zip(cfg, names):
            f.write("%s\t# %s\n" % (repr(v), n))
    with open(os.path.join(dest, "src.txt"), "w") as f:
        f.write("# x y z Lp [f0]\n")
        for s in c["src"]:
            f.write(" ".join("%g" % v for v in s) + "\n")
    with open(os.path.join(dest, "rec.txt"), "w") as f:
        f.write("# x y z\n")
        for r in c["rec"]:
            f.write("%g %g %g\n" % r)
    with open(os.path.join(dest, "case.json"), "w") as f:
        json.dump({"case": case, **{k: v for k, v in c.items()}}, f, indent=1)


REF_EXE = os.path.join(ROOT, "oracle", "_ref", "fases3D")


def run_reference(dest, timeout=600):
    if not os.path.exists(REF_EXE):
        raise SystemExit("reference solver not built: run oracle/build_ref.sh")
    cmd = [REF_EXE, os.path.join(dest, "scene.obj"), os.path.join(dest, "config", "config.txt"),
           os.path.join(dest, "src.txt"), os.path.join(dest, "rec.txt")]
    with open(os.path.join(dest, "reference_stdout.txt"), "w") as log:
        r = subprocess.run(cmd, cwd=dest, stdout=log, stderr=subprocess.STDOUT, timeout=timeout)
    return r.returncode


def run_reference_timed(dest, timeout=1800):
    """Runs the reference solver on dest, stamping each stdout line (the solver line-buffers its
    stdout) with time.perf_counter(); returns (returncode, [(t, line), ...]). The stamps of
    "Will now start" and "Simulation time" bracket its time loop on the wall clock."""
    import time
    if not os.path.exists(REF_EXE):
        raise SystemExit("reference solver not built: run oracle/build_ref.sh")
    cmd = [REF_EXE, os.path.join(dest, "scene.obj"), os.path.join(dest, "config", "config.txt"),
           os.path.join(dest, "src.txt"), os.path.join(dest, "rec.txt")]
    stamped = []
    t_end = time.perf_counter() + timeout
    with subprocess.Popen(cmd, cwd=dest, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                          bufsize=1) as proc:
        for line in proc.stdout:
            stamped.append((time.perf_counter(), line))
            if time.perf_counter() > t_end:
                proc.kill()
                break
        rc = proc.wait(timeout=60)
    with open(os.path.join(dest, "reference_stdout.txt"), "w") as log:
        log.writelines(line for _, line in stamped)
    return rc, stamped


def neutral_paths(dest, prefix=None):
    """The reference writes the absolute path of the project into output/scene_cache.txt,
    output/header.txt and its stdout. The fixtures keep the project-relative form ("./scene.obj"),
    so that no path of the machine that generated them is committed; no test reads those fields
    (the cache key is checked against the live path, which never matches a copied project)."""
    prefix = (prefix or dest).rstrip("/") + "/"
    for rel in (os.path.join("output", "scene_cache.txt"), os.path.join("output", "header.txt"),
                "reference_stdout.txt"):
        p = os.path.join(dest, rel)
        if os.path.exists(p):
            with open(p) as f:
                txt = f.read()
            with open(p, "w") as f:
                f.write(txt.replace(prefix, "./"))


def prune(dest, keep_slices=False):
    """Keep only what the tests read (inputs + FVM outputs; the animation slices if asked)."""
    out = os.path.join(dest, "output")
    keep = {"S.bin", "oid.bin", "scene_cache.txt", "header.txt", "pre_header.txt"}
    if keep_slices:
        keep |= {"pressureX.bin", "pressureY.bin", "pressureZ.bin", "Iy_X.bin", "Iz_X.bin", "Ix_Y.bin",
                 "Iz_Y.bin", "Ix_Z.bin", "Iy_Z.bin"}
    for fn in os.listdir(out):
        if fn in keep or (fn.startswith("IR") or fn.startswith("VEL")) and fn.endswith(".bin"):
            continue
        p = os.path.join(out, fn)
        if os.path.isdir(p):
            shutil.rmtree(p)
        else:
            os.remove(p)
    cdir = os.path.join(dest, "config")
    for fn in os.listdir(cdir):
        if fn not in ("config.txt", "poles.txt", "p_ref.bin"):
            os.remove(os.path.join(cdir, fn))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py OUTPUT_DIR [CASE ...]")
    out_root = os.path.abspath(sys.argv[1])
    rc_all = 0
    for case in (sys.argv[2:] or CASES):
        dest = os.path.join(out_root, case)
        if os.path.exists(dest):
            shutil.rmtree(dest)
        make_project(case, dest)
        rc = run_reference(dest)
        print(case, "reference exit code", rc)
        prune(dest, keep_slices=CASES[case].get("keep_slices", False))
        neutral_paths(dest)
        rc_all |= rc
    sys.exit(rc_all)
