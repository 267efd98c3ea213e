"""Generates the golden fixtures that pin the 2D legacy oracle (and the CUDA 2D legacy scheme) to
the reference's own 2D solver.

For each case it writes a small reference 2D project (a 2D OBJ with a `Boundary` polygon and
named obstacle polygons, config/config.txt, config/poles.txt, input/fit/<layer>.fit,
input/src/src.txt, input/rec/rec.txt), runs the reference 2D solver itself -- built from its own
sources by oracle/build_ref.sh into oracle/_ref/phases2D -- on it, answering its prompts with
"2" (WENO + SSP-RK3), "1" and "1" (2D-solver/core/main.cu:588-589, 680, 700), and keeps the inputs
plus the reference's outputs output/S.bin, output/oid.bin, output/pre_header.txt and
output/IR.bin (the pressure at the receiver node after every step).

    python tests/golden/make_golden_legacy2d.py OUT_DIR   # on a machine with a GPU; then copy
                                                          # OUT_DIR/<case> into tests/golden/<case>

The reference needs a CUDA GPU; the committed fixtures let the CPU tests check the oracle
without one.
"""
import json
import math
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _ngon(cx, cy, r, n):
    return [(cx + r * math.cos(2 * math.pi * k / n), cy + r * math.sin(2 * math.pi * k / n)) for k in range(n)]


CASES = {
    # a reflecting panel and a wedge of a second material; sPML on both y faces and x-high; fluid
    # up to the ghost rows, where the reference's ghost-row copy races with its stage update
    "l2d_panel": dict(L=(0.8, 0.5), h=0.005, t_max=0.0012, temp=22.0, cfl=0.2, pml=(1, 1, 1, 0),
                      polys=[("panel", [(0.40, 0.15), (0.46, 0.15), (0.46, 0.35), (0.40, 0.35)]),
                             ("wedge", [(0.55, 0.05), (0.70, 0.05), (0.62, 0.15)])],
                      fits={"panel": (0.82, [(171.9, 317.2), (-343.5, 3796.2)], [(-21.96, -42.35, 39.14, 348.0)]),
                            "wedge": (0.9, [(120.0, 900.0)], [])},
                      poles=(2, 1), src=(0.15, 0.25, 9.0), rec=(0.30, 0.26)),
    # a channel: solid walls over the bottom and top rows (so the reference's racing ghost-row copy
    # only ever copies never-written wall nodes) and a slanted barrier; sPML on x-low only
    "l2d_channel": dict(L=(0.6, 0.45), h=0.005, t_max=0.0016, temp=18.0, cfl=0.25, pml=(0, 0, 0, 1),
                        polys=[("wall", [(0.0, 0.0), (0.6, 0.0), (0.6, 0.035), (0.0, 0.035)]),
                               ("barrier", [(0.30, 0.10), (0.33, 0.09), (0.38, 0.30), (0.35, 0.31)]),
                               ("ceiling", [(0.0, 0.415), (0.6, 0.415), (0.6, 0.45), (0.0, 0.45)])],
                        fits={"wall": (0.95, [(40.0, 2500.0)], []),
                              "barrier": (0.7, [(250.0, 1500.0)], [(15.0, -30.0, 600.0, 1800.0)]),
                              "ceiling": (0.9, [], [(5.0, 8.0, 900.0, 2600.0)])},
                        poles=(1, 1), src=(0.12, 0.2, 9.0), rec=(0.45, 0.22)),
    # curved and repeated geometry: a 40-gon pillar, a second polygon of the same layer name (one
    # material for both), a 'g' group; solid floor and ceiling rows as in l2d_channel; sPML x-high
    "l2d_pillars": dict(L=(0.7, 0.5), h=0.005, t_max=0.0015, temp=20.0, cfl=0.3, pml=(0, 0, 1, 0),
                        polys=[("floor", [(0.0, 0.0), (0.7, 0.0), (0.7, 0.03), (0.0, 0.03)]),
                               ("pillar", _ngon(0.35, 0.25, 0.06, 40)),
                               ("pillar", [(0.52, 0.10), (0.58, 0.12), (0.55, 0.18)], "g"),
                               ("roof", [(0.0, 0.47), (0.7, 0.47), (0.7, 0.5), (0.0, 0.5)])],
                        fits={"floor": (0.95, [(40.0, 2500.0)], []),
                              "pillar": (0.75, [(200.0, 1200.0), (-80.0, 3000.0)], [(10.0, -20.0, 500.0, 2000.0)]),
                              "roof": (0.9, [], [(5.0, 8.0, 900.0, 2600.0)])},
                        poles=(2, 1), src=(0.12, 0.25, 9.0), rec=(0.25, 0.3)),
}


def write_project(case, dest, spec=None):
    """Writes the reference 2D project of CASES[case] (or of the given spec) into dest."""
    c = spec if spec is not None else CASES[case]
    os.makedirs(os.path.join(dest, "config"), exist_ok=True)
    for d in ("input/fit", "input/src", "input/rec", "output"):
        os.makedirs(os.path.join(dest, d), exist_ok=True)
    Lx, Ly = c["L"]
    lines = ["o Boundary", "v 0.000000 0.000000 0.0", "v %.6f 0.000000 0.0" % Lx, "v %.6f %.6f 0.0" % (Lx, Ly),
             "v 0.000000 %.6f 0.0" % Ly, "f 1 2 3 4"]
    nv = 4
    for poly in c["polys"]:
        name, pts, kind = poly[0], poly[1], (poly[2] if len(poly) > 2 else "o")
        lines.append("%s %s" % (kind, name))
        for x, y in pts:
            lines.append("v %.6f %.6f 0.0" % (x, y))
        lines.append("f " + " ".join(str(nv + k + 1) for k in range(len(pts))))
        nv += len(pts)
    with open(os.path.join(dest, "scene.obj"), "w") as f:
        f.write("\n".join(lines) + "\n")
    conf = [(c["h"], "grid spacing h [m]"), (c["t_max"], "maximum simulation time t_max [s]"),
            (1000.0, "cutoff frequency f_cutoff [Hz]"), (c["temp"], "temperature Temp [C]"),
            (c["cfl"], "Courant-Friedrich-Lewy number C_CFL"), (8, "number of poles for the ADE"),
            (c["pml"][0], "N PML [0,1]"), (c["pml"][1], "S PML [0,1]"), (c["pml"][2], "E PML [0,1]"),
            (c["pml"][3], "W PML [0,1]")]
    with open(os.path.join(dest, "config", "config.txt"), "w") as f:
        for v, what in conf:
            f.write("%s\t# %s\n" % (repr(v), what))
    with open(os.path.join(dest, "config", "poles.txt"), "w") as f:
        f.write("%d %d\n" % c["poles"])
    for name, (rinf, ks, ls) in c["fits"].items():
        with open(os.path.join(dest, "input", "fit", name + ".fit"), "w") as f:
            f.write("# R_inf K L\n%r %d %d\n# A_k zeta_k\n" % (rinf, len(ks), len(ls)))
            for a, z in ks:
                f.write("%r %r\n" % (a, z))
            f.write("# B_l C_l alpha_l beta_l\n")
            for b, cc, al, be in ls:
                f.write("%r %r %r %r\n" % (b, cc, al, be))
    with open(os.path.join(dest, "input", "src", "src.txt"), "w") as f:
        f.write("# pos_x pos_y value\n%r %r %r\n" % c["src"])
    with open(os.path.join(dest, "input", "rec", "rec.txt"), "w") as f:
        f.write("# pos_x pos_y\n%r %r\n" % c["rec"])
    with open(os.path.join(dest, "case.json"), "w") as f:
        json.dump(c, f, indent=1)


def run_reference(dest, exe):
    r = subprocess.run([exe, "scene.obj", "config/config.txt", "input/src/src.txt", "input/rec/rec.txt"],
                       cwd=dest, input="2\n1\n1\n", capture_output=True, text=True, timeout=600)
    with open(os.path.join(dest, "reference_stdout.txt"), "w") as f:
        f.write(r.stdout[-20000:])
        f.write(r.stderr[-5000:])
    if r.returncode != 0:
        raise RuntimeError("reference 2D solver failed (%d): %s" % (r.returncode, r.stderr[-2000:]))
    # the animation frames are not a fixture
    path = os.path.join(dest, "output", "pressure.bin")
    if os.path.exists(path):
        os.remove(path)


def run_reference_timed(dest, timeout=1800):
    """Runs the reference 2D solver on dest, stamping each stdout line with time.perf_counter();
    returns (returncode, [(t, line), ...]). The stamps of "Simulation start" and "Simulation time"
    bracket its time loop on the wall clock (its own figure is process CPU time, main.cu:888-891)."""
    import time
    exe = os.path.join(ROOT, "oracle", "_ref", "phases2D")
    cmd = [exe, "scene.obj", "config/config.txt", "input/src/src.txt", "input/rec/rec.txt"]
    if shutil.which("stdbuf"):
        cmd = ["stdbuf", "-oL"] + cmd  # line-buffered, so each line is stamped when it is printed
    stamped = []
    t_end = time.perf_counter() + timeout
    with subprocess.Popen(cmd, cwd=dest, stdin=subprocess.PIPE, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                          text=True, bufsize=1) as proc:
        proc.stdin.write("2\n1\n1\n")
        proc.stdin.close()
        for line in proc.stdout:
            stamped.append((time.perf_counter(), line))
            if time.perf_counter() > t_end:
                proc.kill()
                break
        rc = proc.wait(timeout=60)
    return rc, stamped


def main(out):
    exe = os.path.join(ROOT, "oracle", "_ref", "phases2D")
    if not os.path.exists(exe):
        raise SystemExit("build the reference first: oracle/build_ref.sh")
    for case in CASES:
        dest = os.path.join(out, case)
        if os.path.exists(dest):
            shutil.rmtree(dest)
        write_project(case, dest)
        run_reference(dest, exe)
        print("made", dest)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])
