"""Command-line drop-in for the FVM part of `fases3D` (3D-solver/core/main3D.cu:26-1449):

    python -m fases_b200.fz3d <scene.obj> <config.txt> <src.txt> <rec.txt> [--fp64]

Reads the same project files through libfz.so (fz_load_project), runs the Nt time steps of the
configuration on the GPU, prints the integer progress lines the GUI parses ("NN%" every 5 %,
functions3D.cuh:1431-1439, parsed by the regex (\\d+)\\s*% in common/gui.py:6713), and writes
output/IR<r>_<s>.bin, output/VEL<r>_<s>.bin and output/header.txt in the reference formats
(config/p_ref.bin and output/pre_header.txt are written by the loader). Geometry comes from the
project's scene cache (output/S.bin, output/oid.bin, output/scene_cache.txt).
"""
import os
import sys
import time

from .solver import Solver


def _project_output_dir(config_path):
    cfg = os.path.abspath(config_path)
    cdir = os.path.dirname(cfg)
    if os.path.basename(cfg) == "config.txt" and os.path.basename(cdir) == "config":
        return os.path.join(os.path.dirname(cdir), "output")
    return os.path.join(os.getcwd(), "output")


def _src_index(config_path):
    vals = []
    for line in open(config_path):
        line = line.split("#", 1)[0].strip()
        if not line:
            continue
        try:
            vals.append(float(line.split()[0]))
        except ValueError:
            continue
    return int(vals[17]) if len(vals) > 17 else 0


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    if len(argv) < 4:
        print("Usage: fz3d <scene> <config> <src> <rec> [--fp64]")
        return 1
    precision = "fp64" if "--fp64" in argv else "fp32"
    scene, config, src, rec = argv[:4]
    s, nt = Solver.from_project(scene, config, src, rec, precision=precision)
    print(f"[OK] Will now start {nt} iterations", flush=True)
    t0 = time.perf_counter()
    s.run_progress(nt, lambda done, total: print("%d%%" % int(100.0 * done / total + 0.5), flush=True), 5)
    print("[OK] Simulation time: %f min" % ((time.perf_counter() - t0) / 60.0), flush=True)
    out = _project_output_dir(config)
    s.write_outputs(out, _src_index(config), os.path.abspath(scene))
    print("[OK] Printed header.txt for plot.py", flush=True)
    s.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
