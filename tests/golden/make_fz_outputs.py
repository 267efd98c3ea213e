"""Writes this library's outputs for the golden projects, for the post-processing test.

For each golden project (tests/golden/box_*), the project is loaded through the C ABI's project
loader (fz_load_project) on the reference's own cached geometry (output/S.bin, output/oid.bin),
stepped for the project's Nt steps in FP32, and its outputs are written in the reference's
formats: output/IR<r>_0.bin, output/VEL<r>_0.bin, output/header.txt (fz_write_outputs) and the
radiated reference pulse config/p_ref.bin (written by the loader). These land in
OUT_DIR/<case>/; copied into tests/golden/<case>/fz_output/, they let tests/test_allirs.py run the
reference's own post-processing (common/allIRs.py) on them on a machine without a GPU.

    python tests/golden/make_fz_outputs.py OUT_DIR     # on a machine with a GPU
"""
import os
import shutil
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CASES = ["box_pcs", "box_ricker", "box_sine", "box_poles"]


def write_case(case, out_root):
    from fases_b200 import Solver
    with tempfile.TemporaryDirectory() as tmp:
        proj = os.path.join(tmp, case)
        shutil.copytree(os.path.join(HERE, case), proj)
        shutil.rmtree(os.path.join(proj, "fz_output"), ignore_errors=True)
        pr = os.path.join(proj, "config", "p_ref.bin")
        if os.path.exists(pr):
            os.remove(pr)  # the reference's copy: the one kept below is the loader's own
        args = (os.path.join(proj, "scene.obj"), os.path.join(proj, "config", "config.txt"),
                os.path.join(proj, "src.txt"), os.path.join(proj, "rec.txt"))
        # the first load rebuilds the scene cache under this path; the reference's arrays are then
        # put back under that key, so the second load steps on the reference's own geometry
        Solver.from_project(*args)[0].close()
        for f in ("S.bin", "oid.bin"):
            shutil.copyfile(os.path.join(HERE, case, "output", f), os.path.join(proj, "output", f))
        s, nt = Solver.from_project(*args)
        s.run(nt)
        dest = os.path.join(out_root, case)
        os.makedirs(os.path.join(dest, "config"), exist_ok=True)
        s.write_outputs(os.path.join(dest, "output"), 0, "./scene.obj")
        s.close()
        if os.path.exists(pr):
            shutil.copyfile(pr, os.path.join(dest, "config", "p_ref.bin"))
    return dest


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_fz_outputs.py OUTPUT_DIR")
    root = os.path.abspath(sys.argv[1])
    for c in CASES:
        print(c, "->", write_case(c, root))
