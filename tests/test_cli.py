"""The fases3D-compatible command line (python -m fases_b200.fz3d) on a copy of a golden project
with no scene cache: it builds the geometry from the OBJ, prints the progress lines the GUI parses,
and writes the reference's output files (IR/VEL traces matching the reference solver's, header.txt,
animation slices); --estimate prints the [MEM] pre-flight line."""
import os
import re
import shutil
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _project(tmp_path, case="box_pcs"):
    proj = str(tmp_path / case)
    shutil.copytree(os.path.join(HERE, "golden", case), proj)
    for f in ("S.bin", "oid.bin", "scene_cache.txt", "header.txt"):
        os.remove(os.path.join(proj, "output", f))
    ref = os.path.join(proj, "reference_output")
    shutil.move(os.path.join(proj, "output"), ref)
    os.makedirs(os.path.join(proj, "output"))
    return proj, ref


def _run(proj, *extra):
    env = dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    cmd = [sys.executable, "-m", "fases_b200.fz3d", "scene.obj", "config/config.txt", "src.txt", "rec.txt", *extra]
    return subprocess.run(cmd, cwd=proj, env=env, capture_output=True, text=True, timeout=600)


def test_cli_usage_message():
    env = dict(os.environ, PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, "-m", "fases_b200.fz3d"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "Usage" in r.stdout


@pytest.mark.gpu
def test_cli_runs_a_project_without_cache(tmp_path):
    proj, ref = _project(tmp_path)
    r = _run(proj)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    pct = [int(m.group(1)) for m in re.finditer(r"^(\d+)%$", r.stdout, re.M)]
    assert pct and pct[-1] == 100 and pct == sorted(pct)
    out = os.path.join(proj, "output")
    for f in ("S.bin", "oid.bin", "scene_cache.txt", "header.txt", "pressureX.bin", "Iz_Y.bin"):
        assert os.path.exists(os.path.join(out, f)), f
    for rr in range(3):
        a = np.fromfile(os.path.join(out, f"IR{rr}_0.bin"), np.float32)
        b = np.fromfile(os.path.join(ref, f"IR{rr}_0.bin"), np.float32)
        assert a.shape == b.shape
        assert np.linalg.norm(a - b) <= 2e-5 * np.linalg.norm(b)
    hdr = open(os.path.join(out, "header.txt")).read().split()
    assert int(hdr[7]) > 0 and int(hdr[8]) >= 1  # frames and anim_step of the slices
    nx, ny, nz = (int(x) for x in hdr[:3])
    assert os.path.getsize(os.path.join(out, "pressureX.bin")) == int(hdr[7]) * ny * nz * 4
    # the estimate pass
    e = _run(proj, "--estimate")
    assert e.returncode == 0
    mem = [ln for ln in e.stdout.splitlines() if ln.startswith("[MEM]")]
    assert mem and "voxels=%d" % (nx * ny * nz) in mem[0]
    assert "[OK] estimate: V =" in e.stdout


def test_stale_outputs_are_purged_like_the_reference(tmp_path):
    # main3D.cu:170-216: slices and headers go, every IR/VEL/HIR/HRT/ARR bin goes; with
    # --keep-other-sources only this source's bins go; the scene cache stays
    from fases_b200.fz3d import purge_outputs
    out = tmp_path / "output"
    out.mkdir()
    names = ["IR0_0.bin", "IR1_0.bin", "IR0_1.bin", "VEL0_1.bin", "HIR0_1_125.bin", "HRT2_0_250.bin", "ARR1_1.bin",
             "pressureX.bin", "Iy_X.bin", "header.txt", "pre_header.txt", "S.bin", "oid.bin", "scene_cache.txt",
             "notes.txt"]
    for n in names:
        (out / n).write_bytes(b"x")
    purge_outputs(str(out), 1, keep_other_sources=True)
    left = sorted(p.name for p in out.iterdir())
    assert left == sorted(["IR0_0.bin", "IR1_0.bin", "HRT2_0_250.bin", "S.bin", "oid.bin", "scene_cache.txt",
                           "notes.txt"])
    purge_outputs(str(out), 1)
    left = sorted(p.name for p in out.iterdir())
    assert left == ["S.bin", "notes.txt", "oid.bin", "scene_cache.txt"]


def test_geometric_acoustics_flags_are_refused():
    from fases_b200.fz3d import main
    assert main(["a.obj", "c.txt", "s.txt", "r.txt", "--ga-only"]) == 2
