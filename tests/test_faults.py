"""Host-side fault injection on the project loader and the adjoint: every fault is made on the host
(a file that is missing, truncated or malformed, a receiver outside the room, a memory need larger
than the device), and each must come back as a status code with a message -- no exit(), no device
fault. The reference exits from inside read_fit_file (common/filterABC.h:24-29, 44-48) and reads
config lines it may not have (main3D.cu:1193-1199); the loader here returns FZ_EIO / FZ_EPARSE /
FZ_EINVAL instead. A scene cache whose arrays are shorter than its key says is rebuilt.

GPU-marked: the loader builds the scene and creates the solver on the device."""
import os

import numpy as np
import pytest

from tests.golden import make_golden as mg

pytestmark = pytest.mark.gpu

SPEC = dict(room=(0.8, 0.6, 0.5), h=0.05, t_max=0.004, f_in=250.0, temp=20.0, cfl=0.5, pml=(0, 0, 1, 0, 0, 0),
            obstacles=[((0.3, 0.2, 0.2), (0.45, 0.35, 0.3))], src_opt=0, glob_f=100.0, src=[(0.2, 0.2, 0.2, 90.0)],
            rec=[(0.6, 0.4, 0.3), (0.5, 0.45, 0.25)], seed=5, open_wall=1, frames=10)


def _project(tmp_path):
    proj = str(tmp_path / "proj")
    mg.make_project("faults", proj, spec=SPEC)
    return proj


def _load(proj):
    from fases_b200 import Solver
    return Solver.from_project(os.path.join(proj, "scene.obj"), os.path.join(proj, "config", "config.txt"),
                               os.path.join(proj, "src.txt"), os.path.join(proj, "rec.txt"))


def _expect(proj, code, fragment):
    from fases_b200 import _abi
    with pytest.raises(_abi.FzError) as ex:
        _load(proj)
    assert ex.value.code == code, str(ex.value)
    assert fragment in str(ex.value), str(ex.value)


def test_intact_project_loads(tmp_path):
    proj = _project(tmp_path)
    s, nt = _load(proj)
    s.run(5)
    assert s.ir().shape == (2, 5)
    s.close()


def test_short_config_is_a_parse_error(tmp_path):
    from fases_b200 import _abi
    proj = _project(tmp_path)
    cfg = os.path.join(proj, "config", "config.txt")
    lines = open(cfg).read().splitlines()[:8]
    open(cfg, "w").write("\n".join(lines) + "\n")
    _expect(proj, _abi.FZ_EPARSE, "at least 12 values")


def test_missing_poles_file(tmp_path):
    from fases_b200 import _abi
    proj = _project(tmp_path)
    os.remove(os.path.join(proj, "config", "poles.txt"))
    _expect(proj, _abi.FZ_EIO, "poles")


@pytest.mark.parametrize("fault", ["missing", "letters", "too_many_poles", "short_rows"])
def test_fit_file_faults(tmp_path, fault):
    from fases_b200 import _abi
    proj = _project(tmp_path)
    fit = os.path.join(proj, "input", "fit", "x_lo.fit")
    if fault == "missing":
        os.remove(fit)
        _expect(proj, _abi.FZ_EIO, "x_lo.fit")
        return
    text = open(fit).read().splitlines()
    data = [ln for ln in text if ln.strip() and not ln.lstrip().startswith("#")]
    if fault == "letters":
        open(fit, "w").write("R_inf is not a number\n")
        _expect(proj, _abi.FZ_EPARSE, "R_inf")
    elif fault == "too_many_poles":
        # K larger than poles.txt's K_m (2)
        open(fit, "w").write("\n".join([data[0], "3 2"] + data[2:]) + "\n")
        _expect(proj, _abi.FZ_EPARSE, "K_local")
    else:
        # the complex-pair rows cut short
        open(fit, "w").write("\n".join(data[:-1]) + "\n")
        _expect(proj, _abi.FZ_EPARSE, "B_l C_l alpha_l beta_l")


def test_missing_source_file_and_receiver_outside(tmp_path):
    from fases_b200 import _abi
    proj = _project(tmp_path)
    os.rename(os.path.join(proj, "src.txt"), os.path.join(proj, "src_moved.txt"))
    _expect(proj, _abi.FZ_EIO, "sources")
    os.rename(os.path.join(proj, "src_moved.txt"), os.path.join(proj, "src.txt"))
    with open(os.path.join(proj, "rec.txt"), "a") as f:
        f.write("25.0 0.3 0.3\n")
    _expect(proj, _abi.FZ_EINVAL, "outside")


def test_truncated_scene_cache_is_rebuilt(tmp_path):
    proj = _project(tmp_path)
    s, _ = _load(proj)  # builds and writes the cache
    s.run(8)
    ir_ref = s.ir()
    s.close()
    out = os.path.join(proj, "output")
    assert os.path.exists(os.path.join(out, "scene_cache.txt"))
    S_full = np.fromfile(os.path.join(out, "S.bin"), np.float32)
    with open(os.path.join(out, "S.bin"), "r+b") as f:
        f.truncate(S_full.nbytes // 2)
    s, _ = _load(proj)  # same key, short array: rebuilt, not read past its end
    s.run(8)
    assert np.array_equal(s.ir(), ir_ref)
    s.close()
    assert np.array_equal(np.fromfile(os.path.join(out, "S.bin"), np.float32), S_full)


def test_adjoint_memory_need_beyond_the_device(tmp_path):
    from fases_b200 import _abi
    proj = _project(tmp_path)
    s, nt = _load(proj)
    info = s.info()
    # ask for a segment far longer than device memory can hold: refused before any allocation
    target = np.zeros((2, 2_000_000), np.float64)
    s2 = _make_long(proj, 2_000_000)
    with pytest.raises(_abi.FzError) as ex:
        s2.misfit_gradient(target, nsteps=2_000_000, segment_steps=2_000_000)
    assert ex.value.code == _abi.FZ_ENOMEM and "MiB" in str(ex.value)
    # the handle stays usable
    s2.run(3)
    assert s2.steps_done() == 3
    s2.close()
    s.close()
    assert info["n_band"] > 0


def _make_long(proj, capacity):
    """The project's room as a plain solver with receivers able to hold `capacity` samples."""
    from fases_b200 import Solver, params
    S = np.fromfile(os.path.join(proj, "output", "S.bin"), np.float32)
    oid = np.fromfile(os.path.join(proj, "output", "oid.bin"), np.uint8)
    dims = [int(x) for x in open(os.path.join(proj, "output", "scene_cache.txt")).read().splitlines()[1].split()[:3]]
    Nx, Ny, Nz = dims
    s = Solver(params(h=SPEC["h"], pml=(0, 0, 1, 0, 0, 0), pml_cells=4))
    s.load_geometry(S.reshape(Nz, Ny, Nx), oid.reshape(Nz, Ny, Nx))
    nm = int(oid[oid != 0xFF].max()) if np.any(oid != 0xFF) else 1
    s.set_materials(np.full(nm, 0.5))
    s.set_receivers(np.array([[Nx // 2, Ny // 2, Nz // 2], [Nx // 2 + 1, Ny // 2, Nz // 2]], np.int32), capacity)
    return s
