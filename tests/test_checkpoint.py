"""Checkpoint / resume (fz_state_save / fz_state_load): a solver that loads a state saved after 30
steps and runs 25 more gives, bit for bit, the receiver traces (all 55 samples) and fields of the
solver that ran 55 steps straight; a solver of another configuration, or with other physics (time
step, materials, cPML thickness), refuses the state."""
import numpy as np
import pytest

from fases_b200 import FzError, _abi
from tests.helpers import run_gpu, small_room


def test_state_entry_points_check_arguments():
    L = _abi.lib()
    assert L.fz_state_bytes(None, None) == _abi.FZ_EINVAL
    assert L.fz_state_save(None, None, 0) == _abi.FZ_EINVAL
    assert L.fz_state_load(None, None, 0) == _abi.FZ_EINVAL


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_resume_continues_bit_for_bit(precision, tmp_path):
    cfg = small_room(seed=81, pml=(1, 0, 1, 0, 0, 0), steps=55)
    a = run_gpu(cfg, precision, run=False)
    a.run(30)
    fields30 = a.fields()
    path = str(tmp_path / "state.bin")
    state = a.save_state(path)
    a.run(25)
    ir_a, f_a = a.ir(), a.fields()
    a.close()

    b = run_gpu(cfg, precision, run=False)
    b.load_state(path)
    assert b.steps_done() == 30
    for x, y in zip(b.fields(), fields30):
        assert np.array_equal(x, y)
    b.run(25)
    assert np.array_equal(b.ir(), ir_a)
    for x, y in zip(b.fields(), f_a):
        assert np.array_equal(x, y)
    b.close()

    # a solver with other receivers (and so another state layout) refuses it
    other = dict(cfg, recs=cfg["recs"][:2])
    c = run_gpu(other, precision, run=False)
    with pytest.raises(FzError) as ei:
        c.load_state(state)
    assert ei.value.code == _abi.FZ_EINVAL
    c.close()

    # so do solvers with the same shapes but other physics: another time step, another material
    # coefficient, another cPML thickness
    mats = {k: np.array(v, dtype=np.float64, copy=True) for k, v in cfg["materials"].items()}
    mats["A"] = mats["A"] * 1.01
    for other, what in ((dict(cfg, dt=cfg["dt"] * 0.9), ("physics",)), (dict(cfg, materials=mats), ("physics",)),
                        (dict(cfg, pml_cells=cfg["pml_cells"] - 1), ("configuration", "wrong size"))):
        c = run_gpu(other, precision, run=False)
        with pytest.raises(FzError) as ei:
            c.load_state(state)
        assert ei.value.code == _abi.FZ_EINVAL
        assert any(w in str(ei.value) for w in what), str(ei.value)
        c.close()
