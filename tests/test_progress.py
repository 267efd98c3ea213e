"""The progress protocol (fz_run_progress): slices of every_percent % of the run, one callback per
slice after a bounded wait, early stop on a nonzero return; results equal a plain fz_run."""
import numpy as np
import pytest

from tests.helpers import run_gpu, small_room


@pytest.mark.gpu
def test_progress_slices_and_early_stop():
    cfg = small_room(seed=31, steps=40)
    ref = run_gpu(cfg, "fp32")
    ir_ref = ref.ir()
    ref.close()

    s = run_gpu(cfg, "fp32", run=False)
    seen = []
    s.run_progress(40, lambda done, total: seen.append((done, total)), every_percent=25)
    assert seen == [(10, 40), (20, 40), (30, 40), (40, 40)]
    assert np.array_equal(s.ir(), ir_ref)
    s.close()

    s = run_gpu(cfg, "fp32", run=False)
    s.run_progress(40, lambda done, total: done >= 20, every_percent=25)
    assert s.steps_done() == 20
    s.close()
