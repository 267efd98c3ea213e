"""Health word (failure detection without a GPU fault): a non-finite value injected through the
API into the state reaches a receiver and makes the next wait return FZ_ENONFINITE; the full-state
scan (fz_check_health) counts non-finite values; a new state from fz_set_fields clears the word."""
import ctypes

import numpy as np
import pytest

from fases_b200 import FzError, _abi
from tests.helpers import run_gpu, small_room


def test_health_entry_point_checks_arguments():
    assert _abi.lib().fz_check_health(None, None) == _abi.FZ_EINVAL


@pytest.mark.gpu
def test_nonfinite_state_is_reported_and_cleared():
    cfg = small_room(seed=71, steps=20)
    s = run_gpu(cfg, "fp32", run=False)
    assert s.check_health() == 0
    p_bad = cfg["p0"].copy()
    i, j, k = cfg["recs"][0]
    p_bad[k, j, i] = np.nan  # a blow-up, injected on the host
    s.set_fields(p=p_bad)
    n = ctypes.c_int64()
    assert _abi.lib().fz_check_health(s._h, ctypes.byref(n)) == _abi.FZ_ENONFINITE
    assert n.value >= 1
    with pytest.raises(FzError) as ei:
        s.run(3)
    assert ei.value.code == _abi.FZ_ENONFINITE
    # a clean state starts over
    s.set_fields(p=cfg["p0"])
    s.run(5)
    assert s.check_health() == 0
    ir = s.ir()
    assert ir.shape[1] == 8 and np.all(np.isfinite(ir[:, 3:]))  # the 3 blown-up samples are kept
    s.close()
