"""CUDA stepper vs the FP64 CPU oracle on seeded small rooms (cPML, obstacle, six ADE walls,
PCS source, Gaussian pulse, receivers). Calls go through the C ABI (libfz.so via ctypes)."""
import numpy as np
import pytest

from tests.helpers import rel_l2, run_gpu, run_oracle, small_room

pytestmark = pytest.mark.gpu

# FP64 GPU vs FP64 oracle: same scheme, only the operation order differs.
TOL_FP64 = 1e-10
# FP32 GPU vs FP64 oracle, receiver traces, relative L2 (the plain-path accuracy target is 1e-5).
TOL_FP32_IR = 1e-5


def _first_mismatch(a, b, tol):
    d = np.abs(a - b)
    scale = np.max(np.abs(b)) + 1e-300
    idx = np.argwhere(d > tol * scale)
    return None if idx.size == 0 else (tuple(idx[0]), a[tuple(idx[0])], b[tuple(idx[0])])


@pytest.mark.parametrize("steps", [1, 3])
def test_fields_fp64_few_steps(steps):
    cfg = small_room(seed=1, steps=steps)
    s = run_gpu(cfg, "fp64")
    o = run_oracle(cfg)
    g = s.fields()
    r = o.fields()
    for name, a, b in zip("puvw", g, r):
        err = rel_l2(a, b)
        assert err < TOL_FP64, (name, err, _first_mismatch(a, b, 1e-9))


def test_ir_fp64_long():
    cfg = small_room(seed=2, steps=120)
    s = run_gpu(cfg, "fp64")
    o = run_oracle(cfg)
    ir_o, vel_o = o.ir()
    ir_g = s.ir()
    assert ir_g.shape == ir_o.shape
    assert rel_l2(ir_g, ir_o) < TOL_FP64
    vel_g = s.vel()
    assert rel_l2(vel_g, vel_o) < 1e-6  # VEL is returned as float32


def test_ir_fp32_vs_fp64_oracle():
    cfg = small_room(seed=3, steps=120)
    s = run_gpu(cfg, "fp32")
    o = run_oracle(cfg)
    ir_o, _ = o.ir()
    ir_g = s.ir()
    errs = [rel_l2(ir_g[r], ir_o[r]) for r in range(ir_o.shape[0])]
    assert max(errs) < TOL_FP32_IR, errs


def test_graph_and_direct_launches_agree():
    cfg = small_room(seed=4, steps=25)  # 2 graphs of 10 steps + 5 direct steps
    a = run_gpu(cfg, "fp32", graph=True)
    b = run_gpu(cfg, "fp32", graph=False)
    assert np.array_equal(a.ir(), b.ir())
    for x, y in zip(a.fields(), b.fields()):
        assert np.array_equal(x, y)


def test_prepared_graphs_give_the_same_solve():
    """fz_prepare instantiates the step graphs of both buffer parities without stepping: the solve
    after it (an odd first run, so both graphs are used) equals one that captured its graphs on
    the way, and preparing again after a tuning pass changes nothing either."""
    cfg = small_room(seed=14, steps=35)
    a = run_gpu(cfg, "fp32", run=False)
    a.prepare()
    assert a.steps_done() == 0
    a.run(5)
    a.autotune(reps=1)
    a.prepare()
    a.run(30)
    b = run_gpu(cfg, "fp32")
    assert np.array_equal(a.ir(), b.ir())
    for x, y in zip(a.fields(), b.fields()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


def test_no_pml_no_source_pulse_only():
    cfg = small_room(seed=5, pml=(0, 0, 0, 0, 0, 0), source=None, steps=40)
    s = run_gpu(cfg, "fp64")
    o = run_oracle(cfg)
    for a, b in zip(s.fields(), o.fields()):
        assert rel_l2(a, b) < TOL_FP64


def test_all_pml_faces():
    cfg = small_room(seed=6, room=(30, 30, 30), pml=(1, 1, 1, 1, 1, 1), pml_cells=5, obstacle=False, steps=40)
    s = run_gpu(cfg, "fp64")
    o = run_oracle(cfg)
    for a, b in zip(s.fields(), o.fields()):
        assert rel_l2(a, b) < TOL_FP64


def test_energy_matches_oracle():
    cfg = small_room(seed=7, steps=30)
    s = run_gpu(cfg, "fp64")
    o = run_oracle(cfg)
    assert abs(s.energy() - o.energy()) <= 1e-10 * abs(o.energy())


@pytest.mark.parametrize("K,L", [(3, 4), (5, 6), (0, 3)])
def test_pole_counts_beyond_two(K, L):
    # the band kernel keeps up to 2 (and up to 4) real poles and complex pairs in fixed-size
    # register arrays and takes a general loop above that: each form against the oracle, FP64 and FP32
    cfg = small_room(seed=40 + K, K=K, L=L, steps=60)
    o = run_oracle(cfg)
    ir_o, _ = o.ir()
    s64 = run_gpu(cfg, "fp64")
    assert rel_l2(s64.ir(), ir_o) < TOL_FP64
    for a, b in zip(s64.fields(), o.fields()):
        assert rel_l2(a, b) < TOL_FP64
    s32 = run_gpu(cfg, "fp32")
    ir_g = s32.ir()
    errs = [rel_l2(ir_g[r], ir_o[r]) for r in range(ir_o.shape[0])]
    assert max(errs) < TOL_FP32_IR, errs


def test_free_field_without_band_cells():
    # all air (no wall, no material: the band list is empty), cPML on every face, a pulse and a
    # PCS source; FP64 against the oracle and the receivers' traces
    from types import SimpleNamespace
    cfg = small_room(seed=9, room=(30, 28, 26), pml=(1, 1, 1, 1, 1, 1), pml_cells=5, obstacle=False, steps=50)
    shape = cfg["scene"].S.shape
    S = np.full(shape, 1.0, np.float32)
    oid = np.full(shape, 0xFF, np.uint8)
    cfg["scene"] = SimpleNamespace(S=S, oid=oid, shape=shape)
    cfg["materials"] = {k: np.asarray(v)[:1] for k, v in cfg["materials"].items()}
    s = run_gpu(cfg, "fp64")
    assert s.info()["n_band"] == 0
    o = run_oracle(cfg)
    ir_o, _ = o.ir()
    assert rel_l2(s.ir(), ir_o) < TOL_FP64
    for a, b in zip(s.fields(), o.fields()):
        assert rel_l2(a, b) < TOL_FP64
