"""Launch-shape autotuner (fz_autotune, fz_group_autotune, fz_set_kz_chunk): tuning mid-solve
leaves the solve exactly where it was, and the results do not depend on the tile depth. Every
comparison is bit for bit against an untuned run of the same steps, with a second source placed
inside the obstacle (a cell the stage kernels skip, whose stale output accumulates the source)."""
import numpy as np
import pytest

from tests.helpers import small_room

# the second source sits inside the obstacle of small_room ((9,7,5)-(14,12,9) in room cells)
SOURCES = np.array([[6, 6, 12], [14, 12, 10]], np.int32)


def _solver(cfg, precision="fp32", batch=1, steps=40):
    from fases_b200 import Solver, params
    s = Solver(params(h=cfg["h"], c=cfg["c"], rho=cfg["rho"], dt=cfg["dt"], pml=cfg["pml"],
                      pml_cells=cfg["pml_cells"], precision=precision, batch=batch))
    s.load_geometry(cfg["scene"].S, cfg["scene"].oid)
    m = cfg["materials"]
    s.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    s.set_sources(SOURCES, np.full(len(SOURCES), cfg["sval"][0]), cfg["src_opt"], u_s=cfg["u_s"])
    s.set_receivers(cfg["recs"], steps)
    if cfg["p0"] is not None:
        p0 = cfg["p0"] if batch == 1 else np.stack([cfg["p0"]] * batch)
        s.set_fields(p=p0)
    return s


def test_tuner_entry_points_check_arguments():
    from fases_b200 import _abi
    L = _abi.lib()
    assert L.fz_autotune(None, 3, None, None) == _abi.FZ_EINVAL
    assert L.fz_group_autotune(None, 3, None, None) == _abi.FZ_EINVAL
    assert L.fz_set_kz_chunk(None, 4) == _abi.FZ_EINVAL
    assert L.fz_set_z_schedule(None, None, 0) == _abi.FZ_EINVAL


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_tuning_mid_solve_changes_nothing(precision):
    cfg = small_room(seed=7, pml=(1, 0, 1, 0, 0, 1), steps=40)
    ref = _solver(cfg, precision)
    ref.run(40)
    ir_ref, f_ref = ref.ir(), ref.fields()
    ref.close()
    s = _solver(cfg, precision)
    s.run(13)
    depth, ms = s.autotune(reps=2)
    cur, heur = s.kz_chunk()
    assert depth == cur and depth >= 1 and heur >= 1 and ms > 0
    s.run(11)
    s.set_kz_chunk(5)  # an odd depth that leaves a short last chunk
    assert s.kz_chunk()[0] == 5
    s.run(7)
    nzi = s.shape[0] - 6
    sched = [nzi - 3, 2, 1] if nzi > 3 else [nzi]  # chunks of unequal length, longest first
    s.set_z_schedule(sched)
    assert s.z_schedule() == sched
    s.run(9)
    assert np.array_equal(s.ir(), ir_ref)
    for a, b in zip(s.fields(), f_ref):
        assert np.array_equal(a, b)
    s.close()


@pytest.mark.gpu
def test_tuning_batched_and_grouped_solves():
    from fases_b200 import Group
    cfg = small_room(seed=9, pml=(0, 0, 1, 0, 0, 0), steps=30)
    ref = _solver(cfg, batch=3, steps=30)
    ref.run(30)
    ir_ref = ref.ir()
    ref.close()
    b = _solver(cfg, batch=3, steps=30)
    b.run(10)
    b.autotune(reps=2)
    b.run(20)
    assert np.array_equal(b.ir(), ir_ref)
    b.close()
    rooms = [(26, 22, 18), (30, 20, 16), (20, 24, 22)]
    cfgs = [small_room(seed=30 + q, room=r, steps=30) for q, r in enumerate(rooms)]
    solos = []
    for c in cfgs:
        s = _solver(c, steps=30)
        s.run(30)
        solos.append(s.ir())
        s.close()
    members = [_solver(c, steps=30) for c in cfgs]
    with Group(members) as g:
        g.run(10)
        depth, ms = g.autotune(reps=2)
        assert depth >= 0 and ms > 0
        g.run(20)
        for s, r in zip(members, solos):
            assert np.array_equal(s.ir(), r)
    for s in members:
        s.close()
