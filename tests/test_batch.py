"""Batched solves (several source positions over one room in the same launches) and groups of
rooms advanced as one CUDA graph: every member must reproduce, bit for bit, the solve it stands
for when run alone, and the FP64 members must match the oracle run with their own source."""
import numpy as np
import pytest

from tests.helpers import rel_l2, run_oracle, small_room

SOURCES = np.array([[6, 6, 12], [18, 14, 5], [12, 17, 9]], np.int32)


def _solver(cfg, precision, batch=1, src_rows=None, members=None, steps=None, p0=None):
    from fases_b200 import Solver, params
    steps = cfg["steps"] if steps is None else steps
    s = Solver(params(h=cfg["h"], c=cfg["c"], rho=cfg["rho"], dt=cfg["dt"], pml=cfg["pml"],
                      pml_cells=cfg["pml_cells"], precision=precision, batch=batch))
    s.load_geometry(cfg["scene"].S, cfg["scene"].oid)
    m = cfg["materials"]
    s.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    rows = SOURCES if src_rows is None else src_rows
    s.set_sources(rows, np.full(len(rows), cfg["sval"][0]), cfg["src_opt"], u_s=cfg["u_s"])
    if members is not None:
        s.set_source_members(members)
    s.set_receivers(cfg["recs"], steps)
    if p0 is not None:
        s.set_fields(p=p0)
    return s


def test_batch_parameter_is_validated():
    import ctypes

    from fases_b200 import _abi, params
    p = params(batch=-2)
    h = ctypes.c_void_p()
    assert _abi.lib().fz_create(ctypes.byref(p), ctypes.byref(h)) == _abi.FZ_EINVAL
    assert "batch" in _abi.last_error()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batched_members_equal_single_source_runs(precision):
    cfg = small_room(seed=11, pml=(1, 0, 1, 0, 0, 1), steps=37, pulse=False)
    nb = len(SOURCES)
    b = _solver(cfg, precision, batch=nb, members=np.arange(nb))
    b.run(cfg["steps"])
    ir_b = b.ir()
    f_b = b.fields()
    assert ir_b.shape == (nb, len(cfg["recs"]), cfg["steps"])
    for m in range(nb):
        s = _solver(cfg, precision, src_rows=SOURCES[m:m + 1])
        s.run(cfg["steps"])
        assert np.array_equal(s.ir(), ir_b[m]), (precision, m)
        for a, fb in zip(s.fields(), f_b):
            assert np.array_equal(a, fb[m]), (precision, m)
        s.close()
    if precision == "fp64":
        for m in range(nb):
            c = dict(cfg, src=SOURCES[m:m + 1])
            ir_o, _ = run_oracle(c).ir()
            for r in range(ir_o.shape[0]):
                assert rel_l2(ir_b[m, r], ir_o[r]) < 1e-10, (m, r)
    b.close()


@pytest.mark.gpu
def test_batched_shared_source_and_initial_fields():
    """Sources with member -1 act in every member; initial fields are set per member."""
    cfg = small_room(seed=12, steps=24)
    nb = 2
    rng = np.random.default_rng(3)
    p0 = np.stack([cfg["p0"], cfg["p0"] * rng.uniform(0.5, 1.5)])
    b = _solver(cfg, "fp32", batch=nb, src_rows=SOURCES[:1], p0=p0)
    b.run(cfg["steps"])
    ir_b = b.ir()
    for m in range(nb):
        s = _solver(cfg, "fp32", src_rows=SOURCES[:1], p0=p0[m])
        s.run(cfg["steps"])
        assert np.array_equal(s.ir(), ir_b[m]), m
        s.close()
    b.close()


@pytest.mark.gpu
def test_group_members_equal_solo_runs():
    from fases_b200 import Group
    rooms = [(26, 22, 18), (30, 20, 16), (20, 24, 22)]
    steps = 23  # two graphs of 10 steps plus 3 single steps
    cfgs = [small_room(seed=20 + q, room=r, steps=steps) for q, r in enumerate(rooms)]
    solos = []
    for c in cfgs:
        s = _solver(c, "fp32", src_rows=SOURCES[:1], p0=c["p0"])
        s.run(steps)
        solos.append(s.ir())
        s.close()
    members = [_solver(c, "fp32", src_rows=SOURCES[:1], p0=c["p0"]) for c in cfgs]
    with Group(members) as g:
        assert g.shared_launches()  # 3D rooms of one precision: shared launches
        g.run(steps)
        for s, ref in zip(members, solos):
            assert s.steps_done() == steps
            assert np.array_equal(s.ir(), ref)
        # a member stays usable alone after group runs
        members[1].run(3)
        assert members[1].steps_done() == steps + 3
    for s in members:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_shared_launch_group_of_unlike_rooms_equals_solo_runs(precision):
    """The shared-launch group path over rooms that differ in every way its tables carry: sizes
    (ragged tiles), cPML faces and thickness, pole counts (the group then takes the general band
    form), a room without obstacles, a batched member with two source positions; the members start
    at different steps, and the group runs ungraphed steps, a tuning pass and a graph."""
    from fases_b200 import Group
    steps = 21
    specs = [dict(seed=40, room=(37, 21, 19), pml=(0, 1, 0, 1, 0, 1), pml_cells=4),
             dict(seed=41, room=(26, 22, 18), pml=(1, 1, 1, 1, 1, 1), pml_cells=5, K=5, L=3),
             dict(seed=42, room=(30, 20, 16), pml=(0, 0, 0, 0, 0, 0), obstacle=False, K=1, L=1),
             dict(seed=43, room=(24, 24, 22), pml=(0, 0, 1, 0, 0, 0))]
    cfgs = [small_room(steps=steps, **kw) for kw in specs]
    batch = [1, 1, 1, 2]

    def make(q):
        c = cfgs[q]
        if batch[q] > 1:
            return _solver(c, precision, batch=2, src_rows=SOURCES[:2], members=np.arange(2))
        return _solver(c, precision, src_rows=SOURCES[:1], p0=c["p0"])

    solos = []
    for q in range(len(cfgs)):
        s = make(q)
        s.run(steps)
        solos.append(s.ir())
        s.close()
    members = [make(q) for q in range(len(cfgs))]
    members[0].run(3)  # members may start at different steps (and buffer parities)
    with Group(members) as g:
        assert g.shared_launches()
        g.run(8)         # graph-free steps of the group
        g.autotune(reps=1)
        g.run(10)        # one 10-step graph
        for s in members[1:]:
            s.run(3)     # the others finish alone
        for q, s in enumerate(members):
            assert s.steps_done() == steps
            assert np.array_equal(s.ir(), solos[q]), q
    for s in members:
        s.close()


@pytest.mark.gpu
def test_group_with_a_sliced_member_uses_graph_branches():
    from fases_b200 import Group
    cfgs = [small_room(seed=50 + q, steps=12) for q in range(2)]
    solo = _solver(cfgs[1], "fp32", src_rows=SOURCES[:1], p0=cfgs[1]["p0"])
    solo.run(12)
    ref = solo.ir()
    solo.close()
    members = [_solver(c, "fp32", src_rows=SOURCES[:1], p0=c["p0"]) for c in cfgs]
    members[0].set_slices(10, 10, 9, 4, 4)
    with Group(members) as g:
        assert not g.shared_launches()
        g.run(12)
        assert np.array_equal(members[1].ir(), ref)
    for s in members:
        s.close()


@pytest.mark.gpu
def test_group_larger_than_one_stage_launch_equals_solo_runs():
    """More members than one stage launch covers (its TMA descriptors are kernel parameters): the
    stage kernels run as several launches over member chunks, the band and receiver kernels as one."""
    from fases_b200 import Group
    steps = 12
    rooms = [(20 + (q % 5), 18 + (q % 3), 15 + (q % 4)) for q in range(30)]
    cfgs = [small_room(seed=60 + q, room=r, steps=steps, obstacle=False) for q, r in enumerate(rooms)]
    src = np.array([[6, 6, 7]], np.int32)
    solos = []
    for c in cfgs:
        s = _solver(c, "fp32", src_rows=src, p0=c["p0"])
        s.run(steps)
        solos.append(s.ir())
        s.close()
    members = [_solver(c, "fp32", src_rows=src, p0=c["p0"]) for c in cfgs]
    with Group(members) as g:
        assert g.shared_launches() and g.branches() == 4  # the default for 30 rooms
        g.run(4)
        g.set_branches(1)  # the launch arrangement changes the launch order, not the results
        assert g.branches() == 1
        g.run(4)
        g.set_branches(-1)  # each member's own launches as graph branches
        assert not g.shared_launches() and g.branches() == 30
        g.run(steps - 8)
        for s, ref in zip(members, solos):
            assert np.array_equal(s.ir(), ref)
    for s in members:
        s.close()
