"""Seeded random rooms against the FP64 oracle: room sizes that leave ragged tiles in x and y, any
subset of cPML faces with a random thickness, 0-2 obstacles, random pole counts, one or two PCS
sources, a Gaussian pulse, and a random stage-kernel tile depth (so z chunks start and end on
every kind of plane). FP64 solves must match the oracle to 1e-10 rel-L2 (fields and traces) and
FP32 solves its traces to 1e-5."""
import numpy as np
import pytest

from tests.helpers import rel_l2, run_oracle, small_room

pytestmark = pytest.mark.gpu


def _case(seed):
    rng = np.random.default_rng(1000 + seed)
    room = tuple(int(x) for x in rng.integers(17, 41, size=3))
    pml_cells = int(rng.integers(3, 6))
    pml = tuple(int(x) for x in (rng.random(6) < 0.4))
    if 2 * pml_cells + 6 > min(room) + 6:
        pml = (0, 0, 0, 0, 0, 0)
    K, L = int(rng.integers(0, 4)), int(rng.integers(0, 4))
    steps = int(rng.integers(20, 45))
    cfg = small_room(seed=seed, room=room, pml=pml, pml_cells=pml_cells, obstacle=bool(rng.random() < 0.6),
                     K=K, L=L, steps=steps)
    # keep the source and receivers inside this room (small_room places them for 26 x 22 x 18)
    lim = np.array(room) + 2
    cfg["src"] = np.minimum(cfg["src"], lim - 4).astype(np.int32)
    cfg["recs"] = np.minimum(cfg["recs"], lim - 4).astype(np.int32)
    p0 = cfg["p0"]
    if p0 is not None:
        p0 = p0.copy()
        p0[cfg["scene"].S < cfg["h"]] = 0.0
        cfg["p0"] = p0
    depth = int(rng.integers(1, room[2] + 1))
    return cfg, depth


def _run(cfg, precision, depth):
    from fases_b200 import Solver, params
    s = Solver(params(h=cfg["h"], c=cfg["c"], rho=cfg["rho"], dt=cfg["dt"], pml=cfg["pml"],
                      pml_cells=cfg["pml_cells"], precision=precision))
    s.load_geometry(cfg["scene"].S, cfg["scene"].oid)
    m = cfg["materials"]
    s.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    s.set_sources(cfg["src"], cfg["sval"], cfg["src_opt"], u_s=cfg["u_s"])
    s.set_receivers(cfg["recs"], cfg["steps"])
    if cfg["p0"] is not None:
        s.set_fields(p=cfg["p0"])
    s.set_kz_chunk(depth)
    s.run(cfg["steps"])
    return s


@pytest.mark.parametrize("seed", range(16))
def test_random_room_matches_oracle(seed):
    cfg, depth = _case(seed)
    o = run_oracle(cfg)
    ir_o, _ = o.ir()
    s = _run(cfg, "fp64", depth)
    assert rel_l2(s.ir(), ir_o) < 1e-10, (seed, cfg["scene"].S.shape, cfg["pml"], depth)
    for a, b in zip(s.fields(), o.fields()):
        assert rel_l2(a, b) < 1e-10, (seed, depth)
    s.close()
    s = _run(cfg, "fp32", depth)
    ir = s.ir()
    for r in range(ir_o.shape[0]):
        if np.linalg.norm(ir_o[r]) > 0:
            assert rel_l2(ir[r], ir_o[r]) < 1e-5, (seed, r, depth)
    s.close()
