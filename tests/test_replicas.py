"""Replica plumbing of bench.py --gpus N (fases_b200.replicas) on CPU with gloo, world size 2: the
slowest rank's time is the job's, the whole-job rate counts every rank's units, and a barrier holds
the ranks together. One process per rank, rendezvous on 127.0.0.1."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from fases_b200.replicas import Replicas
    rep = Replicas(backend="gloo", timeout_s=60)
    rep.barrier()
    t = 1.0 + rank  # rank 1 is the slow one
    out[rank] = (rep.max(t), rep.aggregate_rate(100.0, t), rep.world, rep.rank)
    rep.barrier()
    rep.close()


def test_replicas_gloo_world_two():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(2):
        mx, rate, world, rank = res[r]
        assert world == 2 and rank == r
        assert mx == pytest.approx(2.0)
        assert rate == pytest.approx(2 * 100.0 / 2.0)


def test_single_process_needs_no_group():
    from fases_b200.replicas import Replicas
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        os.environ.pop(k, None)
    rep = Replicas()
    assert rep.pg is None and rep.world == 1
    assert rep.max(3.5) == 3.5
    assert rep.aggregate_rate(10, 2.0) == 5.0
    rep.barrier()
    rep.close()
