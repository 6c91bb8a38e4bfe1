"""Independent systems across ranks (sfr3d_b200/sharding.py): the
assignment, and a world-size-2 gloo run whose gathered results equal the
single-process ones.  The per-rank solve here is the oracle (the checker,
on the CPU); on GPUs it is a GpuBatch of the rank's share."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from sfr3d_b200 import sharding as SH


def test_plan_covers_every_system_once_and_balances():
    rng = np.random.default_rng(3)
    work = list(rng.lognormal(0.0, 1.5, 64))
    for world in (1, 2, 3, 4, 8):
        shares = SH.plan(work, world)
        flat = sorted(i for s in shares for i in s)
        assert flat == list(range(64))
        ld = SH.loads(work, shares)
        # LPT bound: no rank above the mean plus the largest single job
        assert max(ld) <= sum(work) / world + max(work) + 1e-9
    assert SH.plan(work, 4) == SH.plan(list(work), 4)  # deterministic


def test_plan_edge_cases():
    assert SH.plan([], 3) == [[], [], []]
    assert SH.plan([5.0], 2) == [[0], []]
    assert SH.plan([1.0, 1.0], 2) == [[0], [1]]  # ties go to the lower rank
    with pytest.raises(ValueError):
        SH.plan([1.0], 0)
    with pytest.raises(ValueError):
        SH.plan([float("nan")], 2)


def test_estimated_work_grows_with_size():
    assert SH.estimated_work(1000, 6000) < SH.estimated_work(8000, 48000)
    assert SH.estimated_work(1000, 6000, 10) == (12 * 6000 + 112 * 1000) * 10


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _systems():
    from sfr3d_b200 import systems as S
    return S.poisson_batch(6, 4, 9, seed=11)


def _oracle_solve(batch):
    from oracle import oracle as O
    out = []
    for s in batch:
        r = O.pcg(O.CSRD, True, s.ia, s.ja, s.al, s.ad, s.b[0], tol=1e-10)
        out.append((r.x, r.iters))
    return out


def _rank(rank, world, port, result_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        systems = _systems()
        work = [SH.estimated_work(s.neq, s.nnz_full) for s in systems]
        shares = SH.plan(work, world)
        pairs = SH.solve_share(systems, shares[rank], _oracle_solve)
        res = SH.gather(pairs, len(systems))
        if rank == 0:
            np.savez(result_path, *[r[0] for r in res], iters=np.array([r[1] for r in res]))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_gather_equals_single_process(tmp_path):
    path = str(tmp_path / "res.npz")
    mp.start_processes(_rank, args=(2, _free_port(), path), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(path)
    ref = _oracle_solve(_systems())
    assert list(got["iters"]) == [r[1] for r in ref]
    for i, (x, _) in enumerate(ref):
        assert np.array_equal(got[f"arr_{i}"], x)
