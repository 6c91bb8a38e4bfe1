"""Batched uneven systems in one persistent launch (sfr_gpu_batch_*)."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import rel
from oracle import oracle as O
from sfr3d_b200 import solver as sv
from sfr3d_b200 import systems as S

pytestmark = pytest.mark.gpu


def poisson_batch(count, nmin, nmax, seed):
    return S.poisson_batch(count, nmin, nmax, seed=seed)


def make_batch(systems, storage="csrd_full"):
    if storage == "csrd_full":
        g = sv.GpuBatch([(s.neq, s.ia, s.ja) for s in systems], sv.CSRD, True)
        g.set_values([s.al for s in systems], [s.ad for s in systems])
    else:  # CSRC symmetric (lower storage)
        lows = [s.csrd_lower() for s in systems]
        g = sv.GpuBatch([(s.neq, l[0], l[1]) for s, l in zip(systems, lows)], sv.CSRC, False)
        g.set_values([l[2] for l in lows], [s.ad for s in systems])
    return g


@pytest.mark.parametrize("storage", ["csrd_full", "csrc_sym"])
def test_batch_pcg_fp64_matches_reference(cuda, storage):
    systems = poisson_batch(12, 6, 22, seed=7)
    g = make_batch(systems, storage)
    xs, infos = g.solve(sv.PCG, [s.b[0] for s in systems], tol=1e-10)
    for s, x, info in zip(systems, xs, infos):
        ref = O.pcg(O.CSRD, True, s.ia, s.ja, s.al, s.ad, s.b[0], tol=1e-10)
        assert info.status == sv.OK
        assert abs(info.iters - ref.iters) <= 1, (info.iters, ref.iters)
        assert rel(x, ref.x) < 1e-12


def test_batch_mixed_meets_reference_criterion(cuda):
    systems = poisson_batch(16, 6, 28, seed=8)
    g = make_batch(systems)
    xs, infos = g.solve(sv.PCG, [s.b[0] for s in systems], tol=1e-10, precision=sv.MIXED)
    for s, x, info in zip(systems, xs, infos):
        assert info.status == sv.OK
        r = s.b[0] - O.matvec(O.CSRD, True, s.ia, s.ja, s.al, s.ad, x)
        bm = np.sqrt(np.dot(s.b[0], s.b[0] / s.ad))
        assert np.sqrt(np.dot(r, r / s.ad)) < 1e-10 * bm


def test_batch_bicgstab_momentum(cuda):
    systems = [S.momentum(n, seed=20 + n, nrhs=1) for n in (6, 9, 12, 15)]
    g = make_batch(systems)
    for prec in (sv.FP64, sv.MIXED):
        xs, infos = g.solve(sv.PBICGSTAB, [s.b[0] for s in systems], tol=1e-10, precision=prec)
        for s, x, info in zip(systems, xs, infos):
            ref = O.pbicgstab(O.CSRD, True, s.ia, s.ja, s.al, s.ad, s.b[0], tol=1e-10)
            assert info.status == sv.OK
            if prec == sv.FP64:
                assert abs(info.iters - ref.iters) <= 1
                assert rel(x, ref.x) < 1e-12
            else:
                r = s.b[0] - O.matvec(O.CSRD, True, s.ia, s.ja, s.al, s.ad, x)
                assert np.linalg.norm(r) < 1e-10 * np.linalg.norm(s.b[0])


def test_batch_autotune_and_repeat(cuda):
    systems = poisson_batch(24, 6, 30, seed=9)
    g = make_batch(systems)
    bs = [s.b[0] for s in systems]
    ms = g.autotune(sv.PCG, bs, tol=1e-10)
    assert ms > 0
    xs1, i1 = g.solve(sv.PCG, bs, tol=1e-10)
    xs2, i2 = g.solve(sv.PCG, bs, tol=1e-10)
    for a, b, ia, ib in zip(xs1, xs2, i1, i2):
        assert np.array_equal(a, b) and ia.iters == ib.iters and ia.status == sv.OK
    st = g.stats()
    assert st["grid"] >= len(systems)


def test_batch_many_small_systems(cuda):
    systems = poisson_batch(64, 4, 12, seed=10)
    g = make_batch(systems)
    xs, infos = g.solve(sv.PCG, [s.b[0] for s in systems], tol=1e-10)
    for s, x, info in zip(systems, xs, infos):
        ref = O.pcg(O.CSRD, True, s.ia, s.ja, s.al, s.ad, s.b[0], tol=1e-10)
        assert info.status == sv.OK and abs(info.iters - ref.iters) <= 1
        assert rel(x, ref.x) < 1e-12


def test_batch_iteration_cap_is_per_system_status(cuda):
    systems = poisson_batch(6, 8, 20, seed=11)
    g = make_batch(systems)
    xs, infos = g.solve(sv.PCG, [s.b[0] for s in systems], tol=1e-10, maxit=5,
                        raise_on_error=False)
    assert all(i.status == sv.MAXIT for i in infos)
