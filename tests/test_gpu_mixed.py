"""Mixed precision (FP32 matrix and inner Krylov, FP64 reliable updates).

The solution must meet the reference's stopping criterion on the FP64 true
residual, recomputed here on the host with the oracle's FP64 SpMV:
  PCG      sqrt|(r, M^-1 r)| < tol sqrt|(b, M^-1 b)|   (Cg.c:70-74, 145)
  BiCGSTAB ||r||_2 < tol ||b||_2                        (Bicgstab.c:72-80)
and its error against the FP64 oracle solution is bounded by what that
criterion allows (both solutions carry an error of order cond(A) * tol).
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import layouts, rel
from oracle import oracle as O
from sfr3d_b200 import solver as sv
from sfr3d_b200 import systems as S

pytestmark = pytest.mark.gpu

TOL = 1e-10


def true_residual(s, st, un, ia, ja, al, x, b, ad=None):
    ad = s.ad if ad is None else ad
    r = b - O.matvec(st, un, ia, ja, al, ad, x)
    return r, float(np.sqrt(abs(np.dot(r, r / ad)))), float(np.sqrt(abs(np.dot(b, b / ad))))


@pytest.mark.parametrize("kind", ["uniform", "jittered"])
def test_mixed_pcg_meets_reference_criterion(cuda, engine, kind):
    s = S.poisson_uniform(32, seed=1) if kind == "uniform" else S.poisson_jittered(40, seed=2)
    st, un, ia, ja, al, _ = layouts(s)["csrd_full"]
    g = sv.GpuSystem(s.neq, ia, ja, st, un)
    g.set_values(al, s.ad)
    g.set_engine(engine)
    x, info = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    assert info.status == sv.OK, info
    r, rm, bm = true_residual(s, st, un, ia, ja, al, x, s.b[0])
    assert rm < TOL * bm
    assert abs(info.norm_r_m - rm) <= 1e-3 * rm + 1e-300
    ref = O.pcg(st, un, ia, ja, al, s.ad, s.b[0], tol=TOL)
    err = rel(x, ref.x)
    # the two solutions differ by at most what the criterion allows
    assert err < 1e-7, err
    assert info.refinements >= 1
    # inner iterations stay close to the FP64 count
    assert info.iters <= 1.5 * ref.iters + 20, (info.iters, ref.iters)


@pytest.mark.parametrize("dt", [1e-2, 1.0])
def test_mixed_bicgstab_meets_reference_criterion(cuda, engine, dt):
    s = S.build(S.params(kind=S.SFR_SYS_CONVDIFF, n=24, lengths=(np.pi,) * 3,
                         dirichlet=S.ALL_FACES, nrhs=1, rhs_normal=True,
                         peclet=50.0, nu=1e-3, dt=dt, seed=41))
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    g.set_values(s.al, s.ad)
    g.set_engine(engine)
    x, info = g.solve(sv.PBICGSTAB, s.b[0], tol=TOL, precision=sv.MIXED)
    assert info.status == sv.OK, info
    r = s.b[0] - O.matvec(O.CSRD, True, s.ia, s.ja, s.al, s.ad, x)
    assert np.linalg.norm(r) < TOL * np.linalg.norm(s.b[0])
    ref = O.pbicgstab(O.CSRD, True, s.ia, s.ja, s.al, s.ad, s.b[0], tol=TOL)
    assert rel(x, ref.x) < 1e-7


def test_mixed_multi_rhs_per_component_diagonal(cuda, engine):
    s = S.momentum(20, seed=53, nrhs=3)
    ad_k = np.stack([s.ad, 1.1 * s.ad, 0.95 * s.ad])
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    g.set_values(s.al, s.ad)
    g.set_engine(engine)
    xs, infos = g.solve_multi(sv.PBICGSTAB, s.b, ad_k=ad_k, tol=TOL, precision=sv.MIXED)
    for k in range(3):
        assert infos[k].status == sv.OK
        r = s.b[k] - O.matvec(O.CSRD, True, s.ia, s.ja, s.al, ad_k[k], xs[k])
        assert np.linalg.norm(r) < TOL * np.linalg.norm(s.b[k])
    # the single-RHS solve of the first component (shared diagonal = ad_k[0])
    x1, i1 = g.solve(sv.PBICGSTAB, s.b[0], tol=TOL, precision=sv.MIXED)
    assert i1.status == sv.OK
    assert rel(x1, xs[0]) < 1e-8


def test_mixed_iteration_cap_folds_correction(cuda, engine):
    s = S.poisson_jittered(24, seed=9)
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    g.set_values(s.al, s.ad)
    g.set_engine(engine)
    x, info = g.solve(sv.PCG, s.b[0], tol=TOL, maxit=40, precision=sv.MIXED)
    assert info.status == sv.MAXIT
    # x holds the FP64 solution after the last correction: the residual the
    # kernel reports is the residual of the returned x
    r = s.b[0] - O.matvec(O.CSRD, True, s.ia, s.ja, s.al, s.ad, x)
    assert abs(np.linalg.norm(r) - info.norm_r) <= 1e-6 * info.norm_r
