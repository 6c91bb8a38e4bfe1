"""Resident engine (engine 4): mixed-precision Jacobi-PCG whose FP32 inner
iteration runs on the symmetrically scaled operator S A S (S = diag(ad)^-1/2)
held in L2 and shared memory, with FP64 reliable updates (resident.cu).

Bar, as for every mixed result: the FP64 true residual, recomputed on the
host with the oracle's FP64 SpMV, meets the reference's criterion
  sqrt|(r, M^-1 r)| < tol sqrt|(b, M^-1 b)|   (Cg.c:70-74, 145)
and the solution differs from the FP64 oracle's by no more than that
criterion allows on these systems (1e-7 relative at tol 1e-10).
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
ERR = 1e-7


def m_norms(st, un, ia, ja, al, ad, x, b):
    r = b - O.matvec(st, un, ia, ja, al, ad, x)
    return float(np.sqrt(abs(np.dot(r, r / ad)))), float(np.sqrt(abs(np.dot(b, b / ad))))


def resident(s, lay="csrd_full"):
    st, un, ia, ja, al, _ = layouts(s)[lay]
    g = sv.GpuSystem(s.neq, ia, ja, st, un)
    g.set_values(al, s.ad)
    g.set_engine(sv.ENGINE_RESIDENT)
    return g, (st, un, ia, ja, al)


@pytest.mark.parametrize("lay", ["csrd_full", "csrd_sym", "csrc_sym", "ellpack"])
@pytest.mark.parametrize("kind", ["uniform", "jittered"])
def test_resident_meets_reference_criterion(cuda, kind, lay):
    s = S.poisson_uniform(32, seed=1) if kind == "uniform" else S.poisson_jittered(28, seed=2)
    g, (st, un, ia, ja, al) = resident(s, lay)
    x, info = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    assert info.status == sv.OK, info
    rm, bm = m_norms(st, un, ia, ja, al, s.ad, x, s.b[0])
    assert rm < TOL * bm
    assert abs(info.norm_r_m - rm) <= 1e-3 * rm
    ref = O.pcg(st, un, ia, ja, al, s.ad, s.b[0], tol=TOL)
    assert rel(x, ref.x) < ERR
    assert info.refinements >= 1
    assert info.inner_iters <= 1.5 * ref.iters + 20, (info.inner_iters, ref.iters)
    g.close()


def test_resident_anisotropic_boxes(cuda):
    """Boxes of the uneven batch: spacing ratio up to 10 on one axis, one
    Dirichlet face -- the nearly singular systems the diagonal correction of
    the rounded operator exists for."""
    boxes = [s for s in S.poisson_batch(64, 8, 96, seed=4) if s.neq <= 40_000][:6]
    assert len(boxes) >= 3
    for s in boxes:
        g, (st, un, ia, ja, al) = resident(s)
        x, info = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
        assert info.status == sv.OK, info
        rm, bm = m_norms(st, un, ia, ja, al, s.ad, x, s.b[0])
        assert rm < TOL * bm
        ref = O.pcg(st, un, ia, ja, al, s.ad, s.b[0], tol=TOL)
        assert rel(x, ref.x) < ERR
        # FP32 inner iterations on these nearly singular systems take up to
        # ~1.6x the FP64 count; the resident engine stays with the mixed
        # persistent engine (unscaled FP32 operator)
        g.set_engine(sv.ENGINE_PERSISTENT)
        _, other = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
        assert info.inner_iters <= 2 * ref.iters + 20, (info.inner_iters, ref.iters)
        assert info.inner_iters <= 1.15 * other.inner_iters + 20, (info.inner_iters,
                                                                   other.inner_iters)
        g.close()


def test_resident_is_the_automatic_choice_and_deterministic(cuda):
    s = S.poisson_jittered(48, seed=6)  # 110,592 rows: the large-system range
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    g.set_values(s.al, s.ad)
    x0, i0 = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    g.set_engine(sv.ENGINE_RESIDENT)
    x1, i1 = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    x2, i2 = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    assert i1.status == sv.OK
    assert np.array_equal(x1, x2) and np.array_equal(x0, x1)
    assert i0.inner_iters == i1.inner_iters == i2.inner_iters
    rm, bm = m_norms(O.CSRD, True, s.ia, s.ja, s.al, s.ad, x1, s.b[0])
    assert rm < TOL * bm
    g.close()


def test_resident_warm_start(cuda):
    s = S.poisson_jittered(24, seed=8)
    g, _ = resident(s)
    x, info = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    x2, info2 = g.solve(sv.PCG, s.b[0], x0=x, newx=False, tol=TOL, precision=sv.MIXED)
    assert info2.status == sv.OK
    assert info2.inner_iters == 0  # the start already meets the criterion
    assert np.array_equal(x, x2)
    # a start from half the solution converges, to the same bar
    x3, info3 = g.solve(sv.PCG, s.b[0], x0=0.5 * x, newx=False, tol=TOL, precision=sv.MIXED)
    assert info3.status == sv.OK and rel(x3, x) < ERR
    g.close()


def test_resident_iteration_cap_folds_correction(cuda):
    s = S.poisson_jittered(24, seed=9)
    g, _ = resident(s)
    x, info = g.solve(sv.PCG, s.b[0], tol=TOL, maxit=40, precision=sv.MIXED)
    assert info.status == sv.MAXIT
    r = s.b[0] - O.matvec(O.CSRD, True, s.ia, s.ja, s.al, s.ad, x)
    assert abs(np.linalg.norm(r) - info.norm_r) <= 1e-6 * info.norm_r
    g.close()


def test_resident_follows_new_values(cuda):
    """The scaled operator is rebuilt after set_values / set_diagonal."""
    s = S.poisson_jittered(20, seed=10)
    g, _ = resident(s)
    x, _ = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    g.set_values(2.0 * s.al, 2.0 * s.ad)
    x2, i2 = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    assert i2.status == sv.OK and rel(x2, 0.5 * x) < ERR
    ad = 1.5 * s.ad
    g.set_values(s.al, s.ad)
    g.set_diagonal(ad)
    x3, i3 = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    assert i3.status == sv.OK
    rm, bm = m_norms(O.CSRD, True, s.ia, s.ja, s.al, ad, x3, s.b[0])
    assert rm < TOL * bm
    g.close()


def test_resident_refuses_what_it_does_not_run(cuda):
    s = S.poisson_jittered(12, seed=11)
    g, _ = resident(s)
    for solver, prec in ((sv.PCG, sv.FP64), (sv.PBICGSTAB, sv.MIXED)):
        with pytest.raises(sv.SolverError) as e:
            g.solve(solver, s.b[0], tol=TOL, precision=prec)
        assert e.value.status == sv.UNSUPPORTED
    # Jacobi scaling needs a positive diagonal
    bad = s.ad.copy()
    bad[5] = -bad[5]
    g.set_diagonal(bad)
    with pytest.raises(sv.SolverError) as e:
        g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    assert e.value.status == sv.UNSUPPORTED
    g.set_diagonal(s.ad)
    _, info = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    assert info.status == sv.OK
    g.close()


def test_resident_transpose_solve(cuda):
    """The transposed view runs on the resident engine too (symmetric
    matrix: A^T x = b has the forward solution)."""
    s = S.poisson_jittered(20, seed=12)
    g, _ = resident(s)
    x, _ = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    xt, it = g.solve_transpose(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    assert it.status == sv.OK and rel(xt, x) < ERR
    g.close()
