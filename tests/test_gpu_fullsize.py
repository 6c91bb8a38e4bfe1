"""Parity at the benchmarked sizes: the workloads the bench times, each
solved on the GPU and compared with the reference's own solver on the same
seeded system.

  * the 128^3 jittered pressure system (2,097,152 rows), FP64 PCG on the
    graph engine, against the reference's compiled pcgOmp (Cg.c:490-715) with
    every host thread;
  * the same system with the mixed-precision resident engine, against the
    same reference solution;
  * the 128^3 momentum system (Peclet 50), three right-hand sides in one K = 3
    FP64 launch, each against the reference's pbicgstabOmp (Bicgstab.c:554);
  * the 64 uneven Poisson boxes (8..96 cells per axis, 2.92 M rows) in one
    batched launch, FP64 and mixed, each box against the oracle's pcg
    (Cg.c:47-209, bit-identical to the reference's serial solver).

Bars:
  FP64  -- ||x - x_ref|| / ||x_ref|| < 1e-12 at equal iteration count +-1.
           The reference's own OpenMP and serial solves of the 128^3 system
           differ by 9e-14, at 1817 iterations both.
  mixed -- the FP64 true residual, recomputed on the host, meets the
           reference's stopping test (PCG: the M-norm, Cg.c:145), and the
           error against the reference's FP64 solution stays below 1e-6
           (the number is printed: 3e-8 at 128^3).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from helpers import rel
from oracle import oracle as O
from sfr3d_b200 import solver as sv
from sfr3d_b200 import systems as S

pytestmark = pytest.mark.gpu

TOL = 1e-10
TOL_X = 1e-12
MIXED_ERR = 1e-6
THREADS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def pressure128():
    """The headline system and the reference's pcgOmp solution of it (CSRC
    symmetric storage, the reference's default, all host threads)."""
    s = S.poisson_jittered(128, seed=2)
    il, jl, al = s.csrd_lower()
    ref = O.ref_solve(O.PCG, O.CSRC, False, il, jl, al, s.ad, s.b[0], tol=TOL,
                      nthreads=THREADS)
    assert ref.status == 0
    return s, ref


def m_residual(s, x, b):
    """(||b - A x||_M, ||b||_M) with the oracle's FP64 SpMV, M = diag(ad)^-1."""
    r = b - O.matvec(O.CSRD, True, s.ia, s.ja, s.al, s.ad, x)
    return float(np.sqrt(abs(np.dot(r, r / s.ad)))), float(np.sqrt(abs(np.dot(b, b / s.ad))))


@pytest.mark.parametrize("fused", [0, 3, 4])
def test_pressure128_fp64_graph_engine(cuda, pressure128, fused):
    """The three-kernel iteration, the fused one-kernel iteration (mode 3)
    and the whole solve in one launch (mode 4), which the autotuner chooses
    between for this system."""
    s, ref = pressure128
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    g.set_values(s.al, s.ad)
    g.set_engine(sv.ENGINE_GRAPH)
    g.set_fused(fused)
    x, info = g.solve(sv.PCG, s.b[0], tol=TOL)
    g.close()
    err = rel(x, ref.x)
    print(f"128^3 FP64 PCG (fused mode {fused}): {info.iters} iterations (reference "
          f"{ref.iters}), error vs reference {err:.2e}")
    assert info.status == sv.OK
    assert abs(info.iters - ref.iters) <= 1
    assert err < TOL_X
    assert abs(info.xKx - ref.xKx) <= 1e-11 * abs(ref.xKx)


def test_pressure128_fp64_through_solverC(cuda, pressure128, tmp_path):
    """The drop-in with the reference's own storage (CSRC symmetric); the
    iteration count is read from its log line (Cg.c:201-208)."""
    s, ref = pressure128
    il, jl, al = s.csrd_lower()
    x = np.zeros(s.neq)
    libc = ctypes.CDLL(None)
    libc.fopen.restype = ctypes.c_void_p
    libc.fopen.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    libc.fclose.argtypes = [ctypes.c_void_p]
    log = tmp_path / "solv.log"
    f = libc.fopen(str(log).encode(), b"w")
    try:
        rc = sv.solverC(s.neq, s.neq, len(jl), 0, il, jl, al, s.ad, None, s.b[0], x, TOL,
                        100000, storage=sv.CSRC, solver=sv.PCG, fSolvLog=f, fLog=True,
                        newX=True, unSym=False)
    finally:
        libc.fclose(f)
        sv.release_cache()
    assert rc == sv.OK
    words = open(log).read().split()
    assert words[0] == "PCG:"
    iters = int(words[words.index("iteration") + 1])
    err = rel(x, ref.x)
    print(f"128^3 FP64 PCG through sfr_solverC: {iters} iterations, error vs reference {err:.2e}")
    assert abs(iters - ref.iters) <= 1
    assert err < TOL_X


def test_pressure128_mixed_resident_engine(cuda, pressure128):
    s, ref = pressure128
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    g.set_values(s.al, s.ad)
    g.set_engine(sv.ENGINE_RESIDENT)
    x, info = g.solve(sv.PCG, s.b[0], tol=TOL, precision=sv.MIXED)
    g.close()
    assert info.status == sv.OK, info
    rm, bm = m_residual(s, x, s.b[0])
    err = rel(x, ref.x)
    print(f"128^3 mixed PCG (resident): {info.inner_iters} inner iterations, "
          f"{info.refinements} refreshes, M-norm residual {rm / bm:.2e} (criterion {TOL}), "
          f"error vs reference {err:.2e}")
    assert rm < TOL * bm
    assert err < MIXED_ERR
    assert info.inner_iters <= 1.2 * ref.iters


def test_momentum128_k3_fp64(cuda):
    m = S.momentum(128, nrhs=3, seed=3)
    g = sv.GpuSystem(m.neq, m.ia, m.ja, sv.CSRD, True)
    g.set_values(m.al, m.ad)
    xs, infos = g.solve_multi(sv.PBICGSTAB, m.b, tol=TOL)
    g.close()
    for k in range(3):
        ref = O.ref_solve(O.PBICGSTAB, O.CSRD, True, m.ia, m.ja, m.al, m.ad, m.b[k], tol=TOL,
                          nthreads=THREADS)
        assert ref.status == 0
        err = rel(xs[k], ref.x)
        print(f"128^3 momentum RHS {k}: {infos[k].iters} iterations (reference {ref.iters}), "
              f"error vs reference {err:.2e}")
        assert infos[k].status == sv.OK
        assert abs(infos[k].iters - ref.iters) <= 1
        assert err < TOL_X


def test_momentum128_k3_mixed(cuda):
    """The K = 3 mixed launch: BiCGSTAB's criterion ||r||_2 < tol ||b||_2
    (Bicgstab.c:130,155) on the FP64 true residual."""
    m = S.momentum(128, nrhs=3, seed=3)
    g = sv.GpuSystem(m.neq, m.ia, m.ja, sv.CSRD, True)
    g.set_values(m.al, m.ad)
    xs, infos = g.solve_multi(sv.PBICGSTAB, m.b, tol=TOL, precision=sv.MIXED)
    g.close()
    for k in range(3):
        r = m.b[k] - O.matvec(O.CSRD, True, m.ia, m.ja, m.al, m.ad, xs[k])
        rr = float(np.linalg.norm(r) / np.linalg.norm(m.b[k]))
        ref = O.ref_solve(O.PBICGSTAB, O.CSRD, True, m.ia, m.ja, m.al, m.ad, m.b[k], tol=TOL,
                          nthreads=THREADS)
        err = rel(xs[k], ref.x)
        print(f"128^3 momentum RHS {k} mixed: relative residual {rr:.2e}, "
              f"error vs reference {err:.2e}")
        assert infos[k].status == sv.OK
        assert rr < TOL
        assert err < MIXED_ERR


@pytest.fixture(scope="module")
def boxes64():
    systems = S.poisson_batch(64, 8, 96, seed=4)
    refs = [O.pcg(O.CSRD, True, s.ia, s.ja, s.al, s.ad, s.b[0], tol=TOL) for s in systems]
    return systems, refs


def test_batch64_fp64(cuda, boxes64):
    systems, refs = boxes64
    g = sv.GpuBatch([(s.neq, s.ia, s.ja) for s in systems], sv.CSRD, True)
    g.set_values([s.al for s in systems], [s.ad for s in systems])
    xs, infos = g.solve(sv.PCG, [s.b[0] for s in systems], tol=TOL)
    g.close()
    worst = 0.0
    for s, x, info, ref in zip(systems, xs, infos, refs):
        assert info.status == sv.OK
        assert abs(info.iters - ref.iters) <= 1, (s.neq, info.iters, ref.iters)
        worst = max(worst, rel(x, ref.x))
    print(f"64 boxes FP64 batched: worst error vs oracle {worst:.2e}")
    assert worst < TOL_X


def test_batch64_mixed(cuda, boxes64):
    systems, refs = boxes64
    g = sv.GpuBatch([(s.neq, s.ia, s.ja) for s in systems], sv.CSRD, True)
    g.set_values([s.al for s in systems], [s.ad for s in systems])
    xs, infos = g.solve(sv.PCG, [s.b[0] for s in systems], tol=TOL, precision=sv.MIXED)
    g.close()
    worst = 0.0
    for s, x, info, ref in zip(systems, xs, infos, refs):
        assert info.status == sv.OK
        rm, bm = m_residual(s, x, s.b[0])
        assert rm < TOL * bm, (s.neq, rm / bm)
        worst = max(worst, rel(x, ref.x))
    print(f"64 boxes mixed batched: worst error vs oracle {worst:.2e}")
    assert worst < MIXED_ERR
