"""The oracle pinned against the reference.

* golden fixtures (tests/golden/ref_solves.npz, written by the reference's own
  compiled solverC) -> the C restatement reproduces them bit for bit;
* live: the restatement and oracle/_ref agree bit for bit on fresh systems;
* the reference's exit codes on non-convergence (Cg.c:195-200,
  Bicgstab.c:225-231) are recorded in the fixtures.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from helpers import layouts, rel
from oracle import oracle as O
from sfr3d_b200 import systems as S

GOLD_PATH = os.path.join(os.path.dirname(__file__), "golden", "ref_solves.npz")
GOLD = np.load(GOLD_PATH)
CASES = [str(c) for c in GOLD["cases"]]


def case(name):
    g = {k.split("/", 1)[1]: GOLD[k] for k in GOLD.files if k.startswith(name + "/")}
    solver, st, un, maxit, newx = (int(v) for v in g["meta"])
    return g, solver, st, bool(un), maxit, bool(newx), float(g["tol"][0])


@pytest.mark.parametrize("name", CASES)
def test_restatement_reproduces_reference_fixture(name):
    g, solver, st, un, maxit, newx, tol = case(name)
    fn = O.SOLVERS[solver]
    r = fn(st, un, g["ia"], g["ja"], g["al"], g["ad"], g["b"], x0=g["x0"],
           tol=tol, maxit=maxit, newx=newx)
    iters, status = (int(v) for v in g["res"])
    if solver == O.MINRES and r.status == 1:
        # the reference's MINRES only warns at maxIt (Iters.c:525-529)
        assert status == 0 and iters == maxit + 1 == r.iters
        status = 1
    assert (r.status == 0) == (status == 0)
    if status == 0:
        assert r.iters == iters
        xkx, nx = g["log"]
        assert abs(r.xKx - xkx) <= 1e-11 * abs(xkx)
        assert abs(r.norm_x - nx) <= 1e-11 * abs(nx)
    assert np.array_equal(r.x, g["x"])


def test_reference_exit_codes_recorded():
    # PCG exits with EXIT_FAILURE (1), serial BiCGSTAB with EXIT_SOLVER (-2),
    # GMRES and BiCGSTAB(2) with EXIT_FAILURE; MINRES does not exit
    assert int(GOLD["uni8_maxit/res"][1]) == 1
    assert int(GOLD["mom8_maxit/res"][1]) == -2
    assert int(GOLD["jit10_gmres_maxit/res"][1]) == 1
    assert int(GOLD["mom8_bicgl2_maxit/res"][1]) == 1
    assert int(GOLD["jit10_minres_maxit/res"][1]) == 0


def test_restatement_status_on_iteration_cap():
    g, solver, st, un, maxit, newx, tol = case("uni8_maxit")
    r = O.pcg(st, un, g["ia"], g["ja"], g["al"], g["ad"], g["b"], tol=tol, maxit=maxit)
    assert r.status == 1 and r.iters == maxit + 1


needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("kind", ["uniform", "jittered", "momentum", "steady"])
def test_restatement_bit_identical_to_compiled_reference(kind):
    if kind == "uniform":
        s, solver = S.poisson_uniform(16, seed=21), O.PCG
    elif kind == "jittered":
        s, solver = S.poisson_jittered(14, seed=22), O.PCG
    elif kind == "momentum":
        s, solver = S.momentum(14, seed=23, nrhs=1), O.PBICGSTAB
    else:
        s = S.build(S.params(kind=S.SFR_SYS_CONVDIFF, n=12, lengths=(np.pi,) * 3,
                             dirichlet=S.ALL_FACES, rhs_normal=True, peclet=50.0,
                             nu=1e-3, dt=1e3, seed=24))
        solver = O.PBICGSTAB
    fn = O.SOLVERS[solver]
    for lname, (st, un, ia, ja, al, au) in layouts(s).items():
        ref = O.ref_solve(solver, st, un, ia, ja, al, s.ad, s.b[0])
        mine = fn(st, un, ia, ja, al, s.ad, s.b[0])
        assert ref.status == 0, lname
        assert mine.iters == ref.iters, lname
        assert np.array_equal(mine.x, ref.x), lname


@needs_ref
@pytest.mark.parametrize("solver", [O.PBICGSTABL2, O.GMRES, O.MINRES])
@pytest.mark.parametrize("kind", ["jittered", "momentum"])
def test_other_krylov_restatements_bit_identical_to_compiled_reference(kind, solver):
    """BiCGSTAB(2), GMRES(15) and MINRES: the restatement and the
    reference's own solverC agree bit for bit on every layout."""
    if kind == "momentum" and solver == O.MINRES:
        pytest.skip("MINRES needs a symmetric matrix")
    s = (S.poisson_jittered(11, seed=27) if kind == "jittered"
         else S.momentum(11, seed=28, nrhs=1))
    for lname, (st, un, ia, ja, al, au) in layouts(s).items():
        ref = O.ref_solve(solver, st, un, ia, ja, al, s.ad, s.b[0])
        mine = O.SOLVERS[solver](st, un, ia, ja, al, s.ad, s.b[0])
        assert ref.status == 0 and mine.status == 0, lname
        assert mine.iters == ref.iters, lname
        assert np.array_equal(mine.x, ref.x), lname


@needs_ref
def test_reference_openmp_path_close_to_serial():
    s = S.poisson_jittered(16, seed=25)
    il, jl, al = s.csrd_lower()
    ser = O.ref_solve(O.PCG, O.CSRC, False, il, jl, al, s.ad, s.b[0])
    omp = O.ref_solve(O.PCG, O.CSRC, False, il, jl, al, s.ad, s.b[0], nthreads=4)
    assert omp.status == 0 and abs(omp.iters - ser.iters) <= 1
    assert rel(omp.x, ser.x) < 1e-12


def test_matvec_layouts_agree():
    s = S.poisson_jittered(9, seed=26)
    x = np.random.default_rng(0).standard_normal(s.neq)
    base = O.matvec(O.CSRD, True, s.ia, s.ja, s.al, s.ad, x)
    for lname, (st, un, ia, ja, al, au) in layouts(s).items():
        y = O.matvec(st, un, ia, ja, al, s.ad, x)
        # CSRD/CSRC sum each row in the same order; ELLPACK in face order
        if lname == "ellpack":
            assert rel(y, base) < 1e-15
        else:
            assert np.array_equal(y, base), lname
    A = s.dense()
    assert rel(base, A @ x) < 1e-14
