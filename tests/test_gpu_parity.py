"""GPU parity against the oracle (FP64 plain path), through the C ABI.

Bar: SpMV rows bit-identical to the reference's kernels; PCG / BiCGSTAB
solutions within 1e-12 relative (2-norm) of the reference's FP64 solver at
equal iteration count (+-1).
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np
import pytest

from helpers import bits_equal, layouts, rel
from oracle import oracle as O
from sfr3d_b200 import solver as sv
from sfr3d_b200 import systems as S

pytestmark = pytest.mark.gpu

TOL_X = 1e-12  # relative 2-norm error in x, FP64 path vs reference

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_solves.npz"))


def gpu_system(sysx, lname, engine=0):
    st, un, ia, ja, al, au = layouts(sysx)[lname]
    g = sv.GpuSystem(sysx.neq, ia, ja, st, un)
    g.set_values(al, sysx.ad, au)
    g.set_engine(engine)
    return g, (st, un, ia, ja, al)


def reference(solver, st, un, ia, ja, al, ad, b, **kw):
    if O.ref_available():
        return O.ref_solve(solver, st, un, ia, ja, al, ad, b, **kw)
    fn = O.pcg if solver == O.PCG else O.pbicgstab
    return fn(st, un, ia, ja, al, ad, b, **kw)


@pytest.mark.parametrize("kind", ["uniform", "jittered", "momentum"])
def test_spmv_bit_identical(cuda, kind):
    torch = cuda
    s = {"uniform": lambda: S.poisson_uniform(12, seed=31),
         "jittered": lambda: S.poisson_jittered(13, seed=32),
         "momentum": lambda: S.momentum(11, seed=33, nrhs=1)}[kind]()
    x = np.random.default_rng(1).standard_normal(s.neq)
    dx = torch.tensor(x, device="cuda")
    for lname in layouts(s):
        g, (st, un, ia, ja, al) = gpu_system(s, lname)
        dy = torch.empty_like(dx)
        g.spmv(dx.data_ptr(), dy.data_ptr())
        torch.cuda.synchronize()
        want = O.matvec(st, un, ia, ja, al, s.ad, x)
        assert np.array_equal(dy.cpu().numpy(), want), lname
        dot = g.spmv_dot(dx.data_ptr(), dy.data_ptr())
        assert abs(dot - float(np.dot(want, x))) <= 1e-13 * abs(dot)
        g.close()


def test_dot_deterministic(cuda):
    torch = cuda
    a = torch.randn(3_000_001, dtype=torch.float64, device="cuda")
    b = torch.randn(3_000_001, dtype=torch.float64, device="cuda")
    v1 = sv.dot(a.data_ptr(), b.data_ptr(), a.numel())
    v2 = sv.dot(a.data_ptr(), b.data_ptr(), a.numel())
    assert v1 == v2
    assert abs(v1 - float(torch.dot(a, b))) < 1e-10 * a.numel() ** 0.5


@pytest.mark.parametrize("name", [str(c) for c in GOLD["cases"]])
def test_solver_against_reference_fixture(cuda, engine, name):
    g = {k.split("/", 1)[1]: GOLD[k] for k in GOLD.files if k.startswith(name + "/")}
    solver, st, un, maxit, newx = (int(v) for v in g["meta"])
    iters, status = (int(v) for v in g["res"])
    n = len(g["ad"])
    sysg = sv.GpuSystem(n, g["ia"], g["ja"], st, bool(un))
    sysg.set_values(g["al"], g["ad"])
    sysg.set_engine(engine)
    x, info = sysg.solve(solver, g["b"], x0=g["x0"], tol=float(g["tol"][0]),
                         maxit=maxit, newx=bool(newx), raise_on_error=False)
    # GMRES counts iterations in restart cycles of 15 (Iters.c:651)
    slack, x_bar = (15 if solver == sv.GMRES else 1), TOL_X
    if solver in (sv.PBICGSTABL2, sv.GMRES) and status == 0:
        # sensitive to the dot products' summation order: the bar is the
        # spread the reference's own algorithm shows when only that changes
        d_it, d_x = O.order_spread(solver, st, bool(un), g["ia"], g["ja"], g["al"], g["ad"],
                                   g["b"], x0=g["x0"], tol=float(g["tol"][0]),
                                   maxit=maxit, newx=bool(newx))
        slack, x_bar = max(slack, 2 * d_it), max(x_bar, 20 * d_x)
    if solver == sv.MINRES and iters == maxit + 1:
        status = 1  # the reference's MINRES only warns at maxIt (Iters.c:525-529)
    if status == 0:
        assert info.status == sv.OK
        assert abs(info.iters - iters) <= slack
        assert rel(x, g["x"]) < x_bar
    else:
        assert info.status == sv.MAXIT
        if solver == sv.GMRES:
            assert info.iters == 15 * maxit + 1
        else:
            assert info.iters == iters + 1 or info.iters == maxit + 1
        assert rel(x, g["x"]) < 1e-10


@pytest.mark.parametrize("lname", ["csrd_full", "csrd_sym", "csrc_sym", "ellpack"])
def test_pcg_uniform_32(cuda, engine, lname):
    s = S.poisson_uniform(32, seed=1)
    g, (st, un, ia, ja, al) = gpu_system(s, lname, engine)
    x, info = g.solve(sv.PCG, s.b[0], tol=1e-10)
    ref = reference(O.PCG, st, un, ia, ja, al, s.ad, s.b[0], tol=1e-10)
    assert info.status == sv.OK and ref.status == 0
    assert abs(info.iters - ref.iters) <= 1
    assert rel(x, ref.x) < TOL_X
    assert abs(info.xKx - ref.xKx) <= 1e-11 * abs(ref.xKx)


def test_pcg_jittered_contrast(cuda, engine):
    s = S.poisson_jittered(40, seed=2)
    g, (st, un, ia, ja, al) = gpu_system(s, "csrd_full", engine)
    x, info = g.solve(sv.PCG, s.b[0], tol=1e-10)
    ref = O.pcg(st, un, ia, ja, al, s.ad, s.b[0], tol=1e-10)
    assert info.status == sv.OK
    assert abs(info.iters - ref.iters) <= 1
    assert rel(x, ref.x) < TOL_X


def steady_system(n=24, seed=41):
    """Nearly steady upwind convection-diffusion (dt = 1e3, Peclet 50)."""
    return S.build(S.params(kind=S.SFR_SYS_CONVDIFF, n=n, lengths=(np.pi,) * 3,
                            dirichlet=S.ALL_FACES, nrhs=1, rhs_normal=True,
                            peclet=50.0, nu=1e-3, dt=1e3, seed=seed))


@pytest.mark.parametrize("lname", ["csrd_full", "csrc_unsym", "ellpack"])
def test_bicgstab_momentum(cuda, engine, lname):
    # the momentum system as the SIMPLE loop sees it (dt = 1e-2)
    s = S.momentum(24, seed=41, nrhs=1)
    g, (st, un, ia, ja, al) = gpu_system(s, lname, engine)
    x, info = g.solve(sv.PBICGSTAB, s.b[0], tol=1e-10)
    ref = reference(O.PBICGSTAB, st, un, ia, ja, al, s.ad, s.b[0], tol=1e-10)
    assert info.status == sv.OK and ref.status == 0
    assert abs(info.iters - ref.iters) <= 1
    assert rel(x, ref.x) < TOL_X


def reference_spread(solver, s, b):
    """How far the reference moves from its own serial result when only the
    reduction order changes: its OpenMP path (dotOmp reductions, per-thread
    SpMV buffers) at 2, 4 and 8 threads on the CSRD layout."""
    ser = O.ref_solve(solver, O.CSRD, True, s.ia, s.ja, s.al, s.ad, b)
    its, errs = [ser.iters], [0.0]
    for nt in (2, 4, 8):
        o = O.ref_solve(solver, O.CSRD, True, s.ia, s.ja, s.al, s.ad, b, nthreads=nt)
        its.append(o.iters)
        errs.append(rel(o.x, ser.x))
    return ser, min(its), max(its), max(errs)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("lname", ["csrd_full", "csrc_unsym", "ellpack"])
def test_bicgstab_steady_within_reference_spread(cuda, engine, lname):
    # Convection-dominated and nearly steady: the BiCGSTAB residual history
    # is irregular near the threshold, so any change of summation order moves
    # the iteration count by a few and x by up to ~1e-9 -- the reference's
    # own OpenMP path does.  Bar: stay inside that spread (+1 iteration, x 4x).
    s = steady_system()
    g, (st, un, ia, ja, al) = gpu_system(s, lname, engine)
    x, info = g.solve(sv.PBICGSTAB, s.b[0], tol=1e-10)
    ser, lo, hi, err = reference_spread(O.PBICGSTAB, s, s.b[0])
    assert info.status == sv.OK
    assert lo - 1 <= info.iters <= hi + 1
    assert rel(x, ser.x) <= max(TOL_X, 4 * err)


@pytest.mark.parametrize("solver", [sv.PCG, sv.PBICGSTAB])
def test_multi_rhs_matches_single(cuda, engine, solver):
    # K right-hand sides in one launch against K single solves.  The K-RHS
    # kernel may run a different grid (occupancy), i.e. another reduction
    # order, so the bar is the parity bar, not bit equality.
    s = (S.poisson_jittered(24, seed=51) if solver == sv.PCG
         else S.momentum(24, seed=52, nrhs=3))
    b = np.stack([s.b[0], -0.5 * s.b[0] + 0.1, np.cos(np.arange(s.neq))]) \
        if solver == sv.PCG else s.b
    g, _ = gpu_system(s, "csrd_full", engine)
    xs, infos = g.solve_multi(solver, b, tol=1e-10)
    for k in range(3):
        x1, i1 = g.solve(solver, b[k], tol=1e-10)
        assert infos[k].status == sv.OK and i1.status == sv.OK
        assert abs(infos[k].iters - i1.iters) <= 1
        assert rel(xs[k], x1) < TOL_X


def test_multi_rhs_per_component_diagonal(cuda, engine):
    # u, v, w share al/au and differ in ad (Simple.c:2736-2750)
    s = S.momentum(14, seed=53, nrhs=3)
    ad_k = np.stack([s.ad, 1.1 * s.ad, 0.95 * s.ad])
    g, (st, un, ia, ja, al) = gpu_system(s, "csrd_full", engine)
    xs, infos = g.solve_multi(sv.PBICGSTAB, s.b, ad_k=ad_k, tol=1e-10)
    for k in range(3):
        ref = O.pbicgstab(st, un, ia, ja, al, ad_k[k], s.b[k], tol=1e-10)
        assert abs(infos[k].iters - ref.iters) <= 1
        assert rel(xs[k], ref.x) < TOL_X


def test_warm_start_and_repeatability(cuda, engine):
    s = S.poisson_uniform(20, seed=61)
    g, (st, un, ia, ja, al) = gpu_system(s, "csrd_sym", engine)
    x0 = np.linspace(-1, 1, s.neq)
    x1, i1 = g.solve(sv.PCG, s.b[0], x0=x0, newx=False, tol=1e-9)
    x2, i2 = g.solve(sv.PCG, s.b[0], x0=x0, newx=False, tol=1e-9)
    assert np.array_equal(x1, x2) and i1.iters == i2.iters
    ref = O.pcg(st, un, ia, ja, al, s.ad, s.b[0], x0=x0, newx=False, tol=1e-9)
    assert abs(i1.iters - ref.iters) <= 1
    assert rel(x1, ref.x) < TOL_X


def test_breakdown_and_maxit_are_statuses_not_hangs(cuda, engine):
    s = S.poisson_uniform(10, seed=71)
    g, _ = gpu_system(s, "csrd_full", engine)
    b = s.b[0].copy()
    b[5] = np.nan
    _, info = g.solve(sv.PCG, b, tol=1e-10, maxit=50)
    assert info.status in (sv.BREAKDOWN, sv.MAXIT)
    _, info = g.solve(sv.PCG, s.b[0], tol=1e-10, maxit=3)
    assert info.status == sv.MAXIT and info.iters == 4


def test_solverC_dropin_log_line(cuda):
    s = S.poisson_uniform(16, seed=81)
    il, jl, al = s.csrd_lower()
    x = np.zeros(s.neq)
    libc = ctypes.CDLL(None)
    libc.fopen.restype = ctypes.c_void_p
    libc.fopen.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    libc.fclose.argtypes = [ctypes.c_void_p]
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "solv_log.txt")
        f = libc.fopen(path.encode(), b"w")
        b = s.b[0].copy()
        rc = sv.solverC(s.neq, s.neq, len(jl), 0, il, jl, al, s.ad, None, b, x,
                        1e-10, 1000, sv.CSRD, sv.PCG, fSolvLog=f, fLog=True,
                        newX=True, unSym=False, name="pres")
        libc.fclose(f)
        line = open(path).read()
    assert rc == sv.OK
    assert np.array_equal(b, s.b[0])          # b unchanged (Cg.c:41)
    ref = O.pcg(O.CSRD, False, il, jl, al, s.ad, s.b[0], tol=1e-10)
    assert line.startswith("PCG: tol") and f"iteration {ref.iters} " in line
    assert rel(x, ref.x) < TOL_X
    # second call reuses the cached pattern
    x2 = np.zeros(s.neq)
    assert sv.solverC(s.neq, s.neq, len(jl), 0, il, jl, al, s.ad, None, s.b[0],
                      x2, 1e-10, 1000, sv.CSRD, sv.PCG) == sv.OK
    assert np.array_equal(x, x2)
    sv.release_cache()


@pytest.mark.parametrize("eng", [2, 4])
def test_wide_bandwidth_uses_32bit_columns(cuda, eng):
    """Without RCM the bandwidth of a 40^3 system exceeds what 16-bit column
    offsets hold: the graph engine reads 32-bit indices (same FP64 parity
    bar), and the resident engine, which needs offsets, declines the solve."""
    s = S.build(S.params(n=(40, 40, 40), jitter=0.2, log10k=(-2.0, 2.0), permute=True,
                         rcm=False, seed=21))
    g, (st, un, ia, ja, al) = gpu_system(s, "csrd_full", eng)
    assert g.stats()["bandwidth"] > 32767
    if eng == 4:
        with pytest.raises(sv.SolverError) as e:
            g.solve(sv.PCG, s.b[0], tol=1e-10, precision=sv.MIXED)
        assert e.value.status == sv.UNSUPPORTED
        g.set_engine(0)  # the automatic choice falls back to another engine
        x, info = g.solve(sv.PCG, s.b[0], tol=1e-10, precision=sv.MIXED)
        assert info.status == sv.OK
        return
    x, info = g.solve(sv.PCG, s.b[0], tol=1e-10)
    ref = O.pcg(st, un, ia, ja, al, s.ad, s.b[0], tol=1e-10)
    assert info.status == sv.OK
    assert abs(info.iters - ref.iters) <= 1
    assert rel(x, ref.x) < TOL_X


@pytest.mark.parametrize("engine_", [2, 3])
@pytest.mark.parametrize("precision", [sv.FP64, sv.MIXED])
def test_staged_slices_are_bit_identical(cuda, engine_, precision):
    """BiCGSTAB's SpMV phases with the slices staged in shared memory by bulk
    copies do the same arithmetic as the direct loads: on one grid (slices
    per warp fixed, so both run the same blocks and reduction order) x is
    bit-identical, for one and three right-hand sides; and the staged solve
    meets the FP64 bar against the oracle."""
    s = S.momentum(24, seed=54, nrhs=3)
    g, (st, un, ia, ja, al) = gpu_system(s, "csrd_full")
    g.set_engine(engine_, 256, 2)
    maxit = 100000 if engine_ == 2 else 40
    out = {}
    for flag in (1, 0):
        g.set_staging(flag)
        xs, infos = g.solve_multi(sv.PBICGSTAB, s.b, tol=1e-10, maxit=maxit, precision=precision,
                                  raise_on_error=False)
        x1, i1 = g.solve(sv.PBICGSTAB, s.b[1], tol=1e-10, maxit=maxit, precision=precision,
                         raise_on_error=False)
        out[flag] = (xs, [i.iters for i in infos], x1, i1.iters)
    assert bits_equal(out[1][0], out[0][0]) and out[1][1] == out[0][1]
    assert bits_equal(out[1][2], out[0][2]) and out[1][3] == out[0][3]
    if precision == sv.FP64 and engine_ == 2:
        for k in range(3):
            ref = O.pbicgstab(st, un, ia, ja, al, s.ad, s.b[k], tol=1e-10)
            assert abs(out[1][1][k] - ref.iters) <= 1
            assert rel(out[1][0][k], ref.x) < TOL_X
    g.close()


def test_staged_slices_without_off_diagonals(cuda):
    """A diagonal system: every slice is empty, each stage completes on its
    arrival alone (no bytes to wait for)."""
    n = 1000
    ia = np.zeros(n + 1, np.int32)
    ad = np.linspace(1.0, 2.0, n)
    b = np.cos(np.arange(n))
    g = sv.GpuSystem(n, ia, np.zeros(0, np.int32), sv.CSRD, True)
    g.set_values(np.zeros(0), ad)
    g.set_engine(2)
    x, info = g.solve(sv.PBICGSTAB, b, tol=1e-12)
    assert info.status == sv.OK
    assert rel(x, b / ad) < 1e-14
    g.close()
