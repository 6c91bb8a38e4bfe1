"""The partitioned solve on the GPU (csrc/halo.cu through the C ABI) against
the oracle's restatement of mpiPcg / mpiPbicgstab with the same ranks.

A local group runs every rank on one device (the only form a single GPU
can run); an NCCL group of one rank runs the NCCL transport's calls.  Bar:
the matrix rows are the reference's (bit-identical products); each rank's
partial dots are a fixed tree instead of the reference's left-to-right sum,
so iterations agree within one and x to 1e-12 relative (PCG) / within the
tolerance-level spread (BiCGSTAB)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from sfr3d_b200 import halo as H
from sfr3d_b200 import solver as SV
from sfr3d_b200 import systems as S

pytestmark = pytest.mark.gpu


def _ranked(lays, al, ad, b):
    return ([lay.values(al, ad)[0] for lay in lays], [lay.values(al, ad)[1] for lay in lays],
            [lay.rows(b) for lay in lays])


def _global(lays, xs, n):
    x = np.zeros(n)
    for lay, xr in zip(lays, xs):
        x[lay.l2g[:lay.nEqNov]] = xr[:lay.nEqNov]
    return x


def _gpu(lays, al, ad, b, solver, **kw):
    g = H.LocalGroup(len(lays), 0)
    systems = [H.DistSystem(g, lay) for lay in lays]
    a_r, d_r, b_r = _ranked(lays, al, ad, b)
    for s, a, d in zip(systems, a_r, d_r):
        s.set_values(a, d)
    xs, info = H.solve(g, systems, solver, b_r, **kw)
    g.close()
    return xs, info


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("unsym", [True, False])
@pytest.mark.parametrize("nparts", [1, 2, 4])
def test_local_group_pcg_matches_the_oracle(unsym, nparts):
    s = S.poisson_jittered(24, seed=7)
    ia, ja, al = (s.ia, s.ja, s.al) if unsym else s.csrd_lower()
    ad, b = s.ad, s.b[0]
    lays = H.partition(s.neq, ia, ja, unsym, nparts)
    xs_o, ref = O.mpi_solve(O.PCG, lays, *_ranked(lays, al, ad, b), tol=1e-10)
    xs, info = _gpu(lays, al, ad, b, O.PCG, tol=1e-10)
    assert info.status == 0
    assert abs(info.iters - ref.iters) <= 1
    x = _global(lays, xs, s.neq)
    assert _rel(x, ref.x) < 1e-12
    assert abs(info.xKx - ref.xKx) <= 1e-10 * abs(ref.xKx)
    assert abs(info.norm_x - ref.norm_x) <= 1e-10 * ref.norm_x
    assert info.norm_r_m < 3.16 * info.conv
    # ghost entries: the owners' final values
    for lay, xr in zip(lays, xs):
        assert np.array_equal(xr[lay.nEqNov:], x[lay.l2g[lay.nEqNov:]])


@pytest.mark.parametrize("nparts", [1, 3])
def test_local_group_bicgstab_matches_the_oracle(nparts):
    m = S.momentum(20, peclet=50.0, nrhs=1)
    lays = H.partition(m.neq, m.ia, m.ja, True, nparts)
    _, ref = O.mpi_solve(O.PBICGSTAB, lays, *_ranked(lays, m.al, m.ad, m.b[0]), tol=1e-10)
    xs, info = _gpu(lays, m.al, m.ad, m.b[0], O.PBICGSTAB, tol=1e-10)
    assert info.status == 0
    assert abs(info.iters - ref.iters) <= 1
    assert _rel(_global(lays, xs, m.neq), ref.x) < 1e-12


def test_bicgstab_on_a_poisson_system_within_the_order_spread():
    """BiCGSTAB on a symmetric system is sensitive to the summation order:
    the bar is the spread of the oracle itself over partitionings."""
    s = S.poisson_jittered(16, seed=9)
    al, ad, b = s.al, s.ad, s.b[0]
    its, xs_ref = [], []
    for R in (1, 2, 3):
        lays = H.partition(s.neq, s.ia, s.ja, True, R)
        xs, r = O.mpi_solve(O.PBICGSTAB, lays, *_ranked(lays, al, ad, b), tol=1e-10)
        its.append(r.iters)
        xs_ref.append(_global(lays, xs, s.neq))
    lays = H.partition(s.neq, s.ia, s.ja, True, 2)
    xs, info = _gpu(lays, al, ad, b, O.PBICGSTAB, tol=1e-10)
    x = _global(lays, xs, s.neq)
    assert info.status == 0
    assert min(its) - 1 <= info.iters <= max(its) + 1
    spread = max(_rel(v, xs_ref[0]) for v in xs_ref[1:])
    assert _rel(x, xs_ref[1]) <= max(10 * spread, 1e-12)


def test_warm_start_and_maxit():
    s = S.poisson_jittered(16, seed=4)
    lays = H.partition(s.neq, s.ia, s.ja, True, 3)
    rng = np.random.default_rng(2)
    xg0 = rng.standard_normal(s.neq)
    x0 = [xg0[lay.l2g] for lay in lays]
    _, ref = O.mpi_solve(O.PCG, lays, *_ranked(lays, s.al, s.ad, s.b[0]), x0=x0,
                         tol=1e-10, newx=False)
    xs, info = _gpu(lays, s.al, s.ad, s.b[0], O.PCG, x0=x0, tol=1e-10, newx=False)
    assert abs(info.iters - ref.iters) <= 1
    assert _rel(_global(lays, xs, s.neq), ref.x) < 1e-12
    _, ref = O.mpi_solve(O.PCG, lays, *_ranked(lays, s.al, s.ad, s.b[0]), tol=1e-10, maxit=7)
    xs, info = _gpu(lays, s.al, s.ad, s.b[0], O.PCG, tol=1e-10, maxit=7)
    assert info.status == 1 and info.iters == ref.iters == 8
    assert _rel(_global(lays, xs, s.neq), ref.x) < 1e-12


def test_nccl_group_of_one_rank_equals_the_local_group():
    s = S.poisson_jittered(20, seed=6)
    lays = H.partition(s.neq, s.ia, s.ja, True, 1)
    xs_l, info_l = _gpu(lays, s.al, s.ad, s.b[0], O.PCG, tol=1e-10)
    g = H.NcclGroup(1, 0, H.nccl_unique_id(), 0)
    d = H.DistSystem(g, lays[0])
    a, dd = lays[0].values(s.al, s.ad)
    d.set_values(a, dd)
    xs, info = H.solve(g, [d], O.PCG, [lays[0].rows(s.b[0])], tol=1e-10)
    g.close()
    assert info.iters == info_l.iters
    assert np.array_equal(xs[0], xs_l[0])


def test_interface_mismatch_is_an_error_before_any_solve():
    s = S.poisson_jittered(10, seed=3)
    lays = H.partition(s.neq, s.ia, s.ja, True, 2)
    lay = lays[1]
    lay.iaSends = lay.iaSends.copy()
    lay.fMap = lay.fMap[:-1].copy()  # one value fewer sent to rank 0
    lay.iaSends[-1] -= 1
    g = H.LocalGroup(2, 0)
    systems = [H.DistSystem(g, la) for la in lays]
    for sy, la in zip(systems, lays):
        sy.set_values(*la.values(s.al, s.ad))
    with pytest.raises(SV.SolverError, match="interface mismatch"):
        H.solve(g, systems, O.PCG, [la.rows(s.b[0]) for la in lays], tol=1e-10)
    g.close()


def _fopen(path):
    import ctypes
    libc = ctypes.CDLL(None)
    libc.fopen.restype = ctypes.c_void_p
    libc.fopen.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    libc.fclose.argtypes = [ctypes.c_void_p]
    return libc, libc.fopen(path.encode(), b"w")


@pytest.mark.parametrize("solver,head", [(O.PCG, "MPIPCG: tol"), (O.PBICGSTAB, "MPIPBICGSTAB: tol")])
def test_solverC_mpi_branch_on_an_nccl_group(tmp_path, solver, head):
    """solverC with nPrcs > 1 calls mpiPcg / mpiPbicgstab (Solv.c:952-977,
    1070-1093): the drop-in's MPI branch on a one-rank NCCL group, with the
    reference's Interface passed as iNeq and the symmetric MPI CSRD."""
    # PCG on a pressure system (symmetric MPI CSRD), BiCGSTAB on a momentum
    # system (unsymmetric); BiCGSTAB on a symmetric system moves by a few
    # iterations with the summation order alone
    unsym = solver == O.PBICGSTAB
    s = S.momentum(14, peclet=50.0, nrhs=1) if unsym else S.poisson_jittered(14, seed=8)
    il, jl, al = (s.ia, s.ja, s.al) if unsym else s.csrd_lower()
    lay = H.partition(s.neq, il, jl, unsym, 1)[0]
    a, d = lay.values(al, s.ad)
    b = lay.rows(s.b[0])
    _, ref = O.mpi_solve(solver, [lay], [a], [d], [b], tol=1e-10)
    g = H.NcclGroup(1, 0, H.nccl_unique_id(), 0)
    with pytest.raises(SV.SolverError):
        H.set_solverC_group(H.LocalGroup(1, 0))
    H.set_solverC_group(g)
    try:
        libc, f = _fopen(str(tmp_path / "solv.log"))
        x = np.zeros(lay.nEq)
        iface = lay.interface()
        rc = SV.solverC(lay.nEq, lay.nEqNov, lay.nAd, lay.nAdR, lay.ia, lay.ja, a, d, None, b,
                        x, 1e-10, 100000, SV.CSRD, solver, fSolvLog=f, fLog=True, newX=True,
                        unSym=unsym, name="pres", iNeq=iface)
        libc.fclose(f)
        assert rc == 0
        line = open(tmp_path / "solv.log").read()
        assert line.startswith(head)
        assert abs(int(line.split("iteration")[1].split()[0]) - ref.iters) <= 1
        assert _rel(x[:lay.nEqNov], ref.x) < 1e-12
        if not unsym:
            # CSRC symmetric keeps CSRD's symmetric arrays: the same solve
            x2 = np.zeros(lay.nEq)
            rc = SV.solverC(lay.nEq, lay.nEqNov, lay.nAd, lay.nAdR, lay.ia, lay.ja, a, d, None,
                            b, x2, 1e-10, 100000, SV.CSRC, solver, newX=True, unSym=False,
                            iNeq=iface)
            assert rc == 0 and np.array_equal(x2, x)
        # a storage the reference does not build under MPI (CSRDCOO is
        # symmetric only) is its invalid option
        rc = SV.solverC(lay.nEq, lay.nEqNov, lay.nAd, lay.nAdR, lay.ia, lay.ja, a, d, None, b,
                        x, 1e-10, 100000, H.CSRDCOO, solver, newX=True, unSym=True,
                        iNeq=iface)
        assert rc == SV.UNSUPPORTED
    finally:
        H.set_solverC_group(None)
        SV.release_cache()
        g.close()


@pytest.mark.parametrize("nparts", [1, 2, 4])
@pytest.mark.parametrize("storage,unsym", [(SV.CSRC, True), (SV.CSRC, False),
                                           (H.CSRDCOO, False), (H.CSRCCOO, True),
                                           (H.CSRCCOO, False), (SV.ELLPACK, True)])
def test_other_mpi_storages_match_the_oracle(storage, unsym, nparts):
    """The reference's other MPI storages (CSRC, CSRD+COO, CSRC+COO,
    ELLPACK; Datastruct.c:115-420) on the local group against the oracle's
    restatement of their products (mpiMatVecCsrC, mpiMatVecCsrDcooSym,
    mpiMatVecCsrCcoo, mpiMatVecEllPack) at the same ranks."""
    if unsym:
        sysx = S.momentum(16, peclet=50.0, nrhs=1, seed=9)
        solver = O.PBICGSTAB
    else:
        sysx = S.poisson_jittered(20, seed=9)
        solver = O.PCG
    ia, ja, al, ad, b = sysx.ia, sysx.ja, sysx.al, sysx.ad, sysx.b[0]
    full = storage == SV.ELLPACK
    base = H.partition(sysx.neq, *((ia, ja) if full else sysx.csrd_lower()[:2]), full, nparts)
    conv = [H.as_storage(lay, storage, unsym, ia, ja, al, ad) for lay in base]
    lays = [c[0] for c in conv]
    b_r = [lay.rows(b) for lay in base]
    _, ref = O.mpi_solve(solver, lays, [c[1] for c in conv], [c[2] for c in conv], b_r,
                         tol=1e-10)
    g = H.LocalGroup(nparts, 0)
    systems = [H.DistSystem(g, lay) for lay in lays]
    for sy, c in zip(systems, conv):
        sy.set_values(c[1], c[2])
    xs, info = H.solve(g, systems, solver, b_r, tol=1e-10)
    g.close()
    assert info.status == 0 and ref.status == 0
    assert abs(info.iters - ref.iters) <= 1
    assert _rel(_global(lays, xs, sysx.neq), ref.x) < 1e-12
