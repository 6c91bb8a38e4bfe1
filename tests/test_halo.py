"""Row partition of the reference's MPI path (sfr3d_b200/halo.py,
csrc/partition.cpp) and the oracle's restatement of mpiPcg / mpiPbicgstab
(oracle/sfr3d_oracle.c orc_mpi_solve).  No GPU: the layouts against the
global matrix, the oracle at one rank against the reference's own serial
solver, the oracle at several ranks against the serial solve, and the
interface exchange between two gloo processes."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import oracle as O
from sfr3d_b200 import halo as H
from sfr3d_b200 import solver as SV
from sfr3d_b200 import systems as S


def _poisson(n=10, seed=5):
    s = S.poisson_jittered(n, seed=seed)
    return s, s.ia, s.ja, s.al, s.ad, s.b[0]


def _triples_full(neq, ia, ja, unsym):
    """(row, col, src) of the full off-diagonal matrix from CSRD storage."""
    out = set()
    for i in range(neq):
        for k in range(ia[i], ia[i + 1]):
            out.add((i, int(ja[k]), k))
            if not unsym:
                out.add((int(ja[k]), i, k))
    return out


@pytest.mark.parametrize("unsym", [True, False])
@pytest.mark.parametrize("nparts", [1, 2, 3, 4, 7])
def test_layouts_cover_the_matrix(unsym, nparts):
    s, ia, ja, al, ad, b = _poisson(8)
    if not unsym:
        ia, ja, al = s.csrd_lower()
    lays = H.partition(s.neq, ia, ja, unsym, nparts)
    assert H.check_layouts(lays) == []
    owned = np.concatenate([lay.l2g[:lay.nEqNov] for lay in lays])
    assert sorted(owned.tolist()) == list(range(s.neq))
    got = set()
    for lay in lays:
        rows = lay.l2g
        if unsym:
            assert lay.nAdR == 0 and len(lay.ia) == lay.nEqNov + 1
            for i in range(lay.nEqNov):
                for k in range(lay.ia[i], lay.ia[i + 1]):
                    got.add((int(rows[i]), int(rows[lay.ja[k]]), int(lay.src[k])))
        else:
            sq, rect = lay.ia[:lay.nEqNov + 1], lay.ia[lay.nEqNov + 1:]
            for i in range(lay.nEqNov):
                for k in range(sq[i], sq[i + 1]):
                    j = int(lay.ja[k])
                    assert j < i  # strict lower square part
                    got.add((int(rows[i]), int(rows[j]), int(lay.src[k])))
                    got.add((int(rows[j]), int(rows[i]), int(lay.src[k])))
                for k in range(rect[i], rect[i + 1]):
                    j = int(lay.ja[lay.nAd + k])
                    assert j >= lay.nEqNov  # ghost columns only
                    got.add((int(rows[i]), int(rows[j]), int(lay.src[lay.nAd + k])))
    assert got == _triples_full(s.neq, ia, ja, unsym)


def test_numbering_follows_the_reference():
    """Rows in global order, ghosts by neighbour then global number, rows
    sorted by local column, receives into the ghost entries in order, sends
    after the receives in xb (ParallelMpi.c:3341-3418)."""
    s, ia, ja, al, ad, b = _poisson(9)
    rng = np.random.default_rng(1)
    part = rng.integers(0, 4, s.neq)
    lays = H.partition(s.neq, ia, ja, True, 4, part)
    for lay in lays:
        own = lay.l2g[:lay.nEqNov]
        assert np.all(np.diff(own) > 0)
        assert np.all(part[own] == lay.rank)
        gh = lay.l2g[lay.nEqNov:]
        key = list(zip(part[gh].tolist(), gh.tolist()))
        assert key == sorted(key)
        assert np.array_equal(lay.fMap[:lay.nRcvs], np.arange(lay.nEqNov, lay.nEq))
        assert lay.iaRcvs[0] == 0 and lay.iaRcvs[-1] == lay.nRcvs
        assert lay.iaSends[0] == lay.nRcvs and lay.iaSends[-1] == lay.nRcvs + lay.nSends
        assert np.all(np.diff(lay.vizPart) > 0) and lay.rank not in lay.vizPart.tolist()
        for i in range(lay.nEqNov):
            assert np.all(np.diff(lay.ja[lay.ia[i]:lay.ia[i + 1]]) > 0)
    assert H.check_layouts(lays) == []


def test_contiguous_blocks_balance_entries():
    s, ia, ja, al, ad, b = _poisson(12)
    for nparts in (2, 3, 5):
        lays = H.partition(s.neq, ia, ja, True, nparts)
        work = [lay.nEqNov + lay.nAd for lay in lays]
        assert max(work) - min(work) <= 2 * 7 + 1
        firsts = [int(lay.l2g[0]) for lay in lays]
        assert firsts == sorted(firsts)


def test_partition_rejects_bad_input():
    s, ia, ja, al, ad, b = _poisson(5)
    with pytest.raises(SV.SolverError):
        H.partition(s.neq, ia, ja, True, 0)
    with pytest.raises(SV.SolverError):
        H.partition(s.neq, ia, ja, True, 2, np.full(s.neq, 2))
    with pytest.raises(SV.SolverError):
        H.partition(s.neq, ia, ja, False, 2)  # full rows are not strictly lower
    bad = ja.copy()
    bad[0] = s.neq
    with pytest.raises(SV.SolverError):
        H.partition(s.neq, ia, bad, True, 2)


def test_check_layouts_finds_a_planted_mismatch():
    s, ia, ja, al, ad, b = _poisson(6)
    lays = H.partition(s.neq, ia, ja, True, 3)
    lay = lays[1]
    n = 0
    lo, hi = lay.iaSends[n], lay.iaSends[n + 1]
    lay.fMap[lo:hi] = lay.fMap[lo:hi][::-1].copy()  # same values, another order
    msgs = H.check_layouts(lays)
    assert msgs and "another order" in msgs[0]


def _ranked(lays, al, ad, b):
    return ([lay.values(al, ad)[0] for lay in lays], [lay.values(al, ad)[1] for lay in lays],
            [lay.rows(b) for lay in lays])


def _global(lays, xs, n):
    x = np.zeros(n)
    for lay, xr in zip(lays, xs):
        x[lay.l2g[:lay.nEqNov]] = xr[:lay.nEqNov]
    return x


@pytest.mark.parametrize("solver", [O.PCG, O.PBICGSTAB])
@pytest.mark.parametrize("unsym", [True, False])
def test_oracle_one_rank_is_the_reference(solver, unsym):
    """mpiPcg / mpiPbicgstab at one rank take exactly the serial solver's
    steps (comunicateNeq returns at once, the allreduce is the identity):
    the restatement must be bit-identical to the reference's own serial
    solver (oracle/_ref; the serial restatement when it is not built)."""
    s, ia, ja, al, ad, b = _poisson(10)
    if not unsym:
        ia, ja, al = s.csrd_lower()
    lays = H.partition(s.neq, ia, ja, unsym, 1)
    a_r, d_r, b_r = _ranked(lays, al, ad, b)
    xs, res = O.mpi_solve(solver, lays, a_r, d_r, b_r, tol=1e-10)
    x = _global(lays, xs, s.neq)
    ser = O.SOLVERS[solver](O.CSRD, unsym, ia, ja, al, ad, b, tol=1e-10)
    assert res.iters == ser.iters and np.array_equal(x, ser.x)
    assert res.xKx == ser.xKx and res.norm_r == ser.norm_r
    if O.ref_available():
        ref = O.ref_solve(solver, O.CSRD, unsym, ia, ja, al, ad, b, tol=1e-10)
        assert res.iters == ref.iters and np.array_equal(x, ref.x)


@pytest.mark.parametrize("unsym", [True, False])
@pytest.mark.parametrize("nparts", [2, 3, 5])
def test_oracle_ranks_agree_with_the_serial_solve(unsym, nparts):
    """Several ranks change only the summation order of the dots (and of the
    boundary rows' products): PCG within the order spread of the serial
    solver."""
    s, ia, ja, al, ad, b = _poisson(12)
    if not unsym:
        ia, ja, al = s.csrd_lower()
    ser = O.pcg(O.CSRD, unsym, ia, ja, al, ad, b, tol=1e-10)
    d_it, d_x = O.order_spread(O.PCG, O.CSRD, unsym, ia, ja, al, ad, b, tol=1e-10)
    lays = H.partition(s.neq, ia, ja, unsym, nparts)
    xs, res = O.mpi_solve(O.PCG, lays, *_ranked(lays, al, ad, b), tol=1e-10)
    x = _global(lays, xs, s.neq)
    assert abs(res.iters - ser.iters) <= d_it + 1
    assert np.linalg.norm(x - ser.x) / np.linalg.norm(ser.x) <= max(10 * d_x, 1e-12)
    # ghost entries hold their owners' final values (the post-processing
    # product exchanged x)
    xg = x
    for lay, xr in zip(lays, xs):
        assert np.array_equal(xr[lay.nEqNov:], xg[lay.l2g[lay.nEqNov:]])


def test_oracle_bicgstab_ranks_on_the_momentum_system():
    m = S.momentum(12, peclet=50.0, nrhs=1)
    ia, ja, al, ad, b = m.ia, m.ja, m.al, m.ad, m.b[0]
    ser = O.pbicgstab(O.CSRD, True, ia, ja, al, ad, b, tol=1e-10)
    for nparts in (2, 4):
        lays = H.partition(m.neq, ia, ja, True, nparts)
        xs, res = O.mpi_solve(O.PBICGSTAB, lays, *_ranked(lays, al, ad, b), tol=1e-10)
        x = _global(lays, xs, m.neq)
        assert abs(res.iters - ser.iters) <= 1
        assert np.linalg.norm(x - ser.x) / np.linalg.norm(ser.x) < 1e-12


def test_oracle_warm_start_and_maxit():
    s, ia, ja, al, ad, b = _poisson(8)
    lays = H.partition(s.neq, ia, ja, True, 3)
    ranked = _ranked(lays, al, ad, b)
    rng = np.random.default_rng(4)
    xg0 = rng.standard_normal(s.neq)
    x0 = [xg0[lay.l2g] for lay in lays]
    xs, res = O.mpi_solve(O.PCG, lays, *ranked, x0=x0, tol=1e-10, newx=False)
    ser = O.pcg(O.CSRD, True, ia, ja, al, ad, b, x0=xg0, tol=1e-10, newx=False)
    assert abs(res.iters - ser.iters) <= 1
    assert np.linalg.norm(_global(lays, xs, s.neq) - ser.x) <= 1e-12 * np.linalg.norm(ser.x)
    _, res = O.mpi_solve(O.PCG, lays, *ranked, tol=1e-10, maxit=5)
    assert res.status == 1 and res.iters == 6


# ---- two processes over gloo -------------------------------------------

def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _exchange(lay, v, group=None):
    """comunicateNeq over torch.distributed: pack by fMap, one send and one
    receive per neighbour, unpack into the ghost entries."""
    import torch
    import torch.distributed as dist
    xb = np.zeros(lay.nRcvs + lay.nSends)
    xb[lay.nRcvs:] = v[lay.fMap[lay.nRcvs:]]
    reqs, bufs = [], []
    for n, p in enumerate(lay.vizPart.tolist()):
        s0, s1 = lay.iaSends[n], lay.iaSends[n + 1]
        if s1 > s0:
            reqs.append(dist.isend(torch.from_numpy(xb[s0:s1].copy()), p, group=group))
        r0, r1 = lay.iaRcvs[n], lay.iaRcvs[n + 1]
        buf = torch.zeros(r1 - r0, dtype=torch.float64)
        if r1 > r0:
            reqs.append(dist.irecv(buf, p, group=group))
        bufs.append((r0, buf))
    for r in reqs:
        r.wait()
    for r0, buf in bufs:
        xb[r0:r0 + len(buf)] = buf.numpy()
    v[lay.fMap[:lay.nRcvs]] = xb[:lay.nRcvs]
    return v


def _gloo_rank(rank, world, port, out_path, plant):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = S.poisson_jittered(9, seed=3)
        lay = H.partition(s.neq, s.ia, s.ja, True, world)[rank]
        if plant and rank == 1:
            n = 0
            lay.fMap[lay.iaSends[n]] = lay.fMap[lay.iaSends[n] + 1]
        msgs = H.check_interfaces(lay)
        # every rank's ghost entries must receive their global numbers
        v = np.full(lay.nEq, -1.0)
        v[:lay.nEqNov] = lay.l2g[:lay.nEqNov]
        _exchange(lay, v)
        ok = bool(np.array_equal(v[lay.nEqNov:], lay.l2g[lay.nEqNov:].astype(float)))
        np.savez(f"{out_path}.{rank}.npz", ok=ok, nmsg=len(msgs), nrcv=lay.nRcvs)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("plant", [False, True])
def test_gloo_two_ranks_exchange_the_halo(tmp_path, plant):
    path = str(tmp_path / "halo")
    mp.start_processes(_gloo_rank, args=(2, _free_port(), path, plant), nprocs=2, join=True,
                       start_method="spawn")
    res = [np.load(f"{path}.{r}.npz") for r in range(2)]
    assert all(int(r["nrcv"]) > 0 for r in res)
    if plant:
        # both ranks report the mismatch, and the receiver's ghost is wrong
        assert all(int(r["nmsg"]) >= 1 for r in res)
        assert not bool(res[0]["ok"])
    else:
        assert all(int(r["nmsg"]) == 0 for r in res)
        assert all(bool(r["ok"]) for r in res)


# ---- the reference's other MPI storages (Datastruct.c:115-420) -----------

def _momentum(n=8, seed=6):
    m = S.momentum(n, nrhs=1, seed=seed)
    return m, m.ia, m.ja, m.al, m.ad, m.b[0]


@pytest.mark.parametrize("storage,unsym", [(SV.CSRC, True), (SV.CSRC, False),
                                           (H.CSRDCOO, False), (H.CSRCCOO, True),
                                           (H.CSRCCOO, False), (SV.ELLPACK, True)])
def test_other_storages_at_one_rank_are_the_serial_solver(storage, unsym):
    """At one rank nothing is exchanged, and mpiMatVecCsrC, mpiMatVecCsrDcooSym,
    mpiMatVecCsrCcoo and mpiMatVecEllPack take the serial products' steps:
    the oracle's restatement is bit-identical to the reference's own serial
    solver on the same arrays."""
    sysx, ia, ja, al, ad, b = (_momentum() if unsym else _poisson(8))
    solver = O.PBICGSTAB if unsym else O.PCG
    lay = H.partition(sysx.neq, *((ia, ja) if storage == SV.ELLPACK
                                  else sysx.csrd_lower()[:2]),
                      storage == SV.ELLPACK, 1)[0]
    st, a_r, ad_r = H.as_storage(lay, storage, unsym, ia, ja, al, ad)
    _, got = O.mpi_solve(solver, [st], [a_r], [ad_r], [lay.rows(b)], tol=1e-10)
    # the reference's serial storage with the same arrays (COO parts are
    # empty at one rank: the CSRD / CSRC products)
    serial = {H.CSRDCOO: SV.CSRD, H.CSRCCOO: SV.CSRC}.get(storage, storage)
    if serial == SV.ELLPACK:
        sia, sja, sal = st.ia, st.ja, a_r
    else:
        sia, sja = st.ia[:st.nEqNov + 1], st.ja[:st.nAd]
        sal = a_r[: 2 * st.nAd] if unsym and serial == SV.CSRC else a_r[:st.nAd]
    sun = unsym if serial == SV.CSRC else (serial == SV.ELLPACK)
    want = O.ref_solve(solver, serial, sun, sia, sja, sal, ad_r, lay.rows(b), tol=1e-10) \
        if O.ref_available() else None
    if want is None:
        pytest.skip("oracle/_ref not built")
    assert got.iters == want.iters and got.status == want.status == 0
    assert np.array_equal(got.x.view(np.int64), want.x.view(np.int64))


@pytest.mark.parametrize("nparts", [2, 4])
@pytest.mark.parametrize("storage,unsym", [(SV.CSRC, True), (SV.CSRC, False),
                                           (H.CSRDCOO, False), (H.CSRCCOO, True),
                                           (SV.ELLPACK, True)])
def test_other_storages_over_ranks_solve_the_same_system(storage, unsym, nparts):
    """Over several ranks each storage sums its ghost terms in its own order;
    the solve agrees with the serial solve within the summation-order
    spread (x 1e-10, iterations +-2)."""
    sysx, ia, ja, al, ad, b = (_momentum() if unsym else _poisson(8))
    solver = O.PBICGSTAB if unsym else O.PCG
    lays = H.partition(sysx.neq, *((ia, ja) if storage == SV.ELLPACK
                                   else sysx.csrd_lower()[:2]),
                       storage == SV.ELLPACK, nparts)
    conv = [H.as_storage(lay, storage, unsym, ia, ja, al, ad) for lay in lays]
    _, got = O.mpi_solve(solver, [c[0] for c in conv], [c[1] for c in conv],
                         [c[2] for c in conv], [lay.rows(b) for lay in lays], tol=1e-10)
    ser = (O.pbicgstab if unsym else O.pcg)(O.CSRD, True, ia, ja, al, ad, b, tol=1e-10)
    x = np.zeros(sysx.neq)
    off = 0
    for lay in lays:
        x[lay.l2g[:lay.nEqNov]] = got.x[off:off + lay.nEqNov]
        off += lay.nEqNov
    assert got.status == 0
    assert abs(got.iters - ser.iters) <= 2
    assert np.linalg.norm(x - ser.x) <= 1e-10 * np.linalg.norm(ser.x)
