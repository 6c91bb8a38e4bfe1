"""Autotuners: sfr_gpu_autotune (engine and graph launch shape of one
system's solves) and sfr_gpu_batch_autotune (blocks per system of a batched
launch).

What is checked:
  * the tuned choice is deterministic for a fixed system: a second tune of
    the same handle returns the kept choice, and with SFR_TUNE_CACHE a new
    handle of the same system reads the same choice back from the file;
  * solves on the tuned choice still meet the FP64 bar against the oracle
    (1e-12 relative in x, iterations +-1) and repeat bit for bit;
  * the batch tuner keeps the fastest plan it measured and the tuned batch
    meets the same FP64 bar.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from helpers import bits_equal, rel
from oracle import oracle as O
from sfr3d_b200 import solver as sv
from sfr3d_b200 import systems as S

pytestmark = pytest.mark.gpu

TOL = 1e-10


def test_autotune_choice_is_kept_and_solves_at_parity(cuda, tmp_path, monkeypatch):
    s = S.poisson_jittered(48, seed=21)  # 110,592 rows: the graph engine by default
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("SFR_TUNE_CACHE", str(cache))
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    g.set_values(s.al, s.ad)
    first = g.autotune(sv.PCG, s.b[0], tol=TOL)
    assert first["source"] == 0 and first["candidates"] >= 6, first
    assert first["default_engine"] == sv.ENGINE_GRAPH
    assert first["ms"] <= first["default_ms"]
    again = g.autotune(sv.PCG, s.b[0], tol=TOL)
    assert again["source"] == 1
    assert (again["engine"], again["threads"], again["slices_per_warp"]) == \
        (first["engine"], first["threads"], first["slices_per_warp"])
    # the file holds the choice: a new handle of the same system reads it
    assert cache.read_text().count(" -> engine=") == 1
    h = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    h.set_values(s.al, s.ad)
    third = h.autotune(sv.PCG, s.b[0], tol=TOL)
    assert third["source"] == 2
    assert (third["engine"], third["threads"], third["slices_per_warp"]) == \
        (first["engine"], first["threads"], first["slices_per_warp"])
    h.close()
    # solves on the tuned choice: the FP64 bar, and the same bits twice
    ref = O.pcg(O.CSRD, True, s.ia, s.ja, s.al, s.ad, s.b[0], tol=TOL)
    x1, i1 = g.solve(sv.PCG, s.b[0], tol=TOL)
    x2, i2 = g.solve(sv.PCG, s.b[0], tol=TOL)
    assert i1.status == sv.OK and abs(i1.iters - ref.iters) <= 1
    assert rel(x1, ref.x) < 1e-12
    assert bits_equal(x1, x2) and i1.iters == i2.iters
    g.close()


@pytest.mark.parametrize("engine,threads,spw,pf,fused",
                         [(2, 128, 0, 0, 0), (2, 256, 2, 0, 0), (2, 256, 8, 0, 0),
                          (2, 256, 0, 2, 0), (2, 256, 0, 0, 1), (2, 256, 0, 0, 2),
                          (2, 256, 0, 0, 3), (2, 256, 0, 0, 4), (3, 256, 0, 0, 1),
                          (3, 256, 0, 0, 3), (3, 256, 0, 0, 4), (1, 0, 0, 0, 0)])
def test_every_candidate_shape_meets_the_fp64_bar(cuda, engine, threads, spw, pf, fused):
    """Whatever the tuner picks, the arithmetic is the reference's: every
    candidate engine and launch shape (the L2 prefetch, the fused one-kernel
    PCG iteration, also launched from a host loop) solves at the FP64 bar."""
    s = S.poisson_jittered(40, seed=22)
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    g.set_values(s.al, s.ad)
    g.set_engine(engine, threads, spw if spw else -1)
    g.set_prefetch(pf)
    g.set_fused(fused)
    ref = O.pcg(O.CSRD, True, s.ia, s.ja, s.al, s.ad, s.b[0], tol=TOL)
    maxit = ref.iters + 5 if engine == 3 else 100000  # the host loop runs exactly maxit
    x, info = g.solve(sv.PCG, s.b[0], tol=TOL, maxit=maxit)
    assert info.status == sv.OK and abs(info.iters - ref.iters) <= 1
    assert rel(x, ref.x) < 1e-12
    x2, info2 = g.solve(sv.PCG, s.b[0], tol=TOL, maxit=maxit)
    assert bits_equal(x, x2) and info2.iters == info.iters
    m = S.momentum(24, nrhs=3, seed=23)
    gm = sv.GpuSystem(m.neq, m.ia, m.ja, sv.CSRD, True)
    gm.set_values(m.al, m.ad)
    gm.set_engine(engine, threads, spw if spw else -1)
    gm.set_prefetch(pf)
    gm.set_fused(fused)
    xs, infos = gm.solve_multi(sv.PBICGSTAB, m.b, tol=TOL, maxit=200 if engine == 3 else 100000)
    for k in range(3):
        refk = O.pbicgstab(O.CSRD, True, m.ia, m.ja, m.al, m.ad, m.b[k], tol=TOL)
        assert infos[k].status == sv.OK and abs(infos[k].iters - refk.iters) <= 1
        assert rel(xs[k], refk.x) < 1e-12
    g.close()
    gm.close()


def test_fused_loop_matches_fused_iteration_bit_for_bit(cuda):
    """Mode 4 runs mode 3's iteration in one launch on the same blocks, with a
    wait on the neighbouring blocks where the kernel boundary was: the same
    arithmetic in the same order, so the same bits and iteration count."""
    s = S.poisson_jittered(40, seed=25)
    out = {}
    for mode in (3, 4):
        g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
        g.set_values(s.al, s.ad)
        g.set_engine(2, 256, -1)
        g.set_fused(mode)
        out[mode] = g.solve(sv.PCG, s.b[0], tol=TOL)
        g.close()
    (x3, i3), (x4, i4) = out[3], out[4]
    assert i3.status == sv.OK and i4.status == sv.OK and i3.iters == i4.iters
    assert bits_equal(x3, x4)


def _with_long_range_couplings(s, c=1e-3):
    """The CSRD system s with every row i also coupled to row i +- n/2 (value
    -c, the diagonal raised by c, so the matrix stays symmetric positive
    definite): the bandwidth is then about n/2."""
    n = s.neq
    ia, ja, al = [0], [], []
    ad = s.ad.copy()
    for i in range(n):
        j = i + n // 2 if i < n // 2 else i - n // 2
        cols = list(s.ja[s.ia[i]:s.ia[i + 1]])
        vals = list(s.al[s.ia[i]:s.ia[i + 1]])
        if j != i and j not in cols:
            k = int(np.searchsorted(cols, j))
            cols.insert(k, j)
            vals.insert(k, -c)
            ad[i] += c
        ja += cols
        al += vals
        ia.append(len(ja))
    return (np.array(ia, dtype=np.int32), np.array(ja, dtype=np.int32),
            np.array(al, dtype=np.float64), ad)


def test_fused_loop_long_range_couplings_take_the_grid_barrier(cuda):
    """Mode 4 waits after its update of p only on the blocks its rows gather
    from; when those span more blocks than a block has threads (here every
    row reaches n/2 rows away, 592 blocks) it falls back to a grid barrier.
    The bandwidth also rules out 16-bit column offsets, so this runs the
    32-bit-column kernel.  Both at the FP64 bar against the oracle."""
    s = S.poisson_jittered(64, seed=26)
    ia, ja, al, ad = _with_long_range_couplings(s)
    ref = O.pcg(O.CSRD, True, ia, ja, al, ad, s.b[0], tol=TOL)
    out = {}
    for mode in (3, 4):
        g = sv.GpuSystem(s.neq, ia, ja, sv.CSRD, True)
        g.set_values(al, ad)
        g.set_engine(2, 256, -1)
        g.set_fused(mode)
        out[mode] = g.solve(sv.PCG, s.b[0], tol=TOL)
        g.close()
    for mode, (x, info) in out.items():
        assert info.status == sv.OK, mode
        assert abs(info.iters - ref.iters) <= 1, (mode, info.iters, ref.iters)
        assert rel(x, ref.x) < 1e-12, mode
    assert bits_equal(out[3][0], out[4][0])


def test_autotune_mixed_k3_momentum(cuda):
    m = S.momentum(40, nrhs=3, seed=24)
    g = sv.GpuSystem(m.neq, m.ia, m.ja, sv.CSRD, True)
    g.set_values(m.al, m.ad)
    rep = g.autotune(sv.PBICGSTAB, m.b, tol=TOL, precision=sv.MIXED)
    assert rep["source"] == 0 and rep["ms"] <= rep["default_ms"]
    xs, infos = g.solve_multi(sv.PBICGSTAB, m.b, tol=TOL, precision=sv.MIXED)
    for k in range(3):
        assert infos[k].status == sv.OK
        r = m.b[k] - O.matvec(O.CSRD, True, m.ia, m.ja, m.al, m.ad, xs[k])
        assert np.linalg.norm(r) < TOL * np.linalg.norm(m.b[k])
    g.close()


def test_batch_autotune_keeps_the_fastest_plan(cuda):
    systems = S.poisson_batch(16, 6, 40, seed=25)
    g = sv.GpuBatch([(s.neq, s.ia, s.ja) for s in systems], sv.CSRD, True)
    g.set_values([s.al for s in systems], [s.ad for s in systems])
    bs = [s.b[0] for s in systems]
    ms = g.autotune(sv.PCG, bs, tol=TOL)
    rep = g.tune_report()
    assert rep["plans"] >= 2
    assert rep["tuned_ms"] == pytest.approx(ms)
    assert rep["tuned_ms"] <= min(rep["default_ms"], rep["weighted_ms"])
    assert rep["min_team_blocks"] >= 1 and rep["grid"] >= len(systems)
    xs, infos = g.solve(sv.PCG, bs, tol=TOL)
    for s, x, info in zip(systems, xs, infos):
        ref = O.pcg(O.CSRD, True, s.ia, s.ja, s.al, s.ad, s.b[0], tol=TOL)
        assert info.status == sv.OK and abs(info.iters - ref.iters) <= 1
        assert rel(x, ref.x) < 1e-12
    g.close()
