"""Adjoint of the solve: transpose solve parity and gradients.

* The transpose solve A^T lam = g against the reference's BiCGSTAB run on an
  explicitly transposed CSRD (rows with ascending columns): the FP64 parity
  bar of the forward path (1e-12 relative in lam, iterations +-1).
* dJ/db = lam and dJ/da = -lam_i x_j against FP64 central differences of
  J = w.x, step 1e-6 relative to the coefficient, on seeded coefficients
  (off-diagonal and diagonal) and right-hand-side entries: agreement to
  1e-6 relative (entries whose derivative is below 1e-3 of the largest
  sampled one are held to 1e-9 of that largest instead).
* The torch.autograd harness: backward equals the C-ABI adjoint, and
  torch.autograd.gradcheck passes on a small system.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import layouts, rel, transpose_csrd
from oracle import oracle as O
from sfr3d_b200 import adjoint as A
from sfr3d_b200 import solver as sv
from sfr3d_b200 import systems as S

pytestmark = pytest.mark.gpu

TOL_X = 1e-12
TOL_FD = 1e-6


def _reference_transpose(sysx, g, tol):
    t_ia, t_ja, t_al = transpose_csrd(sysx.neq, sysx.ia, sysx.ja, sysx.al)
    if O.ref_available():
        return O.ref_solve(O.PBICGSTAB, O.CSRD, True, t_ia, t_ja, t_al, sysx.ad, g, tol=tol)
    return O.pbicgstab(O.CSRD, True, t_ia, t_ja, t_al, sysx.ad, g, tol=tol)


def _gpu(sysx, lname, engine=0):
    st, un, ia, ja, al, au = layouts(sysx)[lname]
    g = sv.GpuSystem(sysx.neq, ia, ja, st, un)
    g.set_values(al, sysx.ad, au)
    g.set_engine(engine)
    return g, (st, un, ia, ja, al)


@pytest.mark.parametrize("lname", ["csrd_full", "csrc_unsym", "ellpack"])
def test_transpose_solve_matches_reference(cuda, engine, lname):
    s = S.momentum(20, peclet=20.0, seed=61, nrhs=1)
    w = np.random.default_rng(61).standard_normal(s.neq)
    ref = _reference_transpose(s, w, 1e-10)
    assert ref.status == 0
    g, _ = _gpu(s, lname, engine)
    lam, info = g.solve_transpose(sv.PBICGSTAB, w, tol=1e-10)
    assert info.status == sv.OK
    assert abs(info.iters - ref.iters) <= 1
    assert rel(lam, ref.x) <= TOL_X
    # the transpose really is a different system (Peclet 20 is nonsymmetric)
    x, _ = g.solve(sv.PBICGSTAB, w, tol=1e-10)
    assert rel(x, lam) > 1e-6
    g.close()


def test_transpose_of_symmetric_is_forward(cuda, engine):
    s = S.poisson_uniform(12, seed=62)
    b = s.b[0]
    g, _ = _gpu(s, "csrc_sym", engine)
    x, i1 = g.solve(sv.PCG, b, tol=1e-10)
    lam, i2 = g.solve_transpose(sv.PCG, b, tol=1e-10)
    assert i1.iters == i2.iters
    assert rel(lam, x) <= TOL_X
    g.close()


def _sample(sysx, lname, g, ia, ja, al, rng, n_off=24, n_diag=8, n_b=32):
    """Seeded coefficients: off-diagonals with a nonzero value, diagonals, b."""
    nz = np.flatnonzero(np.asarray(al) != 0.0)
    ent = []
    for k in rng.choice(nz, n_off, replace=False):
        ent.append(A.Entry("al", int(k), A.value_positions(g, ia, ja, "al", int(k))))
    for i in rng.choice(sysx.neq, n_diag, replace=False):
        ent.append(A.Entry("ad", int(i), [(int(i), int(i))]))
    for i in rng.choice(sysx.neq, n_b, replace=False):
        ent.append(A.Entry("b", int(i), []))
    return ent


def _fd_errors(adj, fd):
    scale = np.max(np.abs(fd))
    big = np.abs(fd) >= 1e-3 * scale
    rel_err = np.abs(adj[big] - fd[big]) / np.abs(fd[big])
    small_err = np.abs(adj[~big] - fd[~big]) / scale if np.any(~big) else np.zeros(1)
    return float(rel_err.max()), float(small_err.max())


def _adjoint_vs_fd(sysx, lname, solver, precision, seed, engine=0):
    g, (st, un, ia, ja, al) = _gpu(sysx, lname, engine)
    b = sysx.b[0]
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(sysx.neq)
    x, info = g.solve(solver, b, tol=1e-14, maxit=5000, raise_on_error=False)
    assert info.status in (sv.OK, sv.MAXIT)
    lam, g_al, g_ad, g_au, ainfo = g.adjoint(
        solver, x, w, tol=1e-12 if precision == sv.FP64 else 1e-10,
        precision=precision)
    assert ainfo.status == sv.OK
    g_all = np.concatenate([g_al, g_au]) if g_au is not None else g_al
    ent = _sample(sysx, lname, g, ia, ja, al, rng)
    fd = A.central_differences(g, solver, al, sysx.ad, None, b, x, w, ent,
                               rel_step=1e-6, tol=1e-13, maxit=5000)
    arrays = {"al": g_all, "ad": g_ad, "b": lam}
    adj = np.array([arrays[e.array][e.index] for e in ent])
    g.close()
    return adj, fd, ent


@pytest.mark.parametrize("precision", [sv.FP64, sv.MIXED], ids=["fp64", "mixed"])
@pytest.mark.parametrize("lname", ["csrd_full", "csrc_unsym", "ellpack"])
def test_adjoint_gradients_vs_central_differences(cuda, lname, precision):
    s = S.momentum(12, peclet=20.0, seed=63, nrhs=1)
    adj, fd, _ = _adjoint_vs_fd(s, lname, sv.PBICGSTAB, precision, 63)
    r, a = _fd_errors(adj, fd)
    assert r <= TOL_FD and a <= 1e-9, (r, a)


@pytest.mark.parametrize("lname", ["csrd_sym", "csrc_sym"])
def test_adjoint_mirrored_values_vs_central_differences(cuda, lname):
    # strict-lower storage: one stored value is two matrix entries
    s = S.poisson_jittered(10, seed=64)
    adj, fd, _ = _adjoint_vs_fd(s, lname, sv.PCG, sv.FP64, 64)
    r, a = _fd_errors(adj, fd)
    assert r <= TOL_FD and a <= 1e-9, (r, a)


def test_adjoint_graph_engine_matches_persistent(cuda):
    s = S.momentum(16, peclet=20.0, seed=65, nrhs=1)
    w = np.random.default_rng(65).standard_normal(s.neq)
    out = []
    for eng in (1, 2):
        g, _ = _gpu(s, "csrd_full", eng)
        x, _ = g.solve(sv.PBICGSTAB, s.b[0], tol=1e-12)
        out.append(g.adjoint(sv.PBICGSTAB, x, w, tol=1e-12))
        g.close()
    (l1, a1, d1, _, i1), (l2, a2, d2, _, i2) = out
    assert abs(i1.iters - i2.iters) <= 1
    assert rel(l1, l2) <= TOL_X and rel(a1, a2) <= TOL_X and rel(d1, d2) <= TOL_X


def test_autograd_backward_equals_capi(cuda):
    import torch
    s = S.momentum(10, peclet=20.0, seed=66, nrhs=1)
    g, (st, un, ia, ja, al) = _gpu(s, "csrd_full")
    w = torch.from_numpy(np.random.default_rng(66).standard_normal(s.neq))
    t_al = torch.tensor(al, requires_grad=True)
    t_ad = torch.tensor(s.ad, requires_grad=True)
    t_b = torch.tensor(s.b[0], requires_grad=True)
    x = A.linear_solve(g, t_al, t_ad, t_b, tol=1e-13)
    (w * x).sum().backward()
    lam, g_al, g_ad, _, _ = g.adjoint(sv.PBICGSTAB, x.detach().numpy(), w.numpy(), tol=1e-13)
    assert rel(t_b.grad.numpy(), lam) <= 1e-12
    assert rel(t_al.grad.numpy(), g_al) <= 1e-12
    assert rel(t_ad.grad.numpy(), g_ad) <= 1e-12
    g.close()


def test_autograd_gradcheck_small(cuda):
    import torch
    s = S.momentum(3, peclet=20.0, seed=67, nrhs=1)
    g, (st, un, ia, ja, al) = _gpu(s, "csrd_full")
    t_al = torch.tensor(al, requires_grad=True)
    t_ad = torch.tensor(s.ad, requires_grad=True)
    t_b = torch.tensor(s.b[0], requires_grad=True)
    fn = lambda a, d, bb: A.linear_solve(g, a, d, bb, tol=1e-15, maxit=2000)
    assert torch.autograd.gradcheck(fn, (t_al, t_ad, t_b), eps=1e-6, atol=1e-7, rtol=1e-5)
    g.close()


def test_adjoint_config5_full_size(cuda):
    """96^3 convection-diffusion, Peclet 20: 32 coefficients + 32 b entries
    against central differences (FP64 and mixed adjoint), lam against the
    reference's transpose solve."""
    s = S.momentum(96, peclet=20.0, seed=5, nrhs=1)
    w = np.random.default_rng(5).standard_normal(s.neq)
    g, (st, un, ia, ja, al) = _gpu(s, "csrd_full")
    x, info = g.solve(sv.PBICGSTAB, s.b[0], tol=1e-14, maxit=5000, raise_on_error=False)
    assert info.status in (sv.OK, sv.MAXIT)
    ref = _reference_transpose(s, w, 1e-10)
    lam10, i10 = g.solve_transpose(sv.PBICGSTAB, w, tol=1e-10)
    assert abs(i10.iters - ref.iters) <= 1 and rel(lam10, ref.x) <= TOL_X
    rng = np.random.default_rng(5)
    ent = _sample(s, "csrd_full", g, ia, ja, al, rng)
    fd = A.central_differences(g, sv.PBICGSTAB, al, s.ad, None, s.b[0], x, w, ent,
                               rel_step=1e-6, tol=1e-13, maxit=5000)
    for precision, tol in ((sv.FP64, 1e-12), (sv.MIXED, 1e-10)):
        lam, g_al, g_ad, _, ainfo = g.adjoint(sv.PBICGSTAB, x, w, tol=tol, precision=precision)
        assert ainfo.status == sv.OK
        arrays = {"al": g_al, "ad": g_ad, "b": lam}
        adj = np.array([arrays[e.array][e.index] for e in ent])
        r, a = _fd_errors(adj, fd)
        assert r <= TOL_FD and a <= 1e-9, (precision, r, a)
    g.close()
