"""The seeded system generator (sfr3d_b200/csrc/systems.cpp)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from sfr3d_b200 import systems as S

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_solves.npz"))


def test_generator_pinned_by_fixtures():
    uni = S.poisson_uniform(8, seed=11)
    assert np.array_equal(uni.ia, GOLD["uni8_csrd_full/ia"])
    assert np.array_equal(uni.ja, GOLD["uni8_csrd_full/ja"])
    assert np.array_equal(uni.al, GOLD["uni8_csrd_full/al"])
    assert np.array_equal(uni.ad, GOLD["uni8_csrd_full/ad"])
    assert np.array_equal(uni.b[0], GOLD["uni8_csrd_full/b"])
    jit = S.poisson_jittered(10, seed=12)
    assert np.array_equal(jit.al, GOLD["jit10_csrd_full/al"])
    mom = S.momentum(8, peclet=50.0, nrhs=2, seed=13)
    assert np.array_equal(mom.al, GOLD["mom8_csrd_full/al"])
    assert np.array_equal(mom.b[1], GOLD["mom8_rhs1/b"])


def test_uniform_poisson_coefficients():
    n = 6
    s = S.poisson_uniform(n, seed=1)
    h = 1.0 / n
    assert np.allclose(-s.al, h)                      # k A / d = h
    A = s.dense()
    # row sums: 0 inside, 2h for cells touching the Dirichlet face x = 0
    e = s.numbering()
    rs = A.sum(axis=1)
    for c in range(n ** 3):
        i = c % n
        expect = 2 * h if i == 0 else 0.0
        assert abs(rs[e[c]] - expect) < 1e-14


def test_diffusion_is_symmetric_positive_definite():
    s = S.poisson_jittered(7, seed=3)
    A = s.dense()
    assert np.array_equal(A, A.T)
    assert np.linalg.eigvalsh(A)[0] > 0


def test_layouts_match_dense():
    for s in (S.poisson_jittered(6, seed=4), S.momentum(6, seed=5, nrhs=1)):
        A = s.dense()
        n = s.neq
        ja, a = s.ell()
        E = np.zeros_like(A)
        np.add.at(E, (np.repeat(np.arange(n), s.width), ja), a)
        E[np.arange(n), np.arange(n)] += s.ad
        assert np.array_equal(E, A)
        ia, jc, ac = s.csrc()
        rows = np.repeat(np.arange(n), np.diff(ia))
        assert np.array_equal(A[rows, jc], ac[: len(jc)])
        if s.unsym:
            assert np.array_equal(A[jc, rows], ac[len(jc):])
        else:
            il, jl, al = s.csrd_lower()
            assert np.array_equal(il, ia) and np.array_equal(jl, jc)


def test_momentum_peclet_and_divergence():
    s = S.momentum(10, peclet=50.0, seed=6, nrhs=1)
    A = s.dense()
    iu = np.triu_indices(s.neq, 1)
    apn, anp = A[iu], A.T[iu]
    mask = apn != 0
    F = np.abs(apn[mask] - anp[mask])          # |F_f|
    D = -(apn[mask] + anp[mask] + F) / 2.0     # D_f
    assert abs((F / D).max() - 50.0) < 1e-9
    # sum of each row = V/dt + wall terms (the fluxes cancel: div u = 0)
    h = np.pi / 10
    e = s.numbering()
    rs = A.sum(axis=1)
    for c in (0, 555, 999):
        i, j, k = c % 10, (c // 10) % 10, c // 100
        walls = sum(1 for v in (i, j, k) for end in (0, 9) if v == end)
        expect = h ** 3 / 1e-2 + walls * 1e-3 * h * h / (h / 2)
        assert abs(rs[e[c]] - expect) < 1e-12 * expect


def test_rcm_reduces_bandwidth_and_is_permutation():
    p = S.params(n=12, permute=True, rcm=False, seed=7)
    raw = S.build(p)
    p.rcm = 1
    ordered = S.build(p)
    assert ordered.bandwidth < raw.bandwidth / 5
    xadj = raw.ia.astype(np.int32)
    perm = S.rcm(xadj, raw.ja)
    assert np.array_equal(np.sort(perm), np.arange(raw.neq))


def test_batch_parameters():
    ps = S.batch_params(64, 8, 96, seed=4)
    assert len(ps) == 64
    sizes = [(p.nx, p.ny, p.nz) for p in ps]
    assert all(8 <= v <= 96 for t in sizes for v in t)
    assert sizes == [(p.nx, p.ny, p.nz) for p in S.batch_params(64, 8, 96, seed=4)]
    faces = {p.dirichlet_faces for p in ps}
    assert faces <= {1, 2, 4, 8, 16, 32} and len(faces) > 2


def test_invalid_parameters_rejected():
    with pytest.raises(ValueError):
        S.build(S.params(n=(0, 4, 4)))
    with pytest.raises(ValueError):
        S.build(S.params(n=4, jitter=0.7))
