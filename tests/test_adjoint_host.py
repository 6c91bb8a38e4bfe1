"""Host-side pieces of the adjoint check (no GPU): the explicit transpose
used for the reference's transpose solve, and the map from a stored value
to the matrix positions it occupies."""
from __future__ import annotations

import numpy as np

from helpers import layouts, transpose_csrd
from oracle import oracle as O
from sfr3d_b200 import adjoint as A
from sfr3d_b200 import systems as S


class _Pattern:
    """The attributes value_positions reads from a GpuSystem."""

    def __init__(self, neq, storage, unsym):
        self.neq, self.storage, self.unsym = neq, storage, unsym


def _dense_from_csrd(neq, ia, ja, al, ad):
    m = np.diag(np.asarray(ad, dtype=np.float64))
    for i in range(neq):
        for k in range(ia[i], ia[i + 1]):
            m[i, ja[k]] = al[k]
    return m


def test_transpose_csrd_is_dense_transpose():
    s = S.momentum(5, peclet=20.0, seed=71, nrhs=1)
    t_ia, t_ja, t_al = transpose_csrd(s.neq, s.ia, s.ja, s.al)
    dense = s.dense()
    assert np.array_equal(_dense_from_csrd(s.neq, t_ia, t_ja, t_al, s.ad), dense.T)
    for i in range(s.neq):  # ascending columns in every row
        assert np.all(np.diff(t_ja[t_ia[i]:t_ia[i + 1]]) > 0)


def test_oracle_transpose_solve_solves_transpose():
    s = S.momentum(6, peclet=20.0, seed=72, nrhs=1)
    g = np.random.default_rng(72).standard_normal(s.neq)
    t_ia, t_ja, t_al = transpose_csrd(s.neq, s.ia, s.ja, s.al)
    r = O.pbicgstab(O.CSRD, True, t_ia, t_ja, t_al, s.ad, g, tol=1e-12)
    lam = np.linalg.solve(s.dense().T, g)
    assert np.linalg.norm(r.x - lam) <= 1e-9 * np.linalg.norm(lam)


def test_value_positions_cover_the_matrix():
    """Every stored value maps to positions whose dense entries equal it,
    and together the values cover every off-diagonal of the matrix once."""
    for sysx in (S.momentum(4, peclet=20.0, seed=73, nrhs=1), S.poisson_jittered(4, seed=74)):
        dense = sysx.dense()
        for name, (st, un, ia, ja, al, au) in layouts(sysx).items():
            pat = _Pattern(sysx.neq, st, un)
            hit = np.zeros_like(dense, dtype=np.int64)
            for k in range(len(al)):
                for (i, j) in A.value_positions(pat, ia, ja, "al", k):
                    if st == O.ELLPACK and al[k] == 0.0:
                        continue  # ELLPACK padding
                    assert dense[i, j] == al[k], (name, k)
                    hit[i, j] += 1
            off = (dense != 0) & ~np.eye(sysx.neq, dtype=bool)
            assert np.array_equal(hit[off], np.ones(off.sum(), dtype=np.int64)), name
            assert hit[~off].sum() == 0, name
