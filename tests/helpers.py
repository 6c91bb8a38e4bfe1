"""Helpers shared by the test modules."""
from __future__ import annotations

import numpy as np


def rel(a, b) -> float:
    """||a - b||_2 / ||b||_2."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def layouts(sys_):
    """The reference layouts of one generated system, keyed by name:
    (storage, unsym, ia, ja, al, au)."""
    from oracle import oracle as O
    out = {"csrd_full": (O.CSRD, True, sys_.ia, sys_.ja, sys_.al, None)}
    ej, ea = sys_.ell()
    out["ellpack"] = (O.ELLPACK, sys_.unsym, O.ell_ia(sys_.neq, sys_.width), ej, ea, None)
    ia, ja, a = sys_.csrc()
    if sys_.unsym:
        out["csrc_unsym"] = (O.CSRC, True, ia, ja, a, None)
    else:
        il, jl, alo = sys_.csrd_lower()
        out["csrd_sym"] = (O.CSRD, False, il, jl, alo, None)
        out["csrc_sym"] = (O.CSRC, False, ia, ja, a[: len(ja)], None)
    return out


def transpose_csrd(neq, ia, ja, al):
    """Explicit transpose of a full CSRD matrix (off-diagonals only, the
    diagonal is shared): rows of A^T with ascending column indices, the
    order a transposed CSRD built by sorting takes."""
    ia = np.asarray(ia, dtype=np.int64)
    ja = np.asarray(ja, dtype=np.int64)
    al = np.asarray(al, dtype=np.float64)
    base = int(ia[0])
    rows = np.repeat(np.arange(neq), np.diff(ia))
    cols = ja[base:base + len(rows)]
    order = np.lexsort((rows, cols))  # by new row (= col), then new col (= row)
    t_rows = cols[order]
    t_cols = rows[order]
    t_val = al[: len(rows)][order]
    t_ia = np.zeros(neq + 1, dtype=np.int32)
    np.add.at(t_ia, t_rows + 1, 1)
    t_ia = np.cumsum(t_ia).astype(np.int32)
    return t_ia, t_cols.astype(np.int32), t_val
