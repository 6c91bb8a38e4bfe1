"""Generate tests/golden/coo/*: the reference's own Matrix Market dumps
(writeCoo / writeCooB, WriteMtx.c, built with its vendored mmio writer by
`make -C oracle ref`) of a seeded 3x3x3 jittered Poisson system, with the
inputs in inputs.npz: the CSRD full system, its symmetric (strict lower)
storage, the binary graph, and the force vector.

    python tests/golden/make_mtx_golden.py
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from sfr3d_b200 import systems as S  # noqa: E402

OUT = os.path.join(HERE, "coo")


def main():
    os.makedirs(OUT, exist_ok=True)
    L = O.ref_lib()
    L.sfr_ref_write_coo.argtypes = ([ctypes.c_int] * 2 + [ctypes.c_void_p] * 5
                                    + [ctypes.c_int] * 3 + [ctypes.c_char_p])
    L.sfr_ref_write_coo_b.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p]
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    s = S.poisson_jittered(3, seed=1)
    il, jl, al_l = s.csrd_lower()
    inputs = dict(ia=s.ia, ja=s.ja, al=s.al, ad=s.ad, il=il, jl=jl, al_lower=al_l, b=s.b[0])
    np.savez_compressed(os.path.join(OUT, "inputs.npz"), **inputs)
    for name, (ia, ja, al), unsym, binary in (("full", (s.ia, s.ja, s.al), 1, 0),
                                              ("lower", (il, jl, al_l), 0, 0),
                                              ("graph", (s.ia, s.ja, s.al), 1, 1)):
        ia, ja, al = (np.ascontiguousarray(x).copy() for x in (ia, ja, al))
        ad = s.ad.copy()
        rc = L.sfr_ref_write_coo(s.neq, len(ja), p(ia), p(ja), p(al), p(ad), p(al), O.CSRD,
                                 unsym, binary, os.path.join(OUT, f"{name}.mtx").encode())
        assert rc == 0
    b = s.b[0].copy()
    L.sfr_ref_write_coo_b(p(b), s.neq, os.path.join(OUT, "b.mtx").encode())
    for f in sorted(os.listdir(OUT)):
        print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
