"""ctypes wrappers of the parity oracle (test infrastructure only).

``pcg`` / ``pbicgstab`` / ``pbicgstabl2`` / ``gmres`` / ``minres`` /
``matvec`` run the C restatement (sfr3d_oracle.c);
``ref_solve`` runs the reference's own compiled solverC (Solv.c:64) through
ref_harness.c, serial (nthreads=0) or OpenMP (nthreads>=1).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libsfr3d_ref.so")

CSRD, CSRC, ELLPACK = 2, 3, 4
PCG, PBICGSTAB, PBICGSTABL2, GMRES, MINRES = 1, 2, 3, 4, 5  # Define.h:392-396
NKRYLOV = 15  # solverC's GMRES restart length (Solv.c:82)

_P = ctypes.c_void_p


class _Stats(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int), ("status", ctypes.c_int),
                ("xKx", ctypes.c_double), ("norm_x", ctypes.c_double),
                ("norm_r", ctypes.c_double), ("norm_r_m", ctypes.c_double),
                ("conv", ctypes.c_double)]


@dataclass
class SolveResult:
    x: np.ndarray
    iters: int
    status: int
    xKx: float
    norm_x: float
    norm_r: float = float("nan")
    norm_r_m: float = float("nan")
    conv: float = float("nan")
    seconds: float = float("nan")


_libs: dict[str, ctypes.CDLL] = {}


def _load(path):
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"{path} is not built (make -C oracle [ref])")
        _libs[path] = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
    return _libs[path]


def oracle_lib():
    lib = _load(LIB_ORACLE)
    if not getattr(lib, "_typed", False):
        lib.orc_dot.restype = ctypes.c_double
        lib.orc_dot.argtypes = [_P, _P, ctypes.c_int]
        lib.orc_matvec.restype = None
        lib.orc_matvec.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   _P, _P, _P, _P, _P, _P]
        for f in (lib.orc_pcg, lib.orc_pbicgstab, lib.orc_minres, lib.orc_pbicgstabl2):
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _P,
                          _P, _P, _P, ctypes.c_double, ctypes.c_uint,
                          ctypes.c_int, ctypes.POINTER(_Stats)]
        lib.orc_set_dot_order.restype = None
        lib.orc_set_dot_order.argtypes = [ctypes.c_int]
        lib.orc_gmres.restype = ctypes.c_int
        lib.orc_gmres.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P, _P,
                                  _P, _P, _P, ctypes.c_double, ctypes.c_uint,
                                  ctypes.c_int, ctypes.c_int, ctypes.POINTER(_Stats)]
        lib._typed = True
    return lib


def order_spread(solver, storage, unsym, ia, ja, al, ad, b, **kw):
    """How far the reference's own algorithm moves when only the summation
    order of its dot products changes (right to left, pairwise): the largest
    change in the iteration count and the largest relative change in x,
    against the reference order."""
    lib = oracle_lib()
    fn = SOLVERS[solver]
    base = fn(storage, unsym, ia, ja, al, ad, b, **kw)
    d_it, d_x = 0, 0.0
    try:
        for order in (1, 2):
            lib.orc_set_dot_order(order)
            r = fn(storage, unsym, ia, ja, al, ad, b, **kw)
            d_it = max(d_it, abs(r.iters - base.iters))
            d_x = max(d_x, float(np.linalg.norm(r.x - base.x) / np.linalg.norm(base.x)))
    finally:
        lib.orc_set_dot_order(0)
    return d_it, d_x


def ref_available() -> bool:
    return os.path.exists(LIB_REF)


def ref_lib():
    lib = _load(LIB_REF)
    if not getattr(lib, "_typed", False):
        lib.sfr_ref_solve.restype = ctypes.c_int
        lib.sfr_ref_solve.argtypes = (
            [ctypes.c_int, ctypes.c_int] + [_P] * 7 +
            [ctypes.c_double, ctypes.c_uint] + [ctypes.c_int] * 5 + [_P] * 4)
        lib.sfr_ref_smachn.restype = ctypes.c_double
        lib.sfr_ref_max_threads.restype = ctypes.c_int
        lib._typed = True
    return lib


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a):
    return a.ctypes.data_as(_P)


def dot(a, b) -> float:
    a = _c(a, np.float64)
    b = _c(b, np.float64)
    return oracle_lib().orc_dot(_p(a), _p(b), len(a))


def matvec(storage, unsym, ia, ja, al, ad, x) -> np.ndarray:
    ia, ja = _c(ia, np.int32), _c(ja, np.int32)
    al, ad, x = _c(al, np.float64), _c(ad, np.float64), _c(x, np.float64)
    y = np.zeros(len(ad))
    oracle_lib().orc_matvec(storage, int(unsym), len(ad), _p(ia), _p(ja),
                            _p(al), _p(ad), _p(x), _p(y))
    return y


def _solve(fn, storage, unsym, ia, ja, al, ad, b, x0, tol, maxit, newx, *extra):
    ia, ja = _c(ia, np.int32), _c(ja, np.int32)
    al, ad, b = _c(al, np.float64), _c(ad, np.float64), _c(b, np.float64)
    x = np.zeros(len(ad)) if x0 is None else np.array(x0, dtype=np.float64)
    st = _Stats()
    fn(storage, int(unsym), len(ad), _p(ia), _p(ja), _p(al), _p(ad), _p(b),
       _p(x), tol, maxit, int(newx), *extra, ctypes.byref(st))
    return SolveResult(x=x, iters=st.iters, status=st.status, xKx=st.xKx,
                       norm_x=st.norm_x, norm_r=st.norm_r,
                       norm_r_m=st.norm_r_m, conv=st.conv)


def pcg(storage, unsym, ia, ja, al, ad, b, x0=None, tol=1e-10,
        maxit=100000, newx=True) -> SolveResult:
    """Restatement of pcg (Cg.c:47-209)."""
    return _solve(oracle_lib().orc_pcg, storage, unsym, ia, ja, al, ad, b, x0,
                  tol, maxit, newx)


def pbicgstab(storage, unsym, ia, ja, al, ad, b, x0=None, tol=1e-10,
              maxit=100000, newx=True) -> SolveResult:
    """Restatement of pbicgstab (Bicgstab.c:50-245)."""
    return _solve(oracle_lib().orc_pbicgstab, storage, unsym, ia, ja, al, ad,
                  b, x0, tol, maxit, newx)


def minres(storage, unsym, ia, ja, al, ad, b, x0=None, tol=1e-10,
           maxit=100000, newx=True) -> SolveResult:
    """Restatement of pminres (Iters.c:309-558)."""
    return _solve(oracle_lib().orc_minres, storage, unsym, ia, ja, al, ad, b, x0,
                  tol, maxit, newx)


def pbicgstabl2(storage, unsym, ia, ja, al, ad, b, x0=None, tol=1e-10,
                maxit=100000, newx=True) -> SolveResult:
    """Restatement of pbicgstabl2 (Bicgstab.c:1172-1460)."""
    return _solve(oracle_lib().orc_pbicgstabl2, storage, unsym, ia, ja, al, ad,
                  b, x0, tol, maxit, newx)


def gmres(storage, unsym, ia, ja, al, ad, b, x0=None, tol=1e-10,
          maxit=100000, newx=True, nk=NKRYLOV) -> SolveResult:
    """Restatement of gmres (Iters.c:587-800); maxit counts cycles."""
    return _solve(oracle_lib().orc_gmres, storage, unsym, ia, ja, al, ad, b, x0,
                  tol, maxit, newx, int(nk))


SOLVERS = {PCG: pcg, PBICGSTAB: pbicgstab, PBICGSTABL2: pbicgstabl2, GMRES: gmres,
           MINRES: minres}


def ref_solve(solver, storage, unsym, ia, ja, al, ad, b, x0=None, tol=1e-10,
              maxit=100000, newx=True, nthreads=0, au=None) -> SolveResult:
    """The reference's own solverC (Solv.c:64) on one system."""
    lib = ref_lib()
    ia, ja = _c(ia, np.int32).copy(), _c(ja, np.int32).copy()
    al, ad, b = (_c(al, np.float64).copy(), _c(ad, np.float64).copy(),
                 _c(b, np.float64).copy())
    au_p = None if au is None else _p(_c(au, np.float64))
    x = np.zeros(len(ad)) if x0 is None else np.array(x0, dtype=np.float64)
    iters = ctypes.c_int()
    xkx, nx, sec = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    nad = len(ja) if storage != ELLPACK else int(ia[1])
    rc = lib.sfr_ref_solve(len(ad), nad, _p(ia), _p(ja), _p(al), _p(ad), au_p,
                           _p(b), _p(x), tol, maxit, storage, solver,
                           int(newx), int(unsym), nthreads, ctypes.byref(iters),
                           ctypes.byref(xkx), ctypes.byref(nx),
                           ctypes.byref(sec))
    return SolveResult(x=x, iters=iters.value, status=rc, xKx=xkx.value,
                       norm_x=nx.value, seconds=sec.value)


def ell_ia(neq: int, width: int) -> np.ndarray:
    """The ifEllPack header solverC receives as ia for ELLPACK
    (EllPack.c:35-36): [width, neq*width]."""
    return np.array([width, neq * width], dtype=np.int32)
