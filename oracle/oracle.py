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



class _Rank(ctypes.Structure):
    _fields_ = [("nEq", ctypes.c_int), ("nEqNov", ctypes.c_int), ("nAd", ctypes.c_int),
                ("nAdR", ctypes.c_int), ("unsym", ctypes.c_int), ("ia", _P), ("ja", _P),
                ("al", _P), ("ad", _P), ("nRcvs", ctypes.c_int), ("nSends", ctypes.c_int),
                ("nVizPart", ctypes.c_int), ("iaSends", _P), ("iaRcvs", _P), ("fMap", _P),
                ("vizPart", _P), ("storage", ctypes.c_int)]


def mpi_solve(solver, ranks, al, ad, b, x0=None, tol=1e-10, maxit=100000,
              newx=True) -> tuple[list, SolveResult]:
    """Restatement of mpiPcg (Cg.c:256-442) / mpiPbicgstab (Bicgstab.c:298-520)
    with the ranks simulated in one process.  ranks[r] has the attributes
    unsym, nEq, nEqNov, nAd, nAdR, ia, ja, iaSends, iaRcvs, fMap, vizPart and
    optionally storage (the reference's MPI layout -- CSRD by default, or
    CSRC, ELLPACK, CSRDCOO, CSRCCOO -- and its Interface); al[r], ad[r], b[r] its values and
    rows of b; x0[r] its nEq entries.  Returns ([x_r], SolveResult) with
    SolveResult.x the concatenated rows."""
    lib = oracle_lib()
    if not getattr(lib, "_mpi_typed", False):
        lib.orc_mpi_solve.restype = ctypes.c_int
        lib.orc_mpi_solve.argtypes = [ctypes.c_int, ctypes.c_int, _P, _P, _P, ctypes.c_double,
                                      ctypes.c_uint, ctypes.c_int, ctypes.POINTER(_Stats)]
        lib._mpi_typed = True
    n = len(ranks)
    keep = []
    arr = (_Rank * n)()
    xs = []
    for r, q in enumerate(ranks):
        ia, ja = _c(q.ia, np.int32), _c(q.ja, np.int32)
        a, d = _c(al[r], np.float64), _c(ad[r], np.float64)
        ias, iar, fm = _c(q.iaSends, np.int32), _c(q.iaRcvs, np.int32), _c(q.fMap, np.int32)
        vz = _c(q.vizPart, np.int16)
        bb = _c(b[r], np.float64)
        keep += [ia, ja, a, d, ias, iar, fm, vz, bb]
        nrcv = q.nEq - q.nEqNov
        arr[r] = _Rank(q.nEq, q.nEqNov, q.nAd, q.nAdR, int(bool(q.unsym)), _p(ia), _p(ja),
                       _p(a), _p(d), nrcv, len(fm) - nrcv, len(vz), _p(ias), _p(iar),
                       _p(fm), _p(vz), int(getattr(q, "storage", CSRD)))
        xs.append(np.zeros(q.nEq) if x0 is None else np.array(x0[r], dtype=np.float64))
    bp = (_P * n)(*[_p(keep[9 * r + 8]) for r in range(n)])
    xp = (_P * n)(*[_p(x) for x in xs])
    st = _Stats()
    rc = lib.orc_mpi_solve(int(solver), n, ctypes.cast(arr, _P), bp, xp, tol, maxit,
                           int(newx), ctypes.byref(st))
    if rc < 0:
        raise ValueError("orc_mpi_solve: bad interface")
    x = np.concatenate([xs[r][:q.nEqNov] for r, q in enumerate(ranks)])
    return xs, SolveResult(x=x, iters=st.iters, status=st.status, xKx=st.xKx,
                           norm_x=st.norm_x, norm_r=st.norm_r, norm_r_m=st.norm_r_m,
                           conv=st.conv)

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


# ------------------------------------------------ diffusion assembly --
# systFormDif (CellLoop.c:285-455) -> cellDif3D (CellDif.c:312-537)
MAXLOADPAR = 20                                   # Define.h:336
DIRICHLET, NEUMANN, ROBIN, SINBC, INLET, OUTLET = 1, 2, 3, 4, 6, 7  # Define.h:317-323
MOVEWALL, INLETSTAICTPRES, OPEN, INLETTOTALPRES, STATICWALL, FLUXPRES = 8, 9, 10, 13, 14, 15
MAXPROP, DENSITY = 10, 1                                           # Define.h:349, 203
ORTHOGONAL, MINIMAL, ORTHOGONALC, OVERRELAXED = 1, 2, 3, 4        # Define.h:304-307
EULER, BACKWARD = 0, 1                                             # Define.h:191-192


@dataclass
class Load:
    """One entry of the reference's load table (Loads, StructDefine.h:356):
    type, parameters, nTypeVar (0 constant, 1 function)."""
    type: int
    par: tuple = ()
    var: int = 0
    np: int | None = None
    density: float = 0.0

    def arrays(self):
        par = np.zeros(MAXLOADPAR)
        par[:len(self.par)] = self.par
        return self.type, self.var, len(self.par) if self.np is None else self.np, par


@dataclass
class DifCase:
    """Everything one systFormDif call reads besides the pattern: the mesh
    arrays (any object with the attributes of sfr3d_b200.systems.FvMesh),
    the per-cell fields and the options."""
    mesh: object
    facer: np.ndarray            # (numel, maxviz + 1) short
    loads: list
    density: np.ndarray
    cdiff: np.ndarray
    u0: np.ndarray
    gradu0: np.ndarray           # (numel, 3)
    icod: int = ORTHOGONAL
    fres: bool = True
    time_flag: bool = False
    time_type: int = EULER
    dt: float = 1.0
    dt0: float = 1.0
    caltype: np.ndarray | None = None
    mat: np.ndarray | None = None

    def material(self):
        mat = (np.ones(self.mesh.numel, np.int16) if self.mat is None
               else _c(self.mat, np.int16))
        cal = np.ones(1, np.int16) if self.caltype is None else _c(self.caltype, np.int16)
        return cal, mat

    def load_arrays(self):
        n = max(len(self.loads), 1)
        t = np.zeros(n, np.int32)
        v = np.zeros(n, np.int32)
        npar = np.zeros(n, np.int32)
        par = np.zeros((n, MAXLOADPAR))
        for i, ld in enumerate(self.loads):
            t[i], v[i], npar[i], par[i] = ld.arrays()
        return t, v, npar, par


def dif_size(storage, unsym, neq, ia, ja) -> int:
    """Length of the value array the assembly writes (al, al|au, ELL slots)."""
    if storage == ELLPACK:
        return int(ia[1])
    return 2 * len(ja) if (storage == CSRC and unsym) else len(ja)


class _DifMesh(ctypes.Structure):
    _fields_ = [("numel", ctypes.c_int), ("maxviz", ctypes.c_int)] + [
        (n, _P) for n in ("nelcon", "nface", "cellface", "owner", "volume",
                          "dcca", "xmcc", "mksi", "ksi", "area", "normal",
                          "vskew", "caltype", "mat", "id", "facer")]


class _DifLoad(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("var", ctypes.c_int), ("np", ctypes.c_int),
                ("par", ctypes.c_double * MAXLOADPAR), ("density", ctypes.c_double)]


def _load_table(loads):
    arr = (_DifLoad * max(len(loads), 1))()
    for i, ld in enumerate(loads):
        t, v, npar, par = ld.arrays()
        arr[i].type, arr[i].var, arr[i].np = int(t), int(v), int(npar)
        arr[i].par[:] = list(par)
        arr[i].density = ld.density
    return arr


def _load_arrays(loads):
    n = max(len(loads), 1)
    t, v, npar = (np.zeros(n, np.int32) for _ in range(3))
    par, dens = np.zeros((n, MAXLOADPAR)), np.zeros(n)
    for i, ld in enumerate(loads):
        t[i], v[i], npar[i], par[i] = ld.arrays()
        dens[i] = ld.density
    return t, v, npar, par, dens


class _DifOpts(ctypes.Structure):
    _fields_ = [("icod", ctypes.c_int), ("fres", ctypes.c_int),
                ("time_flag", ctypes.c_int), ("time_type", ctypes.c_int),
                ("dt", ctypes.c_double), ("dt0", ctypes.c_double)]


def _dif_out(storage, unsym, neq, ia, ja, numel, fill):
    a = np.full(dif_size(storage, unsym, neq, ia, ja), fill)
    return a, np.full(neq, fill), np.full(neq, fill), np.full(numel, fill)


def dif_assemble(case: DifCase, storage, unsym, ia, ja, neq, forces=True,
                 matrix=True, calrcell=True, fill=0.0):
    """The C restatement of systFormDif: (rc, a, ad, b, rcell)."""
    m = case.mesh
    lib = oracle_lib()
    if not getattr(lib, "_dif_typed", False):
        lib.orc_dif_assemble.restype = ctypes.c_int
        lib.orc_dif_assemble.argtypes = (
            [ctypes.POINTER(_DifMesh), ctypes.POINTER(_DifLoad), ctypes.c_int,
             ctypes.POINTER(_DifOpts)] + [_P] * 4 + [ctypes.c_int] * 4 + [_P] * 6
            + [ctypes.c_int] * 3)
        lib._dif_typed = True
    cal, mat = case.material()
    keep = dict(
        nelcon=_c(m.nelcon, np.int32), nface=_c(m.nviz, np.int16),
        cellface=_c(m.cellface, np.int32), owner=_c(m.owner, np.int32),
        volume=_c(m.volume, np.float64), dcca=_c(m.dcca, np.float64),
        xmcc=_c(m.xmcc, np.float64), mksi=_c(m.mksi, np.float64),
        ksi=_c(m.ksi, np.float64), area=_c(m.area, np.float64),
        normal=_c(m.normal, np.float64), vskew=_c(m.vskew, np.float64),
        caltype=cal, mat=mat, id=_c(m.id, np.int32), facer=_c(case.facer, np.int16))
    dm = _DifMesh(numel=m.numel, maxviz=m.nelcon.shape[1],
                  **{k: _p(v) for k, v in keep.items()})
    loads = _load_table(case.loads)
    o = _DifOpts(icod=case.icod, fres=int(case.fres), time_flag=int(case.time_flag),
                 time_type=case.time_type, dt=case.dt, dt0=case.dt0)
    ia, ja = _c(ia, np.int32), _c(ja, np.int32)
    a, ad, b, rc_ = _dif_out(storage, unsym, neq, ia, ja, m.numel, fill)
    fields = [_c(case.density, np.float64), _c(case.cdiff, np.float64),
              _c(case.u0, np.float64), _c(case.gradu0, np.float64)]
    nad = len(ja) if storage != ELLPACK else 0
    rc = lib.orc_dif_assemble(ctypes.byref(dm), loads, len(case.loads), ctypes.byref(o),
                              *[_p(f) for f in fields], storage, int(unsym), neq, nad,
                              _p(ia), _p(ja), _p(a), _p(ad), _p(b), _p(rc_),
                              int(forces), int(matrix), int(calrcell))
    return rc, a, ad, b, rc_


def ref_dif_assemble(case: DifCase, storage, unsym, ia, ja, neq, forces=True,
                     matrix=True, calrcell=True, fill=0.0):
    """The reference's own systFormDif: (rc, a, ad, b, rcell, seconds)."""
    m = case.mesh
    lib = ref_lib()
    if not getattr(lib, "_dif_typed", False):
        lib.sfr_ref_syst_form_dif.restype = ctypes.c_int
        lib.sfr_ref_syst_form_dif.argtypes = (
            [ctypes.c_int, ctypes.c_int] + [_P] * 29 + [ctypes.c_int] + [_P] * 4
            + [ctypes.c_int] * 4 + [ctypes.c_double] * 2 + [ctypes.c_int] * 7 + [_P])
        lib._dif_typed = True
    cal, mat = case.material()
    cp = lambda x, dt: np.array(x, dtype=dt, copy=True, order="C")  # noqa: E731
    ia, ja = cp(ia, np.int32), cp(ja, np.int32)
    a, ad, b, rcell = _dif_out(storage, unsym, neq, ia, ja, m.numel, fill)
    t, v, npar, par = case.load_arrays()
    sec = ctypes.c_double()
    arrs = [cp(m.nelcon, np.int32), cp(m.nviz, np.int16), cp(m.cellface, np.int32),
            cp(m.owner, np.int32), cp(m.volume, np.float64), cp(m.dcca, np.float64),
            cp(m.xmcc, np.float64), cp(m.mksi, np.float64), cp(m.ksi, np.float64),
            cp(m.eta, np.float64), cp(m.area, np.float64), cp(m.normal, np.float64),
            cp(m.xm, np.float64), cp(m.mvskew, np.float64), cp(m.vskew, np.float64),
            cal.copy(), mat.copy(), cp(case.density, np.float64),
            cp(case.cdiff, np.float64), ia, ja, a, ad, b, cp(m.id, np.int32),
            cp(case.facer, np.int16), cp(case.u0, np.float64),
            cp(case.gradu0, np.float64), rcell]
    nad = len(ja) if storage != ELLPACK else int(ia[1])
    rc = lib.sfr_ref_syst_form_dif(
        m.numel, m.nelcon.shape[1], *[_p(x) for x in arrs], len(case.loads),
        _p(t), _p(v), _p(npar), _p(par), case.icod, int(case.fres),
        int(case.time_flag), case.time_type, case.dt, case.dt0, neq, nad, storage,
        int(forces), int(matrix), int(calrcell), int(unsym), ctypes.byref(sec))
    return rc, a, ad, b, rcell, sec.value


# ------------------------------------------ pressure-correction assembly --
# systFormSimplePres (CellLoopInc.c:471-700) -> cellSimplePres3D (CellPres.c:903)
@dataclass
class PresCase:
    """Everything one systFormSimplePres call reads besides the pattern: the
    mesh arrays, faceVelR / facePresR, the two load tables, the material
    table prop (nmat x MAXPROP, density in column DENSITY), and the cell
    fields pres, gradPres, vel and dField (the momentum D, 3 per cell)."""
    mesh: object
    facevelr: np.ndarray
    facepresr: np.ndarray
    lvel: list
    lpres: list
    prop: np.ndarray
    pres: np.ndarray
    gradpres: np.ndarray
    vel: np.ndarray
    dfield: np.ndarray
    icod: int = ORTHOGONAL
    mat: np.ndarray | None = None
    caltype: np.ndarray | None = None

    def material(self):
        mat = (np.ones(self.mesh.numel, np.int16) if self.mat is None
               else _c(self.mat, np.int16))
        nmat = len(np.asarray(self.prop).reshape(-1, MAXPROP))
        cal = np.ones(nmat, np.int16) if self.caltype is None else _c(self.caltype, np.int16)
        return cal, mat


def pres_assemble(case: PresCase, storage, unsym, ia, ja, neq, forces=True,
                  matrix=True, calrcell=True, fill=0.0):
    """The C restatement of systFormSimplePres: (rc, a, ad, b, rcell)."""
    m = case.mesh
    lib = oracle_lib()
    if not getattr(lib, "_pres_typed", False):
        lib.orc_pres_assemble.restype = ctypes.c_int
        lib.orc_pres_assemble.argtypes = (
            [ctypes.POINTER(_DifMesh), _P, _P, ctypes.c_int, _P, ctypes.c_int, ctypes.c_int]
            + [_P] * 5 + [ctypes.c_int] * 4 + [_P] * 6 + [ctypes.c_int] * 3)
        lib._pres_typed = True
    cal, mat = case.material()
    keep = dict(
        nelcon=_c(m.nelcon, np.int32), nface=_c(m.nviz, np.int16),
        cellface=_c(m.cellface, np.int32), owner=_c(m.owner, np.int32),
        volume=_c(m.volume, np.float64), dcca=_c(m.dcca, np.float64),
        xmcc=_c(m.xmcc, np.float64), mksi=_c(m.mksi, np.float64),
        ksi=_c(m.ksi, np.float64), area=_c(m.area, np.float64),
        normal=_c(m.normal, np.float64), vskew=_c(m.vskew, np.float64),
        caltype=cal, mat=mat, id=_c(m.id, np.int32), facer=_c(case.facepresr, np.int16))
    dm = _DifMesh(numel=m.numel, maxviz=m.nelcon.shape[1],
                  **{k: _p(v) for k, v in keep.items()})
    fvr = _c(case.facevelr, np.int16)
    lv, lp = _load_table(case.lvel), _load_table(case.lpres)
    ia, ja = _c(ia, np.int32), _c(ja, np.int32)
    a, ad, b, rc_ = _dif_out(storage, unsym, neq, ia, ja, m.numel, fill)
    fields = [_c(case.prop, np.float64), _c(case.pres, np.float64),
              _c(case.gradpres, np.float64), _c(case.vel, np.float64),
              _c(case.dfield, np.float64)]
    nad = len(ja) if storage != ELLPACK else 0
    rc = lib.orc_pres_assemble(ctypes.byref(dm), _p(fvr), lv, len(case.lvel), lp,
                               len(case.lpres), case.icod, *[_p(f) for f in fields],
                               storage, int(unsym), neq, nad, _p(ia), _p(ja), _p(a), _p(ad),
                               _p(b), _p(rc_), int(forces), int(matrix), int(calrcell))
    return rc, a, ad, b, rc_


def ref_pres_assemble(case: PresCase, storage, unsym, ia, ja, neq, forces=True,
                      matrix=True, calrcell=True, fill=0.0, nthreads=0):
    """The reference's own systFormSimplePres: (rc, a, ad, b, rcell, seconds)."""
    m = case.mesh
    lib = ref_lib()
    if not getattr(lib, "_pres_typed", False):
        lib.sfr_ref_syst_form_simple_pres.restype = ctypes.c_int
        lib.sfr_ref_syst_form_simple_pres.argtypes = (
            [ctypes.c_int, ctypes.c_int] + [_P] * 31 + [ctypes.c_int] + [_P] * 5
            + [ctypes.c_int] + [_P] * 5 + [ctypes.c_int] * 9 + [_P])
        lib._pres_typed = True
    cal, mat = case.material()
    cp = lambda x, dt: np.array(x, dtype=dt, copy=True, order="C")  # noqa: E731
    ia, ja = cp(ia, np.int32), cp(ja, np.int32)
    a, ad, b, rcell = _dif_out(storage, unsym, neq, ia, ja, m.numel, fill)
    vt = _load_arrays(case.lvel)
    pt = _load_arrays(case.lpres)
    sec = ctypes.c_double()
    arrs = [cp(m.nelcon, np.int32), cp(m.nviz, np.int16), cp(m.cellface, np.int32),
            cp(m.owner, np.int32), cp(m.volume, np.float64), cp(m.dcca, np.float64),
            cp(m.xmcc, np.float64), cp(m.mksi, np.float64), cp(m.ksi, np.float64),
            cp(m.eta, np.float64), cp(m.area, np.float64), cp(m.normal, np.float64),
            cp(m.xm, np.float64), cp(m.mvskew, np.float64), cp(m.vskew, np.float64),
            cal.copy(), mat.copy(), cp(case.prop, np.float64), ia, ja, a, ad, b,
            cp(m.id, np.int32), cp(case.facevelr, np.int16), cp(case.facepresr, np.int16),
            cp(case.pres, np.float64), cp(case.gradpres, np.float64),
            cp(case.vel, np.float64), cp(case.dfield, np.float64), rcell]
    nad = len(ja) if storage != ELLPACK else int(ia[1])
    rc = lib.sfr_ref_syst_form_simple_pres(
        m.numel, m.nelcon.shape[1], *[_p(x) for x in arrs],
        len(case.lvel), *[_p(x) for x in vt], len(case.lpres), *[_p(x) for x in pt],
        case.icod, neq, nad, storage, int(forces), int(matrix), int(calrcell), int(unsym),
        nthreads, ctypes.byref(sec))
    return rc, a, ad, b, rcell, sec.value


# ------------------------------------------------------ momentum assembly --
# systFormSimpleVel (CellLoopInc.c:98-470) -> cellSimpleVel3D (CellSimple.c:106)
SIMPLE, SIMPLEC = 1, 2  # Define.h:223-224
FOUP, CD, SOUP, TVD, NVD, LUST = 1, 2, 3, 4, 5, 6  # advection schemes, Define.h:267-272


@dataclass
class VelCase:
    """What one laminar, first-order-upwind systFormSimpleVel call reads:
    the mesh arrays plus centroids cc (numel, 3) and face centres xm
    (nface, 3), faceVelR / faceRpres, the velocity loads, the material
    table (DYNAMICVISCOSITY column 0, DENSITY 1) and the cell fields (gradvel
    (numel, 3, 3), row i = grad u_i; dfield is updated in place)."""
    mesh: object
    cc: np.ndarray
    facevelr: np.ndarray
    facepresr: np.ndarray
    lvel: list
    prop: np.ndarray
    pres: np.ndarray
    gradpres: np.ndarray
    vel: np.ndarray
    gradvel: np.ndarray
    dfield: np.ndarray
    icod: int = ORTHOGONAL
    fso: bool = True
    fvisc: bool = False
    fres: bool = True
    type_simple: int = SIMPLE
    time_flag: bool = False
    time_type: int = EULER
    dt: float = 1.0
    dt0: float = 1.0
    under: float = 0.7
    mat: np.ndarray | None = None
    caltype: np.ndarray | None = None
    adv: int = FOUP
    eddy: np.ndarray | None = None     # (numel,) eddy viscosity: Turbulence.fTurb
    stress: np.ndarray | None = None   # (numel, 6) residual stress: fTurbStruct
    adv_beta: float = 0.25             # Advection.par[0]: LUST weight
    adv_fn: int = 1                    # Advection.iCod2: NVD function (1 BCD .. 9 ModBCD)
    wallpar: np.ndarray | None = None  # (numel, 4) yPlus, uPlus, uFri, stressW: Turbulence.fWall
    rhie: int = 0                      # fRhieChowInt: 1 D from the call's start, 2 serial order

    def material(self):
        mat = (np.ones(self.mesh.numel, np.int16) if self.mat is None
               else _c(self.mat, np.int16))
        nmat = len(np.asarray(self.prop).reshape(-1, MAXPROP))
        cal = np.ones(nmat, np.int16) if self.caltype is None else _c(self.caltype, np.int16)
        return cal, mat


class _VelOpts(ctypes.Structure):
    _fields_ = [("icod", ctypes.c_int), ("fso", ctypes.c_int), ("fvisc", ctypes.c_int),
                ("fres", ctypes.c_int), ("type_simple", ctypes.c_int),
                ("time_flag", ctypes.c_int), ("time_type", ctypes.c_int),
                ("adv", ctypes.c_int),
                ("dt", ctypes.c_double), ("dt0", ctypes.c_double), ("under", ctypes.c_double),
                ("fturb", ctypes.c_int), ("fstruc", ctypes.c_int), ("eddy", _P), ("stress", _P),
                ("adv_beta", ctypes.c_double), ("adv_fn", ctypes.c_int),
                ("fwall", ctypes.c_int), ("wallpar", _P), ("rhie", ctypes.c_int)]


def _vel_out(storage, unsym, neq, ia, ja, numel, fill):
    a = np.full(dif_size(storage, unsym, neq, ia, ja), fill)
    return a, np.full(3 * neq, fill), np.full(3 * neq, fill), np.full(3 * numel, fill)


def vel_assemble(case: VelCase, storage, unsym, ia, ja, neq, forces=True, matrix=True,
                 calrcell=True, fill=0.0):
    """The C restatement: (rc, a, ad, b, rcell, dfield)."""
    m = case.mesh
    lib = oracle_lib()
    if not getattr(lib, "_vel_typed", False):
        lib.orc_vel_assemble.restype = ctypes.c_int
        lib.orc_vel_assemble.argtypes = (
            [ctypes.POINTER(_DifMesh), _P, _P, _P, _P, ctypes.c_int, ctypes.POINTER(_VelOpts)]
            + [_P] * 6 + [ctypes.c_int] * 4 + [_P] * 6 + [ctypes.c_int] * 3)
        lib._vel_typed = True
    cal, mat = case.material()
    keep = dict(
        nelcon=_c(m.nelcon, np.int32), nface=_c(m.nviz, np.int16),
        cellface=_c(m.cellface, np.int32), owner=_c(m.owner, np.int32),
        volume=_c(m.volume, np.float64), dcca=_c(m.dcca, np.float64),
        xmcc=_c(m.xmcc, np.float64), mksi=_c(m.mksi, np.float64),
        ksi=_c(m.ksi, np.float64), area=_c(m.area, np.float64),
        normal=_c(m.normal, np.float64), vskew=_c(m.vskew, np.float64),
        caltype=cal, mat=mat, id=_c(m.id, np.int32), facer=_c(case.facevelr, np.int16))
    dm = _DifMesh(numel=m.numel, maxviz=m.nelcon.shape[1],
                  **{k: _p(v) for k, v in keep.items()})
    o = _VelOpts(icod=case.icod, fso=int(case.fso), fvisc=int(case.fvisc),
                 fres=int(case.fres), type_simple=case.type_simple,
                 time_flag=int(case.time_flag), time_type=case.time_type, adv=case.adv,
                 dt=case.dt, dt0=case.dt0, under=case.under)
    turb = [None if a is None else _c(a, np.float64) for a in (case.eddy, case.stress)]
    o.fturb, o.fstruc = int(turb[0] is not None), int(turb[1] is not None)
    o.eddy, o.stress = [None if a is None else _p(a) for a in turb]
    o.adv_beta = case.adv_beta
    o.adv_fn = case.adv_fn
    wall = None if case.wallpar is None else _c(case.wallpar, np.float64)
    o.fwall, o.wallpar = int(wall is not None), None if wall is None else _p(wall)
    o.rhie = int(case.rhie)
    ia, ja = _c(ia, np.int32), _c(ja, np.int32)
    a, ad, b, rc_ = _vel_out(storage, unsym, neq, ia, ja, m.numel, fill)
    dfield = np.array(case.dfield, dtype=np.float64, copy=True, order="C")
    fpr = _c(case.facepresr, np.int16)
    cc, xm = _c(case.cc, np.float64), _c(m.xm, np.float64)
    lv = _load_table(case.lvel)
    fields = [_c(case.prop, np.float64), _c(case.pres, np.float64),
              _c(case.gradpres, np.float64), _c(case.vel, np.float64),
              _c(case.gradvel, np.float64), dfield]
    nad = len(ja) if storage != ELLPACK else 0
    rc = lib.orc_vel_assemble(ctypes.byref(dm), _p(fpr), _p(cc), _p(xm), lv, len(case.lvel),
                              ctypes.byref(o), *[_p(f) for f in fields], storage, int(unsym),
                              neq, nad, _p(ia), _p(ja), _p(a), _p(ad), _p(b), _p(rc_),
                              int(forces), int(matrix), int(calrcell))
    return rc, a, ad, b, rc_, dfield


def ref_vel_assemble(case: VelCase, storage, unsym, ia, ja, neq, forces=True, matrix=True,
                     calrcell=True, fill=0.0, nthreads=0):
    """The reference's own systFormSimpleVel: (rc, a, ad, b, rcell, dfield, seconds)."""
    m = case.mesh
    lib = ref_lib()
    if not getattr(lib, "_vel_typed", False):
        lib.sfr_ref_syst_form_simple_vel.restype = ctypes.c_int
        lib.sfr_ref_syst_form_simple_vel.argtypes = (
            [ctypes.c_int, ctypes.c_int] + [_P] * 33 + [ctypes.c_int] + [_P] * 5
            + [ctypes.c_int] * 7 + [ctypes.c_double] * 3 + [ctypes.c_int] * 11 + [_P] * 2
            + [ctypes.c_double, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int, _P])
        lib._vel_typed = True
    cal, mat = case.material()
    cp = lambda x, dt: np.array(x, dtype=dt, copy=True, order="C")  # noqa: E731
    ia, ja = cp(ia, np.int32), cp(ja, np.int32)
    a, ad, b, rcell = _vel_out(storage, unsym, neq, ia, ja, m.numel, fill)
    dfield = cp(case.dfield, np.float64)
    vt = _load_arrays(case.lvel)
    sec = ctypes.c_double()
    eddy = None if case.eddy is None else cp(case.eddy, np.float64)
    stress = None if case.stress is None else cp(case.stress, np.float64)
    arrs = [cp(m.nelcon, np.int32), cp(m.nviz, np.int16), cp(m.cellface, np.int32),
            cp(m.owner, np.int32), cp(m.volume, np.float64), cp(m.dcca, np.float64),
            cp(m.xmcc, np.float64), cp(case.cc, np.float64), cp(m.mksi, np.float64),
            cp(m.ksi, np.float64), cp(m.eta, np.float64), cp(m.area, np.float64),
            cp(m.normal, np.float64), cp(m.xm, np.float64), cp(m.mvskew, np.float64),
            cp(m.vskew, np.float64), cal.copy(), mat.copy(), cp(case.prop, np.float64), ia, ja,
            a, ad, b, cp(m.id, np.int32), cp(case.facevelr, np.int16),
            cp(case.facepresr, np.int16), cp(case.pres, np.float64),
            cp(case.gradpres, np.float64), cp(case.vel, np.float64),
            cp(case.gradvel, np.float64), dfield, rcell]
    nad = len(ja) if storage != ELLPACK else int(ia[1])
    rc = lib.sfr_ref_syst_form_simple_vel(
        m.numel, m.nelcon.shape[1], *[_p(x) for x in arrs], len(case.lvel),
        *[_p(x) for x in vt], case.icod, int(case.fso), int(case.fvisc), int(case.fres),
        case.type_simple, int(case.time_flag), case.time_type, case.dt, case.dt0, case.under,
        neq, nad, storage, int(forces), int(matrix), int(calrcell), int(unsym), nthreads,
        case.adv, int(eddy is not None), int(stress is not None),
        None if eddy is None else _p(eddy), None if stress is None else _p(stress),
        case.adv_beta, case.adv_fn, int(case.wallpar is not None),
        None if case.wallpar is None else _p(cp(case.wallpar, np.float64)), int(case.rhie),
        ctypes.byref(sec))
    return rc, a, ad, b, rcell, dfield, sec.value


# ------------------------------------------------ gradient reconstruction --
# rcGradU (CellLoop.c:4544-4790): Green-Gauss cell or least squares
RCGRADGAUSSC, RCGRADGAUSSN, RCLSQUARE, RCLSQUAREQR = 1, 2, 3, 4  # Define.h:377-380
CONVECTIONHEAT = 11
FLUXPRESC = 16


@dataclass
class GradCase:
    """One rcGradU call: the mesh arrays, faceR of the field (its face loads),
    the loads, the material table (COEFDIF column 0), u (numel, ndf) and the
    previous gradient gradu (numel, ndf, 3), row k = grad u_k."""
    mesh: object
    facer: np.ndarray
    loads: list
    prop: np.ndarray
    u: np.ndarray
    gradu: np.ndarray
    type: int = RCLSQUARE
    mat: np.ndarray | None = None

    @property
    def ndf(self) -> int:
        u = np.asarray(self.u)
        return 1 if u.ndim == 1 else int(u.shape[1])

    def material(self):
        mat = (np.ones(self.mesh.numel, np.int16) if self.mat is None
               else _c(self.mat, np.int16))
        nmat = len(np.asarray(self.prop).reshape(-1, MAXPROP))
        return np.ones(nmat, np.int16), mat


def _grad_mesh(case: GradCase):
    m = case.mesh
    cal, mat = case.material()
    keep = dict(
        nelcon=_c(m.nelcon, np.int32), nface=_c(m.nviz, np.int16),
        cellface=_c(m.cellface, np.int32), owner=_c(m.owner, np.int32),
        volume=_c(m.volume, np.float64), dcca=_c(m.dcca, np.float64),
        xmcc=_c(m.xmcc, np.float64), mksi=_c(m.mksi, np.float64),
        ksi=_c(m.ksi, np.float64), area=_c(m.area, np.float64),
        normal=_c(m.normal, np.float64), vskew=_c(m.vskew, np.float64),
        caltype=cal, mat=mat, id=_c(m.id, np.int32), facer=_c(case.facer, np.int16))
    dm = _DifMesh(numel=m.numel, maxviz=m.nelcon.shape[1],
                  **{k: _p(v) for k, v in keep.items()})
    return dm, keep


def ls_matrix(case: GradCase) -> np.ndarray:
    """leastSquareMatrix (RCLSQUARE) of every cell: (numel, 3, maxviz)."""
    lib = oracle_lib()
    lib.orc_ls_matrix.restype = None
    lib.orc_ls_matrix.argtypes = [ctypes.POINTER(_DifMesh), _P]
    dm, _keep = _grad_mesh(case)
    out = np.zeros((case.mesh.numel, 3, case.mesh.nelcon.shape[1]))
    lib.orc_ls_matrix(ctypes.byref(dm), _p(out))
    return out


def rc_grad(case: GradCase):
    """The C restatement: (rc, gradu (numel, ndf, 3))."""
    lib = oracle_lib()
    lib.orc_rc_grad.restype = ctypes.c_int
    lib.orc_rc_grad.argtypes = [ctypes.POINTER(_DifMesh), _P, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, _P, _P, _P, _P]
    dm, _keep = _grad_mesh(case)
    ndf = case.ndf
    lsq = ls_matrix(case) if case.type == RCLSQUARE else np.zeros(1)
    g = np.array(case.gradu, dtype=np.float64, copy=True, order="C").reshape(case.mesh.numel,
                                                                            ndf, 3)
    u = _c(case.u, np.float64)
    rc = lib.orc_rc_grad(ctypes.byref(dm), _load_table(case.loads), len(case.loads), case.type,
                         ndf, _p(_c(case.prop, np.float64)), _p(lsq), _p(u), _p(g))
    return rc, g


def ref_rc_grad(case: GradCase, nthreads=0):
    """The reference's own rcLeastSquare + rcGradU: (rc, gradu, lsq, seconds)."""
    m = case.mesh
    lib = ref_lib()
    if not getattr(lib, "_grad_typed", False):
        lib.sfr_ref_rc_grad.restype = ctypes.c_int
        lib.sfr_ref_rc_grad.argtypes = ([ctypes.c_int, ctypes.c_int] + [_P] * 20 + [ctypes.c_int]
                                        + [_P] * 5 + [ctypes.c_int] * 2 + [_P] * 3
                                        + [ctypes.c_int, _P])
        lib._grad_typed = True
    cal, mat = case.material()
    cp = lambda x, dt: np.array(x, dtype=dt, copy=True, order="C")  # noqa: E731
    ndf = case.ndf
    g = cp(case.gradu, np.float64).reshape(m.numel, ndf, 3)
    u = cp(case.u, np.float64)
    lsq = np.zeros((m.numel, 3, m.nelcon.shape[1]))
    cc = m.xm[m.cellface[:, 0] - 1] - m.xmcc[:, 0, :]
    arrs = [cp(m.nelcon, np.int32), cp(m.nviz, np.int16), cp(m.cellface, np.int32),
            cp(m.owner, np.int32), cp(m.volume, np.float64), cp(m.dcca, np.float64),
            cp(m.xmcc, np.float64), cp(cc, np.float64), cp(m.mksi, np.float64),
            cp(m.ksi, np.float64), cp(m.eta, np.float64), cp(m.area, np.float64),
            cp(m.normal, np.float64), cp(m.xm, np.float64), cp(m.mvskew, np.float64),
            cp(m.vskew, np.float64), cal.copy(), mat.copy(), cp(case.prop, np.float64),
            cp(case.facer, np.int16)]
    vt = _load_arrays(case.loads)
    sec = ctypes.c_double()
    rc = lib.sfr_ref_rc_grad(m.numel, m.nelcon.shape[1], *[_p(x) for x in arrs],
                             len(case.loads), *[_p(x) for x in vt], case.type, ndf, _p(u),
                             _p(g), _p(lsq), nthreads, ctypes.byref(sec))
    return rc, g, lsq, sec.value
