"""Seeded finite-volume systems in SFR3D's sparse layouts (host side).

Thin ctypes layer over libsfr3d_systems.so (sfr3d_b200/csrc/systems.cpp).
The presets are the workloads the solver is measured on:

* ``poisson_uniform(32)``   7-point FV Laplacian on the unit cube, unit
  diffusivity, Dirichlet p=0 on x=0, Neumann elsewhere, RCM numbering, RHS
  iid U[-1,1].
* ``poisson_jittered(128)`` the same construction with per-cell diffusivity
  10^U(-2,2), harmonic face coefficients, nodes jittered +-20 % of the
  spacing, cells randomly permuted then RCM-numbered.
* ``momentum(128, 50)``     upwind convection-diffusion on [0,pi]^3 with the
  divergence-free field (sin x cos y cos z, -cos x sin y cos z, 0) scaled to a
  maximum cell Peclet number, nu=1e-3, dt=1e-2, no-slip walls, 3 RHS iid
  N(0,1).
* ``poisson_batch(64)``     uneven Poisson boxes (8..96 cells per axis,
  log-uniform), one stretched axis, constant diffusivity 10^U(-1,1),
  Dirichlet on one random face.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native

SFR_SYS_DIFFUSION = 1
SFR_SYS_CONVDIFF = 2
FACE_XMIN, FACE_XMAX, FACE_YMIN, FACE_YMAX, FACE_ZMIN, FACE_ZMAX = (
    1, 2, 4, 8, 16, 32)
ALL_FACES = 63


class SysParams(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("jitter", ctypes.c_double),
        ("log10k_lo", ctypes.c_double), ("log10k_hi", ctypes.c_double),
        ("dirichlet_faces", ctypes.c_int32),
        ("permute", ctypes.c_int32),
        ("rcm", ctypes.c_int32),
        ("nrhs", ctypes.c_int32),
        ("rhs_normal", ctypes.c_int32),
        ("peclet", ctypes.c_double),
        ("nu", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("seed", ctypes.c_uint64),
    ]


class SysInfo(ctypes.Structure):
    _fields_ = [
        ("neq", ctypes.c_int32), ("nnz_full", ctypes.c_int32),
        ("nnz_lower", ctypes.c_int32), ("width", ctypes.c_int32),
        ("nrhs", ctypes.c_int32), ("unsym", ctypes.c_int32),
        ("bandwidth", ctypes.c_int32), ("pad", ctypes.c_int32),
        ("velocity_scale", ctypes.c_double),
    ]


class SysMesh(ctypes.Structure):
    _fields_ = [(name, ctypes.c_void_p) for name in (
        "nelcon", "nviz", "cellface", "volume", "dcca", "xmcc", "cdiff", "id",
        "owner", "mksi", "ksi", "eta", "area", "normal", "xm", "mvskew",
        "vskew")]


_P = ctypes.c_void_p


def _lib():
    lib = _native.load("libsfr3d_systems.so")
    if not getattr(lib, "_typed", False):
        lib.sfr_sys_build.restype = _P
        lib.sfr_sys_build.argtypes = [ctypes.POINTER(SysParams)]
        lib.sfr_sys_free.restype = None
        lib.sfr_sys_free.argtypes = [_P]
        lib.sfr_sys_info.argtypes = [_P, ctypes.POINTER(SysInfo)]
        for name, n in (("sfr_sys_csrd_full", 4), ("sfr_sys_csrd_lower", 3),
                        ("sfr_sys_csrc", 3), ("sfr_sys_ell", 2),
                        ("sfr_sys_rhs", 1), ("sfr_sys_numbering", 1)):
            getattr(lib, name).argtypes = [_P] + [_P] * n
            getattr(lib, name).restype = ctypes.c_int
        lib.sfr_sys_mesh_sizes.argtypes = [_P, _P, _P]
        lib.sfr_sys_mesh.argtypes = [_P, ctypes.POINTER(SysMesh)]
        lib.sfr_rcm.argtypes = [ctypes.c_int32, _P, _P, _P]
        lib.sfr_sys_batch_params.argtypes = [
            ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64,
            ctypes.POINTER(SysParams)]
        lib._typed = True
    return lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


MAX_VIZ = 6  # face slots per hexahedral cell: x-, x+, y-, y+, z-, z+


@dataclass
class FvMesh:
    """The box in the reference's mesh arrays (the geometry inputs of
    systFormDif, CellLoop.c:285-311): 1-based indices, cell arrays by natural
    cell id, maxViz = 6.  Shapes: nelcon/cellface/dcca (numel, 6),
    xmcc (numel, 6, 3), owner (nface, 2), the face vectors (nface, 3)."""
    numel: int
    nface: int
    nelcon: np.ndarray
    nviz: np.ndarray
    cellface: np.ndarray
    volume: np.ndarray
    dcca: np.ndarray
    xmcc: np.ndarray
    cdiff: np.ndarray
    id: np.ndarray
    owner: np.ndarray
    mksi: np.ndarray
    ksi: np.ndarray
    eta: np.ndarray
    area: np.ndarray
    normal: np.ndarray
    xm: np.ndarray
    mvskew: np.ndarray
    vskew: np.ndarray

    def face_r(self, side_load) -> np.ndarray:
        """faceR (numel, maxViz + 1), short: load number + 1 (0 = none) of
        each boundary face from a per-side table (x-, x+, y-, y+, z-, z+),
        and 0 in the cell's own entry (every cell carries an equation)."""
        side = np.asarray(side_load, np.int16)
        fr = np.zeros((self.numel, MAX_VIZ + 1), np.int16)
        bnd = self.nelcon == -1
        fr[:, :MAX_VIZ] = np.where(bnd, side[None, :], 0)
        return fr


@dataclass
class FvSystem:
    """One assembled system.  CSRD-full arrays are always present; the other
    layouts are materialised on first use."""
    params: SysParams
    neq: int
    nnz_full: int
    nnz_lower: int
    width: int
    unsym: bool
    bandwidth: int
    velocity_scale: float
    ia: np.ndarray
    ja: np.ndarray
    al: np.ndarray
    ad: np.ndarray
    b: np.ndarray                      # shape (nrhs, neq)
    _handle: int | None = field(default=None, repr=False)
    _cache: dict = field(default_factory=dict, repr=False)

    def __del__(self):
        h = self._handle
        if h:
            try:
                _lib().sfr_sys_free(h)
            except Exception:
                pass
            self._handle = None

    def _need(self):
        if not self._handle:
            raise RuntimeError("system handle released")
        return self._handle

    def csrd_lower(self):
        """(ia, ja, al) with the strict lower part only: CSRD symmetric storage."""
        if "csrd_lower" not in self._cache:
            ia = np.empty(self.neq + 1, np.int32)
            ja = np.empty(self.nnz_lower, np.int32)
            al = np.empty(self.nnz_lower, np.float64)
            _check(_lib().sfr_sys_csrd_lower(self._need(), _ptr(ia), _ptr(ja), _ptr(al)))
            self._cache["csrd_lower"] = (ia, ja, al)
        return self._cache["csrd_lower"]

    def csrc(self):
        """(ia, ja, a) CSRC: strict lower pattern, a = [al | au] (2*nad)."""
        if "csrc" not in self._cache:
            ia = np.empty(self.neq + 1, np.int32)
            ja = np.empty(self.nnz_lower, np.int32)
            a = np.empty(2 * self.nnz_lower, np.float64)
            _check(_lib().sfr_sys_csrc(self._need(), _ptr(ia), _ptr(ja), _ptr(a)))
            self._cache["csrc"] = (ia, ja, a)
        return self._cache["csrc"]

    def ell(self):
        """(ja, a) ELLPACK row-major neq x width in cell-face order."""
        if "ell" not in self._cache:
            ja = np.empty(self.neq * self.width, np.int32)
            a = np.empty(self.neq * self.width, np.float64)
            _check(_lib().sfr_sys_ell(self._need(), _ptr(ja), _ptr(a)))
            self._cache["ell"] = (ja, a)
        return self._cache["ell"]

    def numbering(self):
        e = np.empty(self.neq, np.int32)
        _check(_lib().sfr_sys_numbering(self._need(), _ptr(e)))
        return e

    def mesh(self) -> FvMesh:
        """The mesh the system was built on, in the reference's arrays."""
        if "mesh" not in self._cache:
            numel = ctypes.c_int32()
            nface = ctypes.c_int64()
            lib = _lib()
            _check(lib.sfr_sys_mesh_sizes(self._need(), ctypes.byref(numel),
                                          ctypes.byref(nface)))
            ne, nf = numel.value, nface.value
            m = FvMesh(
                numel=ne, nface=nf,
                nelcon=np.empty((ne, MAX_VIZ), np.int32),
                nviz=np.empty(ne, np.int16),
                cellface=np.empty((ne, MAX_VIZ), np.int32),
                volume=np.empty(ne), dcca=np.empty((ne, MAX_VIZ)),
                xmcc=np.empty((ne, MAX_VIZ, 3)), cdiff=np.empty(ne),
                id=np.empty(ne, np.int32), owner=np.empty((nf, 2), np.int32),
                mksi=np.empty(nf), ksi=np.empty((nf, 3)), eta=np.empty((nf, 3)),
                area=np.empty(nf), normal=np.empty((nf, 3)), xm=np.empty((nf, 3)),
                mvskew=np.empty(nf), vskew=np.empty((nf, 3)))
            st = SysMesh(**{name: _ptr(getattr(m, name)) for name, _ in SysMesh._fields_})
            _check(lib.sfr_sys_mesh(self._need(), ctypes.byref(st)))
            self._cache["mesh"] = m
        return self._cache["mesh"]

    def release(self):
        """Free the native copy (the CSRD arrays stay)."""
        self.__del__()

    def dense(self) -> np.ndarray:
        """Dense matrix (small systems only; test helper)."""
        n = self.neq
        if n > 20000:
            raise ValueError("dense() is for small systems")
        A = np.zeros((n, n))
        A[np.arange(n), np.arange(n)] = self.ad
        rows = np.repeat(np.arange(n), np.diff(self.ia))
        A[rows, self.ja] = self.al
        return A


def _check(rc):
    if rc != 0:
        raise RuntimeError(f"native system call failed ({rc})")


def build(params: SysParams) -> FvSystem:
    lib = _lib()
    h = lib.sfr_sys_build(ctypes.byref(params))
    if not h:
        raise ValueError("invalid system parameters")
    info = SysInfo()
    _check(lib.sfr_sys_info(h, ctypes.byref(info)))
    n, nnz = info.neq, info.nnz_full
    ia = np.empty(n + 1, np.int32)
    ja = np.empty(nnz, np.int32)
    al = np.empty(nnz, np.float64)
    ad = np.empty(n, np.float64)
    _check(lib.sfr_sys_csrd_full(h, _ptr(ia), _ptr(ja), _ptr(al), _ptr(ad)))
    b = np.empty((info.nrhs, n), np.float64)
    if info.nrhs:
        _check(lib.sfr_sys_rhs(h, _ptr(b)))
    return FvSystem(params=params, neq=n, nnz_full=nnz, nnz_lower=info.nnz_lower,
                    width=info.width, unsym=bool(info.unsym),
                    bandwidth=info.bandwidth,
                    velocity_scale=info.velocity_scale, ia=ia, ja=ja, al=al,
                    ad=ad, b=b, _handle=h)


def params(kind=SFR_SYS_DIFFUSION, n=(8, 8, 8), lengths=(1.0, 1.0, 1.0),
           jitter=0.0, log10k=(0.0, 0.0), dirichlet=FACE_XMIN, permute=False,
           rcm=True, nrhs=1, rhs_normal=False, peclet=0.0, nu=1e-3, dt=1e-2,
           seed=0) -> SysParams:
    if isinstance(n, int):
        n = (n, n, n)
    p = SysParams()
    p.kind = kind
    p.nx, p.ny, p.nz = (int(v) for v in n)
    p.lx, p.ly, p.lz = (float(v) for v in lengths)
    p.jitter = jitter
    p.log10k_lo, p.log10k_hi = log10k
    p.dirichlet_faces = dirichlet
    p.permute = int(permute)
    p.rcm = int(rcm)
    p.nrhs = nrhs
    p.rhs_normal = int(rhs_normal)
    p.peclet = peclet
    p.nu = nu
    p.dt = dt
    p.seed = seed
    return p


# --------------------------------------------------------------- presets --
def poisson_uniform(n: int = 32, seed: int = 1) -> FvSystem:
    return build(params(n=n, seed=seed))


def poisson_jittered(n: int = 128, seed: int = 2) -> FvSystem:
    return build(params(n=n, jitter=0.2, log10k=(-2.0, 2.0), permute=True,
                        seed=seed))


def momentum(n: int = 128, peclet: float = 50.0, nrhs: int = 3,
             seed: int = 3) -> FvSystem:
    return build(params(kind=SFR_SYS_CONVDIFF, n=n,
                        lengths=(math.pi, math.pi, math.pi),
                        dirichlet=ALL_FACES, nrhs=nrhs, rhs_normal=True,
                        peclet=peclet, nu=1e-3, dt=1e-2, seed=seed))


def batch_params(count: int = 64, nmin: int = 8, nmax: int = 96,
                 seed: int = 4) -> list[SysParams]:
    arr = (SysParams * count)()
    _check(_lib().sfr_sys_batch_params(count, nmin, nmax, seed, arr))
    return [arr[i] for i in range(count)]


def poisson_batch(count: int = 64, nmin: int = 8, nmax: int = 96,
                  seed: int = 4) -> list[FvSystem]:
    return [build(p) for p in batch_params(count, nmin, nmax, seed)]


def rcm(xadj: np.ndarray, adj: np.ndarray) -> np.ndarray:
    """Reverse Cuthill-McKee permutation (perm[new] = old)."""
    xadj = np.ascontiguousarray(xadj, np.int32)
    adj = np.ascontiguousarray(adj, np.int32)
    n = len(xadj) - 1
    perm = np.empty(n, np.int32)
    _check(_lib().sfr_rcm(n, _ptr(xadj), _ptr(adj), _ptr(perm)))
    return perm
