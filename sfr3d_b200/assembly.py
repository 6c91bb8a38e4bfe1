"""Device assembly of the diffusion system (host side of assembly.cu).

The reference builds A and b on the host with systFormDif (CellLoop.c:285)
-> cellDif3D (CellDif.c:312) and hands them to solverC.  Here a plan binds a
mesh (the arrays systFormDif reads) to a resident ``GpuSystem`` once; each
``assemble`` then writes the system's values on the GPU, where the next
``solve_device`` reads them, and returns b and the cell residuals.  Results
are bit-identical to the reference's systFormDif on the same inputs.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import solver as _sv

# load types (Define.h:317-323), non-orthogonal schemes (Define.h:304-307),
# time schemes (Define.h:191-192)
DIRICHLET, NEUMANN, ROBIN, SINBC, INLET, OUTLET = 1, 2, 3, 4, 6, 7
MOVEWALL, INLETSTAICTPRES, OPEN, INLETTOTALPRES, STATICWALL, FLUXPRES = 8, 9, 10, 13, 14, 15
MAXPROP, DENSITY = 10, 1  # material table width and the density column (Define.h:349, 203)
ORTHOGONAL, MINIMAL, ORTHOGONALC, OVERRELAXED = 1, 2, 3, 4
EULER, BACKWARD = 0, 1
MAXLOADPAR = 20   # MAXLOADPARAMETER, Define.h:336
MAX_LOADS = 32

_P = ctypes.c_void_p
_I32 = ctypes.c_int32


class DifMeshC(ctypes.Structure):
    _fields_ = [("numel", _I32), ("maxviz", _I32), ("nfaces", ctypes.c_int64),
                ("nmat", _I32), ("pad", _I32)] + [
        (n, _P) for n in ("nelcon", "nviz", "cellface", "owner", "volume",
                          "dcca", "xmcc", "mksi", "ksi", "area", "normal",
                          "vskew", "caltype", "mat", "id", "facer", "cc", "xm")]


class VelOptsC(ctypes.Structure):
    _fields_ = [("icod", _I32), ("fso", _I32), ("fvisc", _I32), ("fres", _I32),
                ("type_simple", _I32), ("time_flag", _I32), ("time_type", _I32),
                ("adv", _I32), ("dt", ctypes.c_double), ("dt0", ctypes.c_double),
                ("under", ctypes.c_double), ("fturb", _I32), ("fstruc", _I32),
                ("adv_beta", ctypes.c_double), ("adv_fn", _I32), ("fwall", _I32),
                ("rhie", _I32)]


class LoadC(ctypes.Structure):
    _fields_ = [("type", _I32), ("var", _I32), ("np", _I32), ("pad", _I32),
                ("par", ctypes.c_double * MAXLOADPAR), ("density", ctypes.c_double)]


class DifOptsC(ctypes.Structure):
    _fields_ = [("icod", _I32), ("fres", _I32), ("time_flag", _I32),
                ("time_type", _I32), ("dt", ctypes.c_double),
                ("dt0", ctypes.c_double)]


def _lib():
    L = _sv.lib()
    if not getattr(L, "_dif_typed", False):
        L.sfr_gpu_dif_plan_create.argtypes = [_P, ctypes.POINTER(DifMeshC), _I32,
                                              ctypes.POINTER(_P)]
        L.sfr_gpu_dif_assemble.argtypes = ([_P, _P, _I32, ctypes.POINTER(DifOptsC)]
                                           + [_P] * 7 + [_I32] * 3)
        L.sfr_gpu_dif_assemble_device.argtypes = (
            [_P, _P, _I32, ctypes.POINTER(DifOptsC)] + [_P] * 7 + [_I32] * 3 + [_P])
        L.sfr_gpu_dif_update_cells.argtypes = [_P, _P, _P, _I32, _P]
        L.sfr_gpu_pres_plan_create.argtypes = [_P, ctypes.POINTER(DifMeshC), _P, _I32,
                                               ctypes.POINTER(_P)]
        L.sfr_gpu_pres_assemble.argtypes = [_P, _P, _I32, _P, _I32] + [_P] * 7 + [_I32] * 3
        L.sfr_gpu_pres_assemble_device.argtypes = ([_P, _P, _I32, _P, _I32] + [_P] * 7
                                                   + [_I32] * 3 + [_P])
        L.sfr_gpu_vel_plan_create.argtypes = [_P, ctypes.POINTER(DifMeshC), _I32,
                                              ctypes.POINTER(_P)]
        L.sfr_gpu_vel_turbulence.argtypes = [_P, _P, _P, _I32]
        L.sfr_gpu_vel_wall.argtypes = [_P, _P, _I32]
        L.sfr_gpu_vel_assemble.argtypes = ([_P, _P, _I32, ctypes.POINTER(VelOptsC)] + [_P] * 9
                                           + [_I32] * 3)
        L.sfr_gpu_vel_assemble_device.argtypes = ([_P, _P, _I32, ctypes.POINTER(VelOptsC)]
                                                  + [_P] * 9 + [_I32] * 3 + [_P])
        L.sfr_gpu_dif_plan_destroy.argtypes = [_P]
        L.sfr_gpu_get_values.argtypes = [_P, _P, _P, _P]
        L._dif_typed = True
    return L


@dataclass
class Load:
    """One load (Loads, StructDefine.h:356): type, parameters, nTypeVar."""
    type: int
    par: tuple = ()
    var: int = 0
    np: int | None = None
    density: float = 0.0


def _loads_c(loads):
    if len(loads) > MAX_LOADS:
        raise ValueError(f"at most {MAX_LOADS} loads")
    arr = (LoadC * max(len(loads), 1))()
    for i, ld in enumerate(loads):
        arr[i].type = ld.type
        arr[i].var = ld.var
        arr[i].np = len(ld.par) if ld.np is None else ld.np
        for j, v in enumerate(ld.par):
            arr[i].par[j] = v
        arr[i].density = ld.density
    return arr


def _c(a, dt):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def _mesh_c(mesh, facer, caltype, mat, nmat=None, cc=None):
    """The sfr_dif_mesh struct of a mesh object (and the arrays it points
    to, which the caller keeps alive for the call)."""
    numel = int(mesh.numel)
    if caltype is None:
        caltype = np.ones(nmat or 1, np.int16)
    cal = _c(caltype, np.int16)
    mt = np.ones(numel, np.int16) if mat is None else _c(mat, np.int16)
    keep = dict(
        nelcon=_c(mesh.nelcon, np.int32), nviz=_c(mesh.nviz, np.int16),
        cellface=_c(mesh.cellface, np.int32), owner=_c(mesh.owner, np.int32),
        volume=_c(mesh.volume, np.float64), dcca=_c(mesh.dcca, np.float64),
        xmcc=_c(mesh.xmcc, np.float64), mksi=_c(mesh.mksi, np.float64),
        ksi=_c(mesh.ksi, np.float64), area=_c(mesh.area, np.float64),
        normal=_c(mesh.normal, np.float64), vskew=_c(mesh.vskew, np.float64),
        caltype=cal, mat=mt, id=_c(mesh.id, np.int32), facer=_c(facer, np.int16))
    if cc is not None:
        keep["cc"] = _c(cc, np.float64)
        keep["xm"] = _c(mesh.xm, np.float64)
    m = DifMeshC(numel=numel, maxviz=int(keep["nelcon"].size // numel),
                 nfaces=int(mesh.mksi.shape[0]), nmat=int(cal.size),
                 **{k: _ptr(v) for k, v in keep.items()})
    return m, keep


class DifPlan:
    """A mesh bound to a resident system for device-side systFormDif.

    ``mesh`` is any object with the attributes of
    ``sfr3d_b200.systems.FvMesh`` (numel, nface, nelcon, nviz, cellface,
    owner, volume, dcca, xmcc, mksi, ksi, area, normal, vskew, id).
    ``facer`` is the reference's faceR, (numel, maxviz + 1) shorts.
    ``caltype``/``mat`` default to one diffusion material.
    """

    def __init__(self, system: "_sv.GpuSystem", mesh, facer, icod: int = ORTHOGONAL,
                 caltype=None, mat=None):
        self.system = system
        self.numel = int(mesh.numel)
        self.neq = system.neq
        self.icod = icod
        m, keep = _mesh_c(mesh, facer, caltype, mat)
        h = _P()
        rc = _lib().sfr_gpu_dif_plan_create(system.h, ctypes.byref(m), icod,
                                            ctypes.byref(h))
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_dif_plan_create: " + _sv.last_error())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _lib().sfr_gpu_dif_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _opts(self, fres, time):
        o = DifOptsC(icod=self.icod, fres=int(fres))
        if time is not None:
            o.time_flag = 1
            o.time_type, o.dt, o.dt0 = int(time[0]), float(time[1]), float(time[2])
        return o

    def assemble(self, loads, u0, cdiff, density=None, gradu0=None, b0=None,
                 fres=True, time=None, forces=True, matrix=True, calrcell=True):
        """One systFormDif call with host arrays: the matrix goes into the
        system (marked as new values); returns (b, rcell) as numpy arrays
        (None where not requested).  time = (type, dt, dt0) or None."""
        u0, cdiff = _c(u0, np.float64), _c(cdiff, np.float64)
        density, gradu0, b0 = (_c(density, np.float64), _c(gradu0, np.float64),
                               _c(b0, np.float64))
        b = np.empty(self.neq) if forces else None
        rcell = np.empty(self.numel) if calrcell else None
        loads_c = _loads_c(loads)
        o = self._opts(fres, time)
        rc = _lib().sfr_gpu_dif_assemble(
            self.h, loads_c, len(loads), ctypes.byref(o), _ptr(density), _ptr(cdiff),
            _ptr(u0), _ptr(gradu0), _ptr(b0), _ptr(b), _ptr(rcell), int(forces),
            int(matrix), int(calrcell))
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_dif_assemble: " + _sv.last_error())
        if matrix:
            self.system.values_version += 1
        return b, rcell

    def assemble_device(self, loads, d_u0: int, d_cdiff: int, d_density: int = 0,
                        d_gradu0: int = 0, d_b0: int = 0, d_b: int = 0, d_rcell: int = 0,
                        fres=True, time=None, forces=True, matrix=True, calrcell=True,
                        stream: int = 0):
        """The same on device pointers (plain integers), asynchronous on
        `stream` (0: the system's stream)."""
        loads_c = _loads_c(loads)
        o = self._opts(fres, time)
        rc = _lib().sfr_gpu_dif_assemble_device(
            self.h, loads_c, len(loads), ctypes.byref(o), d_density or None, d_cdiff,
            d_u0, d_gradu0 or None, d_b0 or None, d_b or None, d_rcell or None,
            int(forces), int(matrix), int(calrcell), stream or None)
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_dif_assemble_device: " + _sv.last_error())
        if matrix:
            self.system.values_version += 1

    def update_cells(self, d_x: int, d_u: int, add: bool, stream: int = 0):
        """u <- x (or u += x) over the cells, updateCellValue on the device."""
        rc = _lib().sfr_gpu_dif_update_cells(self.h, d_x, d_u, int(add), stream or None)
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_dif_update_cells")


class PresPlan(DifPlan):
    """A mesh bound to a resident system for device-side systFormSimplePres
    (the SIMPLE pressure correction, CellLoopInc.c:471).  facepresr /
    facevelr are the reference's facePresR / faceVelR, (numel, maxviz + 1)
    shorts; mat is the material of each cell (1-based) and nmat the number of
    materials in the prop table.  icod: ORTHOGONAL or OVERRELAXED."""

    def __init__(self, system: "_sv.GpuSystem", mesh, facepresr, facevelr,
                 icod: int = ORTHOGONAL, mat=None, nmat: int = 1, caltype=None):
        self.system = system
        self.numel = int(mesh.numel)
        self.neq = system.neq
        self.icod = icod
        self.nmat = nmat
        m, keep = _mesh_c(mesh, facepresr, caltype, mat, nmat)
        fv = _c(facevelr, np.int16)
        h = _P()
        rc = _lib().sfr_gpu_pres_plan_create(system.h, ctypes.byref(m), _ptr(fv), icod,
                                             ctypes.byref(h))
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_pres_plan_create: " + _sv.last_error())
        self.h = h

    def _prop(self, prop):
        prop = np.ascontiguousarray(prop, np.float64).reshape(-1, MAXPROP)
        if prop.shape[0] < self.nmat:
            raise ValueError("prop has fewer rows than materials")
        return prop

    def assemble(self, lvel, lpres, prop, pres, gradpres, vel, dfield, forces=True,
                 matrix=True, calrcell=True):
        """One systFormSimplePres call with host arrays; returns (b, rcell)."""
        prop = self._prop(prop)
        arrs = [_c(a, np.float64) for a in (pres, gradpres, vel, dfield)]
        b = np.empty(self.neq) if forces else None
        rcell = np.empty(self.numel) if calrcell else None
        lv, lp = _loads_c(lvel), _loads_c(lpres)
        rc = _lib().sfr_gpu_pres_assemble(
            self.h, lv, len(lvel), lp, len(lpres), _ptr(prop), *[_ptr(a) for a in arrs],
            _ptr(b), _ptr(rcell), int(forces), int(matrix), int(calrcell))
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_pres_assemble: " + _sv.last_error())
        if matrix:
            self.system.values_version += 1
        return b, rcell

    def assemble_device(self, lvel, lpres, prop, d_pres: int, d_gradpres: int, d_vel: int,
                        d_dfield: int, d_b: int = 0, d_rcell: int = 0, forces=True,
                        matrix=True, calrcell=True, stream: int = 0):
        """The same on device pointers, asynchronous on `stream`."""
        prop = self._prop(prop)
        lv, lp = _loads_c(lvel), _loads_c(lpres)
        rc = _lib().sfr_gpu_pres_assemble_device(
            self.h, lv, len(lvel), lp, len(lpres), _ptr(prop), d_pres, d_gradpres, d_vel,
            d_dfield, d_b or None, d_rcell or None, int(forces), int(matrix), int(calrcell),
            stream or None)
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_pres_assemble_device: " + _sv.last_error())
        if matrix:
            self.system.values_version += 1


SIMPLE, SIMPLEC = 1, 2  # Define.h:223-224
FOUP, CD, SOUP, TVD, NVD, LUST = 1, 2, 3, 4, 5, 6  # advection schemes (Advection.iCod1), Define.h:267-272


class VelPlan(DifPlan):
    """A mesh bound to a resident system for device-side systFormSimpleVel
    (the SIMPLE momentum system: u, v, w share the off-diagonals), laminar,
    advection FoUp, CD or SoUp, without Rhie-Chow.  facevelr is faceVelR; cc the
    cell centroids (numel, 3); the mesh must carry face centres (xm)."""

    def __init__(self, system: "_sv.GpuSystem", mesh, facevelr, cc, icod: int = ORTHOGONAL,
                 mat=None, nmat: int = 1, caltype=None):
        self.system = system
        self.numel = int(mesh.numel)
        self.neq = system.neq
        self.icod = icod
        self.nmat = nmat
        m, keep = _mesh_c(mesh, facevelr, caltype, mat, nmat, cc=cc)
        h = _P()
        rc = _lib().sfr_gpu_vel_plan_create(system.h, ctypes.byref(m), icod, ctypes.byref(h))
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_vel_plan_create: " + _sv.last_error())
        self.h = h

    def turbulence(self, eddy=None, stress=None, on_device: bool = False) -> None:
        """Bind the eddy viscosity (numel) and residual stress (numel, 6)
        that later calls read when fturb / fstruc are set: host arrays
        (copied now) or device pointers (ints, kept)."""
        if on_device:
            rc = _lib().sfr_gpu_vel_turbulence(self.h, eddy or None, stress or None, 1)
        else:
            e = None if eddy is None else _c(eddy, np.float64)
            st = None if stress is None else _c(stress, np.float64)
            rc = _lib().sfr_gpu_vel_turbulence(self.h, _ptr(e), _ptr(st), 0)
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_vel_turbulence: " + _sv.last_error())

    def wall(self, wallpar=None, on_device: bool = False) -> None:
        """Bind the wall model's parameters (numel, 4: yPlus, uPlus, uFri,
        stressW) that later calls with fwall read: a host array (copied now)
        or a device pointer (int, kept)."""
        if on_device:
            rc = _lib().sfr_gpu_vel_wall(self.h, wallpar or None, 1)
        else:
            w = None if wallpar is None else _c(wallpar, np.float64)
            rc = _lib().sfr_gpu_vel_wall(self.h, _ptr(w), 0)
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_vel_wall: " + _sv.last_error())

    def _vopts(self, fso, fvisc, fres, type_simple, time, under, adv=1, fturb=False,
               fstruc=False, adv_beta=0.25, adv_fn=1, fwall=False, rhie=0):
        o = VelOptsC(icod=self.icod, fso=int(fso), fvisc=int(fvisc), fres=int(fres),
                     type_simple=type_simple, under=under, adv=int(adv), fturb=int(fturb),
                     fstruc=int(fstruc), adv_beta=float(adv_beta), adv_fn=int(adv_fn),
                     fwall=int(fwall), rhie=int(rhie))
        if time is not None:
            o.time_flag = 1
            o.time_type, o.dt, o.dt0 = int(time[0]), float(time[1]), float(time[2])
        return o

    def assemble(self, lvel, prop, pres, gradpres, vel, gradvel, dfield, fso=True,
                 fvisc=False, fres=True, type_simple=SIMPLE, time=None, under=0.7,
                 forces=True, matrix=True, calrcell=True, adv=FOUP, fturb=False, fstruc=False,
                 adv_beta=0.25, adv_fn=1, fwall=False, rhie=0):
        """One call with host arrays: returns (ad3, b3, rcell3, dfield), each
        component block after the other (u, v, w).  adv: FOUP, CD, SOUP or LUST
        (weight adv_beta);
        fturb / fstruc read the fields bound by ``turbulence``."""
        prop = np.ascontiguousarray(prop, np.float64).reshape(-1, MAXPROP)
        arrs = [_c(a, np.float64) for a in (pres, gradpres, vel, gradvel)]
        df = np.array(dfield, dtype=np.float64, copy=True, order="C")
        ad3 = np.empty(3 * self.neq) if matrix else None
        b3 = np.empty(3 * self.neq) if forces else None
        rc3 = np.empty(3 * self.numel) if calrcell else None
        lv = _loads_c(lvel)
        o = self._vopts(fso, fvisc, fres, type_simple, time, under, adv, fturb, fstruc, adv_beta,
                        adv_fn, fwall, rhie)
        rc = _lib().sfr_gpu_vel_assemble(
            self.h, lv, len(lvel), ctypes.byref(o), _ptr(prop), *[_ptr(a) for a in arrs],
            _ptr(df), _ptr(ad3), _ptr(b3), _ptr(rc3), int(forces), int(matrix), int(calrcell))
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_vel_assemble: " + _sv.last_error())
        if matrix:
            self.system.values_version += 1
        return ad3, b3, rc3, df

    def assemble_device(self, lvel, prop, d_pres: int, d_gradpres: int, d_vel: int,
                        d_gradvel: int, d_dfield: int, d_ad3: int = 0, d_b3: int = 0,
                        d_rcell3: int = 0, fso=True, fvisc=False, fres=True,
                        type_simple=SIMPLE, time=None, under=0.7, forces=True, matrix=True,
                        calrcell=True, stream: int = 0, adv=FOUP, fturb=False, fstruc=False,
                        adv_beta=0.25, adv_fn=1, fwall=False, rhie=0):
        prop = np.ascontiguousarray(prop, np.float64).reshape(-1, MAXPROP)
        lv = _loads_c(lvel)
        o = self._vopts(fso, fvisc, fres, type_simple, time, under, adv, fturb, fstruc, adv_beta,
                        adv_fn, fwall, rhie)
        rc = _lib().sfr_gpu_vel_assemble_device(
            self.h, lv, len(lvel), ctypes.byref(o), _ptr(prop), d_pres, d_gradpres, d_vel,
            d_gradvel, d_dfield, d_ad3 or None, d_b3 or None, d_rcell3 or None, int(forces),
            int(matrix), int(calrcell), stream or None)
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_vel_assemble_device: " + _sv.last_error())
        if matrix:
            self.system.values_version += 1


RCGRADGAUSSC, RCLSQUARE = 1, 3  # rcGrad.type (Define.h:377-380)


class GradPlan:
    """rcGradU on the device (sfr_gpu_grad_*): Green-Gauss cell
    (RCGRADGAUSSC) or least squares (RCLSQUARE) over ``mesh`` with the
    field's face loads ``facer`` (faceRpres, faceRvel, ...).  ``mat`` gives
    each cell's material (1-based; COEFDIF of ``prop`` column 0 is read by
    NEUMANN faces)."""

    def __init__(self, mesh, facer, type: int = RCLSQUARE, mat=None, nmat: int = 1,
                 device: int = 0):
        self.numel = int(mesh.numel)
        self.type = type
        L = _lib()
        if not getattr(L, "_grad_typed", False):
            L.sfr_gpu_grad_plan_create.argtypes = [_I32, ctypes.POINTER(DifMeshC), _I32,
                                                   ctypes.POINTER(_P)]
            L.sfr_gpu_grad.argtypes = [_P, _P, _I32, _P, _I32, _P, _P]
            L.sfr_gpu_grad_device.argtypes = [_P, _P, _I32, _P, _I32, _P, _P, _P]
            L.sfr_gpu_grad_plan_destroy.argtypes = [_P]
            L._grad_typed = True
        m, _keep = _mesh_c(mesh, facer, None, mat, nmat=nmat)
        h = _P()
        rc = L.sfr_gpu_grad_plan_create(device, ctypes.byref(m), type, ctypes.byref(h))
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_grad_plan_create: " + _sv.last_error())
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            _lib().sfr_gpu_grad_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def grad(self, loads, prop, u, gradu):
        """One rcGradU call with host arrays: u (numel,) or (numel, 3), gradu
        (numel, ndf, 3) the previous gradient; returns the new one."""
        u = _c(u, np.float64)
        ndf = 1 if u.ndim == 1 else int(u.shape[1])
        g = np.array(gradu, dtype=np.float64, copy=True, order="C").reshape(self.numel, ndf, 3)
        lt = _loads_c(loads)
        pr = _c(prop, np.float64)
        rc = _lib().sfr_gpu_grad(self.h, lt, len(loads), _ptr(pr), ndf, _ptr(u), _ptr(g))
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_grad: " + _sv.last_error())
        return g

    def grad_device(self, loads, prop, ndf: int, d_u: int, d_gradu: int, stream: int = 0):
        """The same on device arrays (torch data_ptr values), on ``stream``."""
        lt = _loads_c(loads)
        pr = _c(prop, np.float64)
        rc = _lib().sfr_gpu_grad_device(self.h, lt, len(loads), _ptr(pr), ndf, d_u, d_gradu,
                                        stream or None)
        if rc != _sv.OK:
            raise _sv.SolverError(rc, "sfr_gpu_grad_device: " + _sv.last_error())


def get_values(system: "_sv.GpuSystem"):
    """(al, ad, au) of the system in the reference's layout, copied back
    (au is None unless the storage is unsym CSRC)."""
    nsrc = system._nsrc()
    split = system.storage == _sv.CSRC and system.unsym
    al = np.empty(nsrc // 2 if split else nsrc)
    au = np.empty(nsrc // 2) if split else None
    ad = np.empty(system.neq)
    rc = _lib().sfr_gpu_get_values(system.h, _ptr(al), _ptr(ad), _ptr(au))
    if rc != _sv.OK:
        raise _sv.SolverError(rc, "sfr_gpu_get_values: " + _sv.last_error())
    return al, ad, au
