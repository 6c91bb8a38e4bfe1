"""Host-side mirror of SFR3D's solver interface over libsfr3d_b200.so.

``solverC`` keeps the argument list and meaning of the reference entry point
(Solv.h:59-70, Solv.c:64-501); ``GpuSystem`` is the explicit handle API
(create / set_values / solve / destroy) that keeps a pattern resident on the
GPU.  Every call goes through the C ABI declared in include/sfr3d_b200.h;
there is no CPU implementation behind it.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native

# solver / storage / status codes (include/sfr3d_b200.h; Define.h:392-412)
PCG, PBICGSTAB, PBICGSTABL2, GMRES, MINRES = 1, 2, 3, 4, 5
CSRD, CSRC, ELLPACK = 2, 3, 4
OK, MAXIT, BREAKDOWN = 0, 1, 2
BAD_INPUT, CUDA_ERROR, TIMEOUT, UNSUPPORTED = -1, -2, -3, -4
FP64, MIXED = 0, 1
ENGINE_AUTO, ENGINE_PERSISTENT, ENGINE_GRAPH, ENGINE_LOOP, ENGINE_RESIDENT = 0, 1, 2, 3, 4

_P = ctypes.c_void_p
_I32 = ctypes.c_int32


class SolveInfoC(ctypes.Structure):
    _fields_ = [("iters", _I32), ("status", _I32), ("xKx", ctypes.c_double),
                ("norm_x", ctypes.c_double), ("norm_r", ctypes.c_double),
                ("norm_r_m", ctypes.c_double), ("conv", ctypes.c_double),
                ("seconds", ctypes.c_double), ("refinements", _I32),
                ("inner_iters", _I32), ("relres", ctypes.c_double)]


@dataclass
class SolveInfo:
    iters: int
    status: int
    xKx: float
    norm_x: float
    norm_r: float
    norm_r_m: float
    conv: float
    seconds: float
    refinements: int
    inner_iters: int
    relres: float

    @classmethod
    def from_c(cls, c: SolveInfoC) -> "SolveInfo":
        return cls(**{f: getattr(c, f) for f, _ in SolveInfoC._fields_})


class TuneResultC(ctypes.Structure):
    _fields_ = [("engine", _I32), ("threads", _I32), ("slices_per_warp", _I32),
                ("prefetch", _I32), ("fused", _I32), ("ms", ctypes.c_double),
                ("default_engine", _I32), ("default_threads", _I32),
                ("default_slices_per_warp", _I32), ("default_prefetch", _I32),
                ("default_fused", _I32), ("default_ms", ctypes.c_double),
                ("candidates", _I32), ("source", _I32)]


class BatchTuneC(ctypes.Structure):
    _fields_ = [("default_ms", ctypes.c_double), ("weighted_ms", ctypes.c_double),
                ("tuned_ms", ctypes.c_double), ("plans", _I32), ("kept", _I32),
                ("grid", _I32), ("max_team_blocks", _I32), ("min_team_blocks", _I32)]


def _struct_dict(c):
    return {name: getattr(c, name) for name, _ in c._fields_}


class SolverError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: {status_string(status)} ({last_error()})")
        self.status = status


def lib() -> ctypes.CDLL:
    L = _native.load("libsfr3d_b200.so")
    if getattr(L, "_typed", False):
        return L
    L.sfr_status_string.restype = ctypes.c_char_p
    L.sfr_status_string.argtypes = [ctypes.c_int]
    L.sfr_last_error.restype = ctypes.c_char_p
    L.sfr_gpu_check_device.argtypes = [_I32, _P, _P]
    L.sfr_gpu_wait_selftest.argtypes = [_I32, _I32, ctypes.c_uint32, _P]
    L.sfr_gpu_create.argtypes = [_I32, _I32, _P, _P, _I32, _I32, _I32,
                                 ctypes.POINTER(_P)]
    L.sfr_gpu_set_values.argtypes = [_P, _P, _P, _P]
    L.sfr_gpu_set_diagonal.argtypes = [_P, _P]
    L.sfr_gpu_solve.argtypes = [_P, _I32, _P, _P, ctypes.c_double,
                                ctypes.c_uint32, _I32, _I32, _P]
    L.sfr_gpu_solve_device.argtypes = [_P, _I32, _P, _P, ctypes.c_double,
                                       ctypes.c_uint32, _I32, _I32, _P, _P]
    L.sfr_gpu_solve_multi_device.argtypes = [_P, _I32, _I32, _P, _P, _P, ctypes.c_double,
                                             ctypes.c_uint32, _I32, _I32, _P, _P]
    L.sfr_gpu_solve_multi.argtypes = [_P, _I32, _I32, _P, _P, _P,
                                      ctypes.c_double, ctypes.c_uint32, _I32,
                                      _I32, _P]
    L.sfr_gpu_solve_transpose.argtypes = [_P, _I32, _P, _P, ctypes.c_double,
                                          ctypes.c_uint32, _I32, _I32, _P]
    L.sfr_gpu_adjoint.argtypes = [_P, _I32, _P, _P, _P, _P, _P, _P,
                                  ctypes.c_double, ctypes.c_uint32, _I32, _P]
    L.sfr_gpu_destroy.argtypes = [_P]
    L.sfr_gpu_set_engine.argtypes = [_P, _I32, _I32, _I32]
    L.sfr_gpu_set_prefetch.argtypes = [_P, _I32]
    L.sfr_gpu_set_fused.argtypes = [_P, _I32]
    L.sfr_gpu_set_staging.argtypes = [_P, _I32]
    L.sfr_gpu_spmv.argtypes = [_P, _P, _P, _P]
    L.sfr_gpu_spmv_transpose.argtypes = [_P, _P, _P, _P]
    L.sfr_gpu_spmv_dot.argtypes = [_P, _P, _P, _P, _P]
    L.sfr_gpu_dot.argtypes = [_P, _P, _I32, _P, _P]
    L.sfr_gpu_stats.argtypes = [_P, _P, _P, _P]
    L.sfr_solverC.argtypes = [_P, _I32, _I32, _I32, _I32, _P, _P, _P, _P, _P,
                              _P, _P, _P, _P, ctypes.c_double, ctypes.c_uint32,
                              ctypes.c_int16, ctypes.c_int16, _P, ctypes.c_bool,
                              ctypes.c_bool, ctypes.c_bool, ctypes.c_char_p]
    L.sfr_gpu_batch_create.argtypes = [_I32, _P, _P, _P, _P, _I32, _I32, _I32,
                                       ctypes.POINTER(_P)]
    L.sfr_gpu_batch_set_values.argtypes = [_P, _P, _P, _P]
    L.sfr_gpu_batch_solve.argtypes = [_P, _I32, _P, _P, ctypes.c_double,
                                      ctypes.c_uint32, _I32, _I32, _P]
    L.sfr_gpu_batch_set_weights.argtypes = [_P, _P]
    L.sfr_gpu_batch_autotune.argtypes = [_P, _I32, _P, ctypes.c_double,
                                         ctypes.c_uint32, _I32, _P]
    L.sfr_gpu_batch_stats.argtypes = [_P, _P, _P, _P]
    L.sfr_gpu_batch_tune_report.argtypes = [_P, _P]
    L.sfr_gpu_autotune.argtypes = [_P, _I32, _I32, _P, _P, ctypes.c_double, ctypes.c_uint32,
                                   _I32, _P]
    L.sfr_gpu_autotune_clear.argtypes = [_P]
    L.sfr_gpu_batch_destroy.argtypes = [_P]
    L.sfr_set_exit_on_failure.argtypes = [_I32]
    L.sfr_set_exit_on_failure.restype = None
    L.sfr_set_precision.argtypes = [_I32]
    L.sfr_set_reliable_delta.argtypes = [ctypes.c_double]
    L.sfr_set_reliable_delta.restype = None
    L.sfr_set_solver_reliable_delta.argtypes = [_I32, ctypes.c_double]
    L.sfr_write_coo.argtypes = [ctypes.c_char_p, _I32, _P, _P, _P, _P, _P, _I32, _I32, _I32,
                                _I32]
    L.sfr_write_coo_b.argtypes = [ctypes.c_char_p, _P, _I32]
    L.sfr_gpu_write_coo.argtypes = [_P, ctypes.c_char_p, _P, _P, _I32]
    L.sfr_set_precision.restype = None
    L.sfr_set_autotune.argtypes = [_I32]
    L.sfr_set_autotune.restype = None
    L.sfr_solverC_set_group.argtypes = [_P]
    L.sfr_solverC_release.restype = None
    L.sfr_solverC_release.argtypes = []
    L._typed = True
    return L


def status_string(status: int) -> str:
    return lib().sfr_status_string(status).decode()


def last_error() -> str:
    return lib().sfr_last_error().decode()


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def check_device(device: int = 0) -> tuple[int, int, int]:
    ma, mi = ctypes.c_int32(), ctypes.c_int32()
    rc = lib().sfr_gpu_check_device(device, ctypes.byref(ma), ctypes.byref(mi))
    return rc, ma.value, mi.value


# the device-side waits sfr_gpu_wait_selftest exercises
WAIT_GRID_BARRIER, WAIT_TAG_EXCHANGE, WAIT_RESIDENT_EXCHANGE = 0, 1, 2


def wait_selftest(kind: int, absent: int, spin_limit: int, stream=None) -> int:
    """Run one of the engines' bounded waits on four blocks of which
    `absent` never arrive; SFR_OK when it completed, SFR_TIMEOUT when it
    gave up after `spin_limit` polls."""
    return lib().sfr_gpu_wait_selftest(kind, absent, spin_limit, stream)


class GpuSystem:
    """One sparse pattern resident on a GPU (sfr_gpu_create ... destroy)."""

    def __init__(self, neq: int, ia, ja, storage: int, unsym: bool,
                 nad: int | None = None, device: int = 0):
        self._ia = _i32(ia)
        self._ja = _i32(ja) if ja is not None else None
        if nad is None:
            nad = (int(self._ia[1]) if storage == ELLPACK
                   else int(self._ia[neq] - self._ia[0]))
        self.neq, self.nad, self.storage, self.unsym = neq, nad, storage, unsym
        self.values_version = 0  # bumped by every set_values / set_diagonal
        h = _P()
        rc = lib().sfr_gpu_create(neq, nad, _ptr(self._ia), _ptr(self._ja),
                                  storage, int(unsym), device, ctypes.byref(h))
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().sfr_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_engine(self, engine: int, threads: int = 0, slices_per_warp: int = 0):
        """0 automatic, 1 persistent (one cooperative launch), 2 graph,
        3 graph kernels from a host loop (profilers), 4 resident (mixed
        PCG, one right-hand side, inner iteration held on chip)."""
        rc = lib().sfr_gpu_set_engine(self.h, engine, threads, slices_per_warp)
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_set_engine")

    def set_prefetch(self, rounds: int):
        """Graph engine: L2 prefetch of the SELL slice each warp reaches
        `rounds` rounds later in the SpMV phases (0 off)."""
        rc = lib().sfr_gpu_set_prefetch(self.h, rounds)
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_set_prefetch")

    def set_fused(self, mode: int):
        """Graph engine, FP64 PCG with one right-hand side
        (sfr_gpu_set_fused): 0 three kernels an iteration, 1-3 one cooperative
        kernel an iteration (2: held to 40 registers; 3: tagged exchanges),
        4 (the default) the whole solve in one cooperative launch."""
        rc = lib().sfr_gpu_set_fused(self.h, int(mode))
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_set_fused")

    def set_staging(self, flag: int):
        """Graph engine, BiCGSTAB: SpMV-phase slices staged in shared memory
        by bulk copies (sfr_gpu_set_staging; 1 on, 0 off, the default)."""
        rc = lib().sfr_gpu_set_staging(self.h, int(flag))
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_set_staging")

    def autotune(self, solver: int, b, ad_k=None, tol: float = 1e-10, maxit: int = 100000,
                 precision: int = FP64) -> dict:
        """Time the engines and graph launch shapes on this system's solve
        of b ((neq,) or (k, neq)) and keep the fastest for later automatic
        solves of that kind (sfr_gpu_autotune).  Returns the report as a dict:
        engine, threads, slices_per_warp, ms, the default_* choice and its
        time, candidates timed and source (0 measured, 1 handle, 2 file)."""
        b = _f64(b)
        k = 1 if b.ndim == 1 else b.shape[0]
        ad_k = _f64(ad_k)
        out = TuneResultC()
        rc = lib().sfr_gpu_autotune(self.h, solver, k, _ptr(ad_k), _ptr(b), tol, maxit,
                                    precision, ctypes.byref(out))
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_autotune: " + last_error())
        return _struct_dict(out)

    def autotune_clear(self):
        lib().sfr_gpu_autotune_clear(self.h)

    def set_values(self, al, ad, au=None):
        al, ad, au = _f64(al), _f64(ad), _f64(au)
        rc = lib().sfr_gpu_set_values(self.h, _ptr(al), _ptr(ad), _ptr(au))
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_set_values")
        self.values_version += 1

    def set_diagonal(self, ad):
        ad = _f64(ad)
        rc = lib().sfr_gpu_set_diagonal(self.h, _ptr(ad))
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_set_diagonal")
        self.values_version += 1

    def solve(self, solver: int, b, x0=None, tol: float = 1e-10,
              maxit: int = 100000, newx: bool = True, precision: int = FP64,
              raise_on_error: bool = True):
        """Host-buffer solve (sfr_gpu_solve).  Returns (x, SolveInfo)."""
        b = _f64(b)
        x = np.zeros(self.neq) if x0 is None else np.array(x0, dtype=np.float64)
        info = SolveInfoC()
        rc = lib().sfr_gpu_solve(self.h, solver, _ptr(b), _ptr(x), tol, maxit,
                                 int(newx), precision, ctypes.byref(info))
        if rc < 0 and raise_on_error:
            raise SolverError(rc, "sfr_gpu_solve")
        return x, SolveInfo.from_c(info)

    def solve_multi(self, solver: int, b, x0=None, ad_k=None, tol=1e-10,
                    maxit=100000, newx=True, precision=FP64,
                    raise_on_error=True):
        """k right-hand sides sharing the matrix; b is (k, neq)."""
        b = _f64(b)
        k = b.shape[0]
        x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
        ad_k = _f64(ad_k)
        infos = (SolveInfoC * k)()
        rc = lib().sfr_gpu_solve_multi(self.h, solver, k, _ptr(ad_k), _ptr(b),
                                       _ptr(x), tol, maxit, int(newx),
                                       precision, infos)
        if rc < 0 and raise_on_error:
            raise SolverError(rc, "sfr_gpu_solve_multi")
        return x, [SolveInfo.from_c(infos[i]) for i in range(k)]

    def solve_transpose(self, solver: int, b, x0=None, tol: float = 1e-10,
                        maxit: int = 100000, newx: bool = True,
                        precision: int = FP64, raise_on_error: bool = True):
        """Solve A^T x = b (sfr_gpu_solve_transpose).  Returns (x, SolveInfo)."""
        b = _f64(b)
        x = np.zeros(self.neq) if x0 is None else np.array(x0, dtype=np.float64)
        info = SolveInfoC()
        rc = lib().sfr_gpu_solve_transpose(self.h, solver, _ptr(b), _ptr(x), tol,
                                           maxit, int(newx), precision,
                                           ctypes.byref(info))
        if rc < 0 and raise_on_error:
            raise SolverError(rc, "sfr_gpu_solve_transpose")
        return x, SolveInfo.from_c(info)

    def adjoint(self, solver: int, x, g, tol: float = 1e-12,
                maxit: int = 100000, precision: int = FP64,
                raise_on_error: bool = True):
        """Adjoint of x = A^-1 b for dJ/dx = g (sfr_gpu_adjoint).

        Returns (lam, g_al, g_ad, g_au, SolveInfo): dJ/db = lam and
        dJ/dA_ij = -lam_i x_j in the value layout of set_values (g_au is
        None unless the storage keeps a separate upper array).
        """
        x, g = _f64(x), _f64(g)
        lam = np.zeros(self.neq)
        split = self.storage == CSRC and self.unsym
        nsrc = self._nsrc()
        g_al = np.zeros(nsrc // 2 if split else nsrc)
        g_ad = np.zeros(self.neq)
        g_au = np.zeros(nsrc // 2) if split else None
        info = SolveInfoC()
        rc = lib().sfr_gpu_adjoint(self.h, solver, _ptr(x), _ptr(g), _ptr(lam),
                                   _ptr(g_al), _ptr(g_ad), _ptr(g_au), tol,
                                   maxit, precision, ctypes.byref(info))
        if rc < 0 and raise_on_error:
            raise SolverError(rc, "sfr_gpu_adjoint")
        return lam, g_al, g_ad, g_au, SolveInfo.from_c(info)

    def _nsrc(self) -> int:
        """Number of stored off-diagonal values (al, plus au when split)."""
        if self.storage == ELLPACK:
            return int(self._ia[1])
        n = int(self._ia[self.neq] - self._ia[0])
        return 2 * n if (self.storage == CSRC and self.unsym) else n

    def write_coo(self, path, binary=False):
        """The system's current values as the reference's writeCoo dump
        (CSRD only), e.g. right after a device assembly."""
        rc = lib().sfr_gpu_write_coo(self.h, str(path).encode(), _ptr(self._ia),
                                     _ptr(self._ja), int(binary))
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_write_coo: " + last_error())

    # device-pointer entry points (pointers are plain integers)
    def solve_device(self, solver, d_b: int, d_x: int, tol=1e-10,
                     maxit=100000, newx=True, precision=FP64, stream: int = 0):
        info = SolveInfoC()
        rc = lib().sfr_gpu_solve_device(self.h, solver, d_b, d_x, tol, maxit,
                                        int(newx), precision, stream or None,
                                        ctypes.byref(info))
        if rc < 0:
            raise SolverError(rc, "sfr_gpu_solve_device")
        return SolveInfo.from_c(info)

    def solve_multi_device(self, solver, k: int, d_b: int, d_x: int, d_ad_k: int = 0,
                           tol=1e-10, maxit=100000, newx=True, precision=FP64,
                           stream: int = 0):
        """k right-hand sides on device arrays (b and x k*neq, RHS r at
        offset r*neq; d_ad_k 0 for the system's own diagonal)."""
        infos = (SolveInfoC * k)()
        rc = lib().sfr_gpu_solve_multi_device(self.h, solver, k, d_ad_k or None, d_b, d_x, tol,
                                              maxit, int(newx), precision, stream or None,
                                              infos)
        if rc < 0:
            raise SolverError(rc, "sfr_gpu_solve_multi_device")
        return [SolveInfo.from_c(infos[i]) for i in range(k)]

    def spmv(self, d_x: int, d_y: int, stream: int = 0):
        rc = lib().sfr_gpu_spmv(self.h, d_x, d_y, stream or None)
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_spmv")

    def spmv_transpose(self, d_x: int, d_y: int, stream: int = 0):
        rc = lib().sfr_gpu_spmv_transpose(self.h, d_x, d_y, stream or None)
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_spmv_transpose")

    def spmv_dot(self, d_x: int, d_y: int, stream: int = 0) -> float:
        out = ctypes.c_double()
        rc = lib().sfr_gpu_spmv_dot(self.h, d_x, d_y, ctypes.byref(out),
                                    stream or None)
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_spmv_dot")
        return out.value

    def stats(self):
        b, s, w = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
        lib().sfr_gpu_stats(self.h, ctypes.byref(b), ctypes.byref(s),
                            ctypes.byref(w))
        return {"device_bytes": b.value, "slots": s.value, "bandwidth": w.value}


def _ptr_array(arrays):
    arr = (_P * len(arrays))()
    for i, a in enumerate(arrays):
        arr[i] = None if a is None else a.ctypes.data
    return arr


class GpuBatch:
    """Many independent systems solved in one persistent launch
    (sfr_gpu_batch_*).  `systems` is a list of (neq, ia, ja) in one storage."""

    def __init__(self, systems, storage: int, unsym: bool, device: int = 0):
        self.nsys = len(systems)
        self._keep = []
        neq = np.array([s[0] for s in systems], np.int32)
        ias = [_i32(s[1]) for s in systems]
        jas = [_i32(s[2]) for s in systems]
        nad = np.array([len(j) for j in jas], np.int32)
        self._keep += [neq, nad, ias, jas]
        self.neq = neq
        h = _P()
        rc = lib().sfr_gpu_batch_create(self.nsys, _ptr(neq), _ptr(nad),
                                        _ptr_array(ias), _ptr_array(jas),
                                        storage, int(unsym), device,
                                        ctypes.byref(h))
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_batch_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().sfr_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_values(self, als, ads, aus=None):
        als = [_f64(a) for a in als]
        ads = [_f64(a) for a in ads]
        aus = None if aus is None else [_f64(a) for a in aus]
        rc = lib().sfr_gpu_batch_set_values(self.h, _ptr_array(als), _ptr_array(ads),
                                            None if aus is None else _ptr_array(aus))
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_batch_set_values")

    def solve(self, solver, bs, x0s=None, tol=1e-10, maxit=100000, newx=True,
              precision=FP64, raise_on_error=True):
        bs = [_f64(b) for b in bs]
        xs = ([np.zeros(int(n)) for n in self.neq] if x0s is None
              else [np.array(x, dtype=np.float64) for x in x0s])
        infos = (SolveInfoC * self.nsys)()
        rc = lib().sfr_gpu_batch_solve(self.h, solver, _ptr_array(bs), _ptr_array(xs),
                                       tol, maxit, int(newx), precision, infos)
        if rc < 0 and raise_on_error:
            raise SolverError(rc, "sfr_gpu_batch_solve")
        return xs, [SolveInfo.from_c(infos[i]) for i in range(self.nsys)]

    def set_weights(self, w):
        w = _f64(w)
        rc = lib().sfr_gpu_batch_set_weights(self.h, _ptr(w))
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_batch_set_weights")

    def autotune(self, solver, bs, tol=1e-10, maxit=100000, precision=FP64) -> float:
        bs = [_f64(b) for b in bs]
        ms = ctypes.c_double()
        rc = lib().sfr_gpu_batch_autotune(self.h, solver, _ptr_array(bs), tol, maxit,
                                          precision, ctypes.byref(ms))
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_batch_autotune")
        return ms.value

    def tune_report(self) -> dict:
        """The last autotune's plans and times (sfr_gpu_batch_tune_report)."""
        out = BatchTuneC()
        rc = lib().sfr_gpu_batch_tune_report(self.h, ctypes.byref(out))
        if rc != OK:
            raise SolverError(rc, "sfr_gpu_batch_tune_report")
        return _struct_dict(out)

    def stats(self):
        g, r, b = ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int64()
        lib().sfr_gpu_batch_stats(self.h, ctypes.byref(g), ctypes.byref(r), ctypes.byref(b))
        return {"grid": g.value, "rows": r.value, "device_bytes": b.value}


def dot(d_a: int, d_b: int, n: int, stream: int = 0) -> float:
    out = ctypes.c_double()
    rc = lib().sfr_gpu_dot(d_a, d_b, n, ctypes.byref(out), stream or None)
    if rc != OK:
        raise SolverError(rc, "sfr_gpu_dot")
    return out.value


def solverC(nEq, nEqNov, nAd, nAdR, ia, ja, al, ad, au, b, x, tol, maxIt,
            storage, solver, fSolvLog=None, fLog=False, newX=True,
            unSym=False, name="system", exit_on_failure=False, iNeq=None) -> int:
    """The reference's solverC (Solv.c:64) through sfr_solverC: x is updated
    in place, b is left unchanged.  fSolvLog is a C FILE* (integer) or None.
    Returns the status (the reference returns nothing and exits on failure;
    pass exit_on_failure=True for that behaviour)."""
    L = lib()
    L.sfr_set_exit_on_failure(int(exit_on_failure))
    ia, ja = _i32(ia), _i32(ja)
    al, ad, au, b = _f64(al), _f64(ad), _f64(au), _f64(b)
    if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
        raise TypeError("x must be a C-contiguous float64 array (updated in place)")
    ineq = None if iNeq is None else ctypes.cast(ctypes.pointer(iNeq), _P)
    return L.sfr_solverC(None, nEq, nEqNov, nAd, nAdR, _ptr(ia), _ptr(ja),
                         _ptr(al), _ptr(ad), _ptr(au), _ptr(b), _ptr(x), ineq,
                         None, tol, maxIt, storage, solver, fSolvLog,
                         bool(fLog), bool(newX), bool(unSym), name.encode())


def set_precision(precision: int) -> None:
    lib().sfr_set_precision(precision)


def set_reliable_delta(delta: float, solver: int | None = None) -> None:
    """Mixed precision: the factor the FP32 residual must fall by before an
    FP64 refresh, for one solver or (solver=None) both."""
    if solver is None:
        lib().sfr_set_reliable_delta(delta)
        return
    rc = lib().sfr_set_solver_reliable_delta(solver, delta)
    if rc != OK:
        raise SolverError(rc, "sfr_set_solver_reliable_delta")


def release_cache() -> None:
    lib().sfr_solverC_release()


# ------------------------------------------------------ Matrix Market --
def write_coo(path, ia, ja, ad, al, au=None, storage=CSRD, unsym=True, binary=False):
    """The reference's writeCoo (WriteMtx.c:26): the CSRD system as a Matrix
    Market coordinate file, diagonal first in each row."""
    ia, ja = _i32(ia), _i32(ja)
    ad, al = _f64(ad), _f64(al)
    au = al if au is None else _f64(au)
    rc = lib().sfr_write_coo(str(path).encode(), len(ia) - 1, _ptr(ia), _ptr(ja), _ptr(au),
                             _ptr(ad), _ptr(al), len(ja), storage, int(unsym), int(binary))
    if rc != OK:
        raise SolverError(rc, "sfr_write_coo: " + last_error())


def write_coo_b(path, b):
    """The reference's writeCooB (WriteMtx.c:163): a force vector."""
    b = _f64(b)
    rc = lib().sfr_write_coo_b(str(path).encode(), _ptr(b), len(b))
    if rc != OK:
        raise SolverError(rc, "sfr_write_coo_b: " + last_error())


def read_mtx(path):
    """A Matrix Market file as written by write_coo / write_coo_b (or any
    real coordinate / array file): ("coordinate", rows, cols, (i, j, v)
    0-based, symmetric flag) or ("array", rows, cols, values)."""
    with open(path) as f:
        banner = f.readline().split()
        kind = banner[2]
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        dims = [int(t) for t in line.split()]
        if kind == "coordinate":
            data = np.loadtxt(f, ndmin=2)
            i = data[:, 0].astype(np.int64) - 1
            j = data[:, 1].astype(np.int64) - 1
            return "coordinate", dims[0], dims[1], (i, j, data[:, 2]), banner[4] == "symmetric"
        return "array", dims[0], dims[1], np.loadtxt(f, ndmin=1)
