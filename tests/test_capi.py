"""The C ABI: symbols, validation and status codes (no GPU needed)."""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

from sfr3d_b200 import _native, solver as sv

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sfr_\w+)\s*\(", text)))


@pytest.mark.parametrize("header,lib", [("sfr3d_b200.h", "libsfr3d_b200.so"),
                                        ("sfr3d_systems.h", "libsfr3d_systems.so")])
def test_every_declared_symbol_is_exported(header, lib):
    L = _native.load(lib)
    names = declared(header)
    assert names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_library_built_for_sm100a():
    # the fatbin carries sm_100a code only; the build flags say so
    from sfr3d_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert os.path.exists(build.LIB)


def test_status_strings():
    assert sv.status_string(sv.OK) == "converged"
    assert "maximum" in sv.status_string(sv.MAXIT)
    assert "timed out" in sv.status_string(sv.TIMEOUT)


def _create(neq, ia, ja, storage, unsym):
    h = ctypes.c_void_p()
    ia = np.ascontiguousarray(ia, np.int32)
    ja = np.ascontiguousarray(ja, np.int32)
    rc = sv.lib().sfr_gpu_create(neq, len(ja), ia.ctypes.data_as(ctypes.c_void_p),
                                 ja.ctypes.data_as(ctypes.c_void_p), storage,
                                 int(unsym), 0, ctypes.byref(h))
    return rc


def test_validation_rejects_bad_patterns_before_device_work():
    # ia not monotone
    assert _create(3, [0, 2, 1, 3], [1, 0, 1], sv.CSRD, True) == sv.BAD_INPUT
    # column out of range
    assert _create(2, [0, 1, 2], [5, 0], sv.CSRD, True) == sv.BAD_INPUT
    # upper entry in lower-triangular storage
    assert _create(2, [0, 1, 1], [1], sv.CSRC, False) == sv.BAD_INPUT
    # ELLPACK header inconsistent
    assert _create(2, [3, 5], [0] * 6, sv.ELLPACK, False) == sv.BAD_INPUT
    # unknown storage
    assert _create(2, [0, 0, 0], [], 7, False) == sv.BAD_INPUT
    assert "storage" in sv.last_error()


def test_solverC_rejects_unsupported_solver_without_exiting():
    ia = np.array([0, 0, 1], np.int32)
    ja = np.array([0], np.int32)
    x = np.zeros(2)
    # 6 = PARDISO (Define.h:397): MKL's direct solver, not on this path
    rc = sv.solverC(2, 2, 1, 0, ia, ja, np.ones(1), np.ones(2), None,
                    np.ones(2), x, 1e-10, 10, sv.CSRD, 6, exit_on_failure=False)
    assert rc == sv.UNSUPPORTED


def test_batch_create_validates_every_system():
    good = (2, np.array([0, 0, 1], np.int32), np.array([0], np.int32))
    bad = (2, np.array([0, 1, 0], np.int32), np.array([0], np.int32))
    with pytest.raises(sv.SolverError) as e:
        sv.GpuBatch([good, bad], sv.CSRD, False)
    assert e.value.status == sv.BAD_INPUT
    assert "system 1" in sv.last_error()


def test_reliable_delta_validation():
    from sfr3d_b200 import solver as sv
    assert sv.lib().sfr_set_solver_reliable_delta(sv.PCG, 0.0) == sv.BAD_INPUT
    assert sv.lib().sfr_set_solver_reliable_delta(sv.PCG, 1.0) == sv.BAD_INPUT
    assert sv.lib().sfr_set_solver_reliable_delta(7, 0.1) == sv.BAD_INPUT
    sv.set_reliable_delta(0.1, sv.PCG)
    sv.set_reliable_delta(1e-4, sv.PBICGSTAB)
