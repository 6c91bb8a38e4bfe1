"""sfr_gpu_dot_noalloc -- the dot product for callers that cannot let this
library allocate device memory.

Such callers reserve their GPU memory once and parcel it out themselves (as
SFR3D does with its host arena), or run while another allocator holds the
device's memory; a cudaMalloc inside the library on first use would break
them.  The entry point keeps its reduction scratch in a fixed device array.
This test calls it through the C ABI twice in a row and compares it with the
allocating sfr_gpu_dot.  Both launch the same deterministic kernel with the
same shape, so the two results must agree bit for bit (the 1e-13 relative
tolerance of the other SpMV/dot tests would hide a change of reduction
order).  It sits in its own file, collected last, and passes both alone in a
fresh process and after the rest of the suite.
"""
from __future__ import annotations

import ctypes

import pytest

from sfr3d_b200 import solver as sv

pytestmark = pytest.mark.gpu


def _noalloc():
    L = sv.lib()
    f = L.sfr_gpu_dot_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def test_noalloc_dot_matches_allocating_dot(cuda):
    torch = cuda
    f = _noalloc()
    gen = torch.Generator(device="cuda").manual_seed(7)
    for n in (2_097_152 + 7, 1000):  # two calls in a row, different sizes
        a = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
        b = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
        want = sv.dot(a.data_ptr(), b.data_ptr(), n)
        out = ctypes.c_double(float("nan"))
        rc = f(a.data_ptr(), b.data_ptr(), n, ctypes.addressof(out), None)
        assert rc == sv.OK, sv.status_string(rc)
        assert out.value == want  # same kernel, same launch shape: same bits
        # and against the reduction torch does itself
        assert abs(out.value - float(torch.dot(a, b))) <= 1e-10 * abs(want)


def test_noalloc_dot_empty_is_zero(cuda):
    torch = cuda
    f = _noalloc()
    a = torch.ones(4, dtype=torch.float64, device="cuda")
    out = ctypes.c_double(float("nan"))
    assert f(a.data_ptr(), a.data_ptr(), 0, ctypes.addressof(out), None) == sv.OK
    assert out.value == 0.0


def test_noalloc_dot_rejects_negative_length(cuda):
    torch = cuda
    f = _noalloc()
    a = torch.ones(4, dtype=torch.float64, device="cuda")
    out = ctypes.c_double()
    assert f(a.data_ptr(), a.data_ptr(), -1, ctypes.addressof(out), None) == sv.BAD_INPUT
