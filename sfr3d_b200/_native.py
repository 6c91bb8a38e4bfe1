"""Loading of the package's native libraries (built in-tree by build.py).

A missing library is an error, never a reason to fall back to Python: the
solver path has no CPU implementation.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
_cache: dict[str, ctypes.CDLL] = {}


class NativeLibraryMissing(RuntimeError):
    pass


def lib_path(name: str) -> str:
    return os.path.join(_HERE, name)


def load(name: str) -> ctypes.CDLL:
    """Load `name` (e.g. 'libsfr3d_b200.so') from the package directory."""
    if name in _cache:
        return _cache[name]
    path = lib_path(name)
    if not os.path.exists(path):
        raise NativeLibraryMissing(
            f"{path} is not built; run `python -m sfr3d_b200.build` "
            f"(or __graft_entry__.build()) first")
    lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
    _cache[name] = lib
    return lib
