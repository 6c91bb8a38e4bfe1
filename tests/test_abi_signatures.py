"""The Python bindings declare as many arguments as the C ABI takes (a
mismatch would only show on a GPU call).  No GPU."""
from __future__ import annotations

import os
import re

from sfr3d_b200 import assembly, halo, solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_arity(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(sfr_\w+)\s*\(([^;{]*?)\)\s*;", text):
        args = m.group(2).strip()
        out[m.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_argtypes_match_the_header():
    arity = declared_arity("sfr3d_b200.h")
    lib = solver.lib()
    assembly._lib()
    halo._lib()
    checked = 0
    for name, n in arity.items():
        fn = getattr(lib, name, None)
        if fn is None or fn.argtypes is None:
            continue
        assert len(fn.argtypes) == n, (name, len(fn.argtypes), n)
        checked += 1
    assert checked >= 52
