"""Matrix Market dumps in the reference's own format (writeCoo / writeCooB,
WriteMtx.c): byte for byte against files the reference wrote.  No GPU."""
from __future__ import annotations

import filecmp
import os

import numpy as np
import pytest

from sfr3d_b200 import solver as sv

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "coo")


@pytest.fixture(scope="module")
def inputs():
    return np.load(os.path.join(GOLD, "inputs.npz"))


@pytest.mark.parametrize("name", ["full", "lower", "graph"])
def test_write_coo_matches_reference(tmp_path, inputs, name):
    z = inputs
    if name == "lower":
        ia, ja, al, unsym = z["il"], z["jl"], z["al_lower"], False
    else:
        ia, ja, al, unsym = z["ia"], z["ja"], z["al"], True
    out = tmp_path / f"{name}.mtx"
    sv.write_coo(out, ia, ja, z["ad"], al, unsym=unsym, binary=name == "graph")
    assert filecmp.cmp(out, os.path.join(GOLD, f"{name}.mtx"), shallow=False)


def test_write_coo_b_matches_reference(tmp_path, inputs):
    out = tmp_path / "b.mtx"
    sv.write_coo_b(out, inputs["b"])
    assert filecmp.cmp(out, os.path.join(GOLD, "b.mtx"), shallow=False)


def test_read_back(tmp_path, inputs):
    z = inputs
    out = tmp_path / "a.mtx"
    sv.write_coo(out, z["ia"], z["ja"], z["ad"], z["al"])
    kind, m, n, (i, j, v), sym = sv.read_mtx(out)
    assert kind == "coordinate" and m == n == len(z["ad"]) and not sym
    A = np.zeros((m, n))
    A[i, j] = v
    rows = np.repeat(np.arange(m), np.diff(z["ia"]))
    B = np.diag(z["ad"])
    B[rows, z["ja"]] = z["al"]
    assert np.allclose(A, B, rtol=1e-13, atol=0)   # %30.14e keeps 15 significant digits
    kind, m, n, b = sv.read_mtx(os.path.join(GOLD, "b.mtx"))
    assert kind == "array" and np.allclose(b, z["b"], rtol=1e-13, atol=0)


def test_write_coo_rejects_other_storages(tmp_path, inputs):
    with pytest.raises(sv.SolverError) as e:
        sv.write_coo(tmp_path / "x.mtx", inputs["ia"], inputs["ja"], inputs["ad"], inputs["al"],
                     storage=sv.CSRC)
    assert e.value.status == sv.BAD_INPUT
