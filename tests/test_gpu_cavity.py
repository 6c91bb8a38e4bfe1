"""The GPU solvers on real SIMPLE systems harvested from the reference's own
lid-driven cavity (64,000 cells, WALE LES): pressure correction (PCG, CSRC
symmetric) and momentum (BiCGSTAB, CSRC unsym), against the solutions the
reference's own solver returned."""
from __future__ import annotations

import numpy as np
import pytest

from sfr3d_b200 import solver as sv
from helpers import cavity_systems, rel

pytestmark = pytest.mark.gpu

ITERS = {"pressure": 404, "momentum": 4}


@pytest.fixture(scope="module")
def systems():
    return cavity_systems()


@pytest.mark.parametrize("tag", ["pressure", "momentum"])
def test_fp64_matches_reference(cuda, systems, engine, tag):
    s = systems[tag]
    g = sv.GpuSystem(s["neq"], s["ia"], s["ja"], s["storage"], s["unsym"])
    g.set_values(s["al"], s["ad"], s["au"])
    g.set_engine(engine)
    x, info = g.solve(s["solver"], s["b"], tol=s["tol"], maxit=s["maxit"])
    assert info.status == sv.OK
    assert abs(info.iters - ITERS[tag]) <= 1
    assert rel(x, s["x"]) < 1e-12
    g.close()


@pytest.mark.parametrize("tag", ["pressure", "momentum"])
def test_mixed_meets_tolerance(cuda, systems, tag):
    s = systems[tag]
    g = sv.GpuSystem(s["neq"], s["ia"], s["ja"], s["storage"], s["unsym"])
    g.set_values(s["al"], s["ad"], s["au"])
    x, info = g.solve(s["solver"], s["b"], tol=s["tol"], maxit=s["maxit"],
                      precision=sv.MIXED)
    assert info.status == sv.OK
    assert info.relres < 10 * s["tol"]
    # against the reference's own solution: the systems' conditioning bounds it
    assert rel(x, s["x"]) < 1e-6
    g.close()


def test_solverC_dropin_on_cavity_momentum(cuda, systems):
    """The reference's own argument list: for unsym CSRC, al holds al then au
    (matVecCsrC, HccaBlas.c:4233-4236)."""
    s = systems["momentum"]
    x = np.zeros(s["neq"])
    rc = sv.solverC(s["neq"], s["neq"], len(s["ja"]), 0, s["ia"], s["ja"], s["a"], s["ad"],
                    None, s["b"], x, s["tol"], s["maxit"], s["storage"], s["solver"],
                    newX=True, unSym=True, exit_on_failure=False)
    assert rc == sv.OK
    assert rel(x, s["x"]) < 1e-12
