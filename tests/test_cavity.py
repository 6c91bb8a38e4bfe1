"""Real SIMPLE systems harvested from the reference's own lid-driven cavity
run (tests/golden/make_cavity_golden.py): the oracle reproduces the
reference's solutions bit for bit.  No GPU."""
from __future__ import annotations

import pytest

from oracle import oracle as O
from helpers import bits_equal, cavity_systems


@pytest.mark.parametrize("tag,iters", [("pressure", 404), ("momentum", 4)])
def test_oracle_reproduces_reference_on_cavity(tag, iters):
    s = cavity_systems()[tag]
    assert s["storage"] == O.CSRC
    r = O.SOLVERS[s["solver"]](s["storage"], s["unsym"], s["ia"], s["ja"], s["a"], s["ad"],
                               s["b"], tol=s["tol"], maxit=s["maxit"])
    assert r.status == 0 and r.iters == iters
    assert bits_equal(r.x, s["x"])
