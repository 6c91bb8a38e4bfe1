"""The engines' device-side waits end by themselves when a participant
never arrives.

The reference's solvers wait in MPI_Allreduce without a limit.  Here the
grid barrier, the fused iteration's tagged exchange and the resident
engine's exchange each poll at most `spin_limit` times, then record
SFR_TIMEOUT, and every block leaves the kernel.  sfr_gpu_wait_selftest runs
one such wait on four co-resident blocks and lets `absent` of them leave
before it: with nobody missing the wait completes; with one or three
missing it must give up (a short limit keeps it to well under a second)
and the context must stay usable for the solve that follows.  No fault,
trap or endless loop is involved: the missing block simply returns.
"""
from __future__ import annotations

import numpy as np
import pytest

from sfr3d_b200 import solver as sv
from sfr3d_b200 import systems as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KINDS = [sv.WAIT_GRID_BARRIER, sv.WAIT_TAG_EXCHANGE, sv.WAIT_RESIDENT_EXCHANGE]


@pytest.mark.parametrize("kind", KINDS)
def test_wait_completes_when_every_block_arrives(cuda, kind):
    assert sv.wait_selftest(kind, 0, 1 << 20) == sv.OK


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("absent", [1, 3])
def test_wait_gives_up_when_a_block_never_arrives(cuda, kind, absent):
    rc = sv.wait_selftest(kind, absent, 2000)
    assert rc == sv.TIMEOUT, sv.status_string(rc)
    # the context is still usable: a solve right after is at parity
    s = S.poisson_uniform(8, seed=1)
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    g.set_values(s.al, s.ad)
    x, info = g.solve(sv.PCG, s.b[0], tol=1e-10)
    g.close()
    ref = O.pcg(O.CSRD, True, s.ia, s.ja, s.al, s.ad, s.b[0], tol=1e-10)
    assert info.status == sv.OK and abs(info.iters - ref.iters) <= 1
    assert np.linalg.norm(x - ref.x) <= 1e-12 * np.linalg.norm(ref.x)


def test_wait_selftest_rejects_bad_arguments(cuda):
    assert sv.wait_selftest(3, 0, 100) == sv.BAD_INPUT
    assert sv.wait_selftest(0, 4, 100) == sv.BAD_INPUT
    assert sv.wait_selftest(1, -1, 100) == sv.BAD_INPUT
    assert sv.wait_selftest(2, 0, 0) == sv.BAD_INPUT
