"""The diffusion assembly oracle (systFormDif restated in C) against the
reference's own compiled systFormDif: the committed fixture always, and
live when oracle/_ref is built.  No GPU."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

from oracle import oracle as O
from sfr3d_b200 import systems as S
from helpers import bits_equal, dif_case, dif_fixture, layouts


def test_oracle_matches_reference_fixture():
    mesh, facer, fields, loads, lays, cases = dif_fixture()
    assert len(cases) >= 20
    for c in cases:
        st, un, ia, ja, neq = lays[c["layout"]]
        rc, a, ad, b, rcell = O.dif_assemble(dif_case(mesh, facer, fields, loads, c), st, un,
                                             ia, ja, neq, c["forces"], c["matrix"],
                                             c["calrcell"], fill=0.0)
        assert rc == 0, c["name"]
        for got, want, what in ((a, c["a"], "a"), (ad, c["ad"], "ad"), (b, c["b"], "b"),
                                (rcell, c["rcell"], "rcell")):
            assert bits_equal(got, want), (c["name"], what)


def _random_case(m, rng, icod, fres, time):
    return O.DifCase(
        mesh=m, facer=m.face_r([1, 4, 2, 6, 3, 0]),
        loads=[O.Load(O.DIRICHLET, (0.5,)), O.Load(O.NEUMANN, (0.25,)),
               O.Load(O.ROBIN, (2.0, 1.5)), O.Load(9, (1.0,)), O.Load(0, ()),
               O.Load(O.INLET, (1.0, 0.3, -0.2, 0.1, 1.2))],
        density=rng.uniform(0.5, 2, m.numel), cdiff=m.cdiff * rng.uniform(0.5, 2, m.numel),
        u0=rng.standard_normal(m.numel), gradu0=rng.standard_normal((m.numel, 3)),
        icod=icod, fres=fres, time_flag=time is not None,
        time_type=time[0] if time else 0, dt=0.1, dt0=0.05)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference)")
def test_oracle_matches_reference_live():
    s = S.poisson_jittered(5, seed=4)
    m = s.mesh()
    rng = np.random.default_rng(2)
    lay = layouts(s)
    ia, ja, _ = s.csrc()
    lay["csrc_unsym"] = (O.CSRC, True, ia, ja, None, None)
    n = 0
    for icod, time, fres, flags in itertools.product(
            (1, 2, 3, 4), (None, (O.EULER,), (O.BACKWARD,)), (False, True),
            ((1, 1, 1), (1, 0, 0), (0, 1, 1))):
        case = _random_case(m, rng, icod, fres, time)
        for name, (st, un, ia, ja, _al, _au) in lay.items():
            r1 = O.dif_assemble(case, st, un, ia, ja, s.neq, *flags, fill=7.0)
            r2 = O.ref_dif_assemble(case, st, un, ia, ja, s.neq, *flags, fill=7.0)
            assert r1[0] == r2[0] == 0
            for x, y in zip(r1[1:], r2[1:5]):
                assert bits_equal(x, y), (icod, time, fres, flags, name)
            n += 1
    assert n == 4 * 3 * 2 * 3 * len(lay)


def test_oracle_error_paths():
    s = S.poisson_uniform(4, seed=1)
    m = s.mesh()
    base = dict(mesh=m, facer=m.face_r([1, 0, 0, 0, 0, 0]), density=np.ones(m.numel),
                cdiff=m.cdiff, u0=np.zeros(m.numel), gradu0=np.zeros((m.numel, 3)))
    run = lambda **kw: O.dif_assemble(O.DifCase(**{**base, **kw}), O.CSRD, True,  # noqa: E731
                                      s.ia, s.ja, s.neq)[0]
    assert run(loads=[O.Load(O.DIRICHLET, (1.0,))]) == 0
    assert run(loads=[O.Load(O.SINBC, (1.0,) * 9)]) == -2       # sin of the face centre
    assert run(loads=[O.Load(O.DIRICHLET, (1.0,), var=1)]) == -2  # a function
    assert run(loads=[O.Load(O.OUTLET, ())]) == -1              # needs a velocity
    assert run(loads=[O.Load(O.DIRICHLET, (1.0,))], icod=5) == -1  # the reference exits
    assert run(loads=[O.Load(O.DIRICHLET, (1.0,))], caltype=np.array([2], np.int16)) == -1


def test_mesh_export_geometry():
    s = S.poisson_jittered(6, seed=3)
    m = s.mesh()
    assert m.nface == 3 * 6 * 6 * 7
    # outward area vectors of every cell close
    fid = m.cellface - 1
    ch = np.where(m.owner[fid, 0] - 1 == np.arange(m.numel)[:, None], 1.0, -1.0)
    tot = (ch[..., None] * m.area[fid][..., None] * m.normal[fid]).sum(axis=1)
    assert abs(tot).max() < 1e-14
    # face neighbours = the system's pattern, in equation numbers
    eq = m.id - 1
    for c in range(m.numel):
        r = eq[c]
        nb = m.nelcon[c][m.nelcon[c] > 0] - 1
        assert sorted(eq[nb]) == sorted(s.ja[s.ia[r]:s.ia[r + 1]])
    # ksi is a unit vector pointing from the owner towards the neighbour
    assert np.allclose(np.linalg.norm(m.ksi, axis=1), 1.0)
    assert (np.einsum("ij,ij->i", m.ksi, m.normal) > 0).all()
    # the ELLPACK layout of the system is in the same face order
    ja, _ = s.ell()
    ja = ja.reshape(s.neq, s.width)
    for c in range(0, m.numel, 7):
        for f in range(6):
            want = eq[m.nelcon[c, f] - 1] if m.nelcon[c, f] > 0 else eq[c]
            assert ja[eq[c], f] == want


def test_dif_plan_rejects_too_many_loads():
    from sfr3d_b200 import assembly as A
    with pytest.raises(ValueError):
        A._loads_c([A.Load(A.NEUMANN, (0.0,))] * 33)


# ------------------------------------------------ pressure correction --
from helpers import pres_fixture  # noqa: E402


def test_pres_oracle_matches_reference_fixture():
    mesh, sides, f, lvel, lpres, lays, cases = pres_fixture()
    assert len(cases) >= 20
    for c in cases:
        st, un, ia, ja, neq = lays[c["layout"]]
        fv, fp = sides[c["sides"]]
        case = O.PresCase(mesh=mesh, facevelr=fv, facepresr=fp, lvel=lvel, lpres=lpres,
                          icod=c["icod"], **f)
        rc, a, ad, b, rcell = O.pres_assemble(case, st, un, ia, ja, neq, c["forces"],
                                              c["matrix"], c["calrcell"], fill=0.0)
        assert rc == 0, c["name"]
        for got, want, what in ((a, c["a"], "a"), (ad, c["ad"], "ad"), (b, c["b"], "b"),
                                (rcell, c["rcell"], "rcell")):
            assert bits_equal(got, want), (c["name"], what)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference)")
def test_pres_oracle_matches_reference_live():
    s = S.poisson_jittered(5, seed=8)
    m = s.mesh()
    rng = np.random.default_rng(4)
    lay = layouts(s)
    ia, ja, _ = s.csrc()
    lay["csrc_unsym"] = (O.CSRC, True, ia, ja, None, None)
    prop = np.zeros((3, O.MAXPROP))
    prop[:, O.DENSITY] = (1.0, 0.8, 1.4)
    lvel = [O.Load(O.STATICWALL, ()), O.Load(O.INLET, (0.5, 0.1, -0.2), np=3),
            O.Load(O.OPEN, (), density=1.1), O.Load(O.OUTLET, ())]
    lpres = [O.Load(O.DIRICHLET, (0.0,)), O.Load(O.OPEN, (0.0,))]
    for icod in (O.ORTHOGONAL, O.OVERRELAXED):
        case = O.PresCase(mesh=m, facevelr=m.face_r([1, 2, 3, 4, 1, 1]),
                          facepresr=m.face_r([0, 1, 2, 0, 0, 0]), lvel=lvel, lpres=lpres,
                          prop=prop, mat=rng.integers(1, 4, m.numel).astype(np.int16),
                          pres=rng.standard_normal(m.numel),
                          gradpres=rng.standard_normal((m.numel, 3)),
                          vel=rng.standard_normal((m.numel, 3)),
                          dfield=rng.uniform(0.1, 1.0, (m.numel, 3)), icod=icod)
        for name, (st, un, ia, ja, _al, _au) in lay.items():
            r1 = O.pres_assemble(case, st, un, ia, ja, s.neq, fill=2.0)
            r2 = O.ref_pres_assemble(case, st, un, ia, ja, s.neq, fill=2.0)
            r3 = O.ref_pres_assemble(case, st, un, ia, ja, s.neq, fill=2.0, nthreads=4)
            assert r1[0] == r2[0] == r3[0] == 0
            for x, y, z in zip(r1[1:], r2[1:5], r3[1:5]):
                assert bits_equal(x, y) and bits_equal(x, z), (icod, name)


def test_pres_oracle_rejects_what_the_reference_cannot_take():
    s = S.poisson_uniform(4, seed=1)
    m = s.mesh()
    base = dict(mesh=m, facevelr=m.face_r([1, 0, 0, 0, 0, 0]), facepresr=m.face_r([0] * 6),
                lpres=[], prop=np.array([[0.0, 1.0] + [0.0] * 8]),
                pres=np.zeros(m.numel), gradpres=np.zeros((m.numel, 3)),
                vel=np.zeros((m.numel, 3)), dfield=np.ones((m.numel, 3)))
    run = lambda **kw: O.pres_assemble(O.PresCase(**{**base, **kw}), O.CSRD, True,  # noqa: E731
                                       s.ia, s.ja, s.neq)[0]
    assert run(lvel=[O.Load(O.INLET, (1.0, 0.0, 0.0, 1.0))]) == 0
    assert run(lvel=[O.Load(O.INLET, (1.0, 0.0, 0.0, 1.0), var=1)]) == -2
    assert run(lvel=[O.Load(O.INLET, (1.0, 0.0))]) == -1
    # MINIMAL / ORTHOGONALC leave the split unset in the reference
    assert run(lvel=[O.Load(O.STATICWALL, ())], icod=O.MINIMAL) == -1


# ------------------------------------------------------ momentum --
def _cell_centres(m):
    """Cell centroids consistent with the exported geometry (xm - xmcc)."""
    return m.xm[m.cellface[:, 0] - 1] - m.xmcc[:, 0, :]


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference)")
def test_vel_oracle_matches_reference_live():
    s = S.poisson_jittered(5, seed=4)
    m = s.mesh()
    rng = np.random.default_rng(5)
    lay = layouts(s)
    ia, ja, _ = s.csrc()
    lay["csrc_unsym"] = (O.CSRC, True, ia, ja, None, None)
    del lay["ellpack"]  # csrSimple's ELLPACK branch refuses ndf > 1
    prop = np.zeros((2, O.MAXPROP))
    prop[:, 0] = (1e-3, 2e-3)
    prop[:, 1] = (1.0, 1.2)
    mat = rng.integers(1, 3, m.numel).astype(np.int16)
    lvel = [O.Load(O.STATICWALL, ()), O.Load(O.MOVEWALL, (1.0, 0.2, -0.1, 0.0)),
            O.Load(O.INLET, (0.5, 0.1, 0.0, 1.1))]
    for icod, fso, fvisc, fres, ts, time in itertools.product(
            (1, 4), (0, 1), (0, 1), (0, 1), (O.SIMPLE, O.SIMPLEC), (None, O.EULER, O.BACKWARD)):
        case = O.VelCase(mesh=m, cc=_cell_centres(m), facevelr=m.face_r([1, 1, 2, 1, 3, 1]),
                         facepresr=m.face_r([0] * 6), lvel=lvel, prop=prop, mat=mat,
                         pres=rng.standard_normal(m.numel),
                         gradpres=rng.standard_normal((m.numel, 3)),
                         vel=rng.standard_normal((m.numel, 3)),
                         gradvel=rng.standard_normal((m.numel, 3, 3)),
                         dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=icod, fso=bool(fso),
                         fvisc=bool(fvisc), fres=bool(fres), type_simple=ts,
                         time_flag=time is not None, time_type=time or 0, dt=0.05, dt0=0.04,
                         under=0.7)
        for name, (st, un, ia, ja, _al, _au) in lay.items():
            r1 = O.vel_assemble(case, st, un, ia, ja, s.neq, fill=3.0)
            r2 = O.ref_vel_assemble(case, st, un, ia, ja, s.neq, fill=3.0)
            assert r1[0] == r2[0] == 0
            for x, y in zip(r1[1:], r2[1:6]):
                assert bits_equal(x, y), (icod, fso, fvisc, fres, ts, time, name)
        # its OpenMP cell loop gives the same system (without Rhie-Chow it
        # only writes the D field)
        st, un, ia, ja, _al, _au = lay["csrd_full"]
        r1 = O.vel_assemble(case, st, un, ia, ja, s.neq, fill=3.0)
        r3 = O.ref_vel_assemble(case, st, un, ia, ja, s.neq, fill=3.0, nthreads=4)
        for x, y in zip(r1[1:], r3[1:6]):
            assert bits_equal(x, y)


def test_vel_oracle_advection_schemes_match_reference_live():
    """CD and SoUp (advectiveScheme, CellLib.c:6394-6480): the deferred
    correction p -= cv cvc, on every layout, against the reference's own
    systFormSimpleVel."""
    s = S.poisson_jittered(5, seed=6)
    m = s.mesh()
    rng = np.random.default_rng(7)
    lay = layouts(s)
    ia, ja, _ = s.csrc()
    lay["csrc_unsym"] = (O.CSRC, True, ia, ja, None, None)
    del lay["ellpack"]
    prop = np.zeros((1, O.MAXPROP))
    prop[0, :2] = (1e-3, 1.0)
    lvel = [O.Load(O.STATICWALL, ()), O.Load(O.MOVEWALL, (1.0, 0.2, -0.1, 0.0)),
            O.Load(O.INLET, (0.5, 0.1, 0.0, 1.1))]
    for adv, icod, fso, ts in itertools.product((O.CD, O.SOUP, O.LUST), (1, 4), (0, 1),
                                                (O.SIMPLE, O.SIMPLEC)):
        case = O.VelCase(mesh=m, cc=_cell_centres(m), facevelr=m.face_r([1, 1, 2, 1, 3, 1]),
                         facepresr=m.face_r([0] * 6), lvel=lvel, prop=prop,
                         pres=rng.standard_normal(m.numel),
                         gradpres=rng.standard_normal((m.numel, 3)),
                         vel=rng.standard_normal((m.numel, 3)),
                         gradvel=rng.standard_normal((m.numel, 3, 3)),
                         dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=icod, fso=bool(fso),
                         type_simple=ts, under=0.7, adv=adv, adv_beta=0.25 + 0.1 * icod)
        for name, (st, un, ia, ja, _al, _au) in lay.items():
            r1 = O.vel_assemble(case, st, un, ia, ja, s.neq, fill=3.0)
            r2 = O.ref_vel_assemble(case, st, un, ia, ja, s.neq, fill=3.0)
            assert r1[0] == r2[0] == 0
            for x, y in zip(r1[1:], r2[1:6]):
                assert bits_equal(x, y), (adv, icod, fso, ts, name)
        # NVD with each of its functions (MUSCL and STOIC weigh 0, as in the reference),
    # TVD with each of its limiters
    st, un, ia_, ja_, _al, _au = lay["csrd_full"]
    for adv, fn in [(O.NVD, k) for k in range(1, 10)] + [(O.TVD, k) for k in range(1, 6)]:
        case = O.VelCase(mesh=m, cc=_cell_centres(m), facevelr=m.face_r([1, 1, 2, 1, 3, 1]),
                         facepresr=m.face_r([0] * 6), lvel=lvel, prop=prop,
                         pres=rng.standard_normal(m.numel),
                         gradpres=rng.standard_normal((m.numel, 3)),
                         vel=rng.standard_normal((m.numel, 3)),
                         gradvel=rng.standard_normal((m.numel, 3, 3)) * 0.3,
                         dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=4, under=0.7,
                         adv=adv, adv_fn=fn)
        for name in ("csrd_full", "csrc_unsym"):
            st, un, ia_, ja_, _al, _au = lay[name]
            r1 = O.vel_assemble(case, st, un, ia_, ja_, s.neq, fill=3.0)
            r2 = O.ref_vel_assemble(case, st, un, ia_, ja_, s.neq, fill=3.0)
            assert r1[0] == r2[0] == 0
            for x, y in zip(r1[1:], r2[1:6]):
                assert bits_equal(x, y), (adv, fn, name)
    # the schemes change b (the deferred correction), not the matrix
        f = O.vel_assemble(O.VelCase(**{**case.__dict__, "adv": O.FOUP}), O.CSRD, True,
                           s.ia, s.ja, s.neq)
        c = O.vel_assemble(case, O.CSRD, True, s.ia, s.ja, s.neq)
        assert bits_equal(f[1], c[1]) and not np.array_equal(f[3], c[3])


def test_vel_oracle_turbulence_matches_reference_live():
    """An eddy viscosity field (effective viscosity mu + nu_t, the walls' too)
    and the residual stress tensor's face integral (turbStructIntegral),
    without a wall model, against the reference's own systFormSimpleVel."""
    s = S.poisson_jittered(5, seed=8)
    m = s.mesh()
    rng = np.random.default_rng(9)
    lay = layouts(s)
    ia, ja, _ = s.csrc()
    lay["csrc_unsym"] = (O.CSRC, True, ia, ja, None, None)
    del lay["ellpack"]
    prop = np.zeros((2, O.MAXPROP))
    prop[:, 0] = (1e-3, 2e-3)
    prop[:, 1] = (1.0, 1.2)
    mat = rng.integers(1, 3, m.numel).astype(np.int16)
    lvel = [O.Load(O.STATICWALL, ()), O.Load(O.MOVEWALL, (1.0, 0.2, -0.1, 0.0)),
            O.Load(O.INLET, (0.5, 0.1, 0.0, 1.1))]
    eddy = rng.uniform(0.0, 5e-3, m.numel)
    stress = rng.standard_normal((m.numel, 6)) * 1e-2
    for (te, ts_), adv, fvisc in itertools.product(((True, False), (False, True), (True, True)),
                                                   (O.FOUP, O.SOUP), (0, 1)):
        case = O.VelCase(mesh=m, cc=_cell_centres(m), facevelr=m.face_r([1, 1, 2, 1, 3, 1]),
                         facepresr=m.face_r([0] * 6), lvel=lvel, prop=prop, mat=mat,
                         pres=rng.standard_normal(m.numel),
                         gradpres=rng.standard_normal((m.numel, 3)),
                         vel=rng.standard_normal((m.numel, 3)),
                         gradvel=rng.standard_normal((m.numel, 3, 3)),
                         dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=4, fvisc=bool(fvisc),
                         under=0.7, adv=adv, eddy=eddy if te else None,
                         stress=stress if ts_ else None)
        for name, (st, un, ia, ja, _al, _au) in lay.items():
            r1 = O.vel_assemble(case, st, un, ia, ja, s.neq, fill=3.0)
            r2 = O.ref_vel_assemble(case, st, un, ia, ja, s.neq, fill=3.0)
            assert r1[0] == r2[0] == 0
            for x, y in zip(r1[1:], r2[1:6]):
                assert bits_equal(x, y), (te, ts_, adv, fvisc, name)
    # the fields change the system
    lam = O.vel_assemble(O.VelCase(**{**case.__dict__, "eddy": None, "stress": None}),
                         O.CSRD, True, s.ia, s.ja, s.neq)
    tur = O.vel_assemble(case, O.CSRD, True, s.ia, s.ja, s.neq)
    assert not np.array_equal(lam[1], tur[1]) and not np.array_equal(lam[3], tur[3])


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference)")
def test_vel_oracle_outflow_loads_match_reference_live():
    """OUTLET (stress plus the null normal gradient, sP += m), OPEN (outflow
    as OUTLET without the stress, inflow along the cell's own velocity) and
    INLETTOTALPRES (pLoadSimple, Loads.c:436-672) against the reference's
    own systFormSimpleVel, on every layout, with the cell velocities of
    both signs on each side."""
    s = S.poisson_jittered(5, seed=10)
    m = s.mesh()
    rng = np.random.default_rng(11)
    lay = layouts(s)
    ia, ja, _ = s.csrc()
    lay["csrc_unsym"] = (O.CSRC, True, ia, ja, None, None)
    del lay["ellpack"]
    prop = np.zeros((2, O.MAXPROP))
    prop[:, 0] = (1e-3, 2e-3)
    prop[:, 1] = (1.0, 1.2)
    mat = rng.integers(1, 3, m.numel).astype(np.int16)
    lvel = [O.Load(O.STATICWALL, ()), O.Load(O.OUTLET, ()), O.Load(O.OPEN, (0.0,), density=1.1),
            O.Load(O.INLETTOTALPRES, (1.05, 2.0, 0.6, -0.5, 0.4))]
    for sides, icod, ts, adv in itertools.product(([1, 2, 3, 4, 1, 3], [4, 3, 2, 1, 2, 2]),
                                                  (1, 4), (O.SIMPLE, O.SIMPLEC),
                                                  (O.FOUP, O.SOUP)):
        case = O.VelCase(mesh=m, cc=_cell_centres(m), facevelr=m.face_r(sides),
                         facepresr=m.face_r([0] * 6), lvel=lvel, prop=prop, mat=mat,
                         pres=rng.standard_normal(m.numel),
                         gradpres=rng.standard_normal((m.numel, 3)),
                         vel=rng.standard_normal((m.numel, 3)),
                         gradvel=rng.standard_normal((m.numel, 3, 3)),
                         dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=icod, fvisc=True,
                         type_simple=ts, under=0.7, adv=adv)
        for name, (st, un, ia_, ja_, _al, _au) in lay.items():
            r1 = O.vel_assemble(case, st, un, ia_, ja_, s.neq, fill=3.0)
            r2 = O.ref_vel_assemble(case, st, un, ia_, ja_, s.neq, fill=3.0)
            assert r1[0] == r2[0] == 0
            for x, y in zip(r1[1:], r2[1:6]):
                assert bits_equal(x, y), (sides, icod, ts, adv, name)
    # the outflow loads change the diagonal (sP += m) and b against a wall
    wall = O.vel_assemble(O.VelCase(**{**case.__dict__, "lvel": [lvel[0]] * 4}), O.CSRD, True,
                          s.ia, s.ja, s.neq)
    out = O.vel_assemble(case, O.CSRD, True, s.ia, s.ja, s.neq)
    assert not np.array_equal(wall[2], out[2]) and not np.array_equal(wall[3], out[3])


def test_vel_oracle_inlet_static_pressure_direction():
    """INLETSTAICTPRES (Loads.c:364-392): the reference's getLoads copies no
    parameters for this type (Loads.c:148-150) and reads an uninitialised
    array, so no run of it pins the branch; the restatement takes the load's
    own par[0..2] as the inflow direction.  Checked here by its algebra: the
    force is -m (t . n)^-1 (v . n) t on each inflow face, t the direction."""
    s = S.poisson_uniform(4, seed=12)
    m = s.mesh()
    rng = np.random.default_rng(13)
    prop = np.zeros((1, O.MAXPROP))
    prop[0, :2] = (1e-3, 1.3)
    t = (0.7, -0.2, 0.3)
    base = dict(mesh=m, cc=_cell_centres(m), facevelr=m.face_r([1, 0, 0, 0, 0, 0]),
                facepresr=m.face_r([0] * 6), prop=prop, pres=np.zeros(m.numel),
                gradpres=np.zeros((m.numel, 3)), vel=rng.standard_normal((m.numel, 3)),
                gradvel=np.zeros((m.numel, 3, 3)), dfield=np.ones((m.numel, 3)), under=1.0)
    wall = O.vel_assemble(O.VelCase(**base, lvel=[O.Load(O.STATICWALL, ())]), O.CSRD, True,
                          s.ia, s.ja, s.neq)
    isp = O.vel_assemble(O.VelCase(**base, lvel=[O.Load(O.INLETSTAICTPRES, t + (1.0,))]),
                         O.CSRD, True, s.ia, s.ja, s.neq)
    none = O.vel_assemble(O.VelCase(**{**base, "facevelr": m.face_r([0] * 6)},
                                    lvel=[O.Load(O.STATICWALL, ())]), O.CSRD, True,
                          s.ia, s.ja, s.neq)
    assert wall[0] == isp[0] == none[0] == 0
    # the load touches b only: no diagonal share, as the reference's branch
    assert np.array_equal(isp[1], none[1]) and np.array_equal(isp[2], none[2])
    db = (isp[3] - none[3]).reshape(3, s.neq)
    for c in np.flatnonzero(m.nelcon[:, 0] == -1):
        face = m.cellface[c, 0] - 1
        ch = 1.0 if m.owner[face, 0] - 1 == c else -1.0  # the normal out of cell c
        nrm = ch * np.asarray(m.normal[face])
        row = m.id[c] - 1
        v = base["vel"][c]
        wfn = v @ nrm
        want = -1.3 * wfn * m.area[face] * (wfn / (np.asarray(t) @ nrm)) * np.asarray(t)
        np.testing.assert_allclose(db[:, row], want, rtol=1e-12, atol=1e-14)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference)")
def test_vel_oracle_wall_model_matches_reference_live():
    """The wall model's viscosity on MOVEWALL / STATICWALL faces
    (Turbulence.fWall, Loads.c:300-313): mu yPlus / uPlus where yPlus > 0.01,
    else mu, from a given per-cell (yPlus, uPlus, uFri, stressW) field, with
    and without an eddy viscosity, against the reference's own
    systFormSimpleVel on every layout."""
    s = S.poisson_jittered(5, seed=14)
    m = s.mesh()
    rng = np.random.default_rng(15)
    lay = layouts(s)
    ia, ja, _ = s.csrc()
    lay["csrc_unsym"] = (O.CSRC, True, ia, ja, None, None)
    del lay["ellpack"]
    prop = np.zeros((2, O.MAXPROP))
    prop[:, 0] = (1e-3, 2e-3)
    prop[:, 1] = (1.0, 1.2)
    mat = rng.integers(1, 3, m.numel).astype(np.int16)
    lvel = [O.Load(O.STATICWALL, ()), O.Load(O.MOVEWALL, (1.0, 0.2, -0.1, 0.0)),
            O.Load(O.OUTLET, ())]
    wall = np.stack([rng.uniform(0.0, 40.0, m.numel), rng.uniform(1.0, 20.0, m.numel),
                     rng.uniform(0.0, 1.0, m.numel), rng.uniform(0.0, 1.0, m.numel)], axis=1)
    wall[::3, 0] = rng.uniform(0.0, 0.01, len(wall[::3]))  # below the threshold: mu
    for eddy, adv in itertools.product((None, rng.uniform(0.0, 5e-3, m.numel)),
                                       (O.FOUP, O.SOUP)):
        case = O.VelCase(mesh=m, cc=_cell_centres(m), facevelr=m.face_r([1, 2, 1, 3, 1, 2]),
                         facepresr=m.face_r([0] * 6), lvel=lvel, prop=prop, mat=mat,
                         pres=rng.standard_normal(m.numel),
                         gradpres=rng.standard_normal((m.numel, 3)),
                         vel=rng.standard_normal((m.numel, 3)),
                         gradvel=rng.standard_normal((m.numel, 3, 3)),
                         dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=4, under=0.7, adv=adv,
                         eddy=eddy, wallpar=wall)
        for name, (st, un, ia_, ja_, _al, _au) in lay.items():
            r1 = O.vel_assemble(case, st, un, ia_, ja_, s.neq, fill=3.0)
            r2 = O.ref_vel_assemble(case, st, un, ia_, ja_, s.neq, fill=3.0)
            assert r1[0] == r2[0] == 0
            for x, y in zip(r1[1:], r2[1:6]):
                assert bits_equal(x, y), (eddy is None, adv, name)
    # the wall model changes the walls' diagonal share
    off = O.vel_assemble(O.VelCase(**{**case.__dict__, "wallpar": None}), O.CSRD, True, s.ia,
                         s.ja, s.neq)
    on = O.vel_assemble(case, O.CSRD, True, s.ia, s.ja, s.neq)
    assert not np.array_equal(off[2], on[2])


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference)")
def test_vel_oracle_rhie_chow_matches_reference_live():
    """Rhie-Chow face velocities in the momentum system (fRhieChowInt,
    interpolFaceVel, CellLib.c:6853-6960).  The reference's serial loop
    rewrites each cell's D as it goes, so a cell reads the new D of its
    lower-numbered neighbours and the old D of the others.  The oracle's
    serial mode (rhie 2) reads D the same way and matches the reference's
    systFormSimpleVel bit for bit on every cell and layout; the defined,
    order-independent variant the device runs (rhie 1: every D from the
    call's start) matches it wherever the two read the same D -- the first
    cell, which has no lower-numbered neighbour -- and differs elsewhere."""
    s = S.poisson_jittered(5, seed=16)
    m = s.mesh()
    rng = np.random.default_rng(17)
    lay = layouts(s)
    ia, ja, _ = s.csrc()
    lay["csrc_unsym"] = (O.CSRC, True, ia, ja, None, None)
    del lay["ellpack"]
    prop = np.zeros((1, O.MAXPROP))
    prop[0, :2] = (1e-3, 1.0)
    lvel = [O.Load(O.STATICWALL, ()), O.Load(O.MOVEWALL, (1.0, 0.2, -0.1, 0.0))]
    for adv, ts in itertools.product((O.FOUP, O.SOUP), (O.SIMPLE, O.SIMPLEC)):
        case = O.VelCase(mesh=m, cc=_cell_centres(m), facevelr=m.face_r([1, 1, 1, 1, 1, 2]),
                         facepresr=m.face_r([0] * 6), lvel=lvel, prop=prop,
                         pres=rng.standard_normal(m.numel) * 0.1,
                         gradpres=rng.standard_normal((m.numel, 3)) * 0.1,
                         vel=rng.standard_normal((m.numel, 3)),
                         gradvel=rng.standard_normal((m.numel, 3, 3)) * 0.1,
                         dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=4, under=0.7, adv=adv,
                         type_simple=ts, rhie=2)
        for name, (st, un, ia_, ja_, _al, _au) in lay.items():
            r1 = O.vel_assemble(case, st, un, ia_, ja_, s.neq, fill=3.0)
            r2 = O.ref_vel_assemble(case, st, un, ia_, ja_, s.neq, fill=3.0)
            assert r1[0] == r2[0] == 0
            for x, y in zip(r1[1:], r2[1:6]):
                assert bits_equal(x, y), (adv, ts, name)
        # the order-independent variant against the reference's serial result
        r1 = O.vel_assemble(O.VelCase(**{**case.__dict__, "rhie": 1}), O.CSRD, True, s.ia, s.ja,
                            s.neq)
        r2 = O.ref_vel_assemble(case, O.CSRD, True, s.ia, s.ja, s.neq)
        N, row0 = s.neq, m.id[0] - 1
        assert bits_equal(r1[1][s.ia[row0]:s.ia[row0 + 1]], r2[1][s.ia[row0]:s.ia[row0 + 1]])
        for k in range(3):
            assert r1[2][k * N + row0] == r2[2][k * N + row0]
            assert r1[3][k * N + row0] == r2[3][k * N + row0]
            assert r1[4][k * m.numel] == r2[4][k * m.numel]
        assert bits_equal(r1[5][0], r2[5][0])
        assert not bits_equal(r1[5], r2[5])  # the other cells read other D values


def test_vel_oracle_rejects_what_it_does_not_restate():
    s = S.poisson_uniform(4, seed=1)
    m = s.mesh()
    prop = np.zeros((1, O.MAXPROP))
    prop[0, :2] = (1e-3, 1.0)
    base = dict(mesh=m, cc=_cell_centres(m), facevelr=m.face_r([1, 0, 0, 0, 0, 0]),
                facepresr=m.face_r([0] * 6), prop=prop, pres=np.zeros(m.numel),
                gradpres=np.zeros((m.numel, 3)), vel=np.zeros((m.numel, 3)),
                gradvel=np.zeros((m.numel, 3, 3)), dfield=np.ones((m.numel, 3)))
    run = lambda **kw: O.vel_assemble(O.VelCase(**{**base, **kw}), O.CSRD, True,  # noqa: E731
                                      s.ia, s.ja, s.neq)[0]
    assert run(lvel=[O.Load(O.STATICWALL, ())]) == 0
    assert run(lvel=[O.Load(O.OUTLET, ())]) == 0
    assert run(lvel=[O.Load(O.INLET, (1.0, 0.0, 0.0, 1.0), var=1)]) == -2
    assert run(lvel=[O.Load(O.STATICWALL, ())], type_simple=3) == -1
    assert run(lvel=[O.Load(O.STATICWALL, ())], adv=4, adv_fn=6) == -1  # no such limiter
    assert run(lvel=[O.Load(O.STATICWALL, ())], adv=7) == -1  # no such scheme
    assert run(lvel=[O.Load(O.STATICWALL, ())], adv=5, adv_fn=10) == -1  # no such function
    assert O.vel_assemble(O.VelCase(**base, lvel=[O.Load(O.STATICWALL, ())]), O.ELLPACK, False,
                          O.ell_ia(s.neq, 6), s.ell()[0], s.neq)[0] == -1


# ---------------------------------------------------- gradient reconstruction
GRAD_SCALAR_LOADS = [O.Load(O.DIRICHLET, (0.3,)), O.Load(O.NEUMANN, (0.2,)),
                     O.Load(O.OUTLET, ()), O.Load(O.ROBIN, (2.0, 1.5)),
                     O.Load(O.FLUXPRES, ()), O.Load(O.FLUXPRESC, ())]
GRAD_VEL_LOADS = [O.Load(O.STATICWALL, ()), O.Load(O.MOVEWALL, (1.0, 0.2, -0.1, 0.0)),
                  O.Load(O.INLET, (0.5, 0.1, 0.0, 1.1)), O.Load(O.OUTLET, ()),
                  O.Load(O.OPEN, (0.0,), density=1.1), O.Load(O.DIRICHLET, (0.1, 0.2, 0.3))]


def _grad_cases(m, rng, typ, ndf):
    prop = np.zeros((2, O.MAXPROP))
    prop[:, 0] = (0.7, 1.3)
    prop[:, 1] = (1.0, 1.2)
    mat = rng.integers(1, 3, m.numel).astype(np.int16)
    if ndf == 1:
        loads = GRAD_SCALAR_LOADS
        tables = [[1, 2, 0, 3, 1, 0], [5, 6, 2, 0, 4, 1]]
        if typ == O.RCLSQUARE:
            tables.append([4, 3, 5, 6, 2, 1])
    else:
        loads = GRAD_VEL_LOADS
        tables = [[1, 2, 3, 4, 0, 1], [6, 5, 1, 1, 2, 0]]
    for sides in tables:
        u = rng.standard_normal(m.numel) if ndf == 1 else rng.standard_normal((m.numel, 3))
        yield sides, O.GradCase(mesh=m, facer=m.face_r(sides), loads=loads, prop=prop, u=u,
                                gradu=rng.standard_normal((m.numel, ndf, 3)), type=typ,
                                mat=mat)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference)")
@pytest.mark.parametrize("typ", [O.RCGRADGAUSSC, O.RCLSQUARE])
@pytest.mark.parametrize("ndf", [1, 3])
def test_rc_grad_oracle_matches_reference_live(typ, ndf):
    """rcGradU (Green-Gauss cell or least squares, no limiter) against the
    reference's own rcLeastSquare + rcGradU, bit for bit: the field's face
    loads of every kind each branch takes, faces without a load (the
    previous gradient, or the two-pass least squares), two materials; the
    least-squares matrices too, and the OpenMP cell loop gives the same
    gradient."""
    s = S.poisson_jittered(5, seed=30)
    m = s.mesh()
    rng = np.random.default_rng(31 + typ + ndf)
    for sides, case in _grad_cases(m, rng, typ, ndf):
        r1, g1 = O.rc_grad(case)
        r2, g2, lsq, _sec = O.ref_rc_grad(case)
        assert r1 == r2 == 0, sides
        assert bits_equal(g1, g2), (sides, np.abs(g1 - g2).max())
        if typ == O.RCLSQUARE:
            assert bits_equal(O.ls_matrix(case), lsq)
        r3, g3, _lsq, _sec = O.ref_rc_grad(case, nthreads=4)
        assert r3 == 0 and bits_equal(g1, g3)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built (needs the reference)")
def test_rc_grad_least_squares_staticwall_index_quirk():
    """leastSquare with ndf > 1 compares the load's index, not its type, with
    STATICWALL (CellLib.c:3118): a STATICWALL load elsewhere in the table
    contributes nothing, while whatever load sits at index 14 pins the face
    to zero.  The restatement keeps both, against the reference."""
    s = S.poisson_jittered(4, seed=32)
    m = s.mesh()
    rng = np.random.default_rng(33)
    prop = np.zeros((1, O.MAXPROP))
    prop[0, :2] = (0.7, 1.0)
    loads = [O.Load(O.OUTLET, ())] * 13 + [O.Load(O.OPEN, (0.0,), density=1.0),
                                           O.Load(O.STATICWALL, ())]
    for sides in ([14, 15, 1, 14, 15, 0], [15, 15, 15, 15, 15, 15]):
        case = O.GradCase(mesh=m, facer=m.face_r(sides), loads=loads, prop=prop,
                          u=rng.standard_normal((m.numel, 3)),
                          gradu=rng.standard_normal((m.numel, 3, 3)), type=O.RCLSQUARE)
        r1, g1 = O.rc_grad(case)
        r2, g2, _lsq, _sec = O.ref_rc_grad(case)
        assert r1 == r2 == 0 and bits_equal(g1, g2), sides


def test_rc_grad_oracle_rejects_what_the_reference_leaves_undefined():
    s = S.poisson_uniform(4, seed=34)
    m = s.mesh()
    prop = np.zeros((1, O.MAXPROP))
    prop[0, :2] = (0.7, 1.0)
    run = lambda loads, typ, ndf, p=prop: O.rc_grad(O.GradCase(  # noqa: E731
        mesh=m, facer=m.face_r([1, 0, 0, 0, 0, 0]), loads=loads, prop=p,
        u=np.zeros(m.numel) if ndf == 1 else np.zeros((m.numel, 3)),
        gradu=np.zeros((m.numel, ndf, 3)), type=typ))[0]
    assert run([O.Load(O.DIRICHLET, (1.0,))], O.RCGRADGAUSSC, 1) == 0
    assert run([O.Load(O.DIRICHLET, (1.0,), var=1)], O.RCLSQUARE, 1) == -2
    assert run([O.Load(O.SINBC, (1.0, 1.0, 0.0) * 3)], O.RCGRADGAUSSC, 1) == -2
    assert run([O.Load(O.STATICWALL, ())], O.RCGRADGAUSSC, 1) == -1  # no face value
    assert run([O.Load(O.ROBIN, (1.0, 1.0))], O.RCLSQUARE, 3) == -1  # the reference stops
    zero = prop.copy()
    zero[0, 0] = 0.0
    assert run([O.Load(O.NEUMANN, (1.0,))], O.RCGRADGAUSSC, 1, zero) == -1
    assert run([O.Load(O.NEUMANN, (1.0,))], O.RCLSQUARE, 1, zero) == 0  # du stays 0
    assert run([O.Load(O.STATICWALL, ())], O.RCLSQUARE + 1, 1) == -1  # QR: not restated
