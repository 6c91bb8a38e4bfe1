"""Device assembly of the diffusion system against the reference's
systFormDif: the committed fixture (made by the reference's own compiled
code) and the oracle restatement, bit for bit, then the assembled system
solved on the device."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

from oracle import oracle as O
from sfr3d_b200 import assembly as A
from sfr3d_b200 import solver as sv
from sfr3d_b200 import systems as S
from helpers import bits_equal, dif_case, dif_fixture, layouts, rel

pytestmark = pytest.mark.gpu

LOADS = [O.Load(O.DIRICHLET, (0.5,)), O.Load(O.NEUMANN, (0.25,)), O.Load(O.ROBIN, (2.0, 1.5)),
         O.Load(9, (1.0,)), O.Load(0, ()), O.Load(O.INLET, (1.0, 0.3, -0.2, 0.1, 1.2))]
SIDES = [1, 4, 2, 6, 3, 0]


def _loads(loads):
    return [A.Load(ld.type, tuple(ld.par), var=ld.var, np=ld.np) for ld in loads]


def _time(case):
    return (case.time_type, case.dt, case.dt0) if case.time_flag else None


def _device_assemble(gs, plan, case, flags, fill=0.0):
    """Assemble on the device with host arrays; read back (a, ad, b, rcell)
    in the reference's layout.  The values start from `fill` so that
    entries the reference leaves alone are compared too."""
    forces, matrix, calr = flags
    if matrix or not gs.values_version:
        n = gs._nsrc()
        split = gs.storage == sv.CSRC and gs.unsym
        gs.set_values(np.full(n // 2 if split else n, fill), np.full(gs.neq, fill),
                      np.full(n // 2, fill) if split else None)
    b, rcell = plan.assemble(_loads(case.loads), case.u0, case.cdiff, density=case.density,
                             gradu0=case.gradu0, fres=case.fres, time=_time(case),
                             forces=forces, matrix=matrix, calrcell=calr)
    al, ad, au = A.get_values(gs)
    a = al if au is None else np.concatenate([al, au])
    return a, ad, b, rcell


def test_fixture_replay(cuda):
    mesh, facer, fields, loads, lays, cases = dif_fixture()
    for lname, (st, un, ia, ja, neq) in lays.items():
        gs = sv.GpuSystem(neq, ia, ja, st, un)
        plans = {}
        for c in (c for c in cases if c["layout"] == lname):
            plan = plans.get(c["icod"])
            if plan is None:
                plan = plans[c["icod"]] = A.DifPlan(gs, mesh, facer, icod=c["icod"])
            case = dif_case(mesh, facer, fields, loads, c)
            flags = (c["forces"], c["matrix"], c["calrcell"])
            a, ad, b, rcell = _device_assemble(gs, plan, case, flags)
            if c["matrix"]:
                assert bits_equal(a, c["a"]), c["name"]
                assert bits_equal(ad, c["ad"]), c["name"]
            if c["forces"]:
                assert bits_equal(b, c["b"]), c["name"]
            if c["calrcell"]:
                assert bits_equal(rcell, c["rcell"]), c["name"]


@pytest.fixture(scope="module")
def box():
    s = S.poisson_jittered(7, seed=5)
    lay = layouts(s)
    ia, ja, _ = s.csrc()
    lay["csrc_unsym"] = (O.CSRC, True, ia, ja, None, None)
    return s, s.mesh(), lay


@pytest.mark.parametrize("icod", [1, 2, 3, 4])
def test_every_layout_and_option_matches_oracle(cuda, box, icod):
    s, m, lay = box
    rng = np.random.default_rng(icod)
    for name, (st, un, ia, ja, _al, _au) in lay.items():
        gs = sv.GpuSystem(s.neq, ia, ja, st, un)
        plan = A.DifPlan(gs, m, m.face_r(SIDES), icod=icod)
        for time, fres, flags in itertools.product((None, O.EULER, O.BACKWARD), (False, True),
                                                   ((1, 1, 1), (1, 0, 0), (0, 1, 1))):
            case = O.DifCase(mesh=m, facer=m.face_r(SIDES), loads=LOADS,
                             density=rng.uniform(0.5, 2, m.numel),
                             cdiff=m.cdiff * rng.uniform(0.5, 2, m.numel),
                             u0=rng.standard_normal(m.numel),
                             gradu0=rng.standard_normal((m.numel, 3)), icod=icod, fres=fres,
                             time_flag=time is not None, time_type=time or 0, dt=0.1, dt0=0.05)
            want = O.dif_assemble(case, st, un, ia, ja, s.neq, *flags, fill=3.0)
            assert want[0] == 0
            got = _device_assemble(gs, plan, case, flags, fill=3.0)
            forces, matrix, calr = flags
            if matrix:
                assert bits_equal(got[0], want[1]), (name, time, fres, flags)
                assert bits_equal(got[1], want[2]), (name, time, fres, flags)
            if forces:
                assert bits_equal(got[2], want[3]), (name, time, fres, flags)
            if calr:
                assert bits_equal(got[3], want[4]), (name, time, fres, flags)
        plan.close()
        gs.close()


@pytest.mark.parametrize("icod", [1, 4])
def test_64cubed_matches_oracle(cuda, icod):
    s = S.poisson_jittered(64, seed=6)
    m = s.mesh()
    rng = np.random.default_rng(7)
    case = O.DifCase(mesh=m, facer=m.face_r([1, 0, 2, 0, 0, 3]), loads=LOADS[:3],
                     density=np.ones(m.numel), cdiff=m.cdiff, u0=rng.standard_normal(m.numel),
                     gradu0=rng.standard_normal((m.numel, 3)), icod=icod, fres=True,
                     time_flag=True, time_type=O.EULER, dt=1e-2)
    want = O.dif_assemble(case, O.CSRD, True, s.ia, s.ja, s.neq)
    gs = sv.GpuSystem(s.neq, s.ia, s.ja, O.CSRD, True)
    plan = A.DifPlan(gs, m, case.facer, icod=icod)
    got = _device_assemble(gs, plan, case, (1, 1, 1))
    for g, w in zip(got, want[1:]):
        assert bits_equal(g, w)


def test_b0_and_update_cells(cuda, box):
    torch = cuda
    s, m, lay = box
    st, un, ia, ja, _al, _au = lay["csrd_full"]
    rng = np.random.default_rng(11)
    case = O.DifCase(mesh=m, facer=m.face_r(SIDES), loads=LOADS, density=np.ones(m.numel),
                     cdiff=m.cdiff, u0=rng.standard_normal(m.numel),
                     gradu0=rng.standard_normal((m.numel, 3)), icod=O.MINIMAL)
    want = O.dif_assemble(case, st, un, ia, ja, s.neq)
    b0 = rng.standard_normal(s.neq)
    gs = sv.GpuSystem(s.neq, ia, ja, st, un)
    plan = A.DifPlan(gs, m, case.facer, icod=O.MINIMAL)
    dev = lambda a: torch.tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    d_u0, d_k, d_g, d_b0 = dev(case.u0), dev(case.cdiff), dev(case.gradu0), dev(b0)
    d_b = torch.empty(s.neq, dtype=torch.float64, device="cuda")
    d_r = torch.empty(m.numel, dtype=torch.float64, device="cuda")
    plan.assemble_device(_loads(LOADS), d_u0.data_ptr(), d_k.data_ptr(),
                         d_gradu0=d_g.data_ptr(), d_b0=d_b0.data_ptr(), d_b=d_b.data_ptr(),
                         d_rcell=d_r.data_ptr())
    torch.cuda.synchronize()
    # addVector (b + b0) and updateCellValue (rCell + b0[id - 1]), Diffusion.c:107-118
    assert bits_equal(d_b.cpu().numpy(), want[3] + b0)
    assert bits_equal(d_r.cpu().numpy(), want[4] + b0[m.id - 1])
    x = rng.standard_normal(s.neq)
    d_x = dev(x)
    d_u = d_u0.clone()
    plan.update_cells(d_x.data_ptr(), d_u.data_ptr(), add=True)
    torch.cuda.synchronize()
    assert bits_equal(d_u.cpu().numpy(), case.u0 + x[m.id - 1])
    plan.update_cells(d_x.data_ptr(), d_u.data_ptr(), add=False)
    torch.cuda.synchronize()
    assert bits_equal(d_u.cpu().numpy(), x[m.id - 1])


def test_assembled_system_solves_like_reference(cuda, box):
    """Assemble on the device, solve on the device: the solution of the
    system the oracle assembles, solved by the oracle's PCG."""
    torch = cuda
    s, m, lay = box
    st, un, ia, ja, _al, _au = lay["csrc_sym"]
    rng = np.random.default_rng(12)
    case = O.DifCase(mesh=m, facer=m.face_r([1, 0, 2, 0, 0, 0]), loads=LOADS[:2],
                     density=np.ones(m.numel), cdiff=m.cdiff, u0=rng.standard_normal(m.numel),
                     gradu0=np.zeros((m.numel, 3)), icod=O.ORTHOGONAL)
    rc, a, ad, b, _ = O.dif_assemble(case, st, un, ia, ja, s.neq)
    ref = O.pcg(st, un, ia, ja, a, ad, b, tol=1e-10)
    gs = sv.GpuSystem(s.neq, ia, ja, st, un)
    plan = A.DifPlan(gs, m, case.facer, icod=O.ORTHOGONAL)
    dev = lambda v: torch.tensor(np.ascontiguousarray(v), device="cuda")  # noqa: E731
    d_u0, d_k = dev(case.u0), dev(case.cdiff)
    d_b = torch.empty(s.neq, dtype=torch.float64, device="cuda")
    d_x = torch.zeros(s.neq, dtype=torch.float64, device="cuda")
    plan.assemble_device(_loads(LOADS[:2]), d_u0.data_ptr(), d_k.data_ptr(),
                         d_b=d_b.data_ptr(), calrcell=False)
    info = gs.solve_device(sv.PCG, d_b.data_ptr(), d_x.data_ptr(), tol=1e-10)
    assert abs(info.iters - ref.iters) <= 1
    assert rel(d_x.cpu().numpy(), ref.x) < 1e-12
    # new coefficients reach every engine: the resident mixed path re-derives
    # its scaled operator from the new values
    case2 = O.DifCase(**{**case.__dict__, "cdiff": case.cdiff * 3.0})
    rc, a2, ad2, b2, _ = O.dif_assemble(case2, st, un, ia, ja, s.neq)
    ref2 = O.pcg(st, un, ia, ja, a2, ad2, b2, tol=1e-10)
    plan.assemble_device(_loads(LOADS[:2]), d_u0.data_ptr(), dev(case2.cdiff).data_ptr(),
                         d_b=d_b.data_ptr(), calrcell=False)
    d_x.zero_()
    info = gs.solve_device(sv.PCG, d_b.data_ptr(), d_x.data_ptr(), tol=1e-10,
                           precision=sv.MIXED)
    assert info.relres < 1e-10
    # the residual of the new system (assembled by the oracle) at the GPU's x
    x2 = d_x.cpu().numpy()
    r2 = b2 - O.matvec(st, un, ia, ja, a2, ad2, x2)
    assert np.linalg.norm(r2) / np.linalg.norm(b2) < 2e-10
    assert rel(x2, ref2.x) < 1e-6


def test_plan_and_call_validation(cuda, box):
    s, m, lay = box
    st, un, ia, ja, _al, _au = lay["csrd_full"]
    gs = sv.GpuSystem(s.neq, ia, ja, st, un)
    bad = S.FvMesh(**{**m.__dict__, "id": m.id.copy()})
    bad.id[3] = bad.id[4]
    with pytest.raises(sv.SolverError) as e:
        A.DifPlan(gs, bad, m.face_r(SIDES))
    assert e.value.status == sv.BAD_INPUT and "same equation" in sv.last_error()
    with pytest.raises(sv.SolverError) as e:
        A.DifPlan(gs, m, m.face_r(SIDES), caltype=np.array([3], np.int16))
    assert e.value.status == sv.BAD_INPUT
    plan = A.DifPlan(gs, m, m.face_r(SIDES))
    u0 = np.zeros(m.numel)
    with pytest.raises(sv.SolverError) as e:   # a face names load 6 of 2
        plan.assemble(_loads(LOADS[:2]), u0, m.cdiff)
    assert e.value.status == sv.BAD_INPUT
    with pytest.raises(sv.SolverError) as e:
        plan.assemble([A.Load(A.SINBC, (1.0,) * 9)] + _loads(LOADS[1:]), u0, m.cdiff)
    assert e.value.status == sv.UNSUPPORTED
    with pytest.raises(sv.SolverError) as e:
        plan.assemble([A.Load(A.DIRICHLET, (1.0,), var=1)] + _loads(LOADS[1:]), u0, m.cdiff)
    assert e.value.status == sv.UNSUPPORTED
    with pytest.raises(sv.SolverError) as e:
        plan.assemble([A.Load(A.OUTLET, ())] + _loads(LOADS[1:]), u0, m.cdiff)
    assert e.value.status == sv.BAD_INPUT
    # a load no face names is not checked, as in the reference
    assert 4 not in [v - 1 for v in SIDES if v]
    plan.assemble(_loads(LOADS[:4]) + [A.Load(A.OUTLET, ())] + _loads(LOADS[5:]), u0, m.cdiff)


def test_plan_outliving_its_system_leaves_no_error(cuda, box):
    """Garbage collection may free a system before its plan: destroying the
    plan then must not touch the system (a stale CUDA error would fail the
    next launch check of any handle)."""
    s, m, lay = box
    st, un, ia, ja, al, _au = lay["csrd_full"]
    gs = sv.GpuSystem(s.neq, ia, ja, st, un)
    plan = A.DifPlan(gs, m, m.face_r(SIDES))
    gs.close()
    plan.close()
    g2 = sv.GpuSystem(s.neq, ia, ja, st, un)
    g2.set_values(al, s.ad)
    x, info = g2.solve(sv.PCG, s.b[0], tol=1e-10)
    assert info.status == sv.OK


@pytest.mark.parametrize("name", ["csrd_full", "csrc_unsym", "ellpack", "csrd_sym"])
def test_solver_copy_matches_uploaded_values(cuda, box, name):
    """Where the assembly also writes the solver's SELL copy (full-row
    layouts), FP64 and mixed solves see exactly what an upload of the same
    values gives: bit-identical solutions."""
    s, m, lay = box
    st, un, ia, ja, _al, _au = lay[name]
    rng = np.random.default_rng(13)
    case = O.DifCase(mesh=m, facer=m.face_r([1, 0, 2, 0, 0, 0]), loads=LOADS[:2],
                     density=np.ones(m.numel), cdiff=m.cdiff, u0=rng.standard_normal(m.numel),
                     gradu0=np.zeros((m.numel, 3)), icod=O.ORTHOGONAL, time_flag=True, dt=0.05)
    ga = sv.GpuSystem(s.neq, ia, ja, st, un)
    plan = A.DifPlan(ga, m, case.facer, icod=O.ORTHOGONAL)
    b, _ = plan.assemble(_loads(LOADS[:2]), case.u0, case.cdiff, density=case.density,
                         time=(O.EULER, 0.05, 0.05), calrcell=False)
    al, ad, au = A.get_values(ga)
    gu = sv.GpuSystem(s.neq, ia, ja, st, un)
    gu.set_values(al, ad, au)
    solver = sv.PBICGSTAB if un else sv.PCG
    for prec in (sv.FP64, sv.MIXED):
        xa, ia_ = ga.solve(solver, b, tol=1e-10, precision=prec)
        xu, iu_ = gu.solve(solver, b, tol=1e-10, precision=prec)
        assert ia_.iters == iu_.iters and ia_.status == iu_.status == sv.OK
        assert bits_equal(xa, xu), (name, prec)
    plan.close()


# ------------------------------------------------ pressure correction --
from helpers import pres_fixture  # noqa: E402

PLVEL = [O.Load(O.MOVEWALL, (1.0, 0.0, 0.0, 0.0)), O.Load(O.INLET, (0.5, 0.1, -0.2, 1.1)),
         O.Load(O.OUTLET, ()), O.Load(O.OPEN, (0.0,), density=0.9),
         O.Load(O.INLETSTAICTPRES, (1.0, 0.0, 0.0, 1.0)),
         O.Load(O.INLETTOTALPRES, (1.2, 2.0, 1.0, 0.0, 0.0)), O.Load(O.STATICWALL, ())]
PLPRES = [O.Load(O.DIRICHLET, (0.0,)), O.Load(O.OPEN, (0.0,)),
          O.Load(O.INLETTOTALPRES, (1.2, 2.0, 1.0, 0.0, 0.0)), O.Load(O.FLUXPRES, ())]


def _aloads(loads):
    return [A.Load(ld.type, tuple(ld.par), var=ld.var, np=ld.np, density=ld.density)
            for ld in loads]


def _pres_device(gs, plan, case, flags, fill=0.0):
    forces, matrix, calr = flags
    if matrix or not gs.values_version:
        n = gs._nsrc()
        split = gs.storage == sv.CSRC and gs.unsym
        gs.set_values(np.full(n // 2 if split else n, fill), np.full(gs.neq, fill),
                      np.full(n // 2, fill) if split else None)
    b, rcell = plan.assemble(_aloads(case.lvel), _aloads(case.lpres), case.prop, case.pres,
                             case.gradpres, case.vel, case.dfield, forces=forces,
                             matrix=matrix, calrcell=calr)
    al, ad, au = A.get_values(gs)
    return (al if au is None else np.concatenate([al, au])), ad, b, rcell


def _pres_compare(got, want, flags, what):
    forces, matrix, calr = flags
    if matrix:
        assert bits_equal(got[0], want[1]), what
        assert bits_equal(got[1], want[2]), what
    if forces:
        assert bits_equal(got[2], want[3]), what
    if calr:
        assert bits_equal(got[3], want[4]), what


def test_pres_fixture_replay(cuda):
    mesh, sides, f, lvel, lpres, lays, cases = pres_fixture()
    for lname, (st, un, ia, ja, neq) in lays.items():
        gs = sv.GpuSystem(neq, ia, ja, st, un)
        for c in (c for c in cases if c["layout"] == lname):
            fv, fp = sides[c["sides"]]
            plan = A.PresPlan(gs, mesh, fp, fv, icod=c["icod"], mat=f["mat"],
                              nmat=len(f["prop"]))
            case = O.PresCase(mesh=mesh, facevelr=fv, facepresr=fp, lvel=lvel, lpres=lpres,
                              icod=c["icod"], **f)
            flags = (c["forces"], c["matrix"], c["calrcell"])
            got = _pres_device(gs, plan, case, flags)
            _pres_compare(got, (0, c["a"], c["ad"], c["b"], c["rcell"]), flags, c["name"])
            plan.close()
        gs.close()


@pytest.mark.parametrize("icod", [1, 4])
def test_pres_every_layout_matches_oracle(cuda, box, icod):
    s, m, lay = box
    rng = np.random.default_rng(20 + icod)
    prop = np.zeros((2, O.MAXPROP))
    prop[:, O.DENSITY] = (1.2, 0.9)
    mat = rng.integers(1, 3, m.numel).astype(np.int16)
    for name, (st, un, ia, ja, _al, _au) in lay.items():
        gs = sv.GpuSystem(s.neq, ia, ja, st, un)
        for vs, ps in (((1, 2, 3, 4, 5, 6), (1, 0, 2, 0, 3, 4)),
                       ((7, 3, 0, 4, 6, 2), (0, 0, 0, 0, 0, 1))):
            fv, fp = m.face_r(vs), m.face_r(ps)
            plan = A.PresPlan(gs, m, fp, fv, icod=icod, mat=mat, nmat=2)
            for flags in ((1, 1, 1), (1, 0, 0), (0, 1, 1)):
                case = O.PresCase(mesh=m, facevelr=fv, facepresr=fp, lvel=PLVEL, lpres=PLPRES,
                                  prop=prop, mat=mat, pres=rng.standard_normal(m.numel),
                                  gradpres=rng.standard_normal((m.numel, 3)),
                                  vel=rng.standard_normal((m.numel, 3)),
                                  dfield=rng.uniform(0.1, 1.0, (m.numel, 3)), icod=icod)
                want = O.pres_assemble(case, st, un, ia, ja, s.neq, *flags, fill=4.0)
                assert want[0] == 0
                got = _pres_device(gs, plan, case, flags, fill=4.0)
                _pres_compare(got, want, flags, (name, vs, flags))
            plan.close()
        gs.close()


def test_pres_64cubed_matches_oracle_and_solves(cuda):
    torch = cuda
    s = S.poisson_jittered(64, seed=9)
    m = s.mesh()
    rng = np.random.default_rng(21)
    prop = np.zeros((1, O.MAXPROP))
    prop[0, O.DENSITY] = 1.0
    fv = m.face_r([7, 7, 7, 7, 7, 1])       # static walls, a moving lid
    fp = m.face_r([1, 0, 0, 0, 0, 0])       # pressure fixed on x = 0
    lvel = [O.Load(O.MOVEWALL, (1.0, 0.0, 0.0, 0.0))] + [O.Load(O.STATICWALL, ())] * 6
    lpres = [O.Load(O.DIRICHLET, (0.0,))]
    case = O.PresCase(mesh=m, facevelr=fv, facepresr=fp, lvel=lvel, lpres=lpres, prop=prop,
                      pres=rng.standard_normal(m.numel),
                      gradpres=rng.standard_normal((m.numel, 3)),
                      vel=rng.standard_normal((m.numel, 3)),
                      dfield=rng.uniform(0.5, 1.0, (m.numel, 3)), icod=O.ORTHOGONAL)
    rc, a, ad, b, rcell = O.pres_assemble(case, O.CSRD, True, s.ia, s.ja, s.neq)
    assert rc == 0
    gs = sv.GpuSystem(s.neq, s.ia, s.ja, O.CSRD, True)
    plan = A.PresPlan(gs, m, fp, fv, icod=O.ORTHOGONAL)
    dev = lambda v: torch.tensor(np.ascontiguousarray(v), device="cuda")  # noqa: E731
    d = [dev(x) for x in (case.pres, case.gradpres, case.vel, case.dfield)]
    d_b = torch.empty(s.neq, dtype=torch.float64, device="cuda")
    d_r = torch.empty(m.numel, dtype=torch.float64, device="cuda")
    plan.assemble_device(_aloads(lvel), _aloads(lpres), prop, *[t.data_ptr() for t in d],
                         d_b=d_b.data_ptr(), d_rcell=d_r.data_ptr())
    torch.cuda.synchronize()
    assert bits_equal(d_b.cpu().numpy(), b) and bits_equal(d_r.cpu().numpy(), rcell)
    al, ad_g, _ = A.get_values(gs)
    assert bits_equal(al, a) and bits_equal(ad_g, ad)
    # the pressure correction solved where it was assembled
    ref = O.pcg(O.CSRD, True, s.ia, s.ja, a, ad, b, tol=1e-10)
    d_x = torch.zeros(s.neq, dtype=torch.float64, device="cuda")
    info = gs.solve_device(sv.PCG, d_b.data_ptr(), d_x.data_ptr(), tol=1e-10)
    assert abs(info.iters - ref.iters) <= 1
    assert rel(d_x.cpu().numpy(), ref.x) < 1e-12


def test_pres_validation(cuda, box):
    s, m, lay = box
    st, un, ia, ja, _al, _au = lay["csrd_full"]
    gs = sv.GpuSystem(s.neq, ia, ja, st, un)
    fv, fp = m.face_r([1, 2, 0, 0, 0, 0]), m.face_r([0, 0, 1, 0, 0, 0])
    with pytest.raises(sv.SolverError) as e:
        A.PresPlan(gs, m, fp, fv, icod=O.MINIMAL)
    assert e.value.status == sv.BAD_INPUT
    plan = A.PresPlan(gs, m, fp, fv)
    prop = np.zeros((1, O.MAXPROP))
    prop[0, O.DENSITY] = 1.0
    z1, z3 = np.zeros(m.numel), np.zeros((m.numel, 3))
    lp = [A.Load(A.DIRICHLET, (0.0,))]
    with pytest.raises(sv.SolverError) as e:   # velocity load 2 named, one given
        plan.assemble([A.Load(A.STATICWALL, ())], lp, prop, z1, z3, z3, z3)
    assert e.value.status == sv.BAD_INPUT
    with pytest.raises(sv.SolverError) as e:
        plan.assemble([A.Load(A.STATICWALL, ()), A.Load(A.INLET, (1.0, 0.0, 0.0), var=1)], lp,
                      prop, z1, z3, z3, z3)
    assert e.value.status == sv.UNSUPPORTED
    plan.assemble([A.Load(A.STATICWALL, ()), A.Load(A.INLET, (1.0, 0.0, 0.0))], lp, prop, z1,
                  z3, z3, z3)
    plan.close()
    gs.close()


def test_device_system_dumped_as_the_reference_writes_it(cuda, box, tmp_path):
    """The pcoo macro's dump (writeCoo) of a system assembled on the device:
    byte for byte the dump of the oracle's assembly."""
    s, m, lay = box
    rng = np.random.default_rng(15)
    for name in ("csrd_full", "csrd_sym"):
        st, un, ia, ja, _al, _au = lay[name]
        case = O.DifCase(mesh=m, facer=m.face_r(SIDES), loads=LOADS[:3] + LOADS[3:],
                         density=np.ones(m.numel), cdiff=m.cdiff,
                         u0=rng.standard_normal(m.numel), gradu0=np.zeros((m.numel, 3)))
        rc, a, ad, b, _ = O.dif_assemble(case, st, un, ia, ja, s.neq)
        gs = sv.GpuSystem(s.neq, ia, ja, st, un)
        plan = A.DifPlan(gs, m, case.facer)
        bd, _ = plan.assemble(_loads(case.loads), case.u0, case.cdiff, calrcell=False)
        gs.write_coo(tmp_path / "dev.mtx")
        sv.write_coo(tmp_path / "ref.mtx", ia, ja, ad, a, unsym=un)
        assert (tmp_path / "dev.mtx").read_bytes() == (tmp_path / "ref.mtx").read_bytes()
        sv.write_coo_b(tmp_path / "bd.mtx", bd)
        sv.write_coo_b(tmp_path / "br.mtx", b)
        assert (tmp_path / "bd.mtx").read_bytes() == (tmp_path / "br.mtx").read_bytes()
        plan.close()
        gs.close()


# ------------------------------------------------------------ momentum --
VLOADS = [O.Load(O.STATICWALL, ()), O.Load(O.MOVEWALL, (1.0, 0.2, -0.1, 0.0)),
          O.Load(O.INLET, (0.5, 0.1, 0.0, 1.1))]


def _centres(m):
    return m.xm[m.cellface[:, 0] - 1] - m.xmcc[:, 0, :]


@pytest.mark.parametrize("icod", [1, 4])
def test_vel_matches_oracle(cuda, box, icod):
    s, m, lay = box
    rng = np.random.default_rng(40 + icod)
    prop = np.zeros((2, O.MAXPROP))
    prop[:, 0] = (1e-3, 2e-3)
    prop[:, 1] = (1.0, 1.2)
    mat = rng.integers(1, 3, m.numel).astype(np.int16)
    cc = _centres(m)
    fv = m.face_r([1, 1, 2, 1, 3, 1])
    for name in ("csrd_full", "csrd_sym", "csrc_sym", "csrc_unsym"):
        st, un, ia, ja, _al, _au = lay[name]
        gs = sv.GpuSystem(s.neq, ia, ja, st, un)
        plan = A.VelPlan(gs, m, fv, cc, icod=icod, mat=mat, nmat=2)
        for fso, fvisc, fres, ts, time in itertools.product(
                (0, 1), (0, 1), (0, 1), (A.SIMPLE, A.SIMPLEC), (None, (O.EULER, 0.05, 0.04))):
            case = O.VelCase(mesh=m, cc=cc, facevelr=fv, facepresr=m.face_r([0] * 6),
                             lvel=VLOADS, prop=prop, mat=mat, pres=rng.standard_normal(m.numel),
                             gradpres=rng.standard_normal((m.numel, 3)),
                             vel=rng.standard_normal((m.numel, 3)),
                             gradvel=rng.standard_normal((m.numel, 3, 3)),
                             dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=icod,
                             fso=bool(fso), fvisc=bool(fvisc), fres=bool(fres), type_simple=ts,
                             time_flag=time is not None, time_type=time[0] if time else 0,
                             dt=time[1] if time else 1.0, dt0=time[2] if time else 1.0,
                             under=0.7)
            want = O.vel_assemble(case, st, un, ia, ja, s.neq, fill=0.0)
            assert want[0] == 0
            n = gs._nsrc()
            split = st == sv.CSRC and un
            gs.set_values(np.zeros(n // 2 if split else n), np.zeros(s.neq),
                          np.zeros(n // 2) if split else None)
            ad3, b3, rc3, df = plan.assemble(_aloads(VLOADS), prop, case.pres, case.gradpres,
                                             case.vel, case.gradvel, case.dfield, fso=fso,
                                             fvisc=fvisc, fres=fres, type_simple=ts, time=time,
                                             under=0.7)
            al, ad, au = A.get_values(gs)
            a = al if au is None else np.concatenate([al, au])
            what = (name, fso, fvisc, fres, ts, time)
            assert bits_equal(a, want[1]), what
            assert bits_equal(ad3, want[2]) and bits_equal(ad, want[2][:s.neq]), what
            assert bits_equal(b3, want[3]), what
            assert bits_equal(rc3, want[4]), what
            assert bits_equal(df, want[5]), what
        plan.close()
        gs.close()


@pytest.mark.parametrize("adv", [O.CD, O.SOUP, O.LUST, O.NVD, O.TVD])
def test_vel_advection_schemes_match_oracle(cuda, box, adv):
    s, m, lay = box
    rng = np.random.default_rng(60 + adv)
    prop = np.zeros((1, O.MAXPROP))
    prop[0, :2] = (1e-3, 1.0)
    cc = _centres(m)
    fv = m.face_r([1, 1, 2, 1, 3, 1])
    for name in ("csrd_full", "csrc_unsym"):
        st, un, ia, ja, _al, _au = lay[name]
        gs = sv.GpuSystem(s.neq, ia, ja, st, un)
        plan = A.VelPlan(gs, m, fv, cc, icod=4)
        for fso, ts in itertools.product((0, 1), (A.SIMPLE, A.SIMPLEC)):
            case = O.VelCase(mesh=m, cc=cc, facevelr=fv, facepresr=m.face_r([0] * 6),
                             lvel=VLOADS, prop=prop, pres=rng.standard_normal(m.numel),
                             gradpres=rng.standard_normal((m.numel, 3)),
                             vel=rng.standard_normal((m.numel, 3)),
                             gradvel=rng.standard_normal((m.numel, 3, 3)),
                             dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=4, fso=bool(fso),
                             type_simple=ts, under=0.7, adv=adv, adv_beta=0.3,
                             adv_fn=(3 + fso + 2 * (ts == A.SIMPLEC)) if adv != O.TVD
                             else 1 + fso + 2 * (ts == A.SIMPLEC))
            want = O.vel_assemble(case, st, un, ia, ja, s.neq, fill=0.0)
            assert want[0] == 0
            ad3, b3, rc3, df = plan.assemble(_aloads(VLOADS), prop, case.pres, case.gradpres,
                                             case.vel, case.gradvel, case.dfield, fso=fso,
                                             type_simple=ts, under=0.7, adv=adv, adv_beta=0.3,
                                             adv_fn=case.adv_fn)
            al, ad, au = A.get_values(gs)
            a = al if au is None else np.concatenate([al, au])
            what = (name, adv, fso, ts)
            assert bits_equal(a, want[1]), what
            assert bits_equal(ad3, want[2]) and bits_equal(b3, want[3]), what
            assert bits_equal(rc3, want[4]) and bits_equal(df, want[5]), what
        with pytest.raises(sv.SolverError):
            plan.assemble(_aloads(VLOADS), prop, case.pres, case.gradpres, case.vel,
                          case.gradvel, case.dfield, adv=7)
        plan.close()
        gs.close()


def test_vel_turbulence_matches_oracle(cuda, box):
    """Eddy viscosity and the residual stress integral: bound as host
    arrays or as device arrays, bit-identical to the oracle."""
    import torch
    s, m, lay = box
    rng = np.random.default_rng(70)
    prop = np.zeros((1, O.MAXPROP))
    prop[0, :2] = (1e-3, 1.0)
    cc = _centres(m)
    fv = m.face_r([1, 1, 2, 1, 3, 1])
    eddy = rng.uniform(0.0, 5e-3, m.numel)
    stress = rng.standard_normal((m.numel, 6)) * 1e-2
    d_eddy = torch.tensor(eddy, device="cuda")
    d_stress = torch.tensor(stress, device="cuda")
    for name in ("csrd_full", "csrd_sym"):
        st, un, ia, ja, _al, _au = lay[name]
        gs = sv.GpuSystem(s.neq, ia, ja, st, un)
        plan = A.VelPlan(gs, m, fv, cc, icod=4)
        with pytest.raises(sv.SolverError):  # nothing bound yet
            plan.assemble(_aloads(VLOADS), prop, np.zeros(m.numel), np.zeros((m.numel, 3)),
                          np.zeros((m.numel, 3)), np.zeros((m.numel, 3, 3)),
                          np.ones((m.numel, 3)), fturb=True)
        for on_device, (te, ts_) in itertools.product((False, True),
                                                      ((True, False), (True, True))):
            if on_device:
                plan.turbulence(d_eddy.data_ptr(), d_stress.data_ptr(), on_device=True)
            else:
                plan.turbulence(eddy, stress)
            case = O.VelCase(mesh=m, cc=cc, facevelr=fv, facepresr=m.face_r([0] * 6),
                             lvel=VLOADS, prop=prop, pres=rng.standard_normal(m.numel),
                             gradpres=rng.standard_normal((m.numel, 3)),
                             vel=rng.standard_normal((m.numel, 3)),
                             gradvel=rng.standard_normal((m.numel, 3, 3)),
                             dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=4, fvisc=True,
                             under=0.7, adv=O.SOUP, eddy=eddy if te else None,
                             stress=stress if ts_ else None)
            want = O.vel_assemble(case, st, un, ia, ja, s.neq, fill=0.0)
            assert want[0] == 0
            ad3, b3, rc3, df = plan.assemble(_aloads(VLOADS), prop, case.pres, case.gradpres,
                                             case.vel, case.gradvel, case.dfield, fvisc=True,
                                             under=0.7, adv=O.SOUP, fturb=te, fstruc=ts_)
            al, ad, au = A.get_values(gs)
            what = (name, on_device, te, ts_)
            assert bits_equal(al, want[1]), what
            assert bits_equal(ad3, want[2]) and bits_equal(b3, want[3]), what
            assert bits_equal(rc3, want[4]) and bits_equal(df, want[5]), what
        plan.close()
        gs.close()


def test_vel_wall_model_matches_oracle(cuda, box):
    """The wall model's viscosity on walls (fwall), with the parameters bound
    as a host array or a device array, with and without an eddy viscosity:
    bit-identical to the oracle (itself pinned to the reference)."""
    import torch
    s, m, lay = box
    rng = np.random.default_rng(72)
    prop = np.zeros((2, O.MAXPROP))
    prop[:, 0] = (1e-3, 2e-3)
    prop[:, 1] = (1.0, 1.2)
    mat = rng.integers(1, 3, m.numel).astype(np.int16)
    cc = _centres(m)
    fv = m.face_r([1, 2, 1, 3, 1, 2])
    lvel = [O.Load(O.STATICWALL, ()), O.Load(O.MOVEWALL, (1.0, 0.2, -0.1, 0.0)),
            O.Load(O.OUTLET, ())]
    wall = np.stack([rng.uniform(0.0, 40.0, m.numel), rng.uniform(1.0, 20.0, m.numel),
                     rng.uniform(0.0, 1.0, m.numel), rng.uniform(0.0, 1.0, m.numel)], axis=1)
    wall[::3, 0] = rng.uniform(0.0, 0.01, len(wall[::3]))
    eddy = rng.uniform(0.0, 5e-3, m.numel)
    d_wall = torch.tensor(wall, device="cuda")
    for name in ("csrd_full", "csrc_unsym"):
        st, un, ia, ja, _al, _au = lay[name]
        gs = sv.GpuSystem(s.neq, ia, ja, st, un)
        plan = A.VelPlan(gs, m, fv, cc, icod=4, mat=mat, nmat=2)
        with pytest.raises(sv.SolverError):  # nothing bound yet
            plan.assemble(_aloads(lvel), prop, np.zeros(m.numel), np.zeros((m.numel, 3)),
                          np.zeros((m.numel, 3)), np.zeros((m.numel, 3, 3)),
                          np.ones((m.numel, 3)), fwall=True)
        plan.turbulence(eddy)
        for on_device, te in itertools.product((False, True), (False, True)):
            if on_device:
                plan.wall(d_wall.data_ptr(), on_device=True)
            else:
                plan.wall(wall)
            case = O.VelCase(mesh=m, cc=cc, facevelr=fv, facepresr=m.face_r([0] * 6),
                             lvel=lvel, prop=prop, mat=mat, pres=rng.standard_normal(m.numel),
                             gradpres=rng.standard_normal((m.numel, 3)),
                             vel=rng.standard_normal((m.numel, 3)),
                             gradvel=rng.standard_normal((m.numel, 3, 3)),
                             dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=4, under=0.7,
                             eddy=eddy if te else None, wallpar=wall)
            want = O.vel_assemble(case, st, un, ia, ja, s.neq, fill=0.0)
            assert want[0] == 0
            n = gs._nsrc()
            split = st == sv.CSRC and un
            gs.set_values(np.zeros(n // 2 if split else n), np.zeros(s.neq),
                          np.zeros(n // 2) if split else None)
            ad3, b3, rc3, df = plan.assemble(_aloads(lvel), prop, case.pres, case.gradpres,
                                             case.vel, case.gradvel, case.dfield, under=0.7,
                                             fturb=te, fwall=True)
            al, ad, au = A.get_values(gs)
            a = al if au is None else np.concatenate([al, au])
            what = (name, on_device, te)
            assert bits_equal(a, want[1]), what
            assert bits_equal(ad3, want[2]) and bits_equal(b3, want[3]), what
            assert bits_equal(rc3, want[4]) and bits_equal(df, want[5]), what
        plan.close()
        gs.close()


@pytest.mark.parametrize("adv", [O.FOUP, O.SOUP, O.TVD])
def test_vel_rhie_chow_matches_oracle(cuda, box, adv):
    """Rhie-Chow face velocities (rhie 1: every cell reads the D field as it
    was at the call's start) on the device, bit for bit against the oracle's
    same form, on every CSR layout; the new D field comes out as before.
    The reference's serial order (rhie 2) is SFR_UNSUPPORTED on the device."""
    s, m, lay = box
    rng = np.random.default_rng(74 + adv)
    prop = np.zeros((1, O.MAXPROP))
    prop[0, :2] = (1e-3, 1.0)
    cc = _centres(m)
    fv = m.face_r([1, 1, 1, 1, 1, 2])
    lvel = [O.Load(O.STATICWALL, ()), O.Load(O.MOVEWALL, (1.0, 0.2, -0.1, 0.0))]
    for name in ("csrd_full", "csrd_sym", "csrc_sym", "csrc_unsym"):
        st, un, ia, ja, _al, _au = lay[name]
        gs = sv.GpuSystem(s.neq, ia, ja, st, un)
        plan = A.VelPlan(gs, m, fv, cc, icod=4)
        for ts in (A.SIMPLE, A.SIMPLEC):
            case = O.VelCase(mesh=m, cc=cc, facevelr=fv, facepresr=m.face_r([0] * 6), lvel=lvel,
                             prop=prop, pres=rng.standard_normal(m.numel) * 0.1,
                             gradpres=rng.standard_normal((m.numel, 3)) * 0.1,
                             vel=rng.standard_normal((m.numel, 3)),
                             gradvel=rng.standard_normal((m.numel, 3, 3)) * 0.1,
                             dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=4, under=0.7,
                             adv=adv, adv_fn=1, type_simple=ts, rhie=1)
            want = O.vel_assemble(case, st, un, ia, ja, s.neq, fill=0.0)
            assert want[0] == 0
            n = gs._nsrc()
            split = st == sv.CSRC and un
            gs.set_values(np.zeros(n // 2 if split else n), np.zeros(s.neq),
                          np.zeros(n // 2) if split else None)
            ad3, b3, rc3, df = plan.assemble(_aloads(lvel), prop, case.pres, case.gradpres,
                                             case.vel, case.gradvel, case.dfield, under=0.7,
                                             adv=adv, adv_fn=1, type_simple=ts, rhie=1)
            al, ad, au = A.get_values(gs)
            a = al if au is None else np.concatenate([al, au])
            what = (name, ts)
            assert bits_equal(a, want[1]), what
            assert bits_equal(ad3, want[2]) and bits_equal(b3, want[3]), what
            assert bits_equal(rc3, want[4]) and bits_equal(df, want[5]), what
        with pytest.raises(sv.SolverError) as e:
            plan.assemble(_aloads(lvel), prop, case.pres, case.gradpres, case.vel,
                          case.gradvel, case.dfield, rhie=2)
        assert e.value.status == sv.UNSUPPORTED
        plan.close()
        gs.close()


def test_vel_assembled_momentum_solves_like_reference(cuda):
    """A lid-driven cavity's momentum system assembled and solved (u, v, w
    with their own diagonals) on the device."""
    torch = cuda
    s = S.poisson_jittered(24, seed=9)
    m = s.mesh()
    rng = np.random.default_rng(41)
    prop = np.zeros((1, O.MAXPROP))
    prop[0, :2] = (1e-2, 1.0)
    fv = m.face_r([1, 1, 1, 1, 1, 2])   # static walls, the z-max lid moving
    lvel = [O.Load(O.STATICWALL, ()), O.Load(O.MOVEWALL, (1.0, 0.0, 0.0, 0.0))]
    case = O.VelCase(mesh=m, cc=_centres(m), facevelr=fv, facepresr=m.face_r([0] * 6), lvel=lvel,
                     prop=prop, pres=rng.standard_normal(m.numel) * 1e-2,
                     gradpres=rng.standard_normal((m.numel, 3)) * 1e-2,
                     vel=rng.standard_normal((m.numel, 3)) * 0.1,
                     gradvel=rng.standard_normal((m.numel, 3, 3)) * 0.1,
                     dfield=np.ones((m.numel, 3)), time_flag=True, dt=0.01, fres=False)
    rc, a, ad3, b3, _, _ = O.vel_assemble(case, O.CSRD, True, s.ia, s.ja, s.neq)
    refs = [O.pbicgstab(O.CSRD, True, s.ia, s.ja, a, ad3[k * s.neq:(k + 1) * s.neq],
                        b3[k * s.neq:(k + 1) * s.neq], tol=1e-10) for k in range(3)]
    gs = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    plan = A.VelPlan(gs, m, fv, case.cc)
    dev = lambda v: torch.tensor(np.ascontiguousarray(v), device="cuda")  # noqa: E731
    d = [dev(x) for x in (case.pres, case.gradpres, case.vel, case.gradvel, case.dfield)]
    d_ad3 = torch.empty(3 * s.neq, dtype=torch.float64, device="cuda")
    d_b3 = torch.empty(3 * s.neq, dtype=torch.float64, device="cuda")
    plan.assemble_device(_aloads(lvel), prop, *[t.data_ptr() for t in d], d_ad3=d_ad3.data_ptr(),
                         d_b3=d_b3.data_ptr(), fres=False, time=(O.EULER, 0.01, 0.01),
                         calrcell=False)
    torch.cuda.synchronize()
    assert bits_equal(d_ad3.cpu().numpy(), ad3) and bits_equal(d_b3.cpu().numpy(), b3)
    # the three solves where the systems were assembled
    d_x3 = torch.zeros(3 * s.neq, dtype=torch.float64, device="cuda")
    infos = gs.solve_multi_device(sv.PBICGSTAB, 3, d_b3.data_ptr(), d_x3.data_ptr(),
                                  d_ad_k=d_ad3.data_ptr(), tol=1e-10)
    xs = d_x3.cpu().numpy().reshape(3, -1)
    for k in range(3):
        assert infos[k].status == sv.OK
        assert abs(infos[k].iters - refs[k].iters) <= 1
        assert rel(xs[k], refs[k].x) < 1e-12
    plan.close()
    gs.close()


VOUT = [O.Load(O.STATICWALL, ()), O.Load(O.OUTLET, ()), O.Load(O.OPEN, (0.0,), density=1.1),
        O.Load(O.INLETTOTALPRES, (1.05, 2.0, 0.6, -0.5, 0.4)),
        O.Load(O.INLETSTAICTPRES, (0.7, -0.2, 0.3, 1.0))]


@pytest.mark.parametrize("sides", [[1, 2, 3, 4, 5, 3], [4, 3, 2, 5, 2, 2]])
def test_vel_outflow_loads_match_oracle(cuda, box, sides):
    """OUTLET, OPEN (outflow and inflow faces), INLETTOTALPRES and
    INLETSTAICTPRES on the device, bit for bit against the oracle (whose
    OUTLET, OPEN and INLETTOTALPRES match the reference's own assembly bit
    for bit), on every CSR layout, FoUp and SoUp advection."""
    s, m, lay = box
    rng = np.random.default_rng(44 + sides[0])
    prop = np.zeros((2, O.MAXPROP))
    prop[:, 0] = (1e-3, 2e-3)
    prop[:, 1] = (1.0, 1.2)
    mat = rng.integers(1, 3, m.numel).astype(np.int16)
    cc = _centres(m)
    fv = m.face_r(sides)
    for name in ("csrd_full", "csrd_sym", "csrc_sym", "csrc_unsym"):
        st, un, ia, ja, _al, _au = lay[name]
        gs = sv.GpuSystem(s.neq, ia, ja, st, un)
        plan = A.VelPlan(gs, m, fv, cc, icod=4, mat=mat, nmat=2)
        for adv, ts in itertools.product((O.FOUP, O.SOUP), (A.SIMPLE, A.SIMPLEC)):
            case = O.VelCase(mesh=m, cc=cc, facevelr=fv, facepresr=m.face_r([0] * 6),
                             lvel=VOUT, prop=prop, mat=mat, pres=rng.standard_normal(m.numel),
                             gradpres=rng.standard_normal((m.numel, 3)),
                             vel=rng.standard_normal((m.numel, 3)),
                             gradvel=rng.standard_normal((m.numel, 3, 3)),
                             dfield=rng.uniform(0.1, 1, (m.numel, 3)), icod=4, fso=True,
                             fvisc=True, type_simple=ts, under=0.7, adv=adv)
            want = O.vel_assemble(case, st, un, ia, ja, s.neq, fill=0.0)
            assert want[0] == 0
            n = gs._nsrc()
            split = st == sv.CSRC and un
            gs.set_values(np.zeros(n // 2 if split else n), np.zeros(s.neq),
                          np.zeros(n // 2) if split else None)
            ad3, b3, rc3, df = plan.assemble(_aloads(VOUT), prop, case.pres, case.gradpres,
                                             case.vel, case.gradvel, case.dfield, fso=1,
                                             fvisc=1, type_simple=ts, under=0.7, adv=adv)
            al, ad, au = A.get_values(gs)
            a = al if au is None else np.concatenate([al, au])
            what = (name, adv, ts)
            assert bits_equal(a, want[1]), what
            assert bits_equal(ad3, want[2]), what
            assert bits_equal(b3, want[3]), what
            assert bits_equal(rc3, want[4]), what
            assert bits_equal(df, want[5]), what
        plan.close()
        gs.close()


def test_vel_validation(cuda, box):
    s, m, lay = box
    st, un, ia, ja, _al, _au = lay["ellpack"]
    cc = _centres(m)
    ge = sv.GpuSystem(s.neq, ia, ja, st, un)
    with pytest.raises(sv.SolverError) as e:
        A.VelPlan(ge, m, m.face_r([1] * 6), cc)
    assert e.value.status == sv.BAD_INPUT
    st, un, ia, ja, _al, _au = lay["csrd_full"]
    gs = sv.GpuSystem(s.neq, ia, ja, st, un)
    plan = A.VelPlan(gs, m, m.face_r([1] * 6), cc)
    prop = np.zeros((1, O.MAXPROP))
    prop[0, :2] = (1e-3, 1.0)
    z1, z3, z9 = np.zeros(m.numel), np.zeros((m.numel, 3)), np.zeros((m.numel, 9))
    with pytest.raises(sv.SolverError) as e:
        plan.assemble([A.Load(A.INLET, (1.0, 0.0, 0.0, 1.0), var=1)], prop, z1, z3, z3, z9, z3)
    assert e.value.status == sv.UNSUPPORTED
    with pytest.raises(sv.SolverError) as e:
        plan.assemble([A.Load(A.STATICWALL, ())], prop, z1, z3, z3, z9, z3, type_simple=3)
    assert e.value.status == sv.BAD_INPUT
    plan.assemble([A.Load(A.STATICWALL, ())], prop, z1, z3, z3, z9, z3)
    plan.close()


# ---------------------------------------------------- gradient reconstruction
GSCALAR = [O.Load(O.DIRICHLET, (0.3,)), O.Load(O.NEUMANN, (0.2,)), O.Load(O.OUTLET, ()),
           O.Load(O.ROBIN, (2.0, 1.5)), O.Load(O.FLUXPRES, ()), O.Load(O.FLUXPRESC, ())]
GVEL = [O.Load(O.STATICWALL, ()), O.Load(O.MOVEWALL, (1.0, 0.2, -0.1, 0.0)),
        O.Load(O.INLET, (0.5, 0.1, 0.0, 1.1)), O.Load(O.OUTLET, ()),
        O.Load(O.OPEN, (0.0,), density=1.1), O.Load(O.DIRICHLET, (0.1, 0.2, 0.3))]


@pytest.mark.parametrize("typ", [O.RCGRADGAUSSC, O.RCLSQUARE])
@pytest.mark.parametrize("ndf", [1, 3])
def test_rc_grad_matches_oracle(cuda, box, typ, ndf):
    """rcGradU on the device, bit for bit against the oracle (itself pinned
    to the reference's rcGradU): every load kind each branch takes, faces
    without a load, two materials; host and device-array calls."""
    torch = cuda
    s, m, lay = box
    rng = np.random.default_rng(60 + typ + ndf)
    prop = np.zeros((2, O.MAXPROP))
    prop[:, 0] = (0.7, 1.3)
    prop[:, 1] = (1.0, 1.2)
    mat = rng.integers(1, 3, m.numel).astype(np.int16)
    loads = GSCALAR if ndf == 1 else GVEL
    tables = ([[1, 2, 0, 3, 1, 0], [5, 6, 2, 0, 4, 1]] if ndf == 1
              else [[1, 2, 3, 4, 0, 1], [6, 5, 1, 1, 2, 0]])
    for sides in tables:
        fr = m.face_r(sides)
        plan = A.GradPlan(m, fr, type=typ, mat=mat, nmat=2)
        for _ in range(2):
            u = rng.standard_normal(m.numel) if ndf == 1 else rng.standard_normal((m.numel, 3))
            g0 = rng.standard_normal((m.numel, ndf, 3))
            case = O.GradCase(mesh=m, facer=fr, loads=loads, prop=prop, u=u, gradu=g0, type=typ,
                              mat=mat)
            rc, want = O.rc_grad(case)
            assert rc == 0
            got = plan.grad(_aloads(loads), prop, u, g0)
            assert bits_equal(got, want), (sides, np.abs(got - want).max())
            du = torch.tensor(np.ascontiguousarray(u), device="cuda")
            dg = torch.tensor(g0, device="cuda")
            plan.grad_device(_aloads(loads), prop, ndf, du.data_ptr(), dg.data_ptr())
            torch.cuda.synchronize()
            assert bits_equal(dg.cpu().numpy(), want)
        plan.close()


def test_rc_grad_validation(cuda, box):
    s, m, lay = box
    prop = np.zeros((1, O.MAXPROP))
    prop[0, :2] = (0.7, 1.0)
    fr = m.face_r([1, 0, 0, 0, 0, 0])
    with pytest.raises(sv.SolverError) as e:
        A.GradPlan(m, fr, type=2)
    assert e.value.status == sv.UNSUPPORTED
    gg = A.GradPlan(m, fr, type=A.RCGRADGAUSSC)
    ls = A.GradPlan(m, fr, type=A.RCLSQUARE)
    u1, g1 = np.zeros(m.numel), np.zeros((m.numel, 1, 3))
    u3, g3 = np.zeros((m.numel, 3)), np.zeros((m.numel, 3, 3))
    with pytest.raises(sv.SolverError) as e:  # no face value under Green-Gauss
        gg.grad([A.Load(O.MOVEWALL, (1.0, 0.0, 0.0, 0.0))], prop, u1, g1)
    assert e.value.status == sv.BAD_INPUT
    with pytest.raises(sv.SolverError) as e:
        ls.grad([A.Load(O.ROBIN, (1.0, 1.0))], prop, u3, g3)  # the reference stops
    assert e.value.status == sv.BAD_INPUT
    with pytest.raises(sv.SolverError) as e:
        ls.grad([A.Load(O.DIRICHLET, (1.0,), var=1)], prop, u1, g1)
    assert e.value.status == sv.UNSUPPORTED
    with pytest.raises(sv.SolverError) as e:
        ls.grad([], prop, u1, g1)  # a face names load 1
    assert e.value.status == sv.BAD_INPUT
    zero = prop.copy()
    zero[0, 0] = 0.0
    with pytest.raises(sv.SolverError) as e:
        gg.grad([A.Load(O.NEUMANN, (1.0,))], zero, u1, g1)
    assert e.value.status == sv.BAD_INPUT
    ls.grad([A.Load(O.NEUMANN, (1.0,))], zero, u1, g1)  # leastSquare: du stays 0
    gg.close()
    ls.close()
