"""Generate tests/golden/ref_solves.npz from the reference's own compiled
solver (oracle/_ref/libsfr3d_ref.so, built by `make -C oracle ref` from the
reference checkout).  Each case stores the inputs solverC received and what
the reference returned: x, the iteration count and the exit code, plus
xKx and ||x|| as its log line prints them (12 significant digits).

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from sfr3d_b200 import systems as S  # noqa: E402
sys.path.insert(0, os.path.join(ROOT, "tests"))
from helpers import layouts  # noqa: E402


def cases():
    uni = S.poisson_uniform(8, seed=11)
    jit = S.poisson_jittered(10, seed=12)
    mom = S.momentum(8, peclet=50.0, nrhs=2, seed=13)
    # nearly steady convection-diffusion (dt = 1e3): ~100 BiCGSTAB iterations
    steady = S.build(S.params(kind=S.SFR_SYS_CONVDIFF, n=8,
                              lengths=(np.pi,) * 3, dirichlet=S.ALL_FACES,
                              nrhs=1, rhs_normal=True, peclet=50.0, nu=1e-3,
                              dt=1e3, seed=14))
    for name, sysx, solver in (("uni8", uni, O.PCG), ("jit10", jit, O.PCG),
                               ("mom8", mom, O.PBICGSTAB),
                               ("steady8", steady, O.PBICGSTAB)):
        for lname, (st, un, ia, ja, al, au) in layouts(sysx).items():
            yield (f"{name}_{lname}", solver, st, un, ia, ja, al, sysx.ad,
                   sysx.b[0], None, 1e-10, 100000, True)
    # warm start, tol = 0 (machine epsilon), iteration cap
    st, un, ia, ja, al, _ = layouts(uni)["csrd_sym"]
    yield ("uni8_warm", O.PCG, st, un, ia, ja, al, uni.ad, uni.b[0],
           0.5 * np.ones(uni.neq), 1e-8, 100000, False)
    yield ("uni8_maxit", O.PCG, st, un, ia, ja, al, uni.ad, uni.b[0], None,
           1e-10, 5, True)
    yield ("mom8_maxit", O.PBICGSTAB, O.CSRD, True, mom.ia, mom.ja, mom.al,
           mom.ad, mom.b[1], None, 1e-14, 1, True)
    yield ("mom8_rhs1", O.PBICGSTAB, O.CSRD, True, mom.ia, mom.ja, mom.al,
           mom.ad, mom.b[1], None, 1e-10, 100000, True)
    # the other Krylov methods behind solverC: BiCGSTAB(2), GMRES(15)
    # (maxit counts restart cycles), MINRES (symmetric systems only)
    others = (("jit10", jit, (O.PBICGSTABL2, O.GMRES, O.MINRES)),
              ("mom8", mom, (O.PBICGSTABL2, O.GMRES)),
              ("steady8", steady, (O.PBICGSTABL2, O.GMRES)))
    tags = {O.PBICGSTABL2: "bicgl2", O.GMRES: "gmres", O.MINRES: "minres"}
    for name, sysx, solvers in others:
        for solver in solvers:
            for lname, (st, un, ia, ja, al, au) in layouts(sysx).items():
                yield (f"{name}_{tags[solver]}_{lname}", solver, st, un, ia, ja, al,
                       sysx.ad, sysx.b[0], None, 1e-10, 100000, True)
    st, un, ia, ja, al, _ = layouts(jit)["csrd_sym"]
    yield ("jit10_minres_warm", O.MINRES, st, un, ia, ja, al, jit.ad, jit.b[0],
           0.5 * np.ones(jit.neq), 1e-8, 100000, False)
    # iteration caps: GMRES and BiCGSTAB(2) exit with EXIT_FAILURE; MINRES
    # only warns and reports maxIt + 1 iterations
    yield ("jit10_gmres_maxit", O.GMRES, st, un, ia, ja, al, jit.ad, jit.b[0], None,
           1e-10, 2, True)
    yield ("jit10_minres_maxit", O.MINRES, st, un, ia, ja, al, jit.ad, jit.b[0], None,
           1e-10, 7, True)
    yield ("mom8_bicgl2_maxit", O.PBICGSTABL2, O.CSRD, True, mom.ia, mom.ja, mom.al,
           mom.ad, mom.b[1], None, 1e-14, 1, True)


def main():
    out = {}
    names = []
    for (name, solver, st, un, ia, ja, al, ad, b, x0, tol, maxit, newx) in cases():
        r = O.ref_solve(solver, st, un, ia, ja, al, ad, b, x0=x0, tol=tol,
                        maxit=maxit, newx=newx)
        names.append(name)
        out[f"{name}/meta"] = np.array([solver, st, int(un), maxit, int(newx)], np.int64)
        out[f"{name}/tol"] = np.array([tol])
        out[f"{name}/ia"] = np.asarray(ia, np.int32)
        out[f"{name}/ja"] = np.asarray(ja, np.int32)
        out[f"{name}/al"] = np.asarray(al, np.float64)
        out[f"{name}/ad"] = np.asarray(ad, np.float64)
        out[f"{name}/b"] = np.asarray(b, np.float64)
        out[f"{name}/x0"] = (np.zeros(len(ad)) if x0 is None else np.asarray(x0, np.float64))
        out[f"{name}/x"] = r.x
        out[f"{name}/res"] = np.array([r.iters, r.status], np.int64)
        out[f"{name}/log"] = np.array([r.xKx, r.norm_x])
        print(f"{name:24s} status {r.status:3d} iters {r.iters:5d}")
    out["cases"] = np.array(names)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_solves.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
