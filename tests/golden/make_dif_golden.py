"""Generate tests/golden/dif_assembly.npz from the reference's own compiled
systFormDif (oracle/_ref/libsfr3d_ref.so, built by `make -C oracle ref` from
the reference checkout).

The mesh is a seeded 5x4x3 box with jittered nodes (sfr3d_b200.systems), in
the reference's mesh arrays; the fields (u0, gradU0, diffusivity, density)
and loads are seeded too.  Each case stores the storage layout, the options
and what the reference wrote: the value array (al, al|au or the ELLPACK
slots), ad, b and rCell.  The inputs are stored with the outputs, so the
fixture does not depend on the generator staying the same.

    python tests/golden/make_dif_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from sfr3d_b200 import systems as S  # noqa: E402

MESH_FIELDS = ("nelcon", "nviz", "cellface", "owner", "volume", "dcca", "xmcc",
               "mksi", "ksi", "eta", "area", "normal", "xm", "mvskew", "vskew",
               "id")
LOADS = [O.Load(O.DIRICHLET, (0.5,)), O.Load(O.NEUMANN, (0.25,)),
         O.Load(O.ROBIN, (2.0, 1.5)), O.Load(O.INLET, (1.0, 0.3, -0.2, 0.1, 1.2))]
SIDES = (1, 4, 2, 0, 3, 0)   # load + 1 per box side x-, x+, y-, y+, z-, z+


def problem():
    sysx = S.build(S.params(n=(5, 4, 3), jitter=0.2, log10k=(-1.0, 1.0),
                            permute=True, seed=21))
    m = sysx.mesh()
    rng = np.random.default_rng(22)
    fields = dict(density=rng.uniform(0.5, 2.0, m.numel),
                  cdiff=m.cdiff.copy(), u0=rng.standard_normal(m.numel),
                  gradu0=rng.standard_normal((m.numel, 3)))
    ia, ja, _ = sysx.csrc()
    lay = {"csrd_full": (O.CSRD, True, sysx.ia, sysx.ja),
           "csrd_sym": (O.CSRD, False) + sysx.csrd_lower()[:2],
           "csrc_sym": (O.CSRC, False, ia, ja),
           "csrc_unsym": (O.CSRC, True, ia, ja),
           "ellpack": (O.ELLPACK, False, O.ell_ia(sysx.neq, sysx.width), sysx.ell()[0])}
    return sysx, m, fields, lay


def cases():
    """(name, layout, icod, fres, time(type, dt, dt0) or None, forces, matrix, calrcell)"""
    for lname in ("csrd_full", "csrd_sym", "csrc_sym", "csrc_unsym", "ellpack"):
        for icod in (O.ORTHOGONAL, O.MINIMAL, O.ORTHOGONALC, O.OVERRELAXED):
            yield (f"{lname}_i{icod}", lname, icod, True, None, True, True, True)
    yield ("csrd_full_euler", "csrd_full", O.OVERRELAXED, True, (O.EULER, 0.1, 0.1), True, True, True)
    yield ("csrd_full_backward", "csrd_full", O.MINIMAL, False, (O.BACKWARD, 0.1, 0.05),
           True, True, True)
    yield ("ellpack_forces_only", "ellpack", O.ORTHOGONAL, True, None, True, False, False)
    yield ("csrc_sym_matrix_only", "csrc_sym", O.ORTHOGONALC, False, None, False, True, True)


def main():
    sysx, m, fields, lay = problem()
    out = {f"mesh/{k}": np.asarray(getattr(m, k)) for k in MESH_FIELDS}
    out["mesh/facer"] = m.face_r(SIDES)
    for k, v in fields.items():
        out[f"field/{k}"] = v
    t, v, npar, par = O.DifCase(mesh=m, facer=None, loads=LOADS, density=None,
                                cdiff=None, u0=None, gradu0=None).load_arrays()
    out["loads/type"], out["loads/var"], out["loads/np"], out["loads/par"] = t, v, npar, par
    for lname, (st, un, ia, ja) in lay.items():
        out[f"layout/{lname}/meta"] = np.array([st, int(un), sysx.neq], np.int64)
        out[f"layout/{lname}/ia"] = np.asarray(ia, np.int32)
        out[f"layout/{lname}/ja"] = np.asarray(ja, np.int32)
    names = []
    for (name, lname, icod, fres, time, forces, matrix, calr) in cases():
        st, un, ia, ja = lay[lname]
        case = O.DifCase(mesh=m, facer=out["mesh/facer"], loads=LOADS, icod=icod,
                         fres=fres, time_flag=time is not None,
                         time_type=time[0] if time else 0,
                         dt=time[1] if time else 1.0, dt0=time[2] if time else 1.0,
                         **fields)
        rc, a, ad, b, rcell, _ = O.ref_dif_assemble(case, st, un, ia, ja, sysx.neq,
                                                    forces, matrix, calr, fill=0.0)
        assert rc == 0, (name, rc)
        names.append(name)
        out[f"{name}/meta"] = np.array([icod, int(fres), time is not None,
                                        time[0] if time else 0, forces, matrix, calr],
                                       np.int64)
        out[f"{name}/time"] = np.array([time[1], time[2]] if time else [1.0, 1.0])
        out[f"{name}/layout"] = np.array(lname)
        out[f"{name}/a"], out[f"{name}/ad"] = a, ad
        out[f"{name}/b"], out[f"{name}/rcell"] = b, rcell
        print(f"{name:28s} |b| {np.linalg.norm(b):.6e} |a| {np.linalg.norm(a):.6e}")
    out["cases"] = np.array(names)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dif_assembly.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
