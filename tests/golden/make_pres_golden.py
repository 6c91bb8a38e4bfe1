"""Generate tests/golden/pres_assembly.npz from the reference's own compiled
systFormSimplePres (oracle/_ref/libsfr3d_ref.so, built by `make -C oracle
ref` from the reference checkout).

Same seeded 5x4x3 jittered box as make_dif_golden.py, two materials, seeded
pressure, pressure gradient, velocity and momentum D fields, every velocity
and pressure load type the pressure equation reads.  Each case stores the
layout, the scheme and what the reference wrote (value array, ad, b, rCell);
the inputs are stored with the outputs.

    python tests/golden/make_pres_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from oracle import oracle as O  # noqa: E402
from make_dif_golden import MESH_FIELDS, problem  # noqa: E402

LVEL = [O.Load(O.MOVEWALL, (1.0, 0.0, 0.0, 0.0)), O.Load(O.INLET, (0.5, 0.1, -0.2, 1.1)),
        O.Load(O.OUTLET, ()), O.Load(O.OPEN, (0.0,), density=0.9),
        O.Load(O.INLETSTAICTPRES, (1.0, 0.0, 0.0, 1.0)),
        O.Load(O.INLETTOTALPRES, (1.2, 2.0, 1.0, 0.0, 0.0)), O.Load(O.STATICWALL, ())]
LPRES = [O.Load(O.DIRICHLET, (0.0,)), O.Load(O.OPEN, (0.0,)),
         O.Load(O.INLETTOTALPRES, (1.2, 2.0, 1.0, 0.0, 0.0)), O.Load(O.FLUXPRES, ())]
VSIDES = ((1, 2, 3, 4, 5, 6), (7, 3, 0, 4, 6, 2))   # velocity load + 1 per side
PSIDES = ((1, 0, 2, 0, 3, 4), (0, 0, 0, 0, 0, 1))   # pressure load + 1 per side


def fields(m):
    rng = np.random.default_rng(31)
    prop = np.zeros((2, O.MAXPROP))
    prop[0, O.DENSITY], prop[1, O.DENSITY] = 1.3, 0.7
    return dict(prop=prop, mat=rng.integers(1, 3, m.numel).astype(np.int16),
                pres=rng.standard_normal(m.numel), gradpres=rng.standard_normal((m.numel, 3)),
                vel=rng.standard_normal((m.numel, 3)),
                dfield=rng.uniform(0.1, 1.0, (m.numel, 3)))


def main():
    sysx, m, _, lay = problem()
    f = fields(m)
    out = {f"mesh/{k}": np.asarray(getattr(m, k)) for k in MESH_FIELDS}
    for k, v in f.items():
        out[f"field/{k}"] = v
    for tag, loads in (("lvel", LVEL), ("lpres", LPRES)):
        t, v, npar, par, dens = O._load_arrays(loads)
        out[f"{tag}/type"], out[f"{tag}/var"], out[f"{tag}/np"] = t, v, npar
        out[f"{tag}/par"], out[f"{tag}/density"] = par, dens
    for lname, (st, un, ia, ja) in lay.items():
        out[f"layout/{lname}/meta"] = np.array([st, int(un), sysx.neq], np.int64)
        out[f"layout/{lname}/ia"] = np.asarray(ia, np.int32)
        out[f"layout/{lname}/ja"] = np.asarray(ja, np.int32)
    names = []
    for k, (vs, ps) in enumerate(zip(VSIDES, PSIDES)):
        out[f"sides/{k}/facevelr"] = m.face_r(vs)
        out[f"sides/{k}/facepresr"] = m.face_r(ps)
    for lname, (st, un, ia, ja) in lay.items():
        for icod in (O.ORTHOGONAL, O.OVERRELAXED):
            for k in range(len(VSIDES)):
                flags = (1, 1, 1) if k == 0 else (1, 0, 1)
                case = O.PresCase(mesh=m, facevelr=out[f"sides/{k}/facevelr"],
                                  facepresr=out[f"sides/{k}/facepresr"], lvel=LVEL,
                                  lpres=LPRES, icod=icod, **f)
                rc, a, ad, b, rcell, _ = O.ref_pres_assemble(case, st, un, ia, ja, sysx.neq,
                                                             *flags, fill=0.0)
                assert rc == 0
                name = f"{lname}_i{icod}_s{k}"
                names.append(name)
                out[f"{name}/meta"] = np.array([icod, k, *flags], np.int64)
                out[f"{name}/layout"] = np.array(lname)
                out[f"{name}/a"], out[f"{name}/ad"] = a, ad
                out[f"{name}/b"], out[f"{name}/rcell"] = b, rcell
                print(f"{name:24s} |b| {np.linalg.norm(b):.6e} |ad| {np.linalg.norm(ad):.6e}")
    out["cases"] = np.array(names)
    path = os.path.join(HERE, "pres_assembly.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
