"""Helpers shared by the test modules."""
from __future__ import annotations

import numpy as np


def rel(a, b) -> float:
    """||a - b||_2 / ||b||_2."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def layouts(sys_):
    """The reference layouts of one generated system, keyed by name:
    (storage, unsym, ia, ja, al, au)."""
    from oracle import oracle as O
    out = {"csrd_full": (O.CSRD, True, sys_.ia, sys_.ja, sys_.al, None)}
    ej, ea = sys_.ell()
    out["ellpack"] = (O.ELLPACK, sys_.unsym, O.ell_ia(sys_.neq, sys_.width), ej, ea, None)
    ia, ja, a = sys_.csrc()
    if sys_.unsym:
        out["csrc_unsym"] = (O.CSRC, True, ia, ja, a, None)
    else:
        il, jl, alo = sys_.csrd_lower()
        out["csrd_sym"] = (O.CSRD, False, il, jl, alo, None)
        out["csrc_sym"] = (O.CSRC, False, ia, ja, a[: len(ja)], None)
    return out


def transpose_csrd(neq, ia, ja, al):
    """Explicit transpose of a full CSRD matrix (off-diagonals only, the
    diagonal is shared): rows of A^T with ascending column indices, the
    order a transposed CSRD built by sorting takes."""
    ia = np.asarray(ia, dtype=np.int64)
    ja = np.asarray(ja, dtype=np.int64)
    al = np.asarray(al, dtype=np.float64)
    base = int(ia[0])
    rows = np.repeat(np.arange(neq), np.diff(ia))
    cols = ja[base:base + len(rows)]
    order = np.lexsort((rows, cols))  # by new row (= col), then new col (= row)
    t_rows = cols[order]
    t_cols = rows[order]
    t_val = al[: len(rows)][order]
    t_ia = np.zeros(neq + 1, dtype=np.int32)
    np.add.at(t_ia, t_rows + 1, 1)
    t_ia = np.cumsum(t_ia).astype(np.int32)
    return t_ia, t_cols.astype(np.int32), t_val


class _Bag:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def dif_fixture():
    """tests/golden/dif_assembly.npz as (mesh, fields, loads, layouts, cases):
    mesh an object with the FvMesh attributes, fields a dict of the per-cell
    arrays, loads a list of oracle.Load, layouts {name: (storage, unsym, ia,
    ja, neq)}, cases a list of dicts (name, layout, icod, fres, time, forces,
    matrix, calrcell, a, ad, b, rcell)."""
    import os
    from oracle import oracle as O
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                        "dif_assembly.npz")
    z = np.load(path)
    mk = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith("mesh/")}
    facer = mk.pop("facer")
    numel = len(mk["nviz"])
    mesh = _Bag(numel=numel, nface=len(mk["mksi"]), **mk)
    fields = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith("field/")}
    loads = []
    for i in range(len(z["loads/type"])):
        loads.append(O.Load(int(z["loads/type"][i]), tuple(z["loads/par"][i][:int(z["loads/np"][i])]),
                            var=int(z["loads/var"][i]), np=int(z["loads/np"][i])))
    lays = {}
    for k in z.files:
        if k.startswith("layout/") and k.endswith("/meta"):
            name = k.split("/")[1]
            st, un, neq = (int(v) for v in z[k])
            lays[name] = (st, bool(un), z[f"layout/{name}/ia"], z[f"layout/{name}/ja"], neq)
    cases = []
    for name in z["cases"]:
        name = str(name)
        icod, fres, tf, tt, forces, matrix, calr = (int(v) for v in z[f"{name}/meta"])
        dt, dt0 = (float(v) for v in z[f"{name}/time"])
        cases.append(dict(name=name, layout=str(z[f"{name}/layout"]), icod=icod,
                          fres=bool(fres), time=(tt, dt, dt0) if tf else None,
                          forces=bool(forces), matrix=bool(matrix), calrcell=bool(calr),
                          a=z[f"{name}/a"], ad=z[f"{name}/ad"], b=z[f"{name}/b"],
                          rcell=z[f"{name}/rcell"]))
    return mesh, facer, fields, loads, lays, cases


def dif_case(mesh, facer, fields, loads, c):
    """An oracle.DifCase for one fixture case dict (or any dict with icod,
    fres and time)."""
    from oracle import oracle as O
    t = c["time"]
    return O.DifCase(mesh=mesh, facer=facer, loads=loads, icod=c["icod"], fres=c["fres"],
                     time_flag=t is not None, time_type=t[0] if t else 0,
                     dt=t[1] if t else 1.0, dt0=t[2] if t else 1.0, **fields)


def bits_equal(a, b) -> bool:
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


def pres_fixture():
    """tests/golden/pres_assembly.npz as (mesh, sides, fields, lvel, lpres,
    layouts, cases); sides[k] = (facevelr, facepresr); cases are dicts
    (name, layout, icod, sides, forces, matrix, calrcell, a, ad, b, rcell)."""
    import os
    from oracle import oracle as O
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                        "pres_assembly.npz")
    z = np.load(path)
    mk = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith("mesh/")}
    mesh = _Bag(numel=len(mk["nviz"]), nface=len(mk["mksi"]), **mk)
    fields = {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith("field/")}
    tables = {}
    for tag in ("lvel", "lpres"):
        loads = []
        for i in range(len(z[f"{tag}/type"])):
            npar = int(z[f"{tag}/np"][i])
            loads.append(O.Load(int(z[f"{tag}/type"][i]), tuple(z[f"{tag}/par"][i][:npar]),
                                var=int(z[f"{tag}/var"][i]), np=npar,
                                density=float(z[f"{tag}/density"][i])))
        tables[tag] = loads
    sides = {}
    k = 0
    while f"sides/{k}/facevelr" in z.files:
        sides[k] = (z[f"sides/{k}/facevelr"], z[f"sides/{k}/facepresr"])
        k += 1
    lays = {}
    for key in z.files:
        if key.startswith("layout/") and key.endswith("/meta"):
            name = key.split("/")[1]
            st, un, neq = (int(v) for v in z[key])
            lays[name] = (st, bool(un), z[f"layout/{name}/ia"], z[f"layout/{name}/ja"], neq)
    cases = []
    for name in z["cases"]:
        name = str(name)
        icod, k, forces, matrix, calr = (int(v) for v in z[f"{name}/meta"])
        cases.append(dict(name=name, layout=str(z[f"{name}/layout"]), icod=icod, sides=k,
                          forces=bool(forces), matrix=bool(matrix), calrcell=bool(calr),
                          a=z[f"{name}/a"], ad=z[f"{name}/ad"], b=z[f"{name}/b"],
                          rcell=z[f"{name}/rcell"]))
    return mesh, sides, fields, tables["lvel"], tables["lpres"], lays, cases


def cavity_systems():
    """tests/golden/cavity_systems.npz: {tag: dict(storage, unsym, solver, ia,
    ja, a, al, au, ad, b, x, tol, maxit, neq)} for the harvested pressure and
    momentum systems of the reference's lid-driven cavity; `a` is what the
    oracle takes (al, or al then au for unsym CSRC) and x the reference's own
    solution."""
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                        "cavity_systems.npz")
    z = np.load(path)
    out = {}
    for tag in ("pressure", "momentum"):
        neq, nad, st, solver, unsym, newx, maxit = (int(v) for v in z[f"{tag}/meta"])
        al = z[f"{tag}/al"]
        au = z[f"{tag}/au"] if unsym else None
        out[tag] = dict(storage=st, unsym=bool(unsym), solver=solver, ia=z[f"{tag}/ia"],
                        ja=z[f"{tag}/ja"], al=al, au=au,
                        a=np.concatenate([al, au]) if unsym else al, ad=z[f"{tag}/ad"],
                        b=z[f"{tag}/b"], x=z[f"{tag}/x"], tol=float(z[f"{tag}/tol"][0]),
                        maxit=maxit, neq=neq)
    return out
