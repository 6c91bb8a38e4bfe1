"""Generate tests/golden/cavity_systems.npz: real SIMPLE systems from the
reference's own lid-driven-cavity example (exemplos/lid_driven_cavity,
64,000 hexahedra, WALE LES, second-order upwind), harvested by running the
reference's own program with solverC wrapped (oracle/harvest.c, built by
`make -C oracle harvest`).

Kept: the pressure correction of the first SIMPLE iteration (PCG, CSRC
symmetric, 63,999 rows) and the momentum system of the second iteration's
first velocity solve (BiCGSTAB, CSRC unsym), each with the solution the
reference's own solver returned.

    python tests/golden/make_cavity_golden.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import zipfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# the reference checkout: $SFR3D_REFERENCE, else "reference" beside the repository
REF = os.environ.get("SFR3D_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")
if not os.path.isdir(os.path.join(REF, "src")):
    sys.exit(f"make_cavity_golden: no reference checkout at {REF} (set SFR3D_REFERENCE)")
WORK = os.path.join(ROOT, "oracle", "_ref", "cavity")


def read_system(path):
    b = open(path, "rb").read()
    hdr = np.frombuffer(b, np.int32, 7, 0)
    off = 28
    tol = float(np.frombuffer(b, np.float64, 1, off)[0])
    off += 8
    name = b[off:off + 32].split(b"\0")[0].decode()
    off += 32
    neq, nad = int(hdr[0]), int(hdr[1])
    out = {}
    for key, dt, n in (("ia", np.int32, neq + 1), ("ja", np.int32, nad),
                       ("al", np.float64, nad), ("au", np.float64, nad),
                       ("ad", np.float64, neq), ("b", np.float64, neq),
                       ("x0", np.float64, neq), ("x", np.float64, neq)):
        a = np.frombuffer(b, dt, n, off)
        off += a.nbytes
        out[key] = a.copy()
    assert off == len(b)
    out["meta"] = np.array([neq, nad, hdr[2], hdr[3], hdr[4], hdr[5], hdr[6]], np.int64)
    out["tol"] = np.array([tol])
    out["name"] = np.array(name)
    return out


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "harvest"], check=True)
    os.makedirs(WORK, exist_ok=True)
    zipfile.ZipFile(os.path.join(REF, "exemplos", "lid_driven_cavity.zip")).extractall(WORK)
    case = os.path.join(WORK, "lid_driven_cavity")
    env = dict(os.environ, SFR_HARVEST_CALLS="4", SFR_HARVEST_PREFIX=os.path.join(case, "sys"))
    subprocess.run([os.path.join(ROOT, "oracle", "_ref", "harvest"), "cavidadeQH2.dat", "out"],
                   cwd=case, env=env, check=True, stdin=subprocess.DEVNULL,
                   stdout=subprocess.DEVNULL)
    out = {}
    for tag, k in (("pressure", 2), ("momentum", 3)):
        s = read_system(os.path.join(case, f"sys{k}.bin"))
        if tag == "pressure":
            del s["au"]  # symmetric CSRC: al only
        for key, v in s.items():
            out[f"{tag}/{key}"] = v
        print(tag, s["meta"], s["name"], "|x|", np.linalg.norm(s["x"]))
    path = os.path.join(HERE, "cavity_systems.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    sys.exit(main())
