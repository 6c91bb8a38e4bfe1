"""The drop-in end to end: the reference's own program, built from its own
objects, run on a short copy of its lid-driven-cavity example (64,000
hexahedra; SIMPLE with Rhie-Chow, WALE LES, second-order upwind; two time
steps of three SIMPLE iterations) twice:

  * sfr3d_cpu -- the plain program: the reference's own CPU solvers;
  * sfr3d_gpu -- the same objects linked with -Wl,--wrap=solverC and the
    drop-in glue (oracle/sfr_gpu_glue.c), so every pressure PCG and momentum
    BiCGSTAB (Simple.c:2983,3003,3023,3136) runs through sfr_solverC on the
    GPU.

Checked: the solver logs have the same lines in the same order, every
solve's iteration count within +-1 and xKx and ||x|| within 1e-8
(relative); the SIMPLE residual history and the final cell pressure and
velocity fields agree to 1e-8 (relative 2-norm over the field).

Both programs and the deck are built where the reference checkout is
(`make -C oracle dropin`, run by the build entry point) into oracle/_ref/.
"""
from __future__ import annotations

import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
DECK = os.path.join(REF, "cavity_deck")
RTOL = 1e-8


def run_program(binary, where):
    os.makedirs(where)
    for name in os.listdir(DECK):
        src = os.path.join(DECK, name)
        if name == "mesh":
            os.symlink(src, os.path.join(where, name))
        elif os.path.isdir(src):
            shutil.copytree(src, os.path.join(where, name))
        else:
            shutil.copy(src, where)
    p = subprocess.run([os.path.join(REF, binary), "cavidadeQH2.dat", "out"], cwd=where,
                       stdin=subprocess.DEVNULL, stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, timeout=900)
    assert p.returncode == 0, p.stdout[-3000:].decode(errors="replace")
    return where


def solver_log(where, kind):
    rows = []
    for line in open(os.path.join(where, f"out_fluid_{kind}_n_1_solv_log.txt")):
        w = line.split()
        rows.append((w[0], int(w[w.index("iteration") + 1]), float(w[w.index("xKx") + 1]),
                     float(w[w.index("xKx") + 3])))
    return rows


def vtk_cell_fields(path):
    """ePres and eVel of the reference's ASCII VTK writer."""
    out, want, cur, n = {}, None, None, 0
    with open(path) as f:
        for line in f:
            if line.startswith("CELL_DATA"):
                n = int(line.split()[1])
            head = line.split()[:2]
            if head[:2] in (["SCALARS", "ePres"], ["VECTORS", "eVel"]):
                want, cur = head[1], []
                if head[0] == "SCALARS":
                    next(f)  # LOOKUP_TABLE
                continue
            if want is not None:
                cur.extend(float(v) for v in line.split())
                if len(cur) >= (n if want == "ePres" else 3 * n):
                    out[want] = np.array(cur)
                    want = None
    return out


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_reference_program_runs_on_the_gpu_path(cuda, tmp_path):
    for need in ("sfr3d_cpu", "sfr3d_gpu", os.path.join("cavity_deck", "cavidadeQH2.dat")):
        if not os.path.exists(os.path.join(REF, need)):
            pytest.fail(f"oracle/_ref/{need} missing: build with `make -C oracle dropin` "
                        "where the reference checkout is")
    cpu = run_program("sfr3d_cpu", str(tmp_path / "cpu"))
    gpu = run_program("sfr3d_gpu", str(tmp_path / "gpu"))
    for kind in ("pres", "vel"):
        a, b = solver_log(cpu, kind), solver_log(gpu, kind)
        assert len(a) == len(b) and len(a) > 0, (kind, len(a), len(b))
        for i, (ra, rb) in enumerate(zip(a, b)):
            assert ra[0] == rb[0], (kind, i, ra, rb)          # PCG: / PBICGSTAB:
            assert abs(ra[1] - rb[1]) <= 1, (kind, i, ra, rb)  # iterations
            assert abs(ra[2] - rb[2]) <= RTOL * abs(ra[2]) + 1e-300, (kind, i, ra, rb)
            assert abs(ra[3] - rb[3]) <= RTOL * abs(ra[3]), (kind, i, ra, rb)
    # SIMPLE's residual history (out_n_1_it_simple.txt)
    def history(where):
        vals = []
        for line in open(os.path.join(where, "out_n_1_it_simple.txt")):
            if not line.startswith("istep"):
                vals.append([float(v) for v in line.split()[1:]])
        return np.array(vals)
    ha, hb = history(cpu), history(gpu)
    assert ha.shape == hb.shape and ha.size > 0
    assert np.allclose(ha, hb, rtol=1e-6, atol=1e-14), np.abs(ha - hb).max()
    # the final fields
    steps = sorted(f for f in os.listdir(cpu) if f.startswith("out_3D_step_"))
    assert steps and steps == sorted(f for f in os.listdir(gpu) if f.startswith("out_3D_step_"))
    fa, fb = vtk_cell_fields(os.path.join(cpu, steps[-1])), \
        vtk_cell_fields(os.path.join(gpu, steps[-1]))
    for name in ("ePres", "eVel"):
        err = rel(fb[name], fa[name])
        print(f"{steps[-1]} {name}: relative difference {err:.2e}")
        assert err < RTOL, (name, err)
