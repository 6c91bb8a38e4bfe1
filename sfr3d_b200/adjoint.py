"""Adjoint of the linear solve x = A^-1 b, and a torch.autograd harness.

For a scalar J(x) with g = dJ/dx the adjoint system is A^T lam = g; then
dJ/db = lam and dJ/dA_ij = -lam_i x_j for every (i, j) of the stored
pattern.  The GPU work (transpose solve on the transposed SELL copy, the
gradient scatter into the caller's value layout) is one C-ABI call,
``sfr_gpu_adjoint``; this module only adapts it to torch tensors.

The reference solves forward systems only (Solv.c:64-501, Bicgstab.c:57);
the transpose solve reuses its BiCGSTAB iteration on A^T.  A value that the
layout stores once for two mirrored entries (strict-lower storage of a
symmetric matrix, Csr.c:csrD / csrC with unsym = false) receives both terms,
-lam_i x_j - lam_j x_i.

``central_differences`` is the verification companion: FP64 central
differences of J = w.x with each perturbed system solved by defect
correction from the unperturbed solution, so the O(1) part of J cancels
exactly instead of in floating point.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .solver import (CSRC, CSRD, ELLPACK, FP64, PBICGSTAB, GpuSystem,
                     SolverError)

try:  # torch is the harness's only dependency beyond the C ABI
    import torch
except ImportError:  # pragma: no cover - torch ships with the image
    torch = None


def _np(t):
    if t is None:
        return None
    if torch is not None and isinstance(t, torch.Tensor):
        return t.detach().to("cpu", torch.float64).numpy()
    return np.asarray(t, dtype=np.float64)


if torch is not None:

    class LinearSolve(torch.autograd.Function):
        """x = A(al, ad, au)^-1 b on the pattern of a GpuSystem.

        ``apply(system, solver, opts, al, ad, au, b)``: al / ad / au are the
        value arrays of ``GpuSystem.set_values`` (au may be None), b the
        right-hand side; opts = (tol, maxit, precision) of the forward and
        the adjoint solve.  Forward and backward go through the C ABI;
        tensors are staged through host memory.
        """

        @staticmethod
        def forward(ctx, system, solver, opts, al, ad, au, b):
            tol, maxit, precision = opts
            system.set_values(_np(al), _np(ad), _np(au))
            x, info = system.solve(solver, _np(b), tol=tol, maxit=maxit,
                                   precision=precision)
            if info.status != 0:
                raise SolverError(info.status, "LinearSolve.forward")
            ctx.system, ctx.solver, ctx.opts = system, solver, opts
            ctx.values = (_np(al), _np(ad), _np(au))
            ctx.version = system.values_version
            ctx.has_au = au is not None
            ctx.x = x
            return torch.from_numpy(x).to(b.device)

        @staticmethod
        def backward(ctx, gx):
            system = ctx.system
            tol, maxit, precision = ctx.opts
            if system.values_version != ctx.version:
                system.set_values(*ctx.values)
                ctx.version = system.values_version
            lam, g_al, g_ad, g_au, info = system.adjoint(
                ctx.solver, ctx.x, _np(gx), tol=tol, maxit=maxit,
                precision=precision)
            if info.status != 0:
                raise SolverError(info.status, "LinearSolve.backward")
            dev = gx.device
            t = lambda a: None if a is None else torch.from_numpy(a).to(dev)
            return (None, None, None, t(g_al), t(g_ad),
                    t(g_au) if ctx.has_au else None, t(lam))

    def linear_solve(system: GpuSystem, al, ad, b, au=None,
                     solver: int = PBICGSTAB, tol: float = 1e-12,
                     maxit: int = 100000, precision: int = FP64):
        """Differentiable x = A^-1 b (see LinearSolve)."""
        return LinearSolve.apply(system, solver, (tol, maxit, precision),
                                 al, ad, au, b)


# ---------------------------------------------------------------------------
# Central differences of J = w.x
# ---------------------------------------------------------------------------
@dataclass
class Entry:
    """One coefficient of the stored layout: array ('al', 'ad', 'au', 'b'),
    index into it, and the matrix positions it occupies."""
    array: str
    index: int
    positions: list  # [(row, col)], two for a mirrored strict-lower value


def value_positions(system: GpuSystem, ia, ja, array: str, index: int) -> list:
    """Matrix positions (row, col) of stored value array[index]."""
    storage, unsym = system.storage, system.unsym
    ia = np.asarray(ia)
    if array == "ad":
        return [(index, index)]
    if array == "b":
        return []
    if storage == ELLPACK:
        width = int(ia[0])
        return [(index // width, int(ja[index]))]
    cnt = int(ia[system.neq] - ia[0])
    upper = array == "au"
    if storage == CSRC and unsym and array == "al" and index >= cnt:
        index, upper = index - cnt, True  # al given as [al | au]
    k = int(ia[0]) + index
    row = int(np.searchsorted(ia, k, side="right") - 1)
    col = int(ja[k])
    if storage == CSRD and unsym:  # every entry stored once
        return [(row, col)]
    if upper:  # CSRC unsym: au[k] is the mirrored upper entry
        return [(col, row)]
    if unsym:  # CSRC unsym al: lower entry only
        return [(row, col)]
    return [(row, col), (col, row)]


def central_differences(system: GpuSystem, solver: int, al, ad, au, b, x, w,
                        entries, rel_step: float = 1e-6, tol: float = 1e-12,
                        maxit: int = 100000):
    """dJ/dp for J = w.x by central differences, one value p per entry.

    Step h = rel_step * |p| (rel_step when p = 0).  With x the solution of
    A x = b, the solution of the perturbed system A' x' = b' is
    x' = x + d, A' d = (b' - b) - (A' - A) x.  The right-hand side is exact
    for a single changed coefficient ((A' - A) x = dh * x_j in row i for each
    position (i, j) of the value), so J(p + h) - J(p - h) = w.(d+ - d-)
    without forming the O(1) values of J.  Returns the derivative per entry;
    leaves the system holding the unperturbed values.
    """
    al, ad, au, b, x, w = (None if a is None else np.array(a, dtype=np.float64)
                           for a in (al, ad, au, b, x, w))
    arrays = {"al": al, "ad": ad, "au": au, "b": b}
    out = np.zeros(len(entries))
    changed = False
    for q, e in enumerate(entries):
        p = arrays[e.array][e.index]
        h = rel_step * abs(p) if p != 0.0 else rel_step
        jd = []
        for sgn in (1.0, -1.0):
            dh = sgn * h
            rhs = np.zeros(system.neq)
            if e.array == "b":
                if changed:
                    system.set_values(al, ad, au)
                    changed = False
                rhs[e.index] = dh
            else:
                for (i, j) in e.positions:
                    rhs[i] -= dh * x[j]
                pert = arrays[e.array].copy()
                pert[e.index] += dh
                vals = dict(arrays, **{e.array: pert})
                system.set_values(vals["al"], vals["ad"], vals["au"])
                changed = True
            d, info = system.solve(solver, rhs, tol=tol, maxit=maxit,
                                   raise_on_error=False)
            if info.status < 0:
                raise SolverError(info.status, "central_differences")
            jd.append(float(np.dot(w, d)))
        out[q] = (jd[0] - jd[1]) / (2.0 * h)
    if changed:
        system.set_values(al, ad, au)
    return out
