#!/usr/bin/env python
"""Benchmark: Krylov solve time to 1e-10 on the 128^3 pressure-correction
system (seeded jittered hex mesh, per-cell diffusivity 10^U(-2,2), harmonic
faces, random permutation + RCM), Jacobi-PCG in FP64 on one B200, with the
standalone SpMV's HBM roofline and the mixed-precision path beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

A step is one complete solve (x = 0 to relative M-norm residual 1e-10, the
reference's own stopping test, Cg.c:145) of the system resident in HBM.
Between timed steps L2 is flushed by writing a 256 MiB buffer (outside the
timed events).  Under torchrun (N > 1) every rank solves its own seeded
system of the same size (weak scaling, no collective on the data path);
times are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Krylov solve time to 1e-10 at 128^3; SpMV HBM GB/s %peak; mixed vs FP64 plain"
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=128, help="cells per axis")
    ap.add_argument("--maxit", type=int, default=100000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--profile", choices=["none", "spmv", "solve"], default="none",
                    help="short launch sequence for ncu (no JSON line)")
    ap.add_argument("--engine", type=int, default=0,
                    help="0 auto, 1 persistent, 2 graph, 3 graph kernels from a host "
                         "loop (profiling)")
    ap.add_argument("--spw", type=int, default=0, help="SELL slices per warp (0: default)")
    ap.add_argument("--mixed", action="store_true", help="--profile solve: mixed precision")
    return ap.parse_args(argv)


def peak_hbm():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def committed_traffic(kernel: str):
    """Per-unit DRAM traffic from a committed ncu summary: a line
    `bench-traffic <kernel> <bytes> <unit>` in profiles/*.md."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(pdir, fn)):
            m = re.match(r"\s*bench-traffic\s+(\S+)\s+([0-9.eE+]+)\s+(\S+)", line)
            if m and m.group(1) == kernel:
                return float(m.group(2)), m.group(3)
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200", "-f", self.path],
                stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 8:
                    rows.append(parts)
        finally:
            os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        smax = max(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4)
                          if r[4 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": reasons, "samples": len(rows)}


def spmv_alg_bytes(n, nnz_off):
    # CSRD FP64: values + indices of the off-diagonals, row pointers, diagonal,
    # x and y once each (the SpMV figure of the path's scope table)
    return 12 * nnz_off + 4 * (n + 1) + 24 * n


def pcg_alg_bytes(n, nnz_off, iters):
    # setup and post-processing: two SpMVs; each iteration one SpMV plus the
    # 88 N bytes of its vector updates
    return (iters + 2) * spmv_alg_bytes(n, nnz_off) + iters * 88 * n


# --------------------------------------------------------------- ours ----
def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from sfr3d_b200 import solver as sv
    from sfr3d_b200 import systems as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n = args.n
    s = S.poisson_jittered(n, seed=2 + rank)
    N, nnz = s.neq, s.nnz_full
    g = sv.GpuSystem(N, s.ia, s.ja, sv.CSRD, True, device=local)
    g.set_values(s.al, s.ad)
    g.set_engine(args.engine, 0, args.spw)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    b = torch.tensor(s.b[0], device="cuda")
    x = torch.zeros_like(b)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    if args.profile != "none":
        with torch.cuda.stream(stream):
            if args.profile == "spmv":
                y = torch.empty_like(b)
                for _ in range(args.warmup + args.steps):
                    g.spmv(b.data_ptr(), y.data_ptr(), sptr)
            else:
                for _ in range(args.warmup + args.steps):
                    g.solve_device(sv.PCG, b.data_ptr(), x.data_ptr(), tol=1e-10,
                                   maxit=args.maxit, stream=sptr,
                                   precision=sv.MIXED if args.mixed else sv.FP64)
        torch.cuda.synchronize()
        return None

    def timed_solves(precision, steps, warm):
        for _ in range(warm):
            g.solve_device(sv.PCG, b.data_ptr(), x.data_ptr(), tol=1e-10,
                           maxit=args.maxit, precision=precision, stream=sptr)
        barrier()
        times, infos = [], []
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        for i in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            info = g.solve_device(sv.PCG, b.data_ptr(), x.data_ptr(), tol=1e-10,
                                  maxit=args.maxit, precision=precision, stream=sptr)
            ev[i][1].record(stream)
            infos.append(info)
        barrier()
        times = [a.elapsed_time(c) for a, c in ev]
        return times, infos

    gpu_uuid = str(torch.cuda.get_device_properties(local).uuid)
    clocks = ClockSampler(gpu_uuid if gpu_uuid.startswith("GPU-") else f"GPU-{gpu_uuid}")
    clocks.start()
    t_wall0 = time.perf_counter()
    times, infos = timed_solves(sv.FP64, args.steps, args.warmup)
    t_wall = time.perf_counter() - t_wall0
    clk = clocks.stop()
    ms_step = max_over_ranks(statistics.mean(times))
    iters = infos[-1].iters
    status = infos[-1].status
    if status != sv.OK:
        raise RuntimeError(f"solve did not converge: {sv.status_string(status)}")

    # mixed precision beside it
    mixed = None
    if not args.no_mixed:
        try:
            mt, mi = timed_solves(sv.MIXED, max(2, args.steps // 2), 1)
            mixed = {"ms": max_over_ranks(statistics.mean(mt)),
                     "inner_iters": mi[-1].inner_iters,
                     "refinements": mi[-1].refinements,
                     "relres": mi[-1].relres, "status": mi[-1].status}
        except sv.SolverError as e:
            mixed = {"unavailable": str(e)}

    # standalone SpMV roofline (CUDA events on the launching stream)
    y = torch.empty_like(b)
    for _ in range(3):
        g.spmv(b.data_ptr(), y.data_ptr(), sptr)
    reps = 30
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        g.spmv(b.data_ptr(), y.data_ptr(), sptr)
    e1.record(stream)
    torch.cuda.synchronize()
    spmv_ms = e0.elapsed_time(e1) / reps
    peak, peak_kind = peak_hbm()
    sb = spmv_alg_bytes(N, nnz)
    spmv_gbs = sb / (spmv_ms * 1e-3) / 1e9

    # end to end through the reference-facing drop-in (sfr_solverC) with
    # pinned host buffers: al/ad/b uploaded and x read back every step
    e2e = None
    if not args.no_e2e:
        il, jl, al_l = s.csrd_lower()
        h_ia = torch.from_numpy(il).pin_memory()
        h_ja = torch.from_numpy(jl).pin_memory()
        h_al = torch.from_numpy(al_l).pin_memory()
        h_ad = torch.from_numpy(s.ad).pin_memory()
        h_b = torch.from_numpy(s.b[0]).pin_memory()
        h_x = torch.zeros(N, dtype=torch.float64).pin_memory()
        L = sv.lib()
        L.sfr_set_exit_on_failure(0)

        def call():
            return L.sfr_solverC(None, N, N, len(jl), 0, h_ia.data_ptr(), h_ja.data_ptr(),
                                 h_al.data_ptr(), h_ad.data_ptr(), None, h_b.data_ptr(),
                                 h_x.data_ptr(), None, None, 1e-10, args.maxit, sv.CSRD,
                                 sv.PCG, None, False, True, False, b"pressure")
        for _ in range(max(1, args.warmup // 2)):
            assert call() == sv.OK
        barrier()
        t0 = time.perf_counter()
        e2e_steps = max(2, args.steps // 2)
        for _ in range(e2e_steps):
            rc = call()
            if rc != sv.OK:
                raise RuntimeError(f"drop-in solve failed: {sv.status_string(rc)}")
        barrier()
        e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / e2e_steps)
        e2e = {"value": e2e_ms, "unit": "ms",
               "h2d_bytes_per_step": int(h_al.numel() * 8 + h_ad.numel() * 8 + h_b.numel() * 8),
               "d2h_bytes_per_step": int(h_x.numel() * 8),
               "api": "sfr_solverC (solverC drop-in), CSRD symmetric storage"}
        sv.release_cache()

    # CPU baseline: the reference's own pcgOmp on this host (rank 0, N = 1)
    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        cpu = cpu_baseline(s, iters)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return None

    alg = pcg_alg_bytes(N, nnz, iters)
    achieved = alg / (ms_step * 1e-3) / 1e9
    tr = committed_traffic("pcg_fp64_kernel")
    traffic = None
    if tr is not None:
        traffic = tr[0] * (iters if tr[1] == "per_iteration" else 1)
    line = {
        "metric": METRIC,
        "value": ms_step,
        "unit": "ms",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded jittered 128^3 hex mesh, generated on the host)",
        "config": {"workload": f"pressure-correction Poisson {n}^3 = {N} cells, jittered "
                               f"nodes +-20%, diffusivity 10^U(-2,2), harmonic faces, "
                               f"permuted + RCM; Jacobi-PCG FP64 to 1e-10 (M-norm)",
                   "rows": N, "nnz_offdiag": nnz, "iterations": iters,
                   "format": "SELL-32 (from CSRD)", "l2": "flushed between steps (256 MiB write)",
                   "parallelism": f"replicas{world}" if world > 1 else "single GPU"},
        "iterations": iters,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "kernel": "pcg_fp64_kernel (persistent, one launch per solve)",
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "alg_bytes_per_launch": alg},
        "spmv": {"kernel": "spmv_kernel", "ms": spmv_ms, "alg_bytes": sb, "GB/s": spmv_gbs,
                 "frac_of_peak": spmv_gbs / peak, "peak_source": f"{peak_kind} hbm_gbs"},
        "mixed": mixed,
        "fp64_plain_ms": ms_step,
        "mixed_speedup": (ms_step / mixed["ms"]) if mixed and "ms" in mixed else None,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": args.steps,
        "clocks": clk,
        "wall_s_timed_region": t_wall,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return line


def cpu_baseline(s, iters_full, sample_iters=None):
    """The reference's own pcgOmp (Cg.c:490) with all host threads on the
    same system in CSRC symmetric storage (the reference's default), run to a
    bounded iteration count and scaled to the full solve."""
    try:
        from oracle import oracle as O
    except Exception as e:  # pragma: no cover
        return {"unavailable": f"oracle not importable: {e}"}
    if not O.ref_available():
        return {"unavailable": "oracle/_ref/libsfr3d_ref.so not built"}
    threads = os.cpu_count() or 1
    il, jl, al = s.csrd_lower()
    if sample_iters is None:
        sample_iters = min(iters_full, 300)
    r = O.ref_solve(O.PCG, O.CSRC, False, il, jl, al, s.ad, s.b[0], tol=1e-10,
                    maxit=sample_iters, nthreads=threads)
    per_it = r.seconds / sample_iters if r.status != 0 else r.seconds / max(r.iters, 1)
    return {"value": per_it * iters_full * 1e3, "unit": "ms", "cores": threads,
            "kind": "reference",
            "sample": f"{sample_iters} pcgOmp iterations (CSRC symmetric, {threads} threads) "
                      f"of the same system, scaled to the full solve's {iters_full} iterations",
            "ms_per_iteration": per_it * 1e3}


# ---------------------------------------------------------- reference ----
def run_reference(args):
    """The reference's own CPU path (oracle/_ref: its compiled pcgOmp) on the
    same workload; rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return None
    try:
        from oracle import oracle as O
        if not O.ref_available():
            raise FileNotFoundError("oracle/_ref/libsfr3d_ref.so not built")
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": str(e)}))
        return None
    from sfr3d_b200 import systems as S
    s = S.poisson_jittered(args.n, seed=2)
    il, jl, al = s.csrd_lower()
    threads = os.cpu_count() or 1
    # first warm-up step: a full solve gives the iteration count and its time
    full = O.ref_solve(O.PCG, O.CSRC, False, il, jl, al, s.ad, s.b[0], tol=1e-10,
                       maxit=args.maxit, nthreads=threads)
    iters = full.iters
    sample = iters if full.seconds < 20 else max(50, int(iters * 20 / full.seconds))
    for _ in range(max(0, args.warmup - 1)):
        O.ref_solve(O.PCG, O.CSRC, False, il, jl, al, s.ad, s.b[0], tol=1e-10,
                    maxit=min(sample, 50), nthreads=threads)
    vals = []
    for _ in range(args.steps):
        r = O.ref_solve(O.PCG, O.CSRC, False, il, jl, al, s.ad, s.b[0], tol=1e-10,
                        maxit=sample if sample < iters else args.maxit, nthreads=threads)
        n_it = r.iters if r.status == 0 else sample
        vals.append(r.seconds / n_it * iters * 1e3)
    v = statistics.mean(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "ms",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": v,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"pressure-correction Poisson {args.n}^3, reference pcgOmp "
                                   f"(CSRC symmetric) to 1e-10", "iterations": iters},
            "cpu_baseline": {"value": v, "unit": "ms", "cores": threads, "kind": "reference",
                             "sample": ("full solves" if sample >= iters else
                                        f"{sample} of {iters} iterations per step, scaled")},
            "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return line


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
