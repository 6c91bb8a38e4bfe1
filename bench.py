#!/usr/bin/env python
"""Benchmark: Krylov solve time to 1e-10 on the 128^3 pressure-correction
system (seeded jittered hex mesh, per-cell diffusivity 10^U(-2,2), harmonic
faces, random permutation + RCM), Jacobi-PCG in FP64 on one B200, with the
SpMV's HBM roofline and the mixed-precision path beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

A step is one complete solve (x = 0 to relative M-norm residual 1e-10, the
reference's own stopping test, Cg.c:145) of the system resident in HBM: one
CUDA-graph launch.  Between timed steps L2 is flushed by writing a 256 MiB
buffer (outside the timed events).  Under torchrun (N > 1) every rank solves
its own seeded system of the same size (weak scaling, no collective on the
data path), and the 64 uneven systems are split across the ranks by
estimated work; times are the max over ranks.

Beside the headline (N = 1 only): the mixed-precision solve of the same
system and its error against the FP64 solution; the 128^3 momentum system
(Peclet 50, three right-hand sides) solved one right-hand side at a time in
FP64 and as one K = 3 mixed launch; 64 uneven Poisson systems in one batched
launch; the adjoint of the 96^3 Peclet-20 momentum system with its
central-difference check; the end-to-end drop-in call (host buffers); and
the reference's own OpenMP solver on this host.
"""
from __future__ import annotations

import argparse
import json
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
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the momentum, batched and adjoint legs")
    ap.add_argument("--profile", choices=["none", "spmv", "solve", "bicgstab", "assembly",
                                          "pressure", "momentum", "partitioned", "gradient"],
                    default="none",
                    help="short launch sequence for ncu (no JSON line)")
    ap.add_argument("--engine", type=int, default=0,
                    help="0 auto, 1 persistent, 2 graph, 3 graph kernels from a host "
                         "loop (profiling), 4 resident (mixed PCG)")
    ap.add_argument("--threads", type=int, default=0, help="graph-engine block size (0: default)")
    ap.add_argument("--spw", type=int, default=0, help="SELL slices per warp (0: default)")
    ap.add_argument("--fused", type=int, default=4,
                    help="graph engine FP64 PCG: 0 three kernels an iteration, 1-3 one "
                         "cooperative kernel an iteration, 4 (the library's default) the whole "
                         "solve in one cooperative launch")
    ap.add_argument("--pf", type=int, default=0,
                    help="graph engine SpMV-phase L2 prefetch distance in rounds (0: off)")
    ap.add_argument("--mixed", action="store_true", help="--profile solve: mixed precision")
    ap.add_argument("--nrhs", type=int, default=1,
                    help="--profile bicgstab: right-hand sides sharing the momentum matrix")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the autotuner (untimed) before the timed solves")
    ap.add_argument("--partitioned", action="store_true",
                    help="the row-partitioned solve over the ranks (the default under "
                         "torchrun with N > 1; with N = 1 it runs an NCCL group of one rank)")
    ap.add_argument("--replicas", action="store_true",
                    help="N > 1: independent replicas instead of the partitioned solve")
    ap.add_argument("--weak-n", type=int, default=96,
                    help="partitioned weak-scaling case: n x n x (n * N) cells")
    return ap.parse_args(argv)


def peak_hbm():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def committed_traffic(name: str):
    """DRAM traffic from a committed ncu summary: a line
    `bench-traffic <name> <bytes> <unit>` in profiles/*.md."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(pdir, fn)):
            m = re.match(r"\s*bench-traffic\s+(\S+)\s+([0-9.eE+]+)\s+(\S+)", line)
            if m and m.group(1) == name:
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
    # x and y once each
    return 12 * nnz_off + 4 * (n + 1) + 24 * n


def pcg_alg_bytes(n, nnz_off, iters):
    # setup and post-processing: two SpMVs; each iteration one SpMV plus the
    # 88 N bytes of its vector updates
    return (iters + 2) * spmv_alg_bytes(n, nnz_off) + iters * 88 * n


def pcg_kernel_launches(iters, fused=0):
    # setup, start, three kernels per iteration (fused modes 1-3: one; mode 4:
    # one for the whole loop), post-processing
    if fused == 4:
        return 4
    return (1 if fused else 3) * iters + 3


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

    if (world > 1 and not args.replicas) or args.partitioned:
        if world == 1 and not dist.is_initialized():
            dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        try:
            return run_partitioned(args, world, rank, local, barrier, max_over_ranks)
        finally:
            dist.destroy_process_group()

    n = args.n
    s = S.poisson_jittered(n, seed=2 + rank)
    N, nnz = s.neq, s.nnz_full
    g = sv.GpuSystem(N, s.ia, s.ja, sv.CSRD, True, device=local)
    g.set_values(s.al, s.ad)
    g.set_engine(args.engine, args.threads, args.spw)
    if args.pf:
        g.set_prefetch(args.pf)
    g.set_fused(args.fused)
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
            elif args.profile in ("assembly", "pressure", "momentum"):
                setup = {"assembly": dif_call_setup, "pressure": pres_call_setup,
                         "momentum": vel_call_setup}[args.profile]
                call, close = setup(np, torch, sv, s, sptr)
                for _ in range(args.warmup + args.steps):
                    call()
                close()
            elif args.profile == "gradient":
                from sfr3d_b200 import assembly as A
                m, prop, vel, _pres, lvel, _lpres = gradient_inputs(np, s)
                plan = A.GradPlan(m, m.face_r(PRES_SIDES_VEL), type=A.RCLSQUARE)
                du = torch.tensor(np.ascontiguousarray(vel), device="cuda")
                dg = torch.zeros((m.numel, 3, 3), dtype=torch.float64, device="cuda")
                for _ in range(args.warmup + args.steps):
                    plan.grad_device(lvel, prop, 3, du.data_ptr(), dg.data_ptr(), sptr)
                torch.cuda.synchronize()
                plan.close()
            elif args.profile == "partitioned":
                from sfr3d_b200 import halo as H
                lays = H.partition(N, s.ia, s.ja, True, 2)
                hg = H.LocalGroup(2, local)
                hs = [H.DistSystem(hg, lay) for lay in lays]
                for sy, lay in zip(hs, lays):
                    sy.set_values(*lay.values(s.al, s.ad))
                b_r = [lay.rows(s.b[0]) for lay in lays]
                for _ in range(args.warmup + args.steps):
                    H.solve(hg, hs, sv.PCG, b_r, tol=1e-10, maxit=args.maxit)
                hg.close()
            elif args.profile == "bicgstab":
                m = S.momentum(n, nrhs=args.nrhs, seed=3)
                gm = sv.GpuSystem(m.neq, m.ia, m.ja, sv.CSRD, True, device=local)
                gm.set_values(m.al, m.ad)
                gm.set_engine(args.engine, args.threads, args.spw)
                gm.set_prefetch(args.pf)
                bm = torch.tensor(m.b.reshape(-1), device="cuda")
                xm = torch.zeros_like(bm)
                for _ in range(args.warmup + args.steps):
                    gm.solve_multi_device(sv.PBICGSTAB, args.nrhs, bm.data_ptr(), xm.data_ptr(),
                                          tol=1e-10, maxit=args.maxit, stream=sptr,
                                          precision=sv.MIXED if args.mixed else sv.FP64)
            else:
                for _ in range(args.warmup + args.steps):
                    g.solve_device(sv.PCG, b.data_ptr(), x.data_ptr(), tol=1e-10,
                                   maxit=args.maxit, stream=sptr,
                                   precision=sv.MIXED if args.mixed else sv.FP64)
        torch.cuda.synchronize()
        return None

    def timed_solves(precision, steps, warm, xbuf):
        for _ in range(warm):
            g.solve_device(sv.PCG, b.data_ptr(), xbuf.data_ptr(), tol=1e-10,
                           maxit=args.maxit, precision=precision, stream=sptr)
        barrier()
        infos = []
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        for i in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            info = g.solve_device(sv.PCG, b.data_ptr(), xbuf.data_ptr(), tol=1e-10,
                                  maxit=args.maxit, precision=precision, stream=sptr)
            ev[i][1].record(stream)
            infos.append(info)
        barrier()
        return [a.elapsed_time(c) for a, c in ev], infos

    # the autotuner picks the engine and launch shape on this system
    # (untimed); the timed solves below take its choice
    tune = None
    if args.engine == 0 and not args.no_tune:
        tune = {"headline_fp64": g.autotune(sv.PCG, s.b[0], tol=1e-10, maxit=args.maxit)}
        if not args.no_mixed:
            tune["headline_mixed"] = g.autotune(sv.PCG, s.b[0], tol=1e-10, maxit=args.maxit,
                                                precision=sv.MIXED)

    gpu_uuid = str(torch.cuda.get_device_properties(local).uuid)
    clocks = ClockSampler(gpu_uuid if gpu_uuid.startswith("GPU-") else f"GPU-{gpu_uuid}")
    clocks.start()
    t_wall0 = time.perf_counter()
    times, infos = timed_solves(sv.FP64, args.steps, args.warmup, x)
    t_wall = time.perf_counter() - t_wall0
    clk = clocks.stop()
    ms_step = max_over_ranks(statistics.mean(times))
    iters = infos[-1].iters
    if infos[-1].status != sv.OK:
        raise RuntimeError(f"solve did not converge: {sv.status_string(infos[-1].status)}")

    extras = rank == 0 and world == 1
    peak, peak_kind = peak_hbm()

    # mixed precision on the same system, and its error against FP64
    mixed = None
    if not args.no_mixed:
        xm = torch.zeros_like(b)
        try:
            mt, mi = timed_solves(sv.MIXED, args.steps, 1, xm)
            x64 = x.cpu().numpy()
            x32 = xm.cpu().numpy()
            m_ms = max_over_ranks(statistics.mean(mt))
            inner = max(mi[-1].inner_iters, 1)
            # per inner iteration: FP32 coupling + 16-bit offset per slot, the
            # gather of p and the read and write of p (12 B a row)
            inner_bytes = g.stats()["slots"] * 6 + 12 * N
            mixed = {"ms": m_ms,
                     "engine": ("resident: one cooperative launch, scaled FP32 operator held "
                                "in L2, inner vectors in shared memory" if args.engine in (0, 4)
                                else f"engine {args.engine}"),
                     "inner_iters": mi[-1].inner_iters,
                     "refinements": mi[-1].refinements,
                     "status": mi[-1].status,
                     "stopping_test": "reference's PCG criterion on the FP64 true residual: "
                                      "sqrt|(r, M^-1 r)| < 1e-10 sqrt|(b, M^-1 b)| (Cg.c:145)",
                     "true_relres_Mnorm": (mi[-1].norm_r_m / (mi[-1].conv / 1e-10)
                                           if mi[-1].conv > 0 else None),
                     "true_relres_2norm": mi[-1].relres,
                     "err_vs_fp64_x": float(np.linalg.norm(x32 - x64) / np.linalg.norm(x64)),
                     "speedup_vs_fp64": ms_step / max(m_ms, 1e-9),
                     "us_per_inner_iteration": m_ms * 1e3 / inner,
                     "alg_bytes_per_inner_iteration": inner_bytes,
                     "inner_GB/s_from_L2": inner_bytes / (m_ms * 1e-3 / inner) / 1e9}
        except sv.SolverError as e:
            mixed = {"unavailable": str(e)}

    spmv_ms = spmv_time(torch, g, b, stream)
    sb = spmv_alg_bytes(N, nnz)
    spmv_gbs = sb / (spmv_ms * 1e-3) / 1e9
    sp_tr = committed_traffic("spmv_kernel")

    momentum = batch = adjoint = target = assembly = partitioned = None
    if world > 1 and not args.no_extras:
        batch = batch_leg_sharded(sv, S, rank, world, max_over_ranks)
    other = None
    if extras and not args.no_extras:
        other = other_krylov_leg(sv, S, s, n)
        assembly = assembly_leg(np, torch, sv, s, n, peak, peak_kind)
        assembly["pressure"] = pressure_leg(np, torch, sv, s, n, peak, peak_kind)
        assembly["momentum"] = momentum_assembly_leg(np, torch, sv, s, n, peak, peak_kind)
        assembly["simple_step"] = simple_step_leg(np, torch, sv, s, n)
        assembly["gradient"] = gradient_leg(np, torch, s, n, peak, peak_kind)
        partitioned = partitioned_leg(np, sv, s, n, ms_step, x.cpu().numpy())
        momentum = momentum_leg(np, torch, sv, S, n, local, tune=not args.no_tune)
        batch = batch_leg(sv, S)
        adjoint = adjoint_leg(np, sv, S)
        if mixed and "ms" in mixed and momentum:
            plain = ms_step + momentum["fp64_sequential_ms"]
            fast = mixed["ms"] + momentum["mixed_k3_ms"]
            target = {"what": "128^3 pressure PCG + 128^3 momentum BiCGSTAB (3 RHS) to 1e-10",
                      "plain_fp64_ms": plain, "mixed_batched_ms": fast,
                      "speedup": plain / fast, "goal": 2.0}

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
        # the drop-in tunes the pattern's first solve (a warm-up call)
        L.sfr_set_autotune(0 if args.no_tune or args.engine != 0 else 1)

        def call():
            return L.sfr_solverC(None, N, N, len(jl), 0, h_ia.data_ptr(), h_ja.data_ptr(),
                                 h_al.data_ptr(), h_ad.data_ptr(), None, h_b.data_ptr(),
                                 h_x.data_ptr(), None, None, 1e-10, args.maxit, sv.CSRD,
                                 sv.PCG, None, False, True, False, b"pressure")
        for _ in range(args.warmup):
            assert call() == sv.OK
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            rc = call()
            if rc != sv.OK:
                raise RuntimeError(f"drop-in solve failed: {sv.status_string(rc)}")
        barrier()
        e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.steps)
        e2e = {"value": e2e_ms, "unit": "ms",
               "h2d_bytes_per_step": int(h_al.numel() * 8 + h_ad.numel() * 8 + h_b.numel() * 8),
               "d2h_bytes_per_step": int(h_x.numel() * 8),
               "api": "sfr_solverC (solverC drop-in), CSRD symmetric storage, FP64"}
        L.sfr_set_autotune(0)
        sv.release_cache()

    # CPU baseline: the reference's own pcgOmp on this host (rank 0, N = 1)
    cpu = None
    if not args.no_cpu and extras:
        xs_gpu = {"fp64": x.cpu().numpy()}
        if mixed and "ms" in mixed:
            xs_gpu["mixed"] = xm.cpu().numpy()
        cpu = cpu_baseline(s, iters, n, xs_gpu)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return None

    alg = pcg_alg_bytes(N, nnz, iters)
    achieved = alg / (ms_step * 1e-3) / 1e9
    # the timed solves' engine: the autotuner's choice, or the flags given
    fused = int(tune["headline_fp64"]["fused"]) if tune else int(args.fused)
    tr = committed_traffic("pcg_fp64_fused_loop_iteration" if fused == 4
                           else "pcg_fp64_fused_iteration" if fused else "pcg_fp64_iteration")
    traffic = None
    if tr is not None and tr[1] == "per_iteration_128":
        traffic = tr[0] * (N / 128 ** 3) * iters
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
                   "format": "SELL-32 from CSRD: FP64 values, 16-bit column offsets",
                   "engine": ("CUDA graph, one cooperative kernel for the whole solve "
                              "(k_pcg_fused_loop: per iteration SpMV+dot, exchange, x/r/z "
                              "update+dot, exchange, p update, wait on the neighbouring blocks; "
                              "q and z kept in shared memory)" if fused == 4 else
                              "CUDA graph, device-side WHILE loop, one cooperative kernel per "
                              "iteration (k_pcg_fused: SpMV+dot, grid barrier, x/r/z update+dot, "
                              "grid barrier, p update; q and z kept in shared memory)"
                              if fused else
                              "CUDA graph, device-side WHILE loop (3 kernels per iteration)"),
                   "fused_mode": fused,
                   "l2": "flushed between steps (256 MiB write)",
                   "parallelism": f"replicas{world}" if world > 1 else "single GPU"},
        "iterations": iters,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "frac_on_traffic": (None if traffic is None
                                         else traffic / (ms_step * 1e-3) / 1e9 / peak),
                     "kernel": ("k_pcg_fused_loop (one launch per solve)" if fused == 4 else
                                "PCG solve graph (one launch per solve: k_pcg_fused per "
                                "iteration)" if fused else
                                "PCG solve graph (one launch per solve: k_pcg_a SpMV+dot, "
                                "k_pcg_b update+dot, k_pcg_c direction per iteration)"),
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "alg_bytes_per_launch": alg,
                     "alg_bytes_rule": "(iters+2)*(12 nnz_off + 4(N+1) + 24N) + iters*88N",
                     "alg_bytes_note": "32-bit column indices, as the CSRD formula counts them; "
                                       "the SpMV phases read 16-bit offsets (2 B a slot less), "
                                       "and the fused iterations keep q and z on chip, so the "
                                       "algorithmic fraction can exceed 1; frac_on_traffic is "
                                       "the ncu DRAM bytes of the same iterations over the "
                                       "same time"},
        "spmv": {"kernel": "spmv_kernel", "ms": spmv_ms, "alg_bytes": sb, "GB/s": spmv_gbs,
                 "frac": spmv_gbs / peak, "peak_source": f"{peak_kind} hbm_gbs",
                 "traffic": None if sp_tr is None else sp_tr[0] * (N / 128 ** 3),
                 "timing": "graph of 20 x [256 MiB read, SpMV] minus graph of 20 x [256 MiB read]"},
        "mixed": mixed,
        "momentum": momentum,
        "partitioned": partitioned,
        "batched": batch,
        "adjoint": adjoint,
        "other_krylov": other,
        "assembly": assembly,
        "target_mixed_batched_vs_fp64": target,
        "autotune": tune,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": args.steps * pcg_kernel_launches(iters, fused),
        "clocks": clk,
        "wall_s_timed_region": t_wall,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return line


def run_partitioned(args, world, rank, local, barrier, max_over_ranks):
    """One system row-partitioned over the ranks: the reference's MPI path
    (mpiPcg, Cg.c:256-442, with comunicateNeq, ParallelMpi.c:3346-3420),
    one rank per GPU, the halo and the dot sums over NCCL.

    Strong scaling (the line's value): the 128^3 headline system split into
    N row blocks; the device time of a solve, max over ranks.  Weak scaling
    (`weak_scaling`): an n x n x (n N) box, n^3 rows per rank.  Rank 0 checks
    the partitioned solution against the one-GPU solve of the same system
    (FP64 bar: 1e-12 relative, iterations +-1) outside the timed region."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from sfr3d_b200 import halo as H
    from sfr3d_b200 import solver as sv
    from sfr3d_b200 import systems as S

    n = args.n
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def setup(sysx):
        lays = H.partition(sysx.neq, sysx.ia, sysx.ja, True, world)
        lay = lays[rank]
        problems = H.check_interfaces(lay)
        if problems:
            raise RuntimeError("partition interfaces disagree: " + "; ".join(problems[:3]))
        grp = H.NcclGroup.from_process_group(local)
        d = H.DistSystem(grp, lay)
        d.set_values(*lay.values(sysx.al, sysx.ad))
        return lay, grp, d

    def timed(grp, d, b_r, steps, warm):
        for _ in range(warm):
            H.solve(grp, [d], sv.PCG, [b_r], tol=1e-10, maxit=args.maxit)
        ms, info, x = [], None, None
        for i in range(steps):
            flush.fill_(i & 0xFF)
            barrier()
            x, info = H.solve(grp, [d], sv.PCG, [b_r], tol=1e-10, maxit=args.maxit)
            ms.append(info.seconds * 1e3)
        barrier()
        if info.status != sv.OK:
            raise RuntimeError(f"partitioned solve: {sv.status_string(info.status)}")
        return max_over_ranks(statistics.mean(ms)), info, x[0]

    # ---- strong scaling: the 128^3 headline system over N ranks
    s = S.poisson_jittered(n, seed=2)
    N, nnz = s.neq, s.nnz_full
    lay, grp, d = setup(s)
    b_r = lay.rows(s.b[0])
    gpu_uuid = str(torch.cuda.get_device_properties(local).uuid)
    clocks = ClockSampler(gpu_uuid if gpu_uuid.startswith("GPU-") else f"GPU-{gpu_uuid}")
    clocks.start()
    t_wall0 = time.perf_counter()
    ms_step, info, x_r = timed(grp, d, b_r, args.steps, args.warmup)
    t_wall = time.perf_counter() - t_wall0
    clk = clocks.stop()
    iters = info.iters

    # end to end through the drop-in's MPI branch (sfr_solverC with the
    # rank's MPI CSRD arrays and its Interface as iNeq): al, ad, b uploaded
    # and x read back every call
    e2e = None
    if not args.no_e2e:
        H.set_solverC_group(grp)
        sv.lib().sfr_set_exit_on_failure(0)
        al_r, ad_r = lay.values(s.al, s.ad)
        iface = lay.interface()
        xr = np.zeros(lay.nEq)

        def call():
            return sv.solverC(lay.nEq, lay.nEqNov, lay.nAd, lay.nAdR, lay.ia, lay.ja, al_r, ad_r,
                              None, b_r, xr, 1e-10, args.maxit, storage=sv.CSRD,
                              solver=sv.PCG, newX=True, unSym=True, iNeq=iface)
        for _ in range(max(1, args.warmup)):
            if call() != sv.OK:
                raise RuntimeError("partitioned drop-in solve failed")
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            if call() != sv.OK:
                raise RuntimeError("partitioned drop-in solve failed")
        barrier()
        e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.steps)
        e2e = {"value": e2e_ms, "unit": "ms",
               "h2d_bytes_per_step": int(8 * (len(al_r) + len(ad_r) + len(b_r))),
               "d2h_bytes_per_step": int(8 * lay.nEq),
               "per": "rank 0's share (every rank moves its own rows)",
               "api": "sfr_solverC MPI branch (sfr_solverC_set_group on an NCCL group): "
                      "the rank's MPI CSRD arrays and Interface, FP64"}
        H.set_solverC_group(None)

    # the partitioned x against the one-GPU solve (rank 0), untimed
    gathered = [None] * world if rank == 0 else None
    dist.gather_object((lay.l2g[:lay.nEqNov], x_r[:lay.nEqNov]), gathered, dst=0)
    parity = None
    if rank == 0:
        xg = np.zeros(N)
        for l2g, xv in gathered:
            xg[l2g] = xv
        one = sv.GpuSystem(N, s.ia, s.ja, sv.CSRD, True, device=local)
        one.set_values(s.al, s.ad)
        x1, i1 = one.solve(sv.PCG, s.b[0], tol=1e-10, maxit=args.maxit)
        one.close()
        err = float(np.linalg.norm(xg - x1) / np.linalg.norm(x1))
        parity = {"err_vs_one_gpu_x": err, "iters": iters, "iters_one_gpu": i1.iters,
                  "bar": "1e-12 relative, iterations +-1",
                  "ok": bool(err < 1e-12 and abs(iters - i1.iters) <= 1)}
    barrier()
    d.close()
    grp.close()

    # ---- weak scaling: n_w^3 rows per rank
    weak = None
    if not args.no_extras:
        nw = args.weak_n
        sw = S.build(S.params(n=(nw, nw, nw * world), lengths=(1.0, 1.0, float(world)),
                              jitter=0.2, log10k=(-2.0, 2.0), permute=True, seed=5))
        lw, gw, dw = setup(sw)
        bw = lw.rows(sw.b[0])
        wms, winfo, _ = timed(gw, dw, bw, max(2, args.steps // 2), 1)
        weak = {"workload": f"{nw}x{nw}x{nw * world} jittered Poisson box, {sw.neq} rows, "
                            f"{nw}^3 rows per rank, PCG FP64 to 1e-10",
                "ms": wms, "iterations": winfo.iters,
                "us_per_iteration": wms * 1e3 / max(winfo.iters, 1),
                "rows_per_rank": lw.nEqNov}
        dw.close()
        gw.close()

    if rank != 0:
        return None
    peak, peak_kind = peak_hbm()
    alg = pcg_alg_bytes(N, nnz, iters)
    achieved = alg / world / (ms_step * 1e-3) / 1e9
    line = {
        "metric": METRIC,
        "value": ms_step,
        "unit": "ms",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": False,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded jittered 128^3 hex mesh, generated on the host)",
        "config": {"workload": f"pressure-correction Poisson {n}^3 = {N} cells (jittered, "
                               f"diffusivity 10^U(-2,2), permuted + RCM), row-partitioned over "
                               f"{world} ranks; mpiPcg FP64 to 1e-10 (M-norm)",
                   "rows": N, "nnz_offdiag": nnz, "iterations": iters,
                   "engine": "row blocks balanced by entries; halo by NCCL send/recv into the "
                             "ghost entries, dot sums by NCCL allreduce; iteration loop a CUDA "
                             "graph of 32 iterations",
                   "l2": "flushed before each step (256 MiB write)",
                   "parallelism": f"row partition over {world} GPUs"},
        "iterations": iters,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None,
                     "kernel": "partitioned PCG solve, per GPU",
                     "peak_source": f"{peak_kind} hbm_gbs",
                     "alg_bytes_per_launch": alg,
                     "alg_bytes_rule": "((iters+2)*(12 nnz_off + 4(N+1) + 24N) + iters*88N) / N_gpus"},
        "parity": parity,
        "weak_scaling": weak,
        "cpu_baseline": None,
        "e2e": e2e,
        "gpu_launches": args.steps * (4 * iters + 4),
        "clocks": clk,
        "wall_s_timed_region": t_wall,
    }
    print(json.dumps(line), flush=True)
    return line


def spmv_time(torch, g, x, stream, reps=20):
    """Device time of one SpMV launch with a cold L2: CUDA events around a
    graph of `reps` x [read 256 MiB, SpMV] minus a graph of `reps` x
    [read 256 MiB] (a read leaves L2 clean, so the SpMV pays no write-backs
    of the flush), divided by reps.  Best of three replays each."""
    y = torch.empty_like(x)
    fl = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    sink = torch.empty((), dtype=torch.float32, device="cuda")
    with torch.cuda.stream(stream):
        for _ in range(3):
            torch.sum(fl, dim=0, out=sink)
            g.spmv(x.data_ptr(), y.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    with_spmv, flush_only = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
    with torch.cuda.graph(with_spmv, stream=stream):
        for _ in range(reps):
            torch.sum(fl, dim=0, out=sink)
            g.spmv(x.data_ptr(), y.data_ptr(), stream.cuda_stream)
    with torch.cuda.graph(flush_only, stream=stream):
        for _ in range(reps):
            torch.sum(fl, dim=0, out=sink)
    best = {}
    for name, gr in (("a", with_spmv), ("b", flush_only)) * 3:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            gr.replay()  # warm
            torch.cuda.synchronize()
            e0.record(stream)
            gr.replay()
            e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1)
        best[name] = min(best.get(name, t), t)
    return (best["a"] - best["b"]) / reps


def partitioned_leg(np, sv, s, n, fp64_ms, x64):
    """The row-partitioned PCG (the reference's MPI path, mpiPcg) on the
    headline system, its ranks held by one GPU: device time per solve at 1,
    2 and 4 ranks against the unpartitioned solve."""
    from sfr3d_b200 import halo as H
    out = {"what": f"mpiPcg path, {n}^3 headline system, R ranks in one process on one GPU "
                   "(halo = one device gather, sums in rank order inside the kernels, the "
                   "iteration loop a CUDA graph of 32 iterations); FP64 to 1e-10",
           "timing": "CUDA events inside sfr_gpu_dist_solve, mean of 2 after 1 warm-up"}
    N, nnz = s.neq, s.nnz_full
    for R in (1, 2, 4):
        lays = H.partition(N, s.ia, s.ja, True, R)
        g = H.LocalGroup(R, 0)
        systems = [H.DistSystem(g, lay) for lay in lays]
        for sy, lay in zip(systems, lays):
            sy.set_values(*lay.values(s.al, s.ad))
        b_r = [lay.rows(s.b[0]) for lay in lays]
        H.solve(g, systems, sv.PCG, b_r, tol=1e-10)
        ms = []
        for _ in range(2):
            xs, info = H.solve(g, systems, sv.PCG, b_r, tol=1e-10)
            ms.append(info.seconds * 1e3)
        x = np.zeros(N)
        for lay, xr in zip(lays, xs):
            x[lay.l2g[:lay.nEqNov]] = xr[:lay.nEqNov]
        ghosts = sum(lay.nRcvs for lay in lays)
        alg = pcg_alg_bytes(N, nnz, info.iters) + (info.iters + 2) * 16 * ghosts
        t = statistics.mean(ms)
        out[f"ranks_{R}"] = {"ms": t, "iterations": info.iters, "ghost_entries": ghosts,
                             "vs_unpartitioned": t / fp64_ms,
                             "alg_GB/s": alg / (t * 1e-3) / 1e9,
                             "err_vs_unpartitioned_x": float(np.linalg.norm(x - x64)
                                                             / np.linalg.norm(x64)),
                             "launches_per_iteration": 3 * R + (1 if R > 1 else 0)}
        g.close()
    return out


def momentum_leg(np, torch, sv, S, n, device, tune=True):
    """128^3 momentum (Peclet 50, nu 1e-3, dt 1e-2), three right-hand sides:
    FP64 one right-hand side at a time vs one K = 3 mixed launch.  With
    `tune`, the K = 3 solves run on the autotuner's choice (tuned untimed)."""
    m = S.momentum(n, nrhs=3, seed=3)
    g = sv.GpuSystem(m.neq, m.ia, m.ja, sv.CSRD, True, device=device)
    g.set_values(m.al, m.ad)
    out = {"workload": f"momentum {n}^3 Peclet 50, 3 RHS, Jacobi-BiCGSTAB to 1e-10"}
    if tune:
        out["autotune"] = {
            "k3_fp64": g.autotune(sv.PBICGSTAB, m.b, tol=1e-10),
            "k3_mixed": g.autotune(sv.PBICGSTAB, m.b, tol=1e-10, precision=sv.MIXED)}
    for _ in range(2):  # warm-up: graphs built, clocks up
        for k in range(3):
            g.solve(sv.PBICGSTAB, m.b[k], tol=1e-10)
        g.solve_multi(sv.PBICGSTAB, m.b, tol=1e-10, precision=sv.MIXED)
        g.solve_multi(sv.PBICGSTAB, m.b, tol=1e-10)
    seq, its = 0.0, []
    x64 = []
    for k in range(3):
        xk, info = g.solve(sv.PBICGSTAB, m.b[k], tol=1e-10)
        seq += info.seconds * 1e3
        its.append(info.iters)
        x64.append(xk)
    xs, infos = g.solve_multi(sv.PBICGSTAB, m.b, tol=1e-10, precision=sv.MIXED)
    _, infos64 = g.solve_multi(sv.PBICGSTAB, m.b, tol=1e-10)
    out.update({
        "fp64_sequential_ms": seq, "fp64_iters": its,
        "fp64_k3_ms": infos64[0].seconds * 1e3,
        "mixed_k3_ms": infos[0].seconds * 1e3,
        "mixed_iters": [i.iters for i in infos],
        "mixed_status": [i.status for i in infos],
        "mixed_err_vs_fp64_x": [float(np.linalg.norm(xs[k] - x64[k]) / np.linalg.norm(x64[k]))
                                for k in range(3)],
        "mixed_true_relres": [i.relres for i in infos],
    })
    g.close()
    return out


def batch_leg(sv, S):
    """64 uneven Poisson systems (8..96 cells per axis) in one batched launch,
    block shares autotuned from measured iterations."""
    systems = S.poisson_batch(64, 8, 96, seed=4)
    g = sv.GpuBatch([(s.neq, s.ia, s.ja) for s in systems], sv.CSRD, True)
    g.set_values([s.al for s in systems], [s.ad for s in systems])
    bs = [s.b[0] for s in systems]
    out = {"workload": f"64 Poisson boxes, {sum(s.neq for s in systems)} rows total, PCG to 1e-10"}
    for name, prec in (("fp64", sv.FP64), ("mixed", sv.MIXED)):
        g.solve(sv.PCG, bs, tol=1e-10, precision=prec)
        ms = g.autotune(sv.PCG, bs, tol=1e-10, precision=prec)
        _, infos = g.solve(sv.PCG, bs, tol=1e-10, precision=prec)
        out[name] = {"ms": infos[0].seconds * 1e3, "autotune_best_ms": ms,
                     "autotune": g.tune_report(),
                     "max_iters": max(i.iters for i in infos),
                     "all_converged": all(i.status == sv.OK for i in infos)}
    out["grid_blocks"] = g.stats()["grid"]
    g.close()
    # the plain path: the same systems one at a time, FP64 (device time of
    # each solve, second of two)
    seq = 0.0
    for sy in systems:
        one = sv.GpuSystem(sy.neq, sy.ia, sy.ja, sv.CSRD, True)
        one.set_values(sy.al, sy.ad)
        one.solve(sv.PCG, sy.b[0], tol=1e-10)
        _, info = one.solve(sv.PCG, sy.b[0], tol=1e-10)
        seq += info.seconds * 1e3
        one.close()
    out["fp64_one_at_a_time_ms"] = seq
    out["speedup_mixed_batched_vs_fp64_one_at_a_time"] = seq / out["mixed"]["ms"]
    return out


def batch_leg_sharded(sv, S, rank, world, max_over_ranks):
    """The 64 uneven systems split across ranks by estimated work (no
    collective on the data path); each rank solves its share in one batched
    launch; the time is the max over ranks."""
    from sfr3d_b200 import sharding as SH
    systems = S.poisson_batch(64, 8, 96, seed=4)
    shares = SH.plan([SH.estimated_work(s.neq, s.nnz_full) for s in systems], world)
    mine = [systems[i] for i in shares[rank]]
    ms = {}
    if mine:
        g = sv.GpuBatch([(s.neq, s.ia, s.ja) for s in mine], sv.CSRD, True)
        g.set_values([s.al for s in mine], [s.ad for s in mine])
        bs = [s.b[0] for s in mine]
    for name, prec in (("fp64", sv.FP64), ("mixed", sv.MIXED)):
        t = 0.0
        if mine:
            g.solve(sv.PCG, bs, tol=1e-10, precision=prec)
            g.autotune(sv.PCG, bs, tol=1e-10, precision=prec)
            _, infos = g.solve(sv.PCG, bs, tol=1e-10, precision=prec)
            t = infos[0].seconds * 1e3
        ms[name] = max_over_ranks(t)
    if mine:
        g.close()
    return {"workload": f"64 Poisson boxes across {world} ranks, PCG to 1e-10",
            "rows_this_rank0": sum(systems[i].neq for i in shares[0]),
            "fp64_ms_max_over_ranks": ms["fp64"], "mixed_ms_max_over_ranks": ms["mixed"]}


def other_krylov_leg(sv, S, s, n):
    """The other Krylov methods behind solverC at 128^3, FP64, one
    right-hand side: MINRES on the pressure system (symmetric), BiCGSTAB(2)
    and GMRES(15) on the momentum system.  Device time of the second of two
    solves; the reference's times are in cpu_baseline.other_krylov."""
    m = S.momentum(n, nrhs=1, seed=3)
    gm = sv.GpuSystem(m.neq, m.ia, m.ja, sv.CSRD, True)
    gm.set_values(m.al, m.ad)
    gp = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    gp.set_values(s.al, s.ad)
    out = {}
    for name, g, sysx, solver in (("minres_pressure", gp, s, sv.MINRES),
                                  ("bicgstabl2_momentum", gm, m, sv.PBICGSTABL2),
                                  ("gmres15_momentum", gm, m, sv.GMRES)):
        for _ in range(2):
            _, info = g.solve(solver, sysx.b[0], tol=1e-10, maxit=100000)
        out[name] = {"ms": info.seconds * 1e3, "iters": info.iters, "status": info.status,
                     "us_per_iteration": info.seconds * 1e6 / max(info.iters, 1),
                     "true_relres_2norm": info.norm_r / float((sysx.b[0] ** 2).sum() ** 0.5)}
    gm.close()
    gp.close()
    return out


# algorithmic bytes per row of the ORTHOGONAL diffusion assembly kernel on a
# hexahedral mesh (6 faces), CSRD full: plan row header (cell 4 + face count
# 2), per face the neighbour, raw-destination and SELL-slot words (12) and 3
# geometry doubles (24), the cell's own diffusivity and u0 (16); writes the
# 6 off-diagonals in the reference's layout and in the solver's copy (FP64 +
# FP32: 6 * 20), ad, its FP32 copy, the row compensation, b and rCell (36).
# Neighbour gathers are counted once (they are other rows' own reads).
ASSEMBLY_ALG_BYTES_PER_ROW = 6 + 6 * 36 + 16 + 6 * 20 + 36


def dif_call_setup(np, torch, sv, s, stream):
    """A device systFormDif call on the system's mesh (ORTHOGONAL, Dirichlet
    on x = 0, Neumann elsewhere, residual form, CSRD): (call, close)."""
    from sfr3d_b200 import assembly as A
    m = s.mesh()
    rng = np.random.default_rng(9)
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    plan = A.DifPlan(g, m, m.face_r([1, 0, 0, 0, 0, 0]), icod=A.ORTHOGONAL)
    loads = [A.Load(A.DIRICHLET, (0.0,))]
    dev = lambda a: torch.tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    d_u0, d_k = dev(rng.standard_normal(m.numel)), dev(m.cdiff)
    d_b = torch.empty(s.neq, dtype=torch.float64, device="cuda")
    d_r = torch.empty(m.numel, dtype=torch.float64, device="cuda")

    def call():
        plan.assemble_device(loads, d_u0.data_ptr(), d_k.data_ptr(), d_b=d_b.data_ptr(),
                             d_rcell=d_r.data_ptr(), stream=stream)

    def close():
        plan.close()
        g.close()
    return call, close


# the SIMPLE pressure correction on the same mesh: a lid-driven cavity's
# loads (static walls, the z-max lid moving) with the pressure fixed on x = 0
PRES_SIDES_VEL = [2, 2, 2, 2, 2, 1]
PRES_SIDES_PRES = [1, 0, 0, 0, 0, 0]


def pres_inputs(np, s):
    m = s.mesh()
    rng = np.random.default_rng(10)
    prop = np.zeros((1, 10))
    prop[0, 1] = 1.0
    return m, prop, dict(pres=rng.standard_normal(m.numel),
                         gradpres=rng.standard_normal((m.numel, 3)),
                         vel=rng.standard_normal((m.numel, 3)),
                         dfield=rng.uniform(0.5, 1.0, (m.numel, 3)))


def pres_call_setup(np, torch, sv, s, stream):
    """A device systFormSimplePres call on the system's mesh: (call, close)."""
    from sfr3d_b200 import assembly as A
    m, prop, f = pres_inputs(np, s)
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    plan = A.PresPlan(g, m, m.face_r(PRES_SIDES_PRES), m.face_r(PRES_SIDES_VEL),
                      icod=A.ORTHOGONAL)
    lvel = [A.Load(A.MOVEWALL, (1.0, 0.0, 0.0, 0.0)), A.Load(A.STATICWALL, ())]
    lpres = [A.Load(A.DIRICHLET, (0.0,))]
    dev = {k: torch.tensor(np.ascontiguousarray(v), device="cuda") for k, v in f.items()}
    d_b = torch.empty(s.neq, dtype=torch.float64, device="cuda")
    d_r = torch.empty(m.numel, dtype=torch.float64, device="cuda")

    def call():
        plan.assemble_device(lvel, lpres, prop, dev["pres"].data_ptr(),
                             dev["gradpres"].data_ptr(), dev["vel"].data_ptr(),
                             dev["dfield"].data_ptr(), d_b=d_b.data_ptr(),
                             d_rcell=d_r.data_ptr(), stream=stream)

    def close():
        plan.close()
        g.close()
    return call, close


def time_calls(torch, call, st, reps=10):
    """Median device time of `call` (CUDA events on st, L2 flushed between)."""
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(st):
        for _ in range(3):
            call()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * reps)]
        for i in range(reps):
            flush.fill_(i & 0xFF)
            ev[2 * i].record(st)
            call()
            ev[2 * i + 1].record(st)
    st.synchronize()
    return sorted(ev[2 * i].elapsed_time(ev[2 * i + 1]) for i in range(reps))[reps // 2]


def assembly_leg(np, torch, sv, s, n, peak, peak_kind):
    """systFormDif on the device for the 128^3 pressure mesh (ORTHOGONAL,
    Dirichlet on x = 0, Neumann elsewhere, residual form): one call writes
    A (CSRD) and b where the next solve reads them.  Beside it: the per-call
    upload of A and b the host-assembled path needs, and the host-array
    entry point (fields in, b and rCell out)."""
    from sfr3d_b200 import assembly as A
    st = torch.cuda.Stream()
    t0 = time.perf_counter()
    call, close = dif_call_setup(np, torch, sv, s, st.cuda_stream)
    torch.cuda.synchronize()
    plan_s = time.perf_counter() - t0
    dev_ms = time_calls(torch, call, st)
    close()
    alg = ASSEMBLY_ALG_BYTES_PER_ROW * s.neq
    reps = 10
    # the host-assembled path: A (al, ad) and b uploaded every call
    h_al = torch.from_numpy(s.al).pin_memory()
    h_ad = torch.from_numpy(s.ad).pin_memory()
    h_b = torch.from_numpy(s.b[0]).pin_memory()
    d_al = torch.empty_like(h_al, device="cuda")
    d_ad = torch.empty_like(h_ad, device="cuda")
    d_b = torch.empty_like(h_b, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        d_al.copy_(h_al, non_blocking=True)
        d_ad.copy_(h_ad, non_blocking=True)
        d_b.copy_(h_b, non_blocking=True)
    torch.cuda.synchronize()
    upload_ms = (time.perf_counter() - t0) * 1e3 / reps
    # the host-array entry point: u0 and the diffusivity in, b and rCell out
    m = s.mesh()
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    plan = A.DifPlan(g, m, m.face_r([1, 0, 0, 0, 0, 0]), icod=A.ORTHOGONAL)
    u0 = np.random.default_rng(9).standard_normal(m.numel)
    loads = [A.Load(A.DIRICHLET, (0.0,))]
    plan.assemble(loads, u0, m.cdiff)
    t0 = time.perf_counter()
    for _ in range(3):
        plan.assemble(loads, u0, m.cdiff)
    host_ms = (time.perf_counter() - t0) * 1e3 / 3
    plan.close()
    g.close()
    gbs = alg / (dev_ms * 1e-3) / 1e9
    tr = committed_traffic("dif_assemble_kernel")
    return {"workload": f"systFormDif, diffusion {n}^3 = {s.neq} cells (the pressure mesh), "
                        "ORTHOGONAL, Dirichlet x=0, residual form, CSRD",
            "device_ms": dev_ms, "plan_create_s": plan_s,
            "traffic": None if tr is None else tr[0] * (s.neq / 128 ** 3),
            "alg_bytes_per_call": alg, "alg_bytes_per_row": ASSEMBLY_ALG_BYTES_PER_ROW,
            "GB/s": gbs, "frac": gbs / peak, "peak_source": f"{peak_kind} hbm_gbs",
            "kernel": "dif_assemble_kernel<orthogonal, 6 faces, fused> (one launch: also "
                      "writes the solver's SELL copy, its FP32 copy and compensation)",
            "timing": "CUDA events around one call, 256 MiB L2 flush between calls, median "
                      "of 10",
            "upload_A_b_pinned_ms": upload_ms,
            "host_api_ms": host_ms,
            "host_api": "sfr_gpu_dif_assemble: u0 + diffusivity H2D, b + rCell D2H "
                        "(pageable numpy)"}


# algorithmic bytes per row of the ORTHOGONAL pressure-correction kernel
# (6 faces, CSRD full): row header 6, per face the plan words (12) and 9
# geometry doubles (72), the cell's own pres, gradpres, vel, dfield and
# material (10 doubles + 2), the writes of the diffusion kernel (156).
PRES_ALG_BYTES_PER_ROW = 6 + 6 * (12 + 72) + 82 + 6 * 20 + 36


def pressure_leg(np, torch, sv, s, n, peak, peak_kind):
    """systFormSimplePres on the device for the same mesh (lid-driven cavity
    loads, pressure fixed on x = 0, ORTHOGONAL, CSRD)."""
    st = torch.cuda.Stream()
    call, close = pres_call_setup(np, torch, sv, s, st.cuda_stream)
    dev_ms = time_calls(torch, call, st)
    close()
    alg = PRES_ALG_BYTES_PER_ROW * s.neq
    gbs = alg / (dev_ms * 1e-3) / 1e9
    tr = committed_traffic("pres_assemble_kernel")
    return {"workload": f"systFormSimplePres, {n}^3 = {s.neq} cells, cavity loads (static "
                        "walls, moving lid), pressure fixed on x=0, ORTHOGONAL, CSRD",
            "device_ms": dev_ms, "alg_bytes_per_row": PRES_ALG_BYTES_PER_ROW,
            "traffic": None if tr is None else tr[0] * (s.neq / 128 ** 3),
            "GB/s": gbs, "frac": gbs / peak, "peak_source": f"{peak_kind} hbm_gbs",
            "kernel": "pres_assemble_kernel<orthogonal, 6 faces, fused>"}


def vel_inputs(np, s):
    m = s.mesh()
    rng = np.random.default_rng(11)
    prop = np.zeros((1, 10))
    prop[0, :2] = (1e-3, 1.0)
    cc = m.xm[m.cellface[:, 0] - 1] - m.xmcc[:, 0, :]
    return m, prop, cc, dict(pres=rng.standard_normal(m.numel) * 1e-2,
                             gradpres=rng.standard_normal((m.numel, 3)) * 1e-2,
                             vel=rng.standard_normal((m.numel, 3)) * 0.1,
                             gradvel=rng.standard_normal((m.numel, 3, 3)) * 0.1,
                             dfield=np.ones((m.numel, 3)))


def vel_call_setup(np, torch, sv, s, stream):
    """A device systFormSimpleVel call on the system's mesh (lid-driven
    cavity loads, second-order face pressure, SIMPLE, Euler dt = 1e-2,
    under-relaxation 0.7, CSRD): (call, close)."""
    from sfr3d_b200 import assembly as A
    m, prop, cc, f = vel_inputs(np, s)
    g = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    plan = A.VelPlan(g, m, m.face_r(PRES_SIDES_VEL), cc)
    lvel = [A.Load(A.MOVEWALL, (1.0, 0.0, 0.0, 0.0)), A.Load(A.STATICWALL, ())]
    dev = {k: torch.tensor(np.ascontiguousarray(v), device="cuda") for k, v in f.items()}
    d_ad3 = torch.empty(3 * s.neq, dtype=torch.float64, device="cuda")
    d_b3 = torch.empty(3 * s.neq, dtype=torch.float64, device="cuda")
    d_r3 = torch.empty(3 * m.numel, dtype=torch.float64, device="cuda")

    def call():
        plan.assemble_device(lvel, prop, dev["pres"].data_ptr(), dev["gradpres"].data_ptr(),
                             dev["vel"].data_ptr(), dev["gradvel"].data_ptr(),
                             dev["dfield"].data_ptr(), d_ad3=d_ad3.data_ptr(),
                             d_b3=d_b3.data_ptr(), d_rcell3=d_r3.data_ptr(),
                             time=(0, 1e-2, 1e-2), stream=stream)

    def close():
        plan.close()
        g.close()
    return call, close


# algorithmic bytes per row of the momentum kernel (6 faces, CSRD full): row
# header 6, per face the plan words (8) and 19 geometry doubles (152), the
# cell's own pres, gradpres, vel, gradvel and material (16 doubles + 2), the
# writes: 6 off-diagonals, the u diagonal, 3 diagonals, 3 forces, 3 cell
# residuals and the D field (6 * 8 + 8 + 12 * 8).
VEL_ALG_BYTES_PER_ROW = 6 + 6 * 160 + 130 + 48 + 8 + 96


def momentum_assembly_leg(np, torch, sv, s, n, peak, peak_kind):
    """systFormSimpleVel on the device for the same mesh (the kernel writes
    the raw values; the solver-copy refresh follows as its own launches)."""
    st = torch.cuda.Stream()
    call, close = vel_call_setup(np, torch, sv, s, st.cuda_stream)
    dev_ms = time_calls(torch, call, st)
    close()
    alg = VEL_ALG_BYTES_PER_ROW * s.neq
    gbs = alg / (dev_ms * 1e-3) / 1e9
    return {"workload": f"systFormSimpleVel, {n}^3 = {s.neq} cells, cavity loads, laminar, "
                        "first-order upwind, second-order face pressure, SIMPLE, Euler, CSRD",
            "device_ms": dev_ms, "alg_bytes_per_row": VEL_ALG_BYTES_PER_ROW,
            "GB/s_incl_refresh": gbs, "frac_incl_refresh": gbs / peak,
            "peak_source": f"{peak_kind} hbm_gbs",
            "kernel": "vel_assemble_kernel<6 faces> + the gather/compensation refresh"}


# algorithmic bytes per cell of the least-squares gradient kernel (6 faces):
# per face the neighbour word (4) and the cell matrix's column for it (3
# doubles; xmcc and dcca are read on boundary faces only), the cell's face
# count and material (4), its own u (8 ndf; the neighbours' u come from
# cache) and the new gradient written (24 ndf; least squares starts from zero
# and does not read the previous one)
def grad_alg_bytes(ndf):
    return 6 * (4 + 24) + 4 + 8 * ndf + 24 * ndf


def gradient_inputs(np, s):
    """The cavity fields and face loads of a SIMPLE step: velocity (MOVEWALL
    lid, STATICWALL walls) and pressure (fixed on x = 0)."""
    from sfr3d_b200 import assembly as A
    m = s.mesh()
    rng = np.random.default_rng(13)
    prop = np.zeros((1, 10))
    prop[0, :2] = (1e-3, 1.0)
    vel = rng.standard_normal((m.numel, 3)) * 0.1
    pres = rng.standard_normal(m.numel) * 1e-2
    lvel = [A.Load(A.MOVEWALL, (1.0, 0.0, 0.0, 0.0)), A.Load(A.STATICWALL, ())]
    lpres = [A.Load(A.DIRICHLET, (0.0,))]
    return m, prop, vel, pres, lvel, lpres


def gradient_leg(np, torch, s, n, peak, peak_kind):
    """rcGradU on the device, least squares (the cavity deck's rcGrad): the
    velocity gradient (ndf 3) and the pressure gradient (ndf 1) of the same
    mesh, each on device arrays."""
    from sfr3d_b200 import assembly as A
    m, prop, vel, pres, lvel, lpres = gradient_inputs(np, s)
    out = {"workload": f"rcGradU least squares, {n}^3 = {m.numel} cells, cavity loads",
           "peak_source": f"{peak_kind} hbm_gbs",
           "kernel": "least_squares_kernel<ndf> (one thread a cell, 6 faces)"}
    st = torch.cuda.Stream()
    for name, sides, loads, u, ndf in (("velocity", PRES_SIDES_VEL, lvel, vel, 3),
                                       ("pressure", PRES_SIDES_PRES, lpres, pres, 1)):
        plan = A.GradPlan(m, m.face_r(sides), type=A.RCLSQUARE)
        du = torch.tensor(np.ascontiguousarray(u), device="cuda")
        dg = torch.zeros((m.numel, ndf, 3), dtype=torch.float64, device="cuda")
        ms = time_calls(torch, lambda: plan.grad_device(loads, prop, ndf, du.data_ptr(),
                                                        dg.data_ptr(), st.cuda_stream), st)
        plan.close()
        gbs = grad_alg_bytes(ndf) * m.numel / (ms * 1e-3) / 1e9
        out[name] = {"ndf": ndf, "device_ms": ms, "alg_bytes_per_cell": grad_alg_bytes(ndf),
                     "GB/s": gbs, "frac": gbs / peak}
    return out


def simple_step_leg(np, torch, sv, s, n):
    """The linear-algebra half of one SIMPLE iteration kept on the device:
    the velocity and pressure gradients (rcGradU, least squares), momentum
    assembly, the u, v, w BiCGSTAB solves in one batched launch, the
    pressure-correction assembly from the new D field, and its PCG solve
    (FP64 and mixed), with no host transfer between the steps."""
    from sfr3d_b200 import assembly as A
    m, prop, cc, f = vel_inputs(np, s)
    gvel_plan = A.GradPlan(m, m.face_r(PRES_SIDES_VEL), type=A.RCLSQUARE)
    gpres_plan = A.GradPlan(m, m.face_r(PRES_SIDES_PRES), type=A.RCLSQUARE)
    gv = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    gp = sv.GpuSystem(s.neq, s.ia, s.ja, sv.CSRD, True)
    vplan = A.VelPlan(gv, m, m.face_r(PRES_SIDES_VEL), cc)
    pplan = A.PresPlan(gp, m, m.face_r(PRES_SIDES_PRES), m.face_r(PRES_SIDES_VEL))
    lvel = [A.Load(A.MOVEWALL, (1.0, 0.0, 0.0, 0.0)), A.Load(A.STATICWALL, ())]
    lpres = [A.Load(A.DIRICHLET, (0.0,))]
    dev = {k: torch.tensor(np.ascontiguousarray(v), device="cuda") for k, v in f.items()}
    N = s.neq
    z = lambda k: torch.zeros(k, dtype=torch.float64, device="cuda")  # noqa: E731
    d_ad3, d_b3, d_x3, d_bp, d_xp = z(3 * N), z(3 * N), z(3 * N), z(N), z(N)
    st = torch.cuda.Stream()
    sp = st.cuda_stream
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
    out = {"workload": f"{n}^3 cavity: rcGradU (velocity, pressure; least squares) + "
                       "systFormSimpleVel + 3 momentum BiCGSTAB (one batched launch) + "
                       "systFormSimplePres from the new D + pressure PCG, to 1e-10, all on the "
                       "device"}
    for prec, tag in ((sv.FP64, "fp64"), (sv.MIXED, "mixed")):
        for rep in range(2):  # the second pass is timed (graphs built, clocks up)
            with torch.cuda.stream(st):
                ev[5].record(st)
                gvel_plan.grad_device(lvel, prop, 3, dev["vel"].data_ptr(),
                                      dev["gradvel"].data_ptr(), sp)
                gpres_plan.grad_device(lpres, prop, 1, dev["pres"].data_ptr(),
                                       dev["gradpres"].data_ptr(), sp)
                ev[0].record(st)
                vplan.assemble_device(lvel, prop, dev["pres"].data_ptr(),
                                      dev["gradpres"].data_ptr(), dev["vel"].data_ptr(),
                                      dev["gradvel"].data_ptr(), dev["dfield"].data_ptr(),
                                      d_ad3=d_ad3.data_ptr(), d_b3=d_b3.data_ptr(),
                                      fres=False, time=(0, 1e-2, 1e-2), calrcell=False,
                                      stream=sp)
                ev[1].record(st)
                iv = gv.solve_multi_device(sv.PBICGSTAB, 3, d_b3.data_ptr(), d_x3.data_ptr(),
                                           d_ad_k=d_ad3.data_ptr(), tol=1e-10, precision=prec,
                                           stream=sp)
                ev[2].record(st)
                pplan.assemble_device(lvel, lpres, np.array([[0.0, 1.0] + [0.0] * 8]),
                                      dev["pres"].data_ptr(), dev["gradpres"].data_ptr(),
                                      dev["vel"].data_ptr(), dev["dfield"].data_ptr(),
                                      d_b=d_bp.data_ptr(), calrcell=False, stream=sp)
                ev[3].record(st)
                ip = gp.solve_device(sv.PCG, d_bp.data_ptr(), d_xp.data_ptr(), tol=1e-10,
                                     precision=prec, stream=sp)
                ev[4].record(st)
            st.synchronize()
        t = [ev[i].elapsed_time(ev[i + 1]) for i in range(4)]
        tg = ev[5].elapsed_time(ev[0])
        out[tag] = {"total_ms": sum(t) + tg, "gradients_ms": tg, "momentum_assembly_ms": t[0],
                    "momentum_solves_ms": t[1], "pressure_assembly_ms": t[2],
                    "pressure_solve_ms": t[3], "momentum_iters": [i.iters for i in iv],
                    "pressure_iters": ip.iters,
                    "status": [i.status for i in iv] + [ip.status]}
    vplan.close()
    pplan.close()
    gvel_plan.close()
    gpres_plan.close()
    gv.close()
    gp.close()
    return out


def cpu_assembly(O, s):
    """The reference's own systFormDif (serial, as the reference runs it) on
    the assembly leg's workload."""
    import numpy as np
    m = s.mesh()
    rng = np.random.default_rng(9)
    case = O.DifCase(mesh=m, facer=m.face_r([1, 0, 0, 0, 0, 0]),
                     loads=[O.Load(O.DIRICHLET, (0.0,))], density=np.ones(m.numel),
                     cdiff=m.cdiff, u0=rng.standard_normal(m.numel),
                     gradu0=np.zeros((m.numel, 3)), icod=O.ORTHOGONAL)
    rc, *_, sec = O.ref_dif_assemble(case, O.CSRD, True, s.ia, s.ja, s.neq)
    m, prop, f = pres_inputs(np, s)
    pcase = O.PresCase(mesh=m, facevelr=m.face_r(PRES_SIDES_VEL),
                       facepresr=m.face_r(PRES_SIDES_PRES),
                       lvel=[O.Load(O.MOVEWALL, (1.0, 0.0, 0.0, 0.0)),
                             O.Load(O.STATICWALL, ())],
                       lpres=[O.Load(O.DIRICHLET, (0.0,))], prop=prop, **f)
    threads = os.cpu_count() or 1
    prc, *_, psec = O.ref_pres_assemble(pcase, O.CSRD, True, s.ia, s.ja, s.neq,
                                        nthreads=threads)
    m, prop, cc, f = vel_inputs(np, s)
    vcase = O.VelCase(mesh=m, cc=cc, facevelr=m.face_r(PRES_SIDES_VEL),
                      facepresr=m.face_r([0] * 6),
                      lvel=[O.Load(O.MOVEWALL, (1.0, 0.0, 0.0, 0.0)), O.Load(O.STATICWALL, ())],
                      prop=prop, time_flag=True, dt=1e-2, dt0=1e-2, **f)
    vrc, *_, vsec = O.ref_vel_assemble(vcase, O.CSRD, True, s.ia, s.ja, s.neq,
                                       nthreads=threads)
    # the same SIMPLE linear-algebra step on the host, the reference's way:
    # its own gradient reconstruction, assembly routines and OpenMP solvers
    t0 = time.perf_counter()
    _grc, gvel, _l, _s = O.ref_rc_grad(O.GradCase(
        mesh=m, facer=m.face_r(PRES_SIDES_VEL), loads=vcase.lvel, prop=prop, u=vcase.vel,
        gradu=np.zeros((m.numel, 3, 3)), type=O.RCLSQUARE), nthreads=threads)
    _grc, gpres, _l, _s = O.ref_rc_grad(O.GradCase(
        mesh=m, facer=m.face_r(PRES_SIDES_PRES), loads=pcase.lpres, prop=prop, u=vcase.pres,
        gradu=np.zeros((m.numel, 1, 3)), type=O.RCLSQUARE), nthreads=threads)
    vcase = O.VelCase(**{**vcase.__dict__, "gradvel": gvel, "gradpres": gpres.reshape(-1, 3)})
    vr = O.ref_vel_assemble(O.VelCase(**{**vcase.__dict__, "fres": False}), O.CSRD, True,
                            s.ia, s.ja, s.neq, nthreads=threads, calrcell=False)
    N = s.neq
    mom_iters = []
    for k in range(3):
        r = O.ref_solve(O.PBICGSTAB, O.CSRD, True, s.ia, s.ja, vr[1], vr[2][k * N:(k + 1) * N],
                        vr[3][k * N:(k + 1) * N], tol=1e-10, nthreads=threads)
        mom_iters.append(r.iters)
    pc2 = O.PresCase(**{**pcase.__dict__, "dfield": vr[5], "pres": vcase.pres,
                        "gradpres": gpres.reshape(-1, 3), "vel": vcase.vel})
    pr = O.ref_pres_assemble(pc2, O.CSRD, True, s.ia, s.ja, N, nthreads=threads, calrcell=False)
    rp = O.ref_solve(O.PCG, O.CSRD, True, s.ia, s.ja, pr[1], pr[2], pr[3], tol=1e-10,
                     nthreads=threads)
    step_ms = (time.perf_counter() - t0) * 1e3
    # the reference's rcGradU (least squares) on the same fields and loads
    m, gprop, gvel, gpres, _lv, _lp = gradient_inputs(np, s)
    grad_cpu = {"threads": threads,
                "sample": "one full rcGradU call (least squares) with its OpenMP cell loop "
                          "on all host threads"}
    for name, sides, loads, u, ndf in (
            ("velocity", PRES_SIDES_VEL,
             [O.Load(O.MOVEWALL, (1.0, 0.0, 0.0, 0.0)), O.Load(O.STATICWALL, ())], gvel, 3),
            ("pressure", PRES_SIDES_PRES, [O.Load(O.DIRICHLET, (0.0,))], gpres, 1)):
        gcase = O.GradCase(mesh=m, facer=m.face_r(sides), loads=loads, prop=gprop, u=u,
                           gradu=np.zeros((m.numel, ndf, 3)), type=O.RCLSQUARE)
        grc, _g, _lsq, gsec = O.ref_rc_grad(gcase, nthreads=threads)
        grad_cpu[name] = {"ms": gsec * 1e3, "status": grc}
    return {"ms": sec * 1e3, "threads": 1, "status": rc,
            "simple_step": {"ms": step_ms, "threads": threads, "momentum_iters": mom_iters,
                            "pressure_iters": rp.iters, "status": [vr[0], pr[0], rp.status],
                            "sample": "rcGradU (velocity, pressure) + systFormSimpleVel + 3 "
                                      "pbicgstabOmp + systFormSimplePres + pcgOmp, the device "
                                      "step's inputs"},
            "sample": "one full systFormDif call (the reference's loop is serial)",
            "pressure": {"ms": psec * 1e3, "threads": threads, "status": prc,
                         "sample": "one full systFormSimplePres call with its OpenMP cell "
                                   "loop on all host threads"},
            "momentum": {"ms": vsec * 1e3, "threads": threads, "status": vrc,
                         "sample": "one full systFormSimpleVel call with its OpenMP cell "
                                   "loop on all host threads"},
            "gradient": grad_cpu}


def adjoint_leg(np, sv, S):
    """Adjoint of the 96^3 Peclet-20 momentum system, J = w.x: transpose
    solve time (FP64 and mixed) and the largest relative difference to
    central differences on 32 coefficients + 32 right-hand-side entries."""
    from sfr3d_b200 import adjoint as A
    m = S.momentum(96, peclet=20.0, nrhs=1, seed=5)
    g = sv.GpuSystem(m.neq, m.ia, m.ja, sv.CSRD, True)
    g.set_values(m.al, m.ad)
    w = np.random.default_rng(5).standard_normal(m.neq)
    x, _ = g.solve(sv.PBICGSTAB, m.b[0], tol=1e-14, maxit=5000, raise_on_error=False)
    rng = np.random.default_rng(5)
    nz = np.flatnonzero(m.al != 0.0)
    ent = [A.Entry("al", int(k), A.value_positions(g, m.ia, m.ja, "al", int(k)))
           for k in rng.choice(nz, 24, replace=False)]
    ent += [A.Entry("ad", int(i), [(int(i), int(i))]) for i in rng.choice(m.neq, 8, replace=False)]
    ent += [A.Entry("b", int(i), []) for i in rng.choice(m.neq, 32, replace=False)]
    fd = A.central_differences(g, sv.PBICGSTAB, m.al, m.ad, None, m.b[0], x, w, ent,
                               rel_step=1e-6, tol=1e-13, maxit=5000)
    out = {"workload": "momentum 96^3 Peclet 20, J = w.x, w ~ N(0,1)"}
    for name, prec, tol in (("fp64", sv.FP64, 1e-12), ("mixed", sv.MIXED, 1e-10)):
        g.adjoint(sv.PBICGSTAB, x, w, tol=tol, precision=prec)
        lam, g_al, g_ad, _, info = g.adjoint(sv.PBICGSTAB, x, w, tol=tol, precision=prec)
        arrays = {"al": g_al, "ad": g_ad, "b": lam}
        adj = np.array([arrays[e.array][e.index] for e in ent])
        out[name] = {"transpose_solve_ms": info.seconds * 1e3, "iters": info.iters,
                     "tol": tol,
                     "max_rel_err_vs_central_diff": float(np.max(np.abs(adj - fd) / np.abs(fd)))}
    g.close()
    return out


def cpu_other_krylov(O, s, n, threads):
    """The reference's own BiCGSTAB(2), GMRES(15) (OpenMP variants) and MINRES
    (serial: its OpenMP branch is commented out in callMinRes) on the
    other_krylov workloads: per-iteration time from a bounded sample."""
    from sfr3d_b200 import systems as S
    m = S.momentum(n, nrhs=1, seed=3)
    il, jl, al = s.csrd_lower()
    out = {}
    for name, args, solver, maxit, nth in (
            ("minres_pressure", (O.CSRC, False, il, jl, al, s.ad, s.b[0]), O.MINRES, 100, 0),
            ("bicgstabl2_momentum", (O.CSRD, True, m.ia, m.ja, m.al, m.ad, m.b[0]),
             O.PBICGSTABL2, 100000, threads),
            ("gmres15_momentum", (O.CSRD, True, m.ia, m.ja, m.al, m.ad, m.b[0]),
             O.GMRES, 100000, threads)):
        r = O.ref_solve(solver, *args, tol=1e-10, maxit=maxit, nthreads=nth)
        # MINRES only warns at maxIt and reports maxIt + 1 iterations
        it = maxit if (solver == O.MINRES and r.iters > maxit) else r.iters
        out[name] = {"ms_per_iteration": r.seconds / max(it, 1) * 1e3, "threads": max(nth, 1),
                     "sample": ("full solve" if r.iters <= maxit else f"{maxit} iterations"),
                     "iters": r.iters}
    return out


def cpu_baseline(s, iters_full, n, xs_gpu=None):
    """The reference's pcgOmp on the bench system (cpu_pcg_baseline), plus
    its other Krylov methods on the other_krylov workloads.  xs_gpu: the
    GPU's solutions ({"fp64": x, "mixed": x}), whose error against the
    reference's solution is reported (computed outside every timed region)."""
    res = cpu_pcg_baseline(s, iters_full, xs_gpu)
    if "unavailable" not in res:
        from oracle import oracle as O
        res["other_krylov"] = cpu_other_krylov(O, s, n, res["cores"])
        res["assembly"] = cpu_assembly(O, s)
    return res


def cpu_pcg_baseline(s, iters_full, xs_gpu=None):
    """The reference's own pcgOmp (Cg.c:490) with all host threads on the
    same system in CSRC symmetric storage (the reference's default): a full
    solve when one takes under 30 s, else a bounded sample scaled to the
    full iteration count."""
    try:
        from oracle import oracle as O
    except Exception as e:  # pragma: no cover
        return {"unavailable": f"oracle not importable: {e}"}
    if not O.ref_available():
        return {"unavailable": "oracle/_ref/libsfr3d_ref.so not built"}
    threads = os.cpu_count() or 1
    il, jl, al = s.csrd_lower()
    probe = O.ref_solve(O.PCG, O.CSRC, False, il, jl, al, s.ad, s.b[0], tol=1e-10,
                        maxit=100, nthreads=threads)
    per_it = probe.seconds / 100
    if per_it * iters_full < 30:
        r = O.ref_solve(O.PCG, O.CSRC, False, il, jl, al, s.ad, s.b[0], tol=1e-10,
                        maxit=100000, nthreads=threads)
        out = {"value": r.seconds * 1e3, "unit": "ms", "cores": threads, "kind": "reference",
               "sample": f"one full pcgOmp solve (CSRC symmetric, {threads} threads), "
                         f"{r.iters} iterations",
               "ms_per_iteration": r.seconds / r.iters * 1e3,
               "iterations": r.iters}
        if xs_gpu:
            import numpy as np
            nref = float(np.linalg.norm(r.x))
            out["err_vs_oracle_x"] = {
                k: float(np.linalg.norm(v - r.x) / nref) for k, v in xs_gpu.items()}
            out["err_vs_oracle_x"]["what"] = ("||x_gpu - x_ref||_2 / ||x_ref||_2 against this "
                                              "pcgOmp solve; FP64 bar 1e-12")
        return out
    n_it = max(100, int(30 / per_it))
    r = O.ref_solve(O.PCG, O.CSRC, False, il, jl, al, s.ad, s.b[0], tol=1e-10,
                    maxit=n_it, nthreads=threads)
    per_it = r.seconds / n_it
    return {"value": per_it * iters_full * 1e3, "unit": "ms", "cores": threads,
            "kind": "reference",
            "sample": f"{n_it} pcgOmp iterations (CSRC symmetric, {threads} threads), "
                      f"scaled to the full solve's {iters_full} iterations",
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
            "higher_is_better": False,
            "scaling": "strong" if world > 1 and not args.replicas else "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
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
