"""In-tree build of the native libraries.

    python -m sfr3d_b200.build            # libsfr3d_b200.so + libsfr3d_systems.so
    python -m sfr3d_b200.build --ptxas    # also print -Xptxas -v resource usage

The CUDA library is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) with the CUDA runtime linked
statically, so the .so carries no dependence on the runtime that torch
bundles.  Objects go to sfr3d_b200/_build/, the .so files next to this file.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CUDA_SOURCES = ["krylov.cu", "mixed.cu", "stream_solve.cu", "batched.cu", "device_mem.cu", "halo.cu",
                "noalloc.cu", "adjoint.cu", "resident.cu", "krylov_ext.cu",
                "assembly.cu", "minres_graph.cu", "bicgl2_graph.cu", "gmres_graph.cu",
                "gradient.cu"]
HOST_SOURCES = ["capi.cpp", "sell_build.cpp", "partition.cpp", "autotune.cpp"]
SYSTEM_SOURCES = ["systems.cpp"]

LIB = os.path.join(HERE, "libsfr3d_b200.so")
SYSLIB = os.path.join(HERE, "libsfr3d_systems.so")


def _nccl_include() -> list[str]:
    # nccl.h of the NCCL that torch loads (the library itself is opened at
    # run time); the system header otherwise
    try:
        import nvidia.nccl as _n  # noqa: PLC0415
        for base in _n.__path__:
            inc = os.path.join(base, "include")
            if os.path.exists(os.path.join(inc, "nccl.h")):
                return ["-I", inc]
    except ImportError:
        pass
    return []


def _host_cxx() -> str:
    # the system g++ (the environment's CC/CXX wrappers may lack runtime specs)
    return shutil.which("g++") or "g++"


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
          if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    if r.stderr.strip() and ("-Xptxas" in cmd):
        sys.stderr.write(r.stderr)


def _compile(src: str, ptxas: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    deps = [src] + _headers() + [__file__]
    if not _newer(obj, deps) and not ptxas:
        return obj
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17",
           "-ccbin", _host_cxx(), "-Xcompiler", "-fPIC,-O2",
           "--expt-relaxed-constexpr", "--extended-lambda",
           "-I", INCLUDE, "-I", CSRC, *_nccl_include(), "-c", src, "-o", obj]
    if ptxas and src.endswith(".cu"):
        cmd.insert(1, "-Xptxas")
        cmd.insert(2, "-v")
    _run(cmd)
    return obj


def build_cuda(ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(CSRC, f) for f in CUDA_SOURCES + HOST_SOURCES]
    srcs = [s for s in srcs if os.path.exists(s)]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, ptxas), srcs))
    if _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-ccbin", _host_cxx(),
              *objs, "-ldl", "-o", LIB + ".tmp"])
        os.replace(LIB + ".tmp", LIB)
    return LIB


def build_systems() -> str:
    srcs = [os.path.join(CSRC, f) for f in SYSTEM_SOURCES]
    if _newer(SYSLIB, srcs + _headers() + [__file__]):
        _run([_host_cxx(), "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall",
              "-I", INCLUDE, *srcs, "-o", SYSLIB + ".tmp"])
        os.replace(SYSLIB + ".tmp", SYSLIB)
    return SYSLIB


def build_all(ptxas: bool = False) -> None:
    build_systems()
    build_cuda(ptxas)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ptxas", action="store_true")
    args = ap.parse_args(argv)
    build_all(args.ptxas)
    print(LIB)
    print(SYSLIB)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
