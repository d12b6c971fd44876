"""Build libbbpd (CUDA, sm_100a) and the mexFunction gateways in-tree.

    python -m bb_pd_b200.build          # or __graft_entry__.build()

Outputs (git-ignored, shipped with the source tree):
    bb_pd_b200/lib/libbbpd.so           the C-ABI library (include/bbpd.h)
    bb_pd_b200/mex/<Name>.mexa64        one gateway per reference MEX routine,
                                        compiled against the stub mex.h here;
                                        with MATLAB, compile mex_gateways.c with
                                        `mex -DGW_<Name> mex_gateways.c -lbbpd`
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
MEXDIR = os.path.join(HERE, "mex")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CUDA_SOURCES = ["common.cu", "routines.cu", "solver.cu", "selftest.cu", "damping_noalloc.cu", "builder.cu",
                "static.cu", "beam.cpp"]

# Gateways: (output name, gateway macro). Names are the reference MEX files.
GATEWAYS = [
    "calculatedeformedlengthMex",
    "calculatebsfexponentialMex",
    "calculatebondforcesMex",
    "calculatenodalforcesopenmpMex",
    "calculatenodalforcesMex",
    "timeintegrationeulercromerMex",
    "calculatebondfailureMex",
]


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _newer(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def build_lib(force: bool = False, out: str | None = None) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    out = out or os.path.join(LIBDIR, "libbbpd.so")
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".cpp", ".h"))]
    deps.append(os.path.join(INCLUDE, "bbpd.h"))
    if not force and _newer(out, deps):
        return out
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17",
           # no fused multiply-add in device code: every double operation rounds
           # like the reference's x86-64 code (bit-identical results)
           "-fmad=false",
           "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
           "-Xptxas", "-v" if os.environ.get("BBPD_PTXAS_VERBOSE") else "-O3",
           "-I", INCLUDE, "-I", CSRC,
           "-shared", "-cudart", "static", "-o", out]
    cmd += [f"-D{d}" for d in os.environ.get("BBPD_DEFINES", "").split()]
    cmd += [os.path.join(CSRC, f) for f in CUDA_SOURCES]
    cmd += ["-lpthread"]
    _run(cmd)
    return out


def build_gateways(force: bool = False) -> list[str]:
    os.makedirs(MEXDIR, exist_ok=True)
    src = os.path.join(CSRC, "mex_gateways.c")
    lib = os.path.join(LIBDIR, "libbbpd.so")
    outs = []
    cc = shutil.which("gcc") or "gcc"
    for name in GATEWAYS:
        out = os.path.join(MEXDIR, name + ".mexa64")
        outs.append(out)
        if not force and _newer(out, [src, lib, os.path.join(INCLUDE, "bbpd.h")]):
            continue
        _run([cc, "-O2", "-fPIC", "-shared", "-ffp-contract=off", f"-DGW_{name}",
              "-I", INCLUDE, "-I", os.path.join(CSRC, "mexstub"),
              "-o", out, src, "-L", LIBDIR, "-lbbpd", "-Wl,-rpath,$ORIGIN/../lib"])
    return outs


def build(force: bool = False) -> None:
    build_lib(force)
    build_gateways(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
