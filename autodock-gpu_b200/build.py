"""Builds libadgpu_b200.so in-tree for sm_100a (nvcc), plus the oracle
libraries used by the test suite (oracle/Makefile).

    python autodock-gpu_b200/build.py [--no-oracle]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib", "libadgpu_b200.so")
# bench-only: the FP32 FMA peak probe (csrc/probe), not part of the product library
PROBE_OUT = os.path.join(HERE, "lib", "libadgpu_probe.so")
PROBE_SRC = os.path.join(CSRC, "probe", "fp32_peak.cu")
SOURCES = ["adgpu_api.cu", "adgpu_tables.cu", "adgpu_engine.cu", "adgpu_compat.cu", "adgpu_prep.cpp", "adgpu_frontend.cpp", "adgpu_noalloc.cu", "adgpu_pipeline.cu"]
# Flushed single-precision denormals: part of the -use_fast_math the
# reference builds its CUDA kernels with (Makefile.Cuda:97-103); it takes 7%
# off a scoring (B200, 45 atoms, 777 pairs).  Division, square root and
# sin/cos stay correctly rounded: the fast sin/cos move clashing atoms enough
# to change r^-12 terms by more than 1e-4, and FIRE's step control branches on
# norms.  The front end and the table repacks are host code or use explicitly
# rounded intrinsics.
NVCC_FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-ftz=true",
              "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-warn-spills"]
# Result processing restates the reference's host arithmetic operation by
# operation, so it keeps IEEE denormals and rounds every product and sum
# separately (no fused multiply-add), as the host code does.
IEEE_SOURCES = ["adgpu_result.cu"]
NVCC_FLAGS_IEEE = [f for f in NVCC_FLAGS if f not in ("-ftz=true", "-shared")] + ["-ftz=false", "-fmad=false"]
OBJ_DIR = os.path.join(HERE, "_build")


def nvcc() -> str:
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.exists(p) or p == "nvcc"):
            return p
    return "nvcc"


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def _run(cmd, verbose):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed building libadgpu_b200.so")


def needs_rebuild() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "adgpu_b200.h"),
                                                                 os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_rebuild():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    objs = []
    for src in IEEE_SOURCES:
        obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
        _run([nvcc()] + NVCC_FLAGS_IEEE + ["-c", "-o", obj, os.path.join(CSRC, src)], verbose)
        objs.append(obj)
    _run([nvcc()] + NVCC_FLAGS + ["-o", OUT] + sources() + objs + ["-lcudart"], verbose)
    return OUT


def build_probe(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(PROBE_OUT) and os.path.getmtime(PROBE_OUT) > os.path.getmtime(PROBE_SRC):
        return PROBE_OUT
    os.makedirs(os.path.dirname(PROBE_OUT), exist_ok=True)
    flags = [f for f in NVCC_FLAGS if f != "-ftz=true"]
    _run([nvcc()] + flags + ["-o", PROBE_OUT, PROBE_SRC, "-lcudart"], verbose)
    return PROBE_OUT


def build_oracle() -> None:
    """The oracle libraries; oracle/_ref and the drop-in programs only where the
    reference checkout is present (ADGPU_REFERENCE, default: the checkout this
    build was made against)."""
    ref = os.environ.get("ADGPU_REFERENCE", "/root/reference")
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all", "-j8", f"REF={ref}"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        sys.stdout.write(r.stdout)
        sys.stderr.write(r.stderr)
        raise RuntimeError("oracle build failed")


if __name__ == "__main__":
    build_lib(force="--force" in sys.argv, verbose=True)
    build_probe(force="--force" in sys.argv, verbose=True)
    if "--no-oracle" not in sys.argv:
        build_oracle()
    print(OUT)
