"""The C-ABI library loads and exports every entry point include/adgpu_b200.h
declares, plus the reference's C++-linkage kernel API names; layout structs
match the reference's sizes.  No device calls."""
import ctypes as C
import os
import re
import subprocess

import pytest

from adgpu_b200 import abi, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "adgpu_b200.h")

# host/src/performdocking.cpp.Cuda:40-84, mangled as the reference host objects reference them
REFERENCE_CXX_SYMBOLS = [
    "_Z17SetKernelsGpuDataP7GpuData",
    "_Z17GetKernelsGpuDataP7GpuData",
    "_Z16gpu_calc_initpopjjPfS_",
    "_Z13gpu_sum_evalsjj",
    "_Z24gpu_gen_and_eval_newpopsjjPfS_S_S_",
    "_Z14gpu_perform_LSjjPfS_",
    "_Z18gpu_gradient_minADjjPfS_",
    "_Z20gpu_gradient_minAdamjjPfS_",
]


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:adgpu_status|const char\*|void|int)\s+(adgpu_\w+)\s*\(", text, re.M)))


def test_library_loads_and_exports_header_symbols():
    L = lib.load()
    decl = declared_symbols()
    assert len(decl) >= 12
    for name in decl:
        assert hasattr(L, name), name
    assert set(decl) <= set(lib.exported_symbols())
    assert L.adgpu_version().decode().startswith("adgpu_b200")


def test_reference_cxx_names_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", lib.LIB_PATH], capture_output=True, text=True).stdout
    for s in REFERENCE_CXX_SYMBOLS:
        assert re.search(rf"\sT\s{re.escape(s)}$", out, re.M), s


def test_layout_sizes_match_reference():
    # sizes of the reference structs (host/inc/calcenergy.h:88-136, cuda/GpuData.h:74-136)
    assert C.sizeof(abi.Dockpars) == 34 * 4
    assert C.sizeof(abi.KcInterintra) == 256 * (4 + 4 + 4 + 1)
    assert C.sizeof(abi.KcIntracontrib) == 2 * 256 * 256 * 4
    assert C.sizeof(abi.KcIntra) == 32 * 4 + 32 * 32 * 2 + 3 * 32 * 32 * 4 + 2 * 32 * 4
    assert C.sizeof(abi.KcRotlist) == 256 * 57 * 4
    assert C.sizeof(abi.KcConform) == (3 * 256 + 6 * 57) * 4
    assert C.sizeof(abi.KcGrads) == (2 * 57 + 256 * 57 + 57) * 4


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libadgpu_ref.so")),
                    reason="oracle/_ref not built")
def test_gpudata_matches_reference_gpudata():
    from oracle import refpy
    assert refpy.lib().adgpu_ref_sizeof_gpudata() == C.sizeof(abi.GpuData)
    assert refpy.lib().adgpu_ref_sizeof_refgpudata() == C.sizeof(abi.GpuData)


def test_errors_without_set_data():
    # a call before adgpu_set_kernels_gpu_data reports NOT_READY (no device work)
    L = lib.load()
    st = L.adgpu_sum_evals(1, 64)
    assert st == 3
    assert b"not called" in L.adgpu_last_error()


DROPIN = os.path.join(ROOT, "oracle", "_ref", "autodock_gpu_b200")


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="reference host program not built (make -C oracle dropin)")
def test_reference_host_program_binds_the_library():
    """The reference's host program, built from its own sources, takes the
    kernel API from libadgpu_b200.so: the seven kernel-API names are
    undefined in the program and resolve to this library."""
    und = subprocess.run(["nm", "-D", "--undefined-only", DROPIN], capture_output=True, text=True).stdout
    for s in REFERENCE_CXX_SYMBOLS:
        if s.startswith("_Z17GetKernelsGpuData"):
            continue            # the host program never calls it
        assert s in und, s
    deps = subprocess.run(["ldd", DROPIN], capture_output=True, text=True).stdout
    assert os.path.realpath(lib.LIB_PATH) in {os.path.realpath(p.split("=>")[1].split("(")[0].strip())
                                              for p in deps.splitlines() if "libadgpu_b200" in p}
