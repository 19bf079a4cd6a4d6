"""ctypes binding of libadgpu_b200.so (the C ABI in include/adgpu_b200.h).

The shared library is built in-tree (``build.py``); there is no fallback: if
the library is missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libadgpu_b200.so")

# Every symbol declared in include/adgpu_b200.h, with (restype, argtypes).
_vp, _u32, _u64, _i = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
SIGNATURES = {
    "adgpu_set_kernels_gpu_data": (_i, [_vp]),
    "adgpu_get_kernels_gpu_data": (_i, [_vp]),
    "adgpu_calc_initpop": (_i, [_u32, _u32, _vp, _vp]),
    "adgpu_sum_evals": (_i, [_u32, _u32]),
    "adgpu_gen_and_eval_newpops": (_i, [_u32, _u32, _vp, _vp, _vp, _vp]),
    "adgpu_perform_ls": (_i, [_u32, _u32, _vp, _vp]),
    "adgpu_gradient_minad": (_i, [_u32, _u32, _vp, _vp]),
    "adgpu_gradient_minadam": (_i, [_u32, _u32, _vp, _vp]),
    "adgpu_gradient_minfire": (_i, [_u32, _u32, _vp, _vp]),
    "adgpu_score_genotypes": (_i, [_u32, _vp, _vp, _vp]),
    "adgpu_score_terms": (_i, [_u32, _vp, _vp, _vp]),
    "adgpu_score_genotypes_noalloc": (_i, [_vp, _u32, _vp, _vp, _vp]),
    "adgpu_dock_resident": (_i, [_i, _u32, _u64, _u32, _vp, _vp, _vp, _vp, _vp, _vp]),
    "adgpu_dock_resident_autostop": (_i, [_i, _u32, _u64, _u32, _u32, C.c_float, _u64,
                                          _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "adgpu_dock_stats_get": (_i, [_vp]),
    "adgpu_grid_read": (_i, [C.c_char_p, _vp]),
    "adgpu_grid_from_values": (_i, [_vp, C.c_double, _vp, _i, _vp, _vp, _vp]),
    "adgpu_grid_free": (None, [_vp]),
    "adgpu_grid_save": (_i, [_vp, C.c_char_p]),
    "adgpu_grid_load": (_i, [C.c_char_p, _vp]),
    "adgpu_ligand_prepare_batch": (_i, [_vp, _vp, _vp, C.c_uint32, _vp, _vp, _i, _i, _vp, _vp]),
    "adgpu_grid_info": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "adgpu_grid_reference_layout": (_i, [_vp, _vp, C.c_size_t]),
    "adgpu_dockpars_default": (_i, [_vp, C.c_double, _i]),
    "adgpu_ligand_prepare": (_i, [_vp, C.c_char_p, C.c_char_p, _vp, _vp, _i, _vp]),
    "adgpu_ligand_free": (None, [_vp]),
    "adgpu_ligand_tables": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "adgpu_ligand_population": (_i, [_vp, _vp, C.c_size_t, _vp, C.c_size_t]),
    "adgpu_last_error": (C.c_char_p, []),
    "adgpu_version": (C.c_char_p, []),
}

_lib = None


class AdgpuError(RuntimeError):
    pass


def load():
    """Loads the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise AdgpuError(f"{LIB_PATH} is missing: build it with `python autodock-gpu_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(SIGNATURES)


def check(status: int, what: str = ""):
    if status != 0:
        msg = load().adgpu_last_error().decode()
        raise AdgpuError(f"{what}: {abi.STATUS.get(status, status)}: {msg}")


def call(name: str, *args):
    conv = []
    for a in args:
        if hasattr(a, "data_ptr"):
            conv.append(C.c_void_p(a.data_ptr()))
        elif isinstance(a, np.ndarray):
            conv.append(a.ctypes.data_as(C.c_void_p))
        else:
            conv.append(a)
    st = getattr(load(), name)(*conv)
    check(st, name)
    return st
