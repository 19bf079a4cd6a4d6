"""ctypes bindings of oracle/liboracle.so, the C restatement of the reference's
hot path (oracle/adgpu_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline leg; never by the product.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_PKG = os.path.join(os.path.dirname(HERE), "autodock-gpu_b200")
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)
from adgpu_b200 import abi  # noqa: E402  (layout structs only)

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle oracle)")
        L = C.CDLL(LIB_PATH)
        vp, u32, i = C.c_void_p, C.c_uint32, C.c_int
        L.oracle_score.argtypes = [vp, vp, vp, vp, vp]
        L.oracle_score_batch.argtypes = [vp, u32, vp, vp, vp, i]
        L.oracle_calc_initpop.argtypes = [vp, u32, vp, vp, i]
        L.oracle_sum_evals.argtypes = [vp, u32]
        L.oracle_gen_and_eval_newpops.argtypes = [vp, u32, u32, vp, vp, vp, vp, i]
        for n in ("perform_ls", "gradient_minad", "gradient_minadam", "gradient_minfire"):
            getattr(L, f"oracle_{n}").argtypes = [vp, u32, u32, vp, vp, i]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class HostTables:
    """Reference-layout tables in host memory plus a GpuData pointing at them."""

    def __init__(self, tables: dict, dockpars: abi.Dockpars, grid: np.ndarray):
        self.t = {k: np.ascontiguousarray(v).view(np.uint8).copy() for k, v in tables.items()}
        self.grid = np.ascontiguousarray(grid, dtype=np.float32)
        self.g = abi.GpuData()
        self.g.dockpars = dockpars.copy()
        for k, attr in (("interintra", "pKerconst_interintra"), ("intracontrib", "pKerconst_intracontrib"),
                        ("intra", "pKerconst_intra"), ("rotlist", "pKerconst_rotlist"),
                        ("conform", "pKerconst_conform"), ("grads", "pKerconst_grads")):
            setattr(self.g, attr, self.t[k].ctypes.data)
        off = abi.table_offsets()
        base = self.t["grads"].ctypes.data
        self.g.pMem_rotbonds_const = base + off["rotbonds"]
        self.g.pMem_rotbonds_atoms_const = base + off["rotbonds_atoms"]
        self.g.pMem_num_rotating_atoms_per_rotbond_const = base + off["num_rotating_atoms_per_rotbond"]
        self.g.pMem_fgrids = self.grid.ctypes.data
        self.g.warpmask, self.g.warpbits = 31, 5
        self._state = []

    @property
    def dockpars(self) -> abi.Dockpars:
        return self.g.dockpars

    def bind_state(self, prng: np.ndarray, evals_new: np.ndarray, evals_runs: np.ndarray):
        self._state = [prng, evals_new, evals_runs]
        self.g.pMem_prng_states = prng.ctypes.data
        self.g.pMem_evals_of_new_entities = evals_new.ctypes.data
        self.g.pMem_gpu_evals_of_runs = evals_runs.ctypes.data

    def ptr(self):
        return C.cast(C.pointer(self.g), C.c_void_p)

    # ---- oracle calls ----
    def score(self, genotypes: np.ndarray, gradients: bool, nthreads: int = 1):
        g = np.ascontiguousarray(genotypes, dtype=np.float32)
        n = g.shape[0]
        e = np.zeros(n, np.float32)
        gr = np.zeros((n, abi.GENOTYPE_STRIDE), np.float32) if gradients else None
        lib().oracle_score_batch(self.ptr(), n, _p(g), _p(e), _p(gr), nthreads)
        return (e, gr) if gradients else e

    def score_terms(self, genotype: np.ndarray):
        g = np.ascontiguousarray(genotype, dtype=np.float32).reshape(-1)
        e = np.zeros(1, np.float32)
        gr = np.zeros(abi.GENOTYPE_STRIDE, np.float32)
        terms = np.zeros(8, np.float32)
        lib().oracle_score(self.ptr(), _p(g), _p(e), _p(gr), _p(terms))
        return float(e[0]), gr, terms

    def call(self, name, *args):
        conv = [(_p(a) if isinstance(a, np.ndarray) else a) for a in args]
        return getattr(lib(), f"oracle_{name}")(self.ptr(), *conv)


def tables_from_refjob(job) -> HostTables:
    """HostTables built from an oracle.refpy.RefJob (reference-prepared inputs)."""
    tabs = {k: job.blob(k) for k in ("interintra", "intracontrib", "intra", "rotlist", "conform", "grads")}
    dp = abi.Dockpars.from_bytes(job.blob("dockpars"))
    return HostTables(tabs, dp, job.blob("grid"))
