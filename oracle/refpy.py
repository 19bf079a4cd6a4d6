"""ctypes bindings of oracle/_ref/libadgpu_ref.so -- the reference's own host
front end and CUDA kernel sources, compiled for the CPU (see oracle/Makefile).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline leg; never by the product.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libadgpu_ref.so")

GENOTYPE_STRIDE = 64
NUM_THREADS = 64      # the reference build this oracle emulates (-DN64WI)


class RefInfo(C.Structure):
    _fields_ = [
        ("num_of_atoms", C.c_int), ("true_ligand_atoms", C.c_int), ("num_of_rotbonds", C.c_int),
        ("num_of_genes", C.c_int), ("num_of_intraE_contributors", C.c_int), ("num_of_rotcyc", C.c_int),
        ("pop_size", C.c_int), ("num_of_runs", C.c_int), ("num_of_lsentities", C.c_int),
        ("num_of_map_atypes", C.c_int), ("gridsize", C.c_int * 3), ("spacing", C.c_float),
        ("grid_origin", C.c_float * 3), ("nev", C.c_ulong), ("ngen", C.c_ulong), ("lsmet", C.c_char * 8),
    ]


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle ref)")
        L = C.CDLL(LIB_PATH)
        L.adgpu_ref_job_create.restype = C.c_void_p
        L.adgpu_ref_job_create.argtypes = [C.c_int, C.POINTER(C.c_char_p)]
        L.adgpu_ref_job_free.argtypes = [C.c_void_p]
        L.adgpu_ref_job_info.argtypes = [C.c_void_p, C.POINTER(RefInfo)]
        L.adgpu_ref_job_blob.restype = C.c_void_p
        L.adgpu_ref_job_blob.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_size_t)]
        L.adgpu_ref_job_bind.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.adgpu_ref_sizeof_gpudata.restype = C.c_size_t
        L.adgpu_ref_sizeof_refgpudata.restype = C.c_size_t
        vp = C.c_void_p
        L.adgpu_ref_score.argtypes = [C.c_uint32, C.c_uint32, vp, vp, vp]
        L.adgpu_ref_calc_initpop.argtypes = [C.c_uint32, C.c_uint32, vp, vp]
        L.adgpu_ref_sum_evals.argtypes = [C.c_uint32, C.c_uint32]
        L.adgpu_ref_gen_and_eval_newpops.argtypes = [C.c_uint32, C.c_uint32, vp, vp, vp, vp]
        for n in ("perform_ls", "gradient_minad", "gradient_minadam"):
            getattr(L, f"adgpu_ref_{n}").argtypes = [C.c_uint32, C.c_uint32, vp, vp]
        L.adgpu_ref_fire.argtypes = [vp, C.c_uint32, C.c_uint32, vp, vp]
        L.adgpu_ref_get_gpudata.argtypes = [vp]
        L.adgpu_ref_ocl_score.argtypes = [vp, C.c_uint32, vp, vp, vp]
        L.adgpu_ref_autostop_new.restype = vp
        L.adgpu_ref_autostop_new.argtypes = [C.c_int, C.c_int, C.c_float, C.c_int]
        L.adgpu_ref_autostop_check.restype = C.c_int
        L.adgpu_ref_autostop_check.argtypes = [vp, C.c_int, vp, C.c_ulong]
        L.adgpu_ref_autostop_free.argtypes = [vp]
        L.adgpu_ref_process_result.argtypes = [vp, vp, vp, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int, vp, vp, vp]
        L.adgpu_ref_rescore.argtypes = [vp, vp, C.c_int, C.c_int, vp]
        L.adgpu_ref_read_grid.restype = C.c_long
        L.adgpu_ref_read_grid.argtypes = [C.c_char_p]
        _lib = L
    return _lib


class RefAutoStop:
    """The reference's own AutoStop object (host/inc/autostop.hpp, compiled
    into _ref/libadgpu_ref.so by ref/ref_autostop.cpp)."""

    def __init__(self, pop_size: int, num_runs: int, stopstd: float, as_frequency: int):
        self.h = lib().adgpu_ref_autostop_new(pop_size, num_runs, stopstd, as_frequency)

    def check(self, generation: int, energies: np.ndarray, total_evals: int) -> bool:
        e = np.ascontiguousarray(energies, np.float32)
        return bool(lib().adgpu_ref_autostop_check(self.h, generation, e.ctypes.data_as(C.c_void_p), total_evals))

    def __del__(self):
        if getattr(self, "h", None):
            lib().adgpu_ref_autostop_free(self.h)
            self.h = None


class RefRunResult(C.Structure):
    """One run's Ligandresult fields (host/inc/processresult.h:40-58)."""
    _fields_ = [("inter_e", C.c_float), ("interflex_e", C.c_float), ("inter_e_elec", C.c_float),
                ("intra_e", C.c_float), ("intraflex_e", C.c_float), ("rmsd_from_ref", C.c_float),
                ("rmsd_from_cluster_center", C.c_float), ("cluster_id", C.c_int), ("cluster_subrank", C.c_int),
                ("output", C.c_int), ("run_number", C.c_int)]


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class RefJob:
    """One docking job prepared by the reference front end from a command line
    (e.g. ['--ffile', f, '--lfile', l, '--nrun', '10', '--seed', '1,2,3'])."""

    BLOB_DTYPES = {"grid": np.float32, "initpop": np.float32, "prng": np.uint32, "bonds": np.int32, "rigid": np.int32, "contrib": np.int32}

    def __init__(self, args):
        L = lib()
        argv = [b"autodock_gpu"] + [a.encode() for a in args]
        arr = (C.c_char_p * (len(argv) + 1))(*argv, None)
        self.h = L.adgpu_ref_job_create(len(argv), arr)
        if not self.h:
            raise RuntimeError(f"reference setup failed for {args}")
        self.info = RefInfo()
        L.adgpu_ref_job_info(self.h, C.byref(self.info))
        self._keep = []

    def __del__(self):
        if getattr(self, "h", None):
            lib().adgpu_ref_job_free(self.h)
            self.h = None

    def blob(self, name: str) -> np.ndarray:
        n = C.c_size_t()
        p = lib().adgpu_ref_job_blob(self.h, name.encode(), C.byref(n))
        if not p:
            raise KeyError(name)
        dt = self.BLOB_DTYPES.get(name, np.uint8)
        buf = (C.c_char * n.value).from_address(p)
        return np.frombuffer(buf, dtype=np.uint8).copy().view(dt)

    def bind(self, prng: np.ndarray, evals_new: np.ndarray, evals_runs: np.ndarray, dockpars: bytes | None = None):
        """Points the emulated kernels at this job with caller-owned state arrays."""
        self._keep = [prng, evals_new, evals_runs]
        dp = None
        if dockpars is not None:
            self._dp = C.create_string_buffer(bytes(dockpars), len(dockpars))
            dp = C.cast(self._dp, C.c_void_p)
        lib().adgpu_ref_job_bind(self.h, dp, _ptr(prng), _ptr(evals_new), _ptr(evals_runs))

    # --- result processing (host/src/processresult.cpp), files switched off ---
    def process_result(self, pops: np.ndarray, energies: np.ndarray, rmsd_tol: float = 2.0, symmetry: bool = True,
                       clustering: bool = True, nr_cluster_poses: int = 0):
        """Runs arrange_result + make_resfiles per run and generate_output's
        clustering; returns (sorted pops, sorted energies, runs, xyz, peratom)."""
        P = self.info.pop_size
        p = np.ascontiguousarray(pops, np.float32).reshape(-1, GENOTYPE_STRIDE).copy()
        e = np.ascontiguousarray(energies, np.float32).reshape(-1).copy()
        R = e.size // P
        N = self.info.num_of_atoms
        runs = (RefRunResult * R)()
        xyz = np.zeros((R, N, 3), np.float64)
        per = np.zeros((R, N, 2), np.float32)
        lib().adgpu_ref_process_result(self.h, _ptr(p), _ptr(e), R, rmsd_tol, int(symmetry), int(clustering),
                                       nr_cluster_poses, C.cast(runs, C.c_void_p), _ptr(xyz), _ptr(per))
        return p, e, runs, xyz, per

    def rescore(self, genotypes: np.ndarray, symmetry: bool = True) -> np.ndarray:
        """make_resfiles' per-entity values: [intra, inter, RMSD] per genotype."""
        g = np.ascontiguousarray(genotypes, np.float32).reshape(-1, GENOTYPE_STRIDE)
        out = np.zeros((g.shape[0], 3), np.float32)
        lib().adgpu_ref_rescore(self.h, _ptr(g), g.shape[0], int(symmetry), _ptr(out))
        return out

    # --- emulated reference kernels (host arrays stand in for device memory) ---
    def score(self, genotypes: np.ndarray, gradients: bool, threads: int = NUM_THREADS):
        g = np.ascontiguousarray(genotypes, dtype=np.float32)
        n = g.shape[0]
        e = np.zeros(n, np.float32)
        gr = np.zeros((n, GENOTYPE_STRIDE), np.float32) if gradients else None
        lib().adgpu_ref_score(n, threads, _ptr(g), _ptr(e), _ptr(gr))
        return (e, gr) if gradients else e


def ocl_score(genotypes: np.ndarray):
    """Energies and gene gradients from the reference's OpenCL merged scorer
    (device/calcMergedEneGra.cl) for the bound job."""
    L = lib()
    g = np.ascontiguousarray(genotypes, np.float32)
    n = g.shape[0]
    e = np.zeros(n, np.float32)
    gr = np.zeros((n, GENOTYPE_STRIDE), np.float32)
    gd = C.create_string_buffer(L.adgpu_ref_sizeof_gpudata())
    L.adgpu_ref_get_gpudata(C.cast(gd, C.c_void_p))
    L.adgpu_ref_ocl_score(C.cast(gd, C.c_void_p), n, _ptr(g), _ptr(e), _ptr(gr))
    return e, gr


def call(name, *args):
    L = lib()
    conv = [(_ptr(a) if isinstance(a, np.ndarray) else a) for a in args]
    if name in ("gradient_minfire", "gradient_minfire_asis"):
        # the OpenCL FIRE kernel (device/kernel_fire.cl) takes its tables as
        # arguments: hand it the bound job's GpuData.  "_asis" keeps the
        # kernel's own first gradient, computed on coordinates it never
        # initialises (ref/ref_fire_tu.cpp)
        C.c_int.in_dll(L, "adgpu_ref_fire_first_gradient").value = 0 if name.endswith("_asis") else 1
        gd = C.create_string_buffer(L.adgpu_ref_sizeof_gpudata())
        L.adgpu_ref_get_gpudata(C.cast(gd, C.c_void_p))
        return L.adgpu_ref_fire(C.cast(gd, C.c_void_p), *conv)
    return getattr(L, f"adgpu_ref_{name}")(*conv)


# ---------------------------------------------------------------------------
# The reference's CUDA kernels compiled unchanged for sm_100a
# (oracle/_ref/libadgpu_refcuda.so): same GpuData, device buffers.
# ---------------------------------------------------------------------------
REFCUDA_PATH = os.path.join(HERE, "_ref", "libadgpu_refcuda.so")
_cuda = None


def cuda_available() -> bool:
    return os.path.exists(REFCUDA_PATH)


def cuda_lib():
    global _cuda
    if _cuda is None:
        if not cuda_available():
            raise FileNotFoundError(f"{REFCUDA_PATH} not built (make -C oracle ref)")
        L = C.CDLL(REFCUDA_PATH)
        vp, u32 = C.c_void_p, C.c_uint32
        L.adgpu_refcuda_set_gpudata.argtypes = [vp]
        L.adgpu_refcuda_score.argtypes = [u32, vp, vp, vp]
        L.adgpu_refcuda_score.restype = C.c_int
        L.adgpu_refcuda_calc_initpop.argtypes = [u32, u32, vp, vp]
        L.adgpu_refcuda_sum_evals.argtypes = [u32, u32]
        L.adgpu_refcuda_gen_and_eval_newpops.argtypes = [u32, u32, vp, vp, vp, vp]
        for n in ("perform_ls", "gradient_minad", "gradient_minadam"):
            getattr(L, f"adgpu_refcuda_{n}").argtypes = [u32, u32, vp, vp]
        _cuda = L
    return _cuda


def cuda_call(name, *args):
    conv = []
    for a in args:
        if hasattr(a, "data_ptr"):
            conv.append(C.c_void_p(a.data_ptr()))
        elif isinstance(a, np.ndarray):
            conv.append(a.ctypes.data_as(C.c_void_p))
        else:
            conv.append(a)
    return getattr(cuda_lib(), f"adgpu_refcuda_{name}")(*conv)
