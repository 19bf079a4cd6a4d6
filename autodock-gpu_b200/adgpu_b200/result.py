"""Result processing on the device (include/adgpu_b200.h, "Result
processing"): the computations of the reference's process_result
(host/src/processresult.cpp:1312-1363) -- each run's final population ordered
by energy, the best poses re-scored with the host scorer's arithmetic, their
RMSD from the input ligand, and the runs clustered by RMSD."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import lib


class ResultParams(C.Structure):
    _fields_ = [("rmsd_tolerance", C.c_float), ("handle_symmetry", C.c_int), ("calc_clustering", C.c_int),
                ("nr_cluster_poses", C.c_int), ("free_roaming_ligand", C.c_int), ("rescore_entities", C.c_int),
                ("coeff_tors", C.c_double)]


class RunResult(C.Structure):
    _fields_ = [("inter_e", C.c_float), ("interflex_e", C.c_float), ("inter_e_elec", C.c_float),
                ("intra_e", C.c_float), ("intraflex_e", C.c_float), ("rmsd_from_ref", C.c_float),
                ("rmsd_from_cluster_center", C.c_float), ("energy", C.c_float), ("run_number", C.c_int),
                ("cluster_id", C.c_int), ("cluster_subrank", C.c_int), ("output", C.c_int),
                ("energy_rank", C.c_int)]


class Cluster(C.Structure):
    _fields_ = [("size", C.c_int), ("best_run", C.c_int), ("best_energy", C.c_double), ("sum_energy", C.c_double)]


_vp = C.c_void_p
SIGNATURES = {
    "adgpu_result_params_default": (C.c_int, [_vp]),
    "adgpu_process_result": (C.c_int, [_vp, _vp, _vp, _vp, C.c_uint32, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
}
lib.SIGNATURES.update(SIGNATURES)
_bound = False


def _L():
    global _bound
    L = lib.load()
    if not _bound:
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _bound = True
    return L


def default_params(**overrides) -> ResultParams:
    p = ResultParams()
    lib.check(_L().adgpu_result_params_default(C.byref(p)), "result_params_default")
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


@dataclass
class Processed:
    runs: list                   # RunResult per run (Ligandresult fields)
    clusters: list               # Cluster per cluster, in cluster-id order
    best_xyz: np.ndarray         # [runs, N, 3] best poses, Angstrom
    peratom: np.ndarray          # [runs, N, 2] per-atom vdW and elec of the best poses
    entities: np.ndarray | None  # [runs, pop, 3] intra, inter, RMSD of every entity (rescore_entities)


def process_result(ligand, grid_dev, populations, energies, num_runs: int, params: ResultParams | None = None,
                   natoms: int | None = None) -> Processed:
    """ligand: frontend.Ligand; grid_dev: the device grid of the kernel API
    (torch tensor, reference layout); populations / energies: the final
    populations on the device (torch tensors), ordered in place on return."""
    params = params or default_params()
    N = natoms if natoms is not None else ligand.dockpars.num_of_atoms
    P = ligand.dockpars.pop_size
    runs = (RunResult * num_runs)()
    clusters = (Cluster * num_runs)()
    nclus = C.c_int()
    xyz = np.zeros((num_runs, N, 3), np.float64)
    per = np.zeros((num_runs, N, 2), np.float32)
    ent = np.zeros((num_runs, P, 3), np.float32) if params.rescore_entities else None
    lib.check(_L().adgpu_process_result(ligand.h, grid_dev.data_ptr(), populations.data_ptr(), energies.data_ptr(),
                                        num_runs, C.byref(params), C.cast(runs, _vp), C.cast(clusters, _vp),
                                        C.byref(nclus), xyz.ctypes.data_as(_vp), per.ctypes.data_as(_vp),
                                        ent.ctypes.data_as(_vp) if ent is not None else None), "process_result")
    return Processed(list(runs), list(clusters)[:nclus.value], xyz, per, ent)
