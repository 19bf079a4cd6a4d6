"""ctypes mirror of the layout types in include/adgpu_b200.h.

These structures are byte-identical to the reference's GpuDockparameters,
GpuData and kernelconstant_* (cuda/GpuData.h:74-136,
host/inc/calcenergy.h:88-136); see the header for the mapping.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

MAX_ATOMS = 256
MAX_ATYPES = 32
MAX_ROTBONDS = 57
MAX_INTRAE = MAX_ATOMS * MAX_ATOMS
MAX_ROTATIONS = MAX_ATOMS * MAX_ROTBONDS
MAX_POPSIZE = 2048
MAX_RUNS = 8192
GENOTYPE_STRIDE = 64
MAX_GENES = MAX_ROTBONDS + 6

RLIST_ATOMID_MASK = 0x000000FF
RLIST_RBONDID_MASK = 0x0000FF00
RLIST_RBONDID_SHIFT = 8
RLIST_FIRSTROT_MASK = 0x00010000
RLIST_GENROT_MASK = 0x00020000
RLIST_DUMMY_MASK = 0x00040000

STATUS = {0: "ok", 1: "bad argument", 2: "CUDA error", 3: "not ready", 4: "limit exceeded",
          5: "memory budget exceeded", 6: "invalid state", 7: "device wait timed out"}


class Dockpars(C.Structure):
    _fields_ = [
        ("num_of_atoms", C.c_int), ("true_ligand_atoms", C.c_int), ("num_of_atypes", C.c_int),
        ("num_of_map_atypes", C.c_int), ("num_of_intraE_contributors", C.c_int),
        ("gridsize_x", C.c_int), ("gridsize_y", C.c_int), ("gridsize_z", C.c_int),
        ("gridsize_x_times_y", C.c_int), ("gridsize_x_times_y_times_z", C.c_int),
        ("grid_spacing", C.c_float), ("rotbondlist_length", C.c_int),
        ("coeff_elec", C.c_float), ("elec_min_distance", C.c_float), ("coeff_desolv", C.c_float),
        ("pop_size", C.c_int), ("num_of_genes", C.c_int),
        ("tournament_rate", C.c_float), ("crossover_rate", C.c_float), ("mutation_rate", C.c_float),
        ("abs_max_dmov", C.c_float), ("abs_max_dang", C.c_float), ("lsearch_rate", C.c_float),
        ("smooth", C.c_float), ("num_of_lsentities", C.c_uint), ("rho_lower_bound", C.c_float),
        ("base_dmov_mul_sqrt3", C.c_float), ("base_dang_mul_sqrt3", C.c_float),
        ("cons_limit", C.c_uint), ("max_num_of_iters", C.c_uint), ("qasp", C.c_float),
        ("adam_beta1", C.c_float), ("adam_beta2", C.c_float), ("adam_epsilon", C.c_float),
    ]

    def copy(self) -> "Dockpars":
        d = Dockpars()
        C.memmove(C.byref(d), C.byref(self), C.sizeof(Dockpars))
        return d

    @staticmethod
    def from_bytes(b) -> "Dockpars":
        d = Dockpars()
        C.memmove(C.byref(d), bytes(b), C.sizeof(Dockpars))
        return d


class KcInterintra(C.Structure):
    _fields_ = [("atom_charges_const", C.c_float * MAX_ATOMS),
                ("atom_types_const", C.c_uint32 * MAX_ATOMS),
                ("atom_types_map_const", C.c_uint32 * MAX_ATOMS),
                ("ignore_inter_const", C.c_char * MAX_ATOMS)]


class KcIntracontrib(C.Structure):
    _fields_ = [("intraE_contributors_const", C.c_uint32 * (2 * MAX_INTRAE))]


class KcIntra(C.Structure):
    _fields_ = [("atom_types_reqm_const", C.c_uint * MAX_ATYPES),
                ("VWpars_exp_const", C.c_ushort * (MAX_ATYPES * MAX_ATYPES)),
                ("reqm_AB_const", C.c_float * (MAX_ATYPES * MAX_ATYPES)),
                ("VWpars_AC_const", C.c_float * (MAX_ATYPES * MAX_ATYPES)),
                ("VWpars_BD_const", C.c_float * (MAX_ATYPES * MAX_ATYPES)),
                ("dspars_S_const", C.c_float * MAX_ATYPES),
                ("dspars_V_const", C.c_float * MAX_ATYPES)]


class KcRotlist(C.Structure):
    _fields_ = [("rotlist_const", C.c_int * MAX_ROTATIONS)]


class KcConform(C.Structure):
    _fields_ = [("ref_coords_const", C.c_float * (3 * MAX_ATOMS)),
                ("rotbonds_moving_vectors_const", C.c_float * (3 * MAX_ROTBONDS)),
                ("rotbonds_unit_vectors_const", C.c_float * (3 * MAX_ROTBONDS))]


class KcGrads(C.Structure):
    _fields_ = [("rotbonds", C.c_int * (2 * MAX_ROTBONDS)),
                ("rotbonds_atoms", C.c_int * (MAX_ATOMS * MAX_ROTBONDS)),
                ("num_rotating_atoms_per_rotbond", C.c_int * MAX_ROTBONDS)]


TABLE_TYPES = {
    "interintra": KcInterintra, "intracontrib": KcIntracontrib, "intra": KcIntra,
    "rotlist": KcRotlist, "conform": KcConform, "grads": KcGrads,
}


class GpuData(C.Structure):
    _fields_ = [
        ("devnum", C.c_int), ("devid", C.c_int), ("preallocated_gridsize", C.c_int),
        ("dockpars", Dockpars),
        ("pKerconst_interintra", C.c_void_p), ("pKerconst_intracontrib", C.c_void_p),
        ("pKerconst_intra", C.c_void_p), ("pKerconst_rotlist", C.c_void_p),
        ("pKerconst_conform", C.c_void_p), ("pKerconst_grads", C.c_void_p),
        ("pMem_fgrids", C.c_void_p), ("pMem_evals_of_new_entities", C.c_void_p),
        ("pMem_gpu_evals_of_runs", C.c_void_p), ("pMem_prng_states", C.c_void_p),
        ("pMem_rotbonds_const", C.c_void_p), ("pMem_rotbonds_atoms_const", C.c_void_p),
        ("pMem_num_rotating_atoms_per_rotbond_const", C.c_void_p),
        ("warpmask", C.c_uint), ("warpbits", C.c_uint),
    ]


def table_offsets():
    """Byte offsets of the kernelconstant_grads sub-arrays (used to point the
    pMem_rotbonds*_const members into one uploaded grads table)."""
    return {
        "rotbonds": KcGrads.rotbonds.offset,
        "rotbonds_atoms": KcGrads.rotbonds_atoms.offset,
        "num_rotating_atoms_per_rotbond": KcGrads.num_rotating_atoms_per_rotbond.offset,
    }


def as_bytes_array(x) -> np.ndarray:
    return np.frombuffer(bytes(x), dtype=np.uint8).copy()


class DockStats(C.Structure):
    """adgpu_dock_stats: accounting of the last adgpu_dock_resident call."""
    _fields_ = [("pipelined", C.c_int), ("threads_per_pose", C.c_int), ("pose_groups", C.c_int),
                ("generations", C.c_uint32), ("generations_discarded", C.c_uint32), ("tasks", C.c_uint64),
                ("parks", C.c_uint64), ("evals_executed", C.c_uint64), ("buffers", C.c_int), ("pad", C.c_int),
                ("busy_s", C.c_double), ("span_s", C.c_double)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        if self.pipelined and self.pose_groups and self.span_s > 0:
            d["utilisation"] = self.busy_s / (self.pose_groups * self.span_s)
        return d
