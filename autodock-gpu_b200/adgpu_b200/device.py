"""Device-side plumbing for the reference kernel API: uploads reference-layout
tables, grid and LGA state with torch (device memory only) and fills the
GpuData the kernel API consumes, exactly as the reference host does in
docking_with_gpu (host/src/performdocking.cpp.Cuda:325-463).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import abi, lib

TABLE_NAMES = ("interintra", "intracontrib", "intra", "rotlist", "conform", "grads")


def _dev(a: np.ndarray, device) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


class DeviceJob:
    """One ligand's tables, grid and population buffers on the GPU.

    tables: {name: uint8 array of the reference struct}, dockpars: abi.Dockpars,
    grid: float32 reference-layout grid, runs: number of runs.
    """

    def __init__(self, tables: dict, dockpars: abi.Dockpars, grid: np.ndarray, runs: int,
                 prng: np.ndarray, device="cuda:0"):
        self.device = torch.device(device)
        self.dp = dockpars.copy()
        self.runs = int(runs)
        self.t = {k: _dev(np.asarray(tables[k]).view(np.uint8), self.device) for k in TABLE_NAMES}
        self.grid = _dev(np.asarray(grid, np.float32), self.device)
        P = self.dp.pop_size
        self.prng = _dev(np.asarray(prng, np.uint32).view(np.int32), self.device)
        self.evals_new = torch.zeros(max(abi.MAX_POPSIZE * 1, P * self.runs), dtype=torch.int32, device=self.device)
        self.evals_runs = torch.zeros(self.runs, dtype=torch.int32, device=self.device)
        self.g = abi.GpuData()
        self._fill()

    def _fill(self):
        g = self.g
        g.devnum = 0
        g.devid = self.device.index or 0
        g.dockpars = self.dp
        g.pKerconst_interintra = self.t["interintra"].data_ptr()
        g.pKerconst_intracontrib = self.t["intracontrib"].data_ptr()
        g.pKerconst_intra = self.t["intra"].data_ptr()
        g.pKerconst_rotlist = self.t["rotlist"].data_ptr()
        g.pKerconst_conform = self.t["conform"].data_ptr()
        g.pKerconst_grads = self.t["grads"].data_ptr()
        off = abi.table_offsets()
        base = self.t["grads"].data_ptr()
        g.pMem_rotbonds_const = base + off["rotbonds"]
        g.pMem_rotbonds_atoms_const = base + off["rotbonds_atoms"]
        g.pMem_num_rotating_atoms_per_rotbond_const = base + off["num_rotating_atoms_per_rotbond"]
        g.pMem_fgrids = self.grid.data_ptr()
        g.pMem_evals_of_new_entities = self.evals_new.data_ptr()
        g.pMem_gpu_evals_of_runs = self.evals_runs.data_ptr()
        g.pMem_prng_states = self.prng.data_ptr()
        g.warpmask, g.warpbits = 31, 5

    def set_dockpars(self, dp: abi.Dockpars):
        self.dp = dp.copy()
        self.g.dockpars = self.dp

    def activate(self):
        """SetKernelsGpuData (cuda/kernels.cu:126-132)."""
        lib.call("adgpu_set_kernels_gpu_data", C.cast(C.pointer(self.g), C.c_void_p))

    def population(self, host: np.ndarray | None = None):
        n = self.runs * self.dp.pop_size
        conf = torch.zeros((n, abi.GENOTYPE_STRIDE), dtype=torch.float32, device=self.device)
        if host is not None:
            conf.copy_(torch.from_numpy(np.ascontiguousarray(host[:n], np.float32)))
        return conf, torch.zeros(n, dtype=torch.float32, device=self.device)


def score(genotypes: np.ndarray, gradients: bool, device="cuda:0"):
    """Scores genotypes with the active ligand (adgpu_score_genotypes)."""
    g = torch.from_numpy(np.ascontiguousarray(genotypes, np.float32)).to(device)
    n = g.shape[0]
    e = torch.zeros(n, dtype=torch.float32, device=device)
    gr = torch.zeros((n, abi.GENOTYPE_STRIDE), dtype=torch.float32, device=device) if gradients else None
    lib.call("adgpu_score_genotypes", n, g, e, gr if gr is not None else None)
    torch.cuda.synchronize()
    return (e.cpu().numpy(), gr.cpu().numpy()) if gradients else e.cpu().numpy()


def score_terms(genotypes: np.ndarray, device="cuda:0"):
    """Energies and their eight terms per genotype (adgpu_score_terms): inter
    type / elec / desolv, intra vdW-Hb / elec / desolv / CG-G0, atoms outside
    the grid."""
    g = torch.from_numpy(np.ascontiguousarray(genotypes, np.float32)).to(device)
    n = g.shape[0]
    e = torch.zeros(n, dtype=torch.float32, device=device)
    t = torch.zeros((n, 8), dtype=torch.float32, device=device)
    lib.call("adgpu_score_terms", n, g, e, t)
    torch.cuda.synchronize()
    return e.cpu().numpy(), t.cpu().numpy()
