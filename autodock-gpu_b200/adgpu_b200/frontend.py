"""Python face of the engine's front end (grid maps and ligand preparation,
C ABI in include/adgpu_b200.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, lib


class Grid:
    """Receptor grid maps (host memory)."""

    def __init__(self, handle):
        self.h = handle
        dims = (C.c_int * 3)()
        sp = C.c_double()
        org = (C.c_double * 3)()
        nm = C.c_int()
        lib.check(lib.load().adgpu_grid_info(self.h, dims, C.byref(sp), org, C.byref(nm)), "grid_info")
        self.dims = tuple(dims)
        self.spacing = sp.value
        self.origin = tuple(org)
        self.num_map_atypes = nm.value

    @classmethod
    def read(cls, fld_path: str) -> "Grid":
        h = C.c_void_p()
        lib.check(lib.load().adgpu_grid_read(fld_path.encode(), C.byref(h)), f"grid_read {fld_path}")
        return cls(h)

    @classmethod
    def load(cls, cache_path: str) -> "Grid":
        """A grid from its binary cache (see save)."""
        h = C.c_void_p()
        lib.check(lib.load().adgpu_grid_load(cache_path.encode(), C.byref(h)), f"grid_load {cache_path}")
        return cls(h)

    def save(self, cache_path: str) -> None:
        """Writes the parsed maps as a binary cache that load() reads in one pass."""
        lib.check(lib.load().adgpu_grid_save(self.h, cache_path.encode()), f"grid_save {cache_path}")

    @classmethod
    def from_maps(cls, maps: dict, types: list, spacing: float, origin) -> "Grid":
        """maps: {type: float32 [z, y, x]} for the type maps and 'e', 'd'."""
        order = list(types) + ["e", "d"]
        vals = np.ascontiguousarray(np.stack([np.asarray(maps[t], np.float32) for t in order]))
        nz, ny, nx = vals.shape[1:]
        dims = (C.c_int * 3)(nx, ny, nz)
        org = (C.c_double * 3)(*origin)
        names = (C.c_char_p * len(order))(*[t.encode() for t in order])
        h = C.c_void_p()
        lib.check(lib.load().adgpu_grid_from_values(dims, spacing, org, len(order), names,
                                                    vals.ctypes.data_as(C.c_void_p), C.byref(h)), "grid_from_values")
        g = cls(h)
        g._keep = vals
        return g

    def reference_layout(self) -> np.ndarray:
        n = 4 * (self.num_map_atypes + 2) * self.dims[0] * self.dims[1] * self.dims[2]
        out = np.empty(n, np.float32)
        lib.check(lib.load().adgpu_grid_reference_layout(self.h, out.ctypes.data_as(C.c_void_p), n), "grid layout")
        return out

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib.load().adgpu_grid_free(self.h)
            except Exception:
                pass
            self.h = None


def default_dockpars(spacing: float, pop_size: int = 150) -> abi.Dockpars:
    dp = abi.Dockpars()
    lib.check(lib.load().adgpu_dockpars_default(C.byref(dp), spacing, pop_size), "dockpars_default")
    return dp


class Ligand:
    """A ligand (and optional flexible residues) prepared against a grid."""

    def __init__(self, grid: Grid, ligand_pdbqt: str | None, flexres_pdbqt: str | None = None,
                 run: abi.Dockpars | None = None, seed=(305419896, 2271560481, 3735928559), num_runs: int = 10):
        run = run or default_dockpars(grid.spacing)
        s = (C.c_uint32 * 3)(*seed)
        h = C.c_void_p()
        lib.check(lib.load().adgpu_ligand_prepare(
            grid.h, ligand_pdbqt.encode() if ligand_pdbqt else None,
            flexres_pdbqt.encode() if flexres_pdbqt else None, C.byref(run), s, num_runs, C.byref(h)),
            "ligand_prepare")
        self._adopt(h, num_runs)

    @classmethod
    def prepare_batch(cls, grid: Grid, ligand_pdbqts, flexres_pdbqt: str | None = None, run: abi.Dockpars | None = None,
                      seeds=None, num_runs: int = 10, nthreads: int = 0) -> list:
        """Prepares many ligands on nthreads host threads (0: all cores); seeds:
        one (a, b, c) triple per ligand (default: the same triple for all)."""
        run = run or default_dockpars(grid.spacing)
        n = len(ligand_pdbqts)
        seeds = seeds or [(305419896, 2271560481, 3735928559)] * n
        texts = (C.c_char_p * n)(*[t.encode() if t else None for t in ligand_pdbqts])
        flex = (C.c_char_p * n)(*([flexres_pdbqt.encode()] * n)) if flexres_pdbqt else None
        sd = (C.c_uint32 * (3 * n))(*[int(x) for s in seeds for x in s])
        out = (C.c_void_p * n)()
        st = (C.c_int * n)()
        rc = lib.load().adgpu_ligand_prepare_batch(grid.h, texts, flex, n, C.byref(run), sd, num_runs, nthreads, out, st)
        ligs = []
        for i in range(n):
            if out[i]:
                lg = cls.__new__(cls)
                lg._adopt(C.c_void_p(out[i]), num_runs)
                ligs.append(lg)
        lib.check(rc, "ligand_prepare_batch")
        return ligs

    def _adopt(self, h, num_runs: int):
        self.h = h
        self.num_runs = num_runs
        self.dockpars = abi.Dockpars()
        t = {k: abi.TABLE_TYPES[k]() for k in abi.TABLE_TYPES}
        lib.check(lib.load().adgpu_ligand_tables(self.h, C.byref(self.dockpars), *(C.byref(t[k]) for k in
                  ("interintra", "intracontrib", "intra", "rotlist", "conform", "grads"))), "ligand_tables")
        self.tables = {k: abi.as_bytes_array(v) for k, v in t.items()}
        n = num_runs * self.dockpars.pop_size * abi.GENOTYPE_STRIDE
        self.initpop = np.zeros(n, np.float32)
        self.prng = np.zeros(n, np.uint32)
        if num_runs > 0:
            lib.check(lib.load().adgpu_ligand_population(self.h, self.initpop.ctypes.data_as(C.c_void_p), n,
                                                         self.prng.ctypes.data_as(C.c_void_p), n), "population")
        self.initpop = self.initpop.reshape(-1, abi.GENOTYPE_STRIDE)

    def __del__(self):
        if getattr(self, "h", None):
            try:
                lib.load().adgpu_ligand_free(self.h)
            except Exception:
                pass
            self.h = None
