"""Python face of the batch / serving engine (include/adgpu_b200.h, layer 2)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi, lib
from .frontend import Grid, Ligand

LSMET = {"sw": 0, "ad": 1, "adam": 2, "fire": 3}


class EngineConfig(C.Structure):
    _fields_ = [("memory_budget_bytes", C.c_size_t), ("threads_per_pose", C.c_int),
                ("gens_per_tick", C.c_int), ("device", C.c_int), ("tick_ms", C.c_float),
                ("idle_timeout_ms", C.c_float), ("priority", C.c_int)]


class RequestParams(C.Structure):
    _fields_ = [("receptor", C.c_int), ("lsmet", C.c_int), ("max_evals", C.c_uint64), ("max_gens", C.c_uint32)]


class EngineStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("cancelled", C.c_uint64), ("ticks", C.c_uint64),
                ("bytes_used", C.c_size_t), ("bytes_budget", C.c_size_t), ("active", C.c_int),
                ("worker_busy_s", C.c_double), ("worker_span_s", C.c_double), ("tasks", C.c_uint64),
                ("kernel_s", C.c_double)]


_vp = C.c_void_p
SIGNATURES = {
    "adgpu_engine_create": (C.c_int, [_vp, _vp]),
    "adgpu_engine_destroy": (None, [_vp]),
    "adgpu_engine_add_receptor": (C.c_int, [_vp, _vp, _vp]),
    "adgpu_engine_submit": (C.c_int, [_vp, _vp, _vp, _vp]),
    "adgpu_engine_tick": (C.c_int, [_vp, _vp]),
    "adgpu_engine_run": (C.c_int, [_vp]),
    "adgpu_engine_poll": (C.c_int, [_vp, C.c_uint64, _vp]),
    "adgpu_engine_result": (C.c_int, [_vp, C.c_uint64, _vp, _vp, _vp, _vp, _vp]),
    "adgpu_engine_stats_get": (C.c_int, [_vp, _vp]),
    "adgpu_engine_cancel": (C.c_int, [_vp, C.c_uint64]),
    "adgpu_engine_inject_stall": (C.c_int, [_vp, C.c_uint64]),
    "adgpu_engine_request_info": (C.c_int, [_vp, C.c_uint64, _vp, _vp]),
    "adgpu_engine_process_result": (C.c_int, [_vp, C.c_uint64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
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


@dataclass
class Result:
    best_energies: np.ndarray     # [runs]
    best_genotypes: np.ndarray    # [runs, 64]
    evals: np.ndarray             # [runs]
    generations: np.ndarray       # [runs]
    latency_s: float


class Engine:
    def __init__(self, memory_budget_bytes: int = 0, threads_per_pose: int = 0, gens_per_tick: int = 0,
                 device: int = 0, tick_ms: float = 0.0, idle_timeout_ms: float = 0.0, priority: int = 0):
        cfg = EngineConfig(memory_budget_bytes, threads_per_pose, gens_per_tick, device, tick_ms, idle_timeout_ms,
                           priority)
        h = C.c_void_p()
        lib.check(_L().adgpu_engine_create(C.byref(cfg), C.byref(h)), "engine_create")
        self.h = h
        self._keep = []
        self._pop_size = {}

    def close(self):
        if getattr(self, "h", None):
            _L().adgpu_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_receptor(self, grid: Grid) -> int:
        rid = C.c_int()
        lib.check(_L().adgpu_engine_add_receptor(self.h, grid.h, C.byref(rid)), "add_receptor")
        self._keep.append(grid)
        return rid.value

    def submit(self, ligand: Ligand, receptor: int, lsmet: str = "ad", max_evals: int = 2_500_000,
               max_gens: int = 0, raise_on_budget: bool = True):
        rp = RequestParams(receptor, LSMET[lsmet], max_evals, max_gens)
        rid = C.c_uint64()
        st = _L().adgpu_engine_submit(self.h, ligand.h, C.byref(rp), C.byref(rid))
        if st == 5 and not raise_on_budget:
            return None
        lib.check(st, "engine_submit")
        self._pop_size[rid.value] = ligand.dockpars.pop_size
        return rid.value

    def tick(self) -> int:
        c = C.c_int()
        lib.check(_L().adgpu_engine_tick(self.h, C.byref(c)), "engine_tick")
        return c.value

    def run(self):
        lib.check(_L().adgpu_engine_run(self.h), "engine_run")

    def cancel(self, request_id: int):
        """Drops a request (finished or not) between ticks."""
        lib.check(_L().adgpu_engine_cancel(self.h, request_id), "engine_cancel")
        self._pop_size.pop(request_id, None)

    def inject_stall(self, request_id: int):
        """Test hook: the request's runs stop handing out tasks (the next tick
        times out after idle_timeout_ms)."""
        lib.check(_L().adgpu_engine_inject_stall(self.h, request_id), "engine_inject_stall")

    def done(self, request_id: int) -> bool:
        d = C.c_int()
        lib.check(_L().adgpu_engine_poll(self.h, request_id, C.byref(d)), "engine_poll")
        return bool(d.value)

    def info(self, request_id: int):
        t, r = C.c_int(), C.c_int()
        lib.check(_L().adgpu_engine_request_info(self.h, request_id, C.byref(t), C.byref(r)), "request_info")
        return t.value, r.value

    def result(self, request_id: int) -> Result:
        _, runs = self.info(request_id)
        be = np.zeros(runs, np.float32)
        bg = np.zeros((runs, abi.GENOTYPE_STRIDE), np.float32)
        ev = np.zeros(runs, np.int32)
        gn = np.zeros(runs, np.uint32)
        lat = C.c_double()
        lib.check(_L().adgpu_engine_result(self.h, request_id, be.ctypes.data_as(_vp), bg.ctypes.data_as(_vp),
                                           ev.ctypes.data_as(_vp), gn.ctypes.data_as(_vp), C.byref(lat)),
                  "engine_result")
        return Result(be, bg, ev, gn, lat.value)

    def process_result(self, request_id: int, natoms: int, params=None, final_population: bool = False):
        """Result processing of a finished request on the device (ordering,
        re-scoring, RMSD, clustering); call before result(), which frees the
        request.  Returns (result.Processed, final populations, final energies)."""
        from . import result as _res
        params = params or _res.default_params()
        _, runs = self.info(request_id)
        rr = (_res.RunResult * runs)()
        cl = (_res.Cluster * runs)()
        nclus = C.c_int()
        xyz = np.zeros((runs, natoms, 3), np.float64)
        per = np.zeros((runs, natoms, 2), np.float32)
        pop = self._pop_size.get(request_id, 0)
        ent = np.zeros((runs, pop, 3), np.float32) if params.rescore_entities else None
        fp = np.zeros((runs * pop, abi.GENOTYPE_STRIDE), np.float32) if final_population else None
        fe = np.zeros(runs * pop, np.float32) if final_population else None
        ptr = (lambda a: a.ctypes.data_as(_vp) if a is not None else None)
        lib.check(_L().adgpu_engine_process_result(self.h, request_id, C.byref(params), C.cast(rr, _vp),
                                                   C.cast(cl, _vp), C.byref(nclus), ptr(xyz), ptr(per), ptr(ent),
                                                   ptr(fp), ptr(fe)), "engine_process_result")
        return _res.Processed(list(rr), list(cl)[:nclus.value], xyz, per, ent), fp, fe

    def stats(self) -> EngineStats:
        s = EngineStats()
        lib.check(_L().adgpu_engine_stats_get(self.h, C.byref(s)), "engine_stats")
        return s
