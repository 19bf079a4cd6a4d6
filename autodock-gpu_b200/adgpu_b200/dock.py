"""Plain per-ligand docking through the reference kernel API: the call
sequence of docking_with_gpu (host/src/performdocking.cpp.Cuda:640-831) --
initial population, eval sums, then the generation loop -- with the loop
resident on the device (adgpu_dock_resident)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import abi, lib
from .device import DeviceJob

LSMET = {"sw": 0, "ad": 1, "adam": 2, "fire": 3}
REF_THREADS = 64


@dataclass
class DockResult:
    conformations: torch.Tensor     # final population [runs*pop, 64]
    energies: torch.Tensor          # [runs*pop]
    evals_per_run: np.ndarray       # [runs]
    generations: int
    autostopped: bool = False


@dataclass
class AutoStopParams:
    """The reference's --asfreq, --stopstd and the heuristics' minimum evaluations."""
    as_frequency: int = 5
    stopstd: float = 0.15
    min_evals: int = 0


def dock_host_loop(job: DeviceJob, initpop: np.ndarray | torch.Tensor, lsmet: str = "ad", nev: int = 2_500_000,
                   ngen: int = 42_000, autostop=None) -> DockResult:
    """The reference host's own generation loop (docking_with_gpu,
    host/src/performdocking.cpp.Cuda:640-831) over the kernel API: one
    synchronous call per kernel per generation and a host-side progress check
    on the per-run eval counters -- how a drop-in user drives the kernels.
    `autostop`: (as_frequency, min_evals, check) with check(generation,
    energies, total_evals) -> bool an AutoStop test run on the host every
    as_frequency generations (:689-698)."""
    R, P = job.runs, job.dp.pop_size
    cur, ecur = job.population()
    nxt, enxt = job.population()
    cur.copy_(initpop[:R * P] if isinstance(initpop, torch.Tensor)
              else torch.from_numpy(np.ascontiguousarray(initpop[:R * P], np.float32)))
    job.evals_runs.zero_()
    T = REF_THREADS
    lib.call("adgpu_calc_initpop", R * P, T, cur, ecur)
    lib.call("adgpu_sum_evals", R, T)
    ls = {"sw": "adgpu_perform_ls", "ad": "adgpu_gradient_minad", "adam": "adgpu_gradient_minadam",
          "fire": "adgpu_gradient_minfire"}[lsmet]
    L = job.dp.num_of_lsentities
    gen = 0
    stopped = False
    while True:
        total = int(job.evals_runs.sum().item())                  # check_progress (:908-942)
        progress = max(total / R / nev * 100.0, gen / ngen * 100.0)
        if progress >= 100.0:
            break
        if autostop is not None and gen % autostop[0] == 0:
            if autostop[2](gen, ecur[:R * P].cpu().numpy(), total) and total > autostop[1]:
                stopped = True
                break
        lib.call("adgpu_gen_and_eval_newpops", R * P, T, cur, ecur, nxt, enxt)
        lib.call(ls, R * L, T, nxt, enxt)
        lib.call("adgpu_sum_evals", R, T)
        gen += 1
        cur, nxt = nxt, cur
        ecur, enxt = enxt, ecur
    return DockResult(cur, ecur, job.evals_runs.cpu().numpy().copy(), gen, stopped)


def dock(job: DeviceJob, initpop: np.ndarray | torch.Tensor, lsmet: str = "ad", nev: int = 2_500_000,
         ngen: int = 42_000, buffers=None, autostop: AutoStopParams | None = None) -> DockResult:
    """Docks the active ligand: runs*pop entities from `initpop`, until the
    mean evaluations per run reach `nev` or `ngen` generations have run, or,
    with `autostop`, the reference's AutoStop test (run on the device) is
    satisfied."""
    R, P = job.runs, job.dp.pop_size
    if buffers is None:
        c1, e1 = job.population()
        c2, e2 = job.population()
    else:
        c1, e1, c2, e2 = buffers
    if isinstance(initpop, torch.Tensor):
        c1.copy_(initpop[:R * P])
    else:
        c1.copy_(torch.from_numpy(np.ascontiguousarray(initpop[:R * P], np.float32)))
    job.evals_runs.zero_()
    lib.call("adgpu_calc_initpop", R * P, REF_THREADS, c1, e1)
    lib.call("adgpu_sum_evals", R, REF_THREADS)
    fin = C.c_int(0)
    gens = C.c_uint32(0)
    stopped = C.c_int(0)
    if autostop is None:
        lib.call("adgpu_dock_resident", LSMET[lsmet], R, int(nev), int(ngen), c1, e1, c2, e2, C.byref(fin), C.byref(gens))
    else:
        lib.call("adgpu_dock_resident_autostop", LSMET[lsmet], R, int(nev), int(ngen), int(autostop.as_frequency),
                 float(autostop.stopstd), int(autostop.min_evals), c1, e1, c2, e2, C.byref(fin), C.byref(gens),
                 C.byref(stopped))
    c, e = (c2, e2) if fin.value else (c1, e1)
    return DockResult(c, e, job.evals_runs.cpu().numpy().copy(), gens.value, bool(stopped.value))


def last_stats() -> dict:
    """Accounting of the last docking through adgpu_dock_resident: whether the
    pipelined loop ran, its pose groups, tasks, their summed busy time, the
    launch span and the resulting utilisation of the pose groups."""
    st = abi.DockStats()
    lib.call("adgpu_dock_stats_get", C.byref(st))
    return st.as_dict()
