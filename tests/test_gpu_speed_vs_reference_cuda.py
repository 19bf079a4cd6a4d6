"""Throughput against the reference's own CUDA kernels (cuda/*.cu compiled
unchanged for sm_100a with the reference's flags, oracle/_ref) on the same
GPU: the cfg2 ligand (40 heavy atoms, 10 torsions), 100 runs x 150
entities, the same GpuData and population: the ADADELTA local search, the GA
generation and the scorer launch by launch, and a whole docking (500k
evaluations per run) through each side's own generation loop.  Prints one
JSON line with both rates; fails if the engine is slower than the reference
in any of the local search, the GA or the docking."""
import ctypes as C
import json
import os

import numpy as np
import pytest
import torch

import helpers
from adgpu_b200 import device, lib
from oracle import refpy

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refpy.cuda_available(), reason="reference CUDA kernels not built")]
T = 64


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    d = tmp_path_factory.mktemp("speed")
    return helpers.make_case(str(d / "cfg2"), 60, ["C", "A", "N", "OA", "HD"], 40, 10, 100, config_id=2)


def _timed(fn, reps=3):
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / 1e3 / reps


def test_kernels_faster_than_reference_cuda(case):
    dp = case.dockpars
    R, P, L = case.runs, dp.pop_size, dp.num_of_lsentities
    me = device.DeviceJob(case.tables, dp, case.grid, R, case.prng)
    me.activate()
    ref = device.DeviceJob(case.tables, dp, case.grid, R, case.prng)
    refpy.cuda_lib().adgpu_refcuda_set_gpudata(C.cast(C.pointer(ref.g), C.c_void_p))
    cur, ecur = me.population(case.initpop)
    lib.call("adgpu_calc_initpop", R * P, T, cur, ecur)
    out = {"workload": f"cfg2 ligand ({dp.num_of_atoms} atoms, {dp.num_of_intraE_contributors} pairs), "
                       f"{R} runs x {L} local-search entities, pop {P}"}
    # ADADELTA local search from the same population (evaluations as counted by the kernels)
    for name, job, call in (("engine", me, lambda c, e: lib.call("adgpu_gradient_minad", R * L, T, c, e)),
                            ("reference_cuda", ref, lambda c, e: refpy.cuda_call("gradient_minad", R * L, T, c, e))):
        job.evals_new.zero_()
        bufs = [(cur.clone(), ecur.clone()) for _ in range(4)]
        it = iter(bufs)
        call(*next(it))                          # warm-up
        job.evals_new.zero_()
        dt = _timed(lambda: call(*next(it)))
        evals = int(job.evals_new.sum().item()) / 3
        out[f"ls_ad_{name}_evals_per_s"] = evals / dt
        out[f"ls_ad_{name}_ms"] = dt * 1e3
    # GA generation (one energy evaluation per entity)
    n1, e1 = me.population()
    for name, call in (("engine", lambda: lib.call("adgpu_gen_and_eval_newpops", R * P, T, cur, ecur, n1, e1)),
                       ("reference_cuda", lambda: refpy.cuda_call("gen_and_eval_newpops", R * P, T, cur, ecur, n1, e1))):
        call()
        dt = _timed(call)
        out[f"ga_{name}_entities_per_s"] = R * P / dt
    # scorer alone, energy + gradient, 15,000 in-box poses
    g = torch.from_numpy(helpers.in_box_genotypes(case, 15000, seed=5)).cuda()
    e = torch.zeros(len(g), device="cuda")
    gr = torch.zeros_like(g)
    for name, call in (("engine", lambda: lib.call("adgpu_score_genotypes", len(g), g, e, gr)),
                       ("reference_cuda", lambda: refpy.cuda_call("score", len(g), g, e, gr))):
        call()
        dt = _timed(call)
        out[f"score_grad_{name}_evals_per_s"] = len(g) / dt
    # a whole docking of the same ligand (100 runs, 500k evaluations per run,
    # ADADELTA): the reference's generation loop over its own kernels, one
    # synchronous call per kernel per generation (docking_with_gpu,
    # host/src/performdocking.cpp.Cuda:684-831), against adgpu_dock_resident
    nev = 500_000
    for name in ("engine", "reference_cuda"):
        job = device.DeviceJob(case.tables, dp, case.grid, R, case.prng)
        cur, ecur = job.population(case.initpop)
        nxt, enxt = job.population()
        if name == "engine":
            job.activate()
            lib.call("adgpu_calc_initpop", R * P, T, cur, ecur)
            lib.call("adgpu_sum_evals", R, T)
        else:
            refpy.cuda_lib().adgpu_refcuda_set_gpudata(C.cast(C.pointer(job.g), C.c_void_p))
            refpy.cuda_call("calc_initpop", R * P, T, cur, ecur)
            refpy.cuda_call("sum_evals", R, T)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        if name == "engine":
            fin, gn = C.c_int(0), C.c_uint32(0)
            lib.call("adgpu_dock_resident", 1, R, nev, 42000, cur, ecur, nxt, enxt, C.byref(fin), C.byref(gn))
            gens = gn.value
        else:
            gens = 0
            while job.evals_runs.sum().item() / R < nev:
                refpy.cuda_call("gen_and_eval_newpops", R * P, T, cur, ecur, nxt, enxt)
                refpy.cuda_call("gradient_minad", R * L, T, nxt, enxt)
                refpy.cuda_call("sum_evals", R, T)
                gens += 1
                cur, nxt, ecur, enxt = nxt, cur, enxt, ecur
        b.record()
        torch.cuda.synchronize()
        dt = a.elapsed_time(b) / 1e3
        out[f"docking_{name}_s"] = dt
        out[f"docking_{name}_evals_per_s"] = (int(job.evals_runs.sum().item()) - R * P) / dt
        out[f"docking_{name}_generations"] = gens
    line = json.dumps(out)
    print(line)
    if os.environ.get("ADGPU_SPEED_OUT"):
        with open(os.environ["ADGPU_SPEED_OUT"], "w") as f:
            f.write(line + "\n")
    assert out["ls_ad_engine_evals_per_s"] > out["ls_ad_reference_cuda_evals_per_s"]
    assert out["ga_engine_entities_per_s"] > out["ga_reference_cuda_entities_per_s"]
    assert out["docking_engine_evals_per_s"] > out["docking_reference_cuda_evals_per_s"]
