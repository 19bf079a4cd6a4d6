"""Throughput against the reference's own CUDA kernels (cuda/*.cu compiled
unchanged for sm_100a with the reference's flags, oracle/_ref) on the same
GPU: the cfg2 ligand (40 heavy atoms, 10 torsions), 100 runs x 150
entities, the same GpuData and population.  Prints one JSON line with both
rates; fails if the engine's kernels are slower than the reference's."""
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
    line = json.dumps(out)
    print(line)
    if os.environ.get("ADGPU_SPEED_OUT"):
        with open(os.environ["ADGPU_SPEED_OUT"], "w") as f:
            f.write(line + "\n")
    assert out["ls_ad_engine_evals_per_s"] > out["ls_ad_reference_cuda_evals_per_s"]
    assert out["ga_engine_entities_per_s"] > out["ga_reference_cuda_entities_per_s"]
