"""Whole dockings against whole dockings of the reference's own CUDA kernels
(cuda/*.cu compiled unchanged for sm_100a, oracle/_ref), same ligand, same
initial population and PRNG seeds, on the same GPU.  Trajectories diverge
after the first rounding difference, so the comparison is statistical: the
best energies of the runs come from the same distribution (two-sample
Kolmogorov-Smirnov), and the top-ranked binding modes after result
processing (ordering, re-scoring, RMSD clustering at 2 A) agree: the best
pose of each side's lowest-energy cluster lies within 2 A of the best pose of
one of the other side's three lowest-energy clusters.  (One docking is one
sample: where two binding modes lie a fraction of a kcal/mol apart, either
can rank first in a given docking, for the reference against itself too.)"""
import ctypes as C
import json

import numpy as np
import pytest
import torch

import helpers
from adgpu_b200 import device, dock
from oracle import refpy

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (refpy.cuda_available() and refpy.available()),
                                 reason="reference CUDA kernels / host oracle not built")]
T = 64
LS_ENTRY = {"ad": "gradient_minad", "sw": "perform_ls", "adam": "gradient_minadam"}


def reference_docking(case, lsmet, nev, ngen=42000):
    """docking_with_gpu's generation loop (host/src/performdocking.cpp.Cuda:
    684-831) over the reference's CUDA kernels: initial population, then GA
    generation, local search and eval sums until the mean evaluations per
    run reach nev (check_progress, :908-942)."""
    dp = case.dockpars
    R, P, L = case.runs, dp.pop_size, dp.num_of_lsentities
    job = device.DeviceJob(case.tables, dp, case.grid, R, case.prng)
    refpy.cuda_lib().adgpu_refcuda_set_gpudata(C.cast(C.pointer(job.g), C.c_void_p))
    cur, ecur = job.population(case.initpop)
    nxt, enxt = job.population()
    refpy.cuda_call("calc_initpop", R * P, T, cur, ecur)
    refpy.cuda_call("sum_evals", R, T)
    gens = 0
    while job.evals_runs.sum().item() / R < nev and gens < ngen:
        refpy.cuda_call("gen_and_eval_newpops", R * P, T, cur, ecur, nxt, enxt)
        refpy.cuda_call(LS_ENTRY[lsmet], R * L, T, nxt, enxt)
        refpy.cuda_call("sum_evals", R, T)
        gens += 1
        cur, nxt, ecur, enxt = nxt, cur, enxt, ecur
    torch.cuda.synchronize()
    return cur, ecur, gens, job


def engine_docking(case, lsmet, nev):
    dp = case.dockpars
    job = device.DeviceJob(case.tables, dp, case.grid, case.runs, case.prng)
    job.activate()
    r = dock.dock(job, case.initpop, lsmet, nev)
    torch.cuda.synchronize()
    return r.conformations, r.energies, r.generations, job


def top_clusters(case, pops, energies, k=3):
    """The reference's own process_result (host oracle) on a final
    population: best energy per run (scorer), and the best pose of each of the
    k lowest-energy clusters (cluster 1 first) with its re-scored energy."""
    P = case.info.pop_size
    p = pops.cpu().numpy().reshape(-1, 64)
    e = energies.cpu().numpy().reshape(-1)
    sp, se, runs, xyz, per = case.job.process_result(p, e)
    tops = []
    for cid in range(1, k + 1):
        i = next((i for i, r in enumerate(runs) if r.cluster_id == cid and r.cluster_subrank == 1), None)
        if i is not None:
            tops.append((xyz[i], runs[i].inter_e + runs[i].intra_e))
    return tops, se.reshape(-1, P)[:, 0]


def sym_rmsd(a, b, types):
    d2 = ((a[:, None, :] - b[None, :, :]) ** 2).sum(-1)
    d2 = np.where(types[:, None] == types[None, :], d2, np.inf)
    return float(np.sqrt(d2.min(axis=1).mean()))


@pytest.mark.parametrize("lsmet,size", [("ad", "cfg1"), ("sw", "cfg1"), ("adam", "cfg1"), ("ad", "cfg2")])
def test_docking_matches_reference_cuda_statistically(tmp_path, lsmet, size):
    """cfg1: 16 heavy atoms / 4 torsions on 40^3 maps, 48 runs of 1M
    evaluations; cfg2: the benchmark's docking, 40 heavy atoms / 10 torsions
    on 60^3 maps, 100 runs of 2.5M evaluations."""
    from scipy import stats
    if size == "cfg1":
        case = helpers.make_case(str(tmp_path), 40, ["C", "A", "N", "OA", "HD"], 16, 4, 48, config_id=1, lsmet=lsmet)
        nev = 1_000_000
    else:
        case = helpers.make_case(str(tmp_path), 60, ["C", "A", "N", "OA", "HD"], 40, 10, 100, config_id=2, lsmet=lsmet)
        nev = 2_500_000
    rc, re_, rgen, _ = reference_docking(case, lsmet, nev)
    ec, ee, egen, _ = engine_docking(case, lsmet, nev)
    r_tops, r_scorer = top_clusters(case, rc, re_)
    e_tops, e_scorer = top_clusters(case, ec, ee)
    ks = stats.ks_2samp(e_scorer, r_scorer)
    N = case.info.true_ligand_atoms
    types = case.tables["interintra"][1024:2048].view(np.uint32)[:N]

    def d(a, b):
        return sym_rmsd(a[0][:N], b[0][:N], types)
    e_in_r = min(d(e_tops[0], t) for t in r_tops)
    r_in_e = min(d(r_tops[0], t) for t in e_tops)
    print(json.dumps({"lsmet": lsmet, "size": size, "generations": [egen, rgen],
                      "best_energy_median": [float(np.median(e_scorer)), float(np.median(r_scorer))],
                      "best_energy_min": [float(e_scorer.min()), float(r_scorer.min())], "ks_p": float(ks.pvalue),
                      "top_pose_rmsd": d(e_tops[0], r_tops[0]), "engine_top_in_reference_top3": e_in_r,
                      "reference_top_in_engine_top3": r_in_e,
                      "top_cluster_energies": [[float(t[1]) for t in e_tops], [float(t[1]) for t in r_tops]]}))
    assert abs(egen - rgen) <= max(3, 0.1 * rgen)          # the same evaluation budget spent alike
    assert ks.pvalue > 1e-3, ks
    assert e_in_r < 2.0 and r_in_e < 2.0, (e_in_r, r_in_e)


def oracle_docking(case, lsmet, nev, nthreads=8):
    """docking_with_gpu's loop over the oracle's kernels on the host (the
    oracle's FIRE is pinned to the reference's OpenCL kernel,
    tests/test_oracle_pins.py; the reference has no CUDA FIRE to run)."""
    dp = case.dockpars
    R, P, L = case.runs, dp.pop_size, dp.num_of_lsentities
    ht = case.host
    ht.g.dockpars = dp
    prng = case.prng.copy()
    en, er = np.zeros(R * P, np.int32), np.zeros(R, np.int32)
    ht.bind_state(prng, en, er)
    cur = case.initpop[:R * P].copy()
    ecur = np.zeros(R * P, np.float32)
    nxt, enxt = np.zeros_like(cur), np.zeros_like(ecur)
    ht.call("calc_initpop", R * P, cur, ecur, nthreads)
    ht.call("sum_evals", R)
    gens = 0
    while er.sum() / R < nev:
        ht.call("gen_and_eval_newpops", R * P, T, cur, ecur, nxt, enxt, nthreads)
        ht.call(f"gradient_min{lsmet}", R * L, T, nxt, enxt, nthreads)
        ht.call("sum_evals", R)
        gens += 1
        cur, nxt, ecur, enxt = nxt, cur, enxt, ecur
    return torch.from_numpy(cur), torch.from_numpy(ecur), gens


def test_fire_docking_matches_oracle_statistically(tmp_path):
    """FIRE whole dockings (cfg1 ligand, 32 runs of 2.5M evaluations) against
    the oracle's, which follows the reference's OpenCL FIRE: same generation
    count, run best energies from the same distribution, top binding modes
    within 2 A of each other's three best clusters."""
    from scipy import stats
    case = helpers.make_case(str(tmp_path), 40, ["C", "A", "N", "OA", "HD"], 16, 4, 32, config_id=1, lsmet="fire")
    nev = 2_500_000
    rc, re_, rgen = oracle_docking(case, "fire", nev)
    ec, ee, egen, _ = engine_docking(case, "fire", nev)
    r_tops, r_scorer = top_clusters(case, rc, re_)
    e_tops, e_scorer = top_clusters(case, ec, ee)
    ks = stats.ks_2samp(e_scorer, r_scorer)
    N = case.info.true_ligand_atoms
    types = case.tables["interintra"][1024:2048].view(np.uint32)[:N]
    e_in_r = min(sym_rmsd(e_tops[0][0][:N], t[0][:N], types) for t in r_tops)
    r_in_e = min(sym_rmsd(r_tops[0][0][:N], t[0][:N], types) for t in e_tops)
    print(json.dumps({"lsmet": "fire", "generations": [egen, rgen], "ks_p": float(ks.pvalue),
                      "best_energy_median": [float(np.median(e_scorer)), float(np.median(r_scorer))],
                      "top": [e_in_r, r_in_e]}))
    assert abs(egen - rgen) <= max(3, 0.1 * rgen)
    assert ks.pvalue > 1e-3, ks
    assert e_in_r < 2.0 and r_in_e < 2.0
