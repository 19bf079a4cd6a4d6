"""Generates the golden vectors in tests/golden/ from the reference's OWN code
(oracle/_ref: the reference's host front end and its CUDA kernel sources run
on the CPU under the SIMT emulator).  Needs the reference checkout (only in
the build container); the output files are committed so the oracle and the
engine can be checked against them anywhere.

    python tests/golden/make_golden.py

Each fixture holds the reference-prepared tables of a seeded synthetic case
(the grid is regenerated from its seed by adgpu_b200.synth), seeded
genotypes with the reference scorer's energies and gradients, one GA
generation and short local searches (Solis-Wets, ADADELTA, ADAM from its CUDA
kernels, FIRE from its OpenCL kernel) with the PRNG states before and after.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "autodock-gpu_b200"), os.path.join(ROOT, "tests")]

import helpers  # noqa: E402
from adgpu_b200 import abi  # noqa: E402
from oracle import refpy  # noqa: E402

CASES = {
    "cfg1_small": dict(npts=24, types=["C", "A", "N", "OA", "HD"], n_heavy=10, n_tors=3, nrun=2, config_id=1, flexres=0),
    "flex_small": dict(npts=24, types=["C", "A", "N", "NA", "OA", "SA", "HD"], n_heavy=8, n_tors=2, nrun=2,
                       config_id=4, flexres=1),
}
T = 64


def sanitize(tables, dp, nrot):
    """Zeroes the table entries the kernels never read (the reference fills
    them from uninitialised host memory), so the fixtures compress."""
    N, NT, Q = dp.num_of_atoms, dp.num_of_atypes, dp.num_of_intraE_contributors
    t = {k: abi.TABLE_TYPES[k].from_buffer_copy(bytes(v)) for k, v in tables.items()}
    ii = t["interintra"]
    for a in range(N, abi.MAX_ATOMS):
        ii.atom_charges_const[a] = 0.0
        ii.atom_types_const[a] = 0
        ii.atom_types_map_const[a] = 0
    C = abi.C if hasattr(abi, "C") else None  # noqa: F841
    ic = np.frombuffer(bytes(t["intracontrib"]), np.uint32).copy()
    ic[2 * Q:] = 0
    kin = t["intra"]
    for k in range(NT, abi.MAX_ATYPES):
        kin.atom_types_reqm_const[k] = 0
        kin.dspars_S_const[k] = 0.0
        kin.dspars_V_const[k] = 0.0
    for k in range(NT * NT, abi.MAX_ATYPES * abi.MAX_ATYPES):
        kin.VWpars_exp_const[k] = 0
        kin.reqm_AB_const[k] = 0.0
        kin.VWpars_AC_const[k] = 0.0
        kin.VWpars_BD_const[k] = 0.0
    rl = np.frombuffer(bytes(t["rotlist"]), np.int32).copy()
    rl[dp.rotbondlist_length:] = 0
    cf = t["conform"]
    for k in range(3 * N, 3 * abi.MAX_ATOMS):
        cf.ref_coords_const[k] = 0.0
    for k in range(3 * nrot, 3 * abi.MAX_ROTBONDS):
        cf.rotbonds_moving_vectors_const[k] = 0.0
        cf.rotbonds_unit_vectors_const[k] = 0.0
    gr = t["grads"]
    rba = np.frombuffer(bytes(gr), np.int32).copy()
    off = abi.KcGrads.rotbonds_atoms.offset // 4
    for r in range(abi.MAX_ROTBONDS):
        n = gr.num_rotating_atoms_per_rotbond[r] if r < nrot else 0
        rba[off + r * abi.MAX_ATOMS + n: off + (r + 1) * abi.MAX_ATOMS] = 0
    for k in range(2 * nrot, 2 * abi.MAX_ROTBONDS):
        rba[k] = 0
    noff = abi.KcGrads.num_rotating_atoms_per_rotbond.offset // 4
    rba[noff + nrot: noff + abi.MAX_ROTBONDS] = 0
    return {"interintra": np.frombuffer(bytes(ii), np.uint8), "intracontrib": ic.view(np.uint8),
            "intra": np.frombuffer(bytes(kin), np.uint8), "rotlist": rl.view(np.uint8),
            "conform": np.frombuffer(bytes(cf), np.uint8), "grads": rba.view(np.uint8)}


def make(name, kw, tmp):
    case = helpers.make_case(os.path.join(tmp, name), kw["npts"], kw["types"], kw["n_heavy"], kw["n_tors"], kw["nrun"],
                             config_id=kw["config_id"], flexres=kw["flexres"], pop=16)
    job = case.job
    R, P = case.runs, case.dockpars.pop_size
    out = sanitize(case.tables, case.dockpars, case.info.num_of_rotbonds)
    out["dockpars"] = np.frombuffer(bytes(case.dockpars), np.uint8)
    out["grid_spec"] = np.array([kw["npts"], 12345 + kw["config_id"]], np.int64)
    out["map_types"] = np.array(kw["types"])
    out["initpop"] = case.initpop
    out["prng"] = case.prng
    # scorer
    g = helpers.in_box_genotypes(case, 64, seed=5, spread=1.5)
    pr = case.prng.copy(); en = np.zeros(R * P, np.int32); er = np.zeros(R, np.int32)
    job.bind(pr, en, er)
    e, gr = job.score(g, True)
    out["score_genotypes"], out["score_energy"], out["score_grad"] = g, e, gr
    # one GA generation on the initial population
    pop = case.initpop[:R * P].copy()
    e0 = np.zeros(R * P, np.float32)
    refpy.call("calc_initpop", R * P, T, pop, e0)
    out["initpop_energy"] = e0.copy()
    cn, enx = np.zeros_like(pop), np.zeros_like(e0)
    prng_before = pr.copy()
    refpy.call("gen_and_eval_newpops", R * P, T, pop, e0, cn, enx)
    out["ga_prng_before"], out["ga_prng_after"] = prng_before, pr.copy()
    out["ga_next"], out["ga_next_energy"], out["ga_evals_new"] = cn, enx, en.copy()
    # short local searches (4 iterations) from the GA offspring
    dp = abi.Dockpars.from_bytes(bytes(case.dockpars))
    dp.max_num_of_iters = 4
    # FIRE: the reference's OpenCL kernel (device/kernel_fire.cl) with its first
    # gradient from its merged scorer (its own first call reads coordinates it
    # never initialises, oracle/ref/ref_fire_tu.cpp)
    for meth in ("perform_ls", "gradient_minad", "gradient_minadam", "gradient_minfire"):
        pr2 = out["ga_prng_after"].copy()
        en2 = np.zeros(R * P, np.int32)
        job.bind(pr2, en2, er.copy(), dockpars=bytes(dp))
        c, ee = cn.copy(), enx.copy()
        refpy.call(meth, R * dp.num_of_lsentities, T, c, ee)
        out[f"{meth}_conf"], out[f"{meth}_energy"], out[f"{meth}_prng"], out[f"{meth}_evals"] = c, ee, pr2, en2
    out["ls_dockpars"] = np.frombuffer(bytes(dp), np.uint8)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, {k: v.shape for k, v in out.items() if k.startswith("score")})


if __name__ == "__main__":
    import tempfile
    with tempfile.TemporaryDirectory() as tmp:
        for name, kw in CASES.items():
            make(name, kw, tmp)
