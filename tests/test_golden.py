"""The oracle and, on a GPU, the engine against the golden vectors that
tests/golden/make_golden.py produced with the reference's own code."""
import glob
import os

import numpy as np
import pytest

from adgpu_b200 import abi, frontend, synth
from oracle import oraclepy

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
T = 64
TABLES = ("interintra", "intracontrib", "intra", "rotlist", "conform", "grads")


def load(path, tmp_path):
    f = dict(np.load(path))
    npts, seed = (int(x) for x in f["grid_spec"])
    types = [str(t) for t in f["map_types"]]
    spec = synth.grid_spec(npts, types, seed=seed)
    synth.write_maps(spec, synth.make_maps(spec), str(tmp_path))
    grid = frontend.Grid.read(str(tmp_path / "receptor.maps.fld")).reference_layout()
    dp = abi.Dockpars.from_bytes(f["dockpars"].tobytes())
    return f, dp, grid


def _quanta(dp, ng):
    q = np.ones(ng) / 1024.0
    q[3:] *= dp.grid_spacing ** 2 / 0.0174533 ** 2
    return q


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_oracle_against_golden(path, tmp_path):
    f, dp, grid = load(path, tmp_path)
    ht = oraclepy.HostTables({k: f[k] for k in TABLES}, dp, grid)
    R = f["initpop"].shape[0] // (dp.pop_size)
    P = dp.pop_size
    ng = dp.num_of_genes
    # scorer
    e, gr = ht.score(f["score_genotypes"], True)
    ref_e, ref_g = f["score_energy"], f["score_grad"]
    assert np.all(np.abs(e - ref_e) <= 1e-5 * np.abs(ref_e) + 1e-4)
    d = np.abs(gr[:, :ng] - ref_g[:, :ng])
    assert (d > 2.5 * _quanta(dp, ng) + 1e-4 * np.abs(ref_g[:, :ng])).mean() < 0.01
    # initial population energies
    st = [f["prng"].copy(), np.zeros(R * P, np.int32), np.zeros(R, np.int32)]
    ht.bind_state(*st)
    pop = f["initpop"][:R * P].copy()
    e0 = np.zeros(R * P, np.float32)
    ht.call("calc_initpop", R * P, pop, e0, 1)
    assert np.all(np.abs(e0 - f["initpop_energy"]) <= 1e-5 * np.abs(f["initpop_energy"]) + 1e-4)
    # one GA generation from the golden energies: bit-exact genes and PRNG states
    st[0][:] = f["ga_prng_before"]
    st[1][:] = 0
    cn, en = np.zeros_like(pop), np.zeros_like(e0)
    ht.call("gen_and_eval_newpops", R * P, T, pop, f["initpop_energy"].copy(), cn, en, 1)
    assert np.array_equal(st[0], f["ga_prng_after"])
    assert np.array_equal(cn[:, :ng], f["ga_next"][:, :ng])
    assert np.array_equal(st[1], f["ga_evals_new"])
    # short local searches from the golden offspring
    ldp = abi.Dockpars.from_bytes(f["ls_dockpars"].tobytes())
    ht.g.dockpars = ldp
    # FIRE's golden vectors come from the reference's OpenCL kernel, whose
    # merged scorer sums the translation gradient over the flexible residues'
    # atoms too (calcMergedEneGra.cl:635, against the CUDA scorer's ligand
    # atoms, calcMergeEneGra.cu:618, which the oracle and the engine follow):
    # compared on rigid-receptor fixtures only
    meths = ("perform_ls", "gradient_minad", "gradient_minadam")
    if dp.true_ligand_atoms == dp.num_of_atoms:
        meths += ("gradient_minfire",)
    for meth in (m for m in meths if f"{m}_conf" in f):
        st[0][:] = f["ga_prng_after"]
        st[1][:] = 0
        c, ee = f["ga_next"].copy(), f["ga_next_energy"].copy()
        ht.call(meth, R * ldp.num_of_lsentities, T, c, ee, 1)
        close = np.abs(c[:, :ng] - f[f"{meth}_conf"][:, :ng]).max(axis=1) <= 1e-2
        assert close.mean() >= 0.95, meth
        if meth != "perform_ls":
            assert np.array_equal(st[0], f[f"{meth}_prng"])
            assert np.array_equal(st[1], f[f"{meth}_evals"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p) for p in FIXTURES])
def test_engine_against_golden(path, tmp_path):
    """The CUDA path through the C ABI against the reference's own outputs
    (no oracle in between): scorer energies and gradients, one GA generation
    bit-exact, short local searches entity by entity."""
    import torch
    from adgpu_b200 import device, lib
    f, dp, grid = load(path, tmp_path)
    R = f["initpop"].shape[0] // dp.pop_size
    P, ng = dp.pop_size, dp.num_of_genes
    tables = {k: f[k] for k in TABLES}
    job = device.DeviceJob(tables, dp, grid, R, f["prng"])
    job.activate()
    e, gr = device.score(f["score_genotypes"], True)
    ref_e, ref_g = f["score_energy"], f["score_grad"]
    assert np.all(np.abs(e - ref_e) <= 1e-4 * np.abs(ref_e) + 1e-4)
    # gradients: 1e-4 relative plus one quantum per quantised term feeding the
    # gene; the orientation genes pass through a 1e-3 rad difference of angles
    # (cuda/calcMergeEneGra.cu:695-815), which amplifies that by up to 1e3
    d = np.abs(gr[:, :ng] - ref_g[:, :ng])
    bound = 1e-4 * np.abs(ref_g[:, :ng]) + _quanta(dp, ng) * (dp.num_of_atoms + 2 * dp.num_of_intraE_contributors)
    bound[:, 3:6] *= 1e3 / 1024.0 * 8.0
    assert np.all(d <= bound), (d / bound).max(axis=0)
    # one GA generation from the golden energies and PRNG states
    job.prng.copy_(torch.from_numpy(f["ga_prng_before"].view(np.int32)).cuda())
    cur, ecur = job.population(f["initpop"])
    ecur.copy_(torch.from_numpy(f["initpop_energy"]).cuda())
    nxt, enxt = job.population()
    job.evals_new.zero_()
    lib.call("adgpu_gen_and_eval_newpops", R * P, T, cur, ecur, nxt, enxt)
    torch.cuda.synchronize()
    assert np.array_equal(job.prng.cpu().numpy().view(np.uint32), f["ga_prng_after"])
    assert np.array_equal(nxt.cpu().numpy()[:, :ng], f["ga_next"][:, :ng])
    assert np.array_equal(job.evals_new.cpu().numpy()[:R * P], f["ga_evals_new"])
    # short local searches from the golden offspring
    ldp = abi.Dockpars.from_bytes(f["ls_dockpars"].tobytes())
    meths = [("perform_ls", "adgpu_perform_ls"), ("gradient_minad", "adgpu_gradient_minad"),
             ("gradient_minadam", "adgpu_gradient_minadam")]
    if dp.true_ligand_atoms == dp.num_of_atoms:
        meths.append(("gradient_minfire", "adgpu_gradient_minfire"))
    for meth, entry in meths:
        if f"{meth}_conf" not in f:
            continue
        lj = device.DeviceJob(tables, ldp, grid, R, f["ga_prng_after"])
        lj.activate()
        c, ee = lj.population(f["ga_next"])
        ee.copy_(torch.from_numpy(f["ga_next_energy"]).cuda())
        lib.call(entry, R * ldp.num_of_lsentities, T, c, ee)
        torch.cuda.synchronize()
        # 32 entities: a rounding difference can flip an accept/reject
        # decision of one or two of them
        close = np.abs(c.cpu().numpy()[:, :ng] - f[f"{meth}_conf"][:, :ng]).max(axis=1) <= 1e-2
        assert close.mean() >= 0.9, meth
        if meth != "perform_ls":
            assert np.array_equal(lj.prng.cpu().numpy().view(np.uint32), f[f"{meth}_prng"]), meth
            assert np.array_equal(lj.evals_new.cpu().numpy()[:R * P], f[f"{meth}_evals"]), meth
