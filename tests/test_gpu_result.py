"""Result processing on the device against the reference's own process_result
(oracle/_ref: arrange_result + make_resfiles + generate_output's clustering,
host/src/processresult.cpp, compiled from the reference sources for the CPU).

The device code follows the host arithmetic operation by operation, so the
ordering, cluster assignments and subranks must be identical and the
energies, RMSDs and coordinates equal up to the last-place rounding of the
device's double sin/cos (tolerances below: coordinates 1e-9 A, energies
1e-5 relative, RMSDs 1e-5 A); most values come out bit-identical and the
tests require at least 90 % of them to."""
import numpy as np
import pytest
import torch

import helpers
from adgpu_b200 import frontend, result, synth
from oracle import refpy

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refpy.available(), reason="oracle/_ref not built (needs the reference checkout)")]


def product_inputs(tmp_path, case, flex=False):
    g = frontend.Grid.read(str(tmp_path / "receptor.maps.fld"))
    lig = (tmp_path / "ligand0.pdbqt").read_text()
    fr = (tmp_path / "flexres.pdbqt").read_text() if flex else None
    seed = tuple(int(s) for s in helpers.SEEDS.split(","))
    L = frontend.Ligand(g, lig, fr, run=frontend.default_dockpars(g.spacing), seed=seed, num_runs=case.runs)
    grid_dev = torch.from_numpy(g.reference_layout()).cuda()
    return L, grid_dev


def clustered_population(case, nbase=3, seed=0, spread=0.15):
    """Runs whose entities lie around a few base poses (so that runs cluster),
    with seeded energies that include ties and NaNs."""
    R, P = case.runs, case.info.pop_size
    rng = np.random.default_rng(seed)
    base = helpers.in_box_genotypes(case, nbase, seed=seed + 1, spread=1.0)
    pops = np.repeat(base[np.arange(R) % nbase], P, axis=0).reshape(R * P, -1).copy()
    G = case.ngenes
    pops[:, :3] += rng.normal(0.0, spread, (R * P, 3)).astype(np.float32)
    pops[:, 3:G] += rng.normal(0.0, 4.0 * spread, (R * P, G - 3)).astype(np.float32)
    en = rng.normal(-6.0, 2.0, R * P).astype(np.float32)
    en[7] = en[9]                       # a tie
    if R > 2:
        en[P + 5] = np.nan              # a NaN inside run 1: splits its ordering
        en[2 * P] = np.nan              # a NaN first in run 2: stays the run's entity 0
    return pops, en


def frac_equal(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.mean((a == b) | (np.isnan(a) & np.isnan(b))))


def run_both(tmp_path, case, pops, en, flex=False, **kw):
    L, grid_dev = product_inputs(tmp_path, case, flex)
    R = case.runs
    ref_pops, ref_en, ref_runs, ref_xyz, ref_per = case.job.process_result(
        pops, en, rmsd_tol=kw.get("rmsd_tolerance", 2.0), symmetry=bool(kw.get("handle_symmetry", 1)),
        clustering=bool(kw.get("calc_clustering", 1)), nr_cluster_poses=kw.get("nr_cluster_poses", 0))
    params = result.default_params(**kw)
    dp = torch.from_numpy(pops.copy()).cuda()
    de = torch.from_numpy(en.copy()).cuda()
    out = result.process_result(L, grid_dev, dp, de, R, params)
    torch.cuda.synchronize()
    return (ref_pops, ref_en, ref_runs, ref_xyz, ref_per), out, dp.cpu().numpy(), de.cpu().numpy(), L, grid_dev


def check_against_reference(ref, out, dev_pops, dev_en, R):
    ref_pops, ref_en, ref_runs, ref_xyz, ref_per = ref
    # arrange_result: a permutation, so bit-identical
    assert np.array_equal(dev_pops, ref_pops)
    assert np.array_equal(dev_en, ref_en, equal_nan=True)
    fields = ("inter_e", "interflex_e", "inter_e_elec", "intra_e", "intraflex_e")
    got = np.array([[getattr(r, f) for f in fields] for r in out.runs], np.float64)
    want = np.array([[getattr(r, f) for f in fields] for r in ref_runs], np.float64)
    assert np.allclose(got, want, rtol=1e-5, atol=1e-5), np.abs(got - want).max()
    rm = np.array([r.rmsd_from_ref for r in out.runs]), np.array([r.rmsd_from_ref for r in ref_runs])
    assert np.allclose(rm[0], rm[1], atol=1e-5)
    assert np.allclose(out.best_xyz, ref_xyz, rtol=0, atol=1e-9)
    assert np.allclose(out.peratom, ref_per, rtol=1e-5, atol=1e-5)
    # generate_output: identical clusters, subranks and output flags
    for a, b in zip(out.runs, ref_runs):
        assert (a.cluster_id, a.cluster_subrank, a.output, a.run_number) == \
            (b.cluster_id, b.cluster_subrank, b.output, b.run_number)
        assert abs(a.rmsd_from_cluster_center - b.rmsd_from_cluster_center) <= 1e-5
    assert [r.energy for r in out.runs] == pytest.approx(list(ref_en.reshape(R, -1)[:, 0]), nan_ok=True)
    exact = np.mean([frac_equal(got, want), frac_equal(out.best_xyz, ref_xyz), frac_equal(out.peratom, ref_per)])
    assert exact >= 0.9, exact
    return exact


@pytest.mark.parametrize("name,kw", [
    ("cfg1", dict(npts=40, types=synth.MAP_TYPES_5, n_heavy=16, n_tors=4, config_id=1, nrun=12)),
    ("cfg2", dict(npts=60, types=synth.MAP_TYPES_5, n_heavy=40, n_tors=10, config_id=2, nrun=20)),
    ("rigid", dict(npts=40, types=synth.MAP_TYPES_5, n_heavy=12, n_tors=0, config_id=3, nrun=9)),
])
def test_process_result_matches_reference(tmp_path, name, kw):
    kw = dict(kw)
    case = helpers.make_case(str(tmp_path), kw.pop("npts"), kw.pop("types"), kw.pop("n_heavy"), kw.pop("n_tors"),
                             kw.pop("nrun"), **kw)
    pops, en = clustered_population(case)
    ref, out, dev_pops, dev_en, _, _ = run_both(tmp_path, case, pops, en)
    check_against_reference(ref, out, dev_pops, dev_en, case.runs)
    # clusters formed (several runs share a base pose) and their statistics
    ids = [r.cluster_id for r in out.runs]
    assert max(ids) == len(out.clusters) and len(out.clusters) < case.runs
    sizes = np.bincount(ids)[1:]
    assert [c.size for c in out.clusters] == sizes.tolist()
    tors = 0.2983 * case.info.num_of_rotbonds
    for c_id, c in enumerate(out.clusters, 1):
        members = sorted((r for r in out.runs if r.cluster_id == c_id), key=lambda r: r.cluster_subrank)
        e = [np.float64(np.float32(r.inter_e) + np.float32(r.interflex_e)) + tors for r in members]
        assert c.best_run == members[0].run_number
        assert c.best_energy == e[0]
        assert c.sum_energy == pytest.approx(sum(e), rel=1e-12)


def test_process_result_flexres_options(tmp_path):
    """Ligand plus two flexible residues (interflex / intraflex terms), with
    symmetry off, a tighter tolerance and at most two poses per cluster."""
    case = helpers.make_case(str(tmp_path), 40, synth.MAP_TYPES_7, 14, 3, 12, config_id=4, flexres=2)
    pops, en = clustered_population(case, nbase=2, seed=4)
    kw = dict(handle_symmetry=0, rmsd_tolerance=1.0, nr_cluster_poses=2)
    ref, out, dev_pops, dev_en, _, _ = run_both(tmp_path, case, pops, en, flex=True, **kw)
    check_against_reference(ref, out, dev_pops, dev_en, case.runs)
    assert any(r.interflex_e != 0.0 for r in out.runs) or any(r.intraflex_e != 0.0 for r in out.runs)


def test_process_result_without_clustering_and_entity_rescoring(tmp_path):
    """calc_clustering off; every entity re-scored as the final-population
    report does, against make_resfiles' per-entity body."""
    case = helpers.make_case(str(tmp_path), 40, synth.MAP_TYPES_5, 16, 4, 6, config_id=1)
    pops, en = clustered_population(case, seed=9)
    ref, out, dev_pops, dev_en, L, grid_dev = run_both(tmp_path, case, pops, en, calc_clustering=0)
    check_against_reference(ref, out, dev_pops, dev_en, case.runs)
    assert all(r.cluster_id == 0 and r.output == 1 for r in out.runs) and out.clusters == []
    params = result.default_params(rescore_entities=1)
    dp = torch.from_numpy(dev_pops.copy()).cuda()
    de = torch.from_numpy(dev_en.copy()).cuda()
    out2 = result.process_result(L, grid_dev, dp, de, case.runs, params)
    want = case.job.rescore(dev_pops).reshape(case.runs, -1, 3)
    assert np.allclose(out2.entities, want, rtol=1e-5, atol=1e-5), np.abs(out2.entities - want).max()
    assert frac_equal(out2.entities, want) >= 0.9


def test_process_result_argument_errors(tmp_path):
    case = helpers.make_case(str(tmp_path), 40, synth.MAP_TYPES_5, 16, 4, 2, config_id=1)
    L, grid_dev = product_inputs(tmp_path, case)
    dp = torch.zeros(2 * 150 * 64, device="cuda")
    de = torch.zeros(2 * 150, device="cuda")
    with pytest.raises(Exception):
        result.process_result(L, grid_dev, dp, de, 2, result.default_params(nr_cluster_poses=-1))
    with pytest.raises(Exception):
        result.process_result(L, grid_dev, dp, de, 0)


def test_engine_process_result_matches_reference(tmp_path):
    """The engine's result processing (resident cell-record maps, final
    populations gathered from its double buffers) on a docked request, against
    the reference's process_result on the same final populations."""
    from adgpu_b200 import engine
    case = helpers.make_case(str(tmp_path), 40, synth.MAP_TYPES_5, 16, 4, 8, config_id=1)
    L, _ = product_inputs(tmp_path, case)
    g = frontend.Grid.read(str(tmp_path / "receptor.maps.fld"))
    en = engine.Engine(memory_budget_bytes=1 << 30)
    rec = en.add_receptor(g)
    rid = en.submit(L, rec, "ad", max_evals=60_000)
    en.run()
    out, fp, fe = en.process_result(rid, case.info.num_of_atoms, final_population=True)
    en.result(rid)
    assert np.all(np.diff(fe.reshape(case.runs, -1), axis=1) >= 0)      # ordered per run
    ref_pops, ref_en, ref_runs, ref_xyz, ref_per = case.job.process_result(fp, fe)
    assert np.array_equal(ref_pops, fp) and np.array_equal(ref_en, fe)   # already in arrange_result's order
    check_against_reference((ref_pops, ref_en, ref_runs, ref_xyz, ref_per), out, fp, fe, case.runs)
    en.close()


def test_process_result_maximum_size(tmp_path):
    """252 atoms, 57 torsions, 29,104 pairs: the largest ligand the reference
    accepts, runs clustered around two poses near the input conformation."""
    case = helpers.make_case(str(tmp_path), 80, synth.MAP_TYPES_5, 226, 57, 6, config_id=3)
    R, P = case.runs, case.info.pop_size
    rng = np.random.default_rng(6)
    base = helpers.in_box_genotypes(case, 2, seed=8, spread=1.0)
    base[:, 6:case.ngenes] = rng.normal(0.0, 5.0, (2, case.ngenes - 6)).astype(np.float32)
    pops = np.repeat(base[np.arange(R) % 2], P, axis=0).copy()
    pops[:, :case.ngenes] += rng.normal(0.0, 0.05, (R * P, case.ngenes)).astype(np.float32)
    en = rng.normal(-6.0, 2.0, R * P).astype(np.float32)
    ref, out, dev_pops, dev_en, _, _ = run_both(tmp_path, case, pops, en)
    check_against_reference(ref, out, dev_pops, dev_en, R)
