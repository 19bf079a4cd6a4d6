"""Per-pose parity of the CUDA scorer with the oracle (energy and gene
gradients for identical genotypes), through the C ABI."""
import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    d = tmp_path_factory.mktemp("scorer")
    return {
        "cfg1": helpers.make_case(str(d / "cfg1"), 40, ["C", "A", "N", "OA", "HD"], 16, 4, 4, config_id=1),
        "cfg2": helpers.make_case(str(d / "cfg2"), 60, ["C", "A", "N", "OA", "HD"], 40, 10, 4, config_id=2),
        "flex": helpers.make_case(str(d / "flex"), 60, ["C", "A", "N", "NA", "OA", "SA", "HD"], 30, 8, 2,
                                  config_id=4, flexres=2),
    }


def _activate(case):
    from adgpu_b200 import device
    dj = device.DeviceJob(case.tables, case.dockpars, case.grid, case.runs, case.prng)
    dj.activate()
    return dj


@pytest.mark.parametrize("name", ["cfg1", "cfg2", "flex"])
@pytest.mark.parametrize("tpp", [32, 64, 128])
def test_energy_and_gradient_parity(cases, name, tpp, monkeypatch):
    from adgpu_b200 import device
    monkeypatch.setenv("ADGPU_THREADS_PER_POSE", str(tpp))
    case = cases[name]
    dj = _activate(case)
    g = helpers.in_box_genotypes(case, 2000 if name != "cfg1" else 1000, seed=7)
    e_gpu, gr_gpu = device.score(g, True)
    e_ref, gr_ref = case.host.score(g, True, nthreads=8)
    # the stated rule: |dE| <= 1e-4 |E| + 1e-6 * sum of |terms|
    tol = helpers.energy_contract(e_ref, helpers.oracle_terms(case, g))
    bad = np.abs(e_gpu - e_ref) > tol
    assert bad.sum() == 0, f"{bad.sum()} energies off, worst {np.abs(e_gpu - e_ref).max()}"
    e_only = device.score(g, False)
    assert np.all(np.abs(e_only - e_ref) <= tol)
    ng = case.ngenes
    diff = np.abs(gr_gpu[:, :ng] - gr_ref[:, :ng])
    # tier 1 (typical pose): 1e-4 relative plus a few fixed-point quanta
    frac_bad = (diff > helpers.gradient_tolerance(case, gr_ref)).mean(axis=0)
    assert frac_bad[:3].max() <= 0.002
    assert frac_bad[6:].max() <= 0.002 if ng > 6 else True
    # orientation genes pass through an infinitesimal-rotation difference of angles
    assert frac_bad[3:6].max() <= 0.01
    # tier 2 (every pose, clashes included): the per-term rule |d| <= 1e-4|ref| + n_terms/1024
    # in gene units, n_terms = quantised terms feeding a gene (atoms + both ends of every pair)
    assert np.all(diff <= helpers.gradient_bound(case, gr_ref)), diff.max(axis=0)
    del dj


def test_out_of_grid_penalty(cases):
    from adgpu_b200 import device
    case = cases["cfg1"]
    _activate(case)
    g = helpers.in_box_genotypes(case, 64, seed=3)
    g[:32, 0] = -5.0     # far outside the box
    e_gpu, gr_gpu = device.score(g, True)
    e_ref, gr_ref = case.host.score(g, True)
    assert np.all(e_gpu[:32] > 1.6e7)
    assert np.allclose(e_gpu, e_ref, rtol=1e-5)
    assert np.allclose(gr_gpu[:32, :3], gr_ref[:32, :3])


def test_large_ligand_parity(tmp_path):
    """Near the reference's limits: 110 heavy atoms (plus polar H), 30
    torsions, some 6,400 intramolecular pairs."""
    from adgpu_b200 import device
    case = helpers.make_case(str(tmp_path / "big"), 60, ["C", "A", "N", "OA", "HD"], 110, 30, 2, config_id=2,
                             lig_index=7)
    dj = _activate(case)
    g = helpers.in_box_genotypes(case, 300, seed=3)
    e_gpu, gr_gpu = device.score(g, True)
    e_ref, gr_ref = case.host.score(g, True, nthreads=8)
    tol = helpers.energy_contract(e_ref, helpers.oracle_terms(case, g))
    assert np.all(np.abs(e_gpu - e_ref) <= tol), np.abs(e_gpu - e_ref).max()
    ng = case.ngenes
    assert np.all(np.abs(gr_gpu[:, :ng] - gr_ref[:, :ng]) <= helpers.gradient_bound(case, gr_ref))
    del dj


def test_maximum_size_parity(tmp_path):
    """At the reference's limits: 252 atoms (226 heavy plus polar H), 57
    torsions (MAX_NUM_OF_ROTBONDS), 29,104 intramolecular pairs, 80^3 maps;
    poses near the input conformation so that the terms stay finite."""
    from adgpu_b200 import device
    case = helpers.make_case(str(tmp_path / "max"), 80, ["C", "A", "N", "OA", "HD"], 226, 57, 2, config_id=3)
    assert case.info.num_of_rotbonds == 57 and case.info.num_of_atoms > 240
    dj = _activate(case)
    g = helpers.in_box_genotypes(case, 200, seed=3, spread=1.0)
    g[:, 6:case.ngenes] = np.random.default_rng(4).normal(0.0, 5.0, (200, case.ngenes - 6)).astype(np.float32)
    e_gpu, gr_gpu = device.score(g, True)
    e_ref, gr_ref = case.host.score(g, True, nthreads=8)
    tol = helpers.energy_contract(e_ref, helpers.oracle_terms(case, g))
    assert np.all(np.abs(e_gpu - e_ref) <= tol), np.abs(e_gpu - e_ref).max()
    ng = case.ngenes
    assert np.all(np.abs(gr_gpu[:, :ng] - gr_ref[:, :ng]) <= helpers.gradient_bound(case, gr_ref))
    del dj


@pytest.mark.parametrize("name", ["cfg1", "cfg2", "flex"])
def test_per_term_energies(cases, name):
    """Each energy term against the oracle's, for identical genotypes: the
    three intermolecular maps and the four intramolecular terms, each within
    1e-4 relative plus a floor of 1e-6 of the pose's summed |terms| (the
    oracle sums in another order); the out-of-grid count exactly."""
    from adgpu_b200 import device
    case = cases[name]
    _activate(case)
    g = helpers.in_box_genotypes(case, 400, seed=17)
    g[:20, 0] = -3.0                      # some atoms outside the grid
    e, t = device.score_terms(g)
    ref = np.array([case.host.score_terms(x)[2] for x in g])
    assert np.array_equal(t[:, 7], ref[:, 7])
    scale = np.abs(ref[:, :7]).sum(axis=1, keepdims=True)
    tol = 1e-4 * np.abs(ref[:, :7]) + 1e-6 * scale + 1e-5
    assert np.all(np.abs(t[:, :7] - ref[:, :7]) <= tol), np.abs(t[:, :7] - ref[:, :7]).max(axis=0)
    # the terms add up to the energy (plus the out-of-grid penalties)
    total = t[:, :7].astype(np.float64).sum(axis=1) + 16777216.0 * t[:, 7]
    assert np.allclose(total, e, rtol=1e-5, atol=1e-3)


@pytest.mark.parametrize("tpp", [32, 64])
def test_modified_pair_exponents(tmp_path, tpp, monkeypatch):
    """Modified vdW pair potentials (the reference's --modpair: C-C as 13-7,
    C-A as 12-8) are scored by the general-exponent pair loop next to the AD4
    pairs: energies, gradients and the per-term split by the same rules as
    the AD4 pairs."""
    from adgpu_b200 import device
    monkeypatch.setenv("ADGPU_THREADS_PER_POSE", str(tpp))
    case = helpers.make_case(str(tmp_path / "mod"), 40, ["C", "A", "N", "OA", "HD"], 16, 4, 2, config_id=1,
                             extra_args=("--modpair", "C:C,4.00,0.150,13,7/C:A,4.00,0.150,12,8"))
    assert helpers.generic_pairs(case) > 20
    dj = _activate(case)
    g = helpers.in_box_genotypes(case, 1000, seed=11)
    e_gpu, gr_gpu = device.score(g, True)
    e_ref, gr_ref = case.host.score(g, True, nthreads=8)
    tol = helpers.energy_contract(e_ref, helpers.oracle_terms(case, g))
    assert np.all(np.abs(e_gpu - e_ref) <= tol), np.abs(e_gpu - e_ref).max()
    ng = case.ngenes
    assert np.all(np.abs(gr_gpu[:, :ng] - gr_ref[:, :ng]) <= helpers.gradient_bound(case, gr_ref))
    e, t = device.score_terms(g[:200])
    ref = np.array([case.host.score_terms(x)[2] for x in g[:200]])
    scale = np.abs(ref[:, :7]).sum(axis=1, keepdims=True)
    assert np.all(np.abs(t[:, :7] - ref[:, :7]) <= 1e-4 * np.abs(ref[:, :7]) + 1e-6 * scale + 1e-5)
    del dj
