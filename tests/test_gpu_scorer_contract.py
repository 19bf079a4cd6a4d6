"""The scorer contract at the plain GPU configuration: 10^4 seeded genotypes
of the cfg2 ligand (40 heavy atoms, 10 torsions, 60^3 maps) with translations
uniform over the grid box, orientations uniform on SO(3) and torsions uniform
in [-180, 180), scored through the C ABI, against the oracle:

  energy    |dE| <= 1e-4 |E| + 1e-6 * sum |terms|
  gradient  |dg| <= 1e-4 |g| + n_terms / 1024   (gene units)

The same genotypes are scored by the reference's own CUDA kernels
(cuda/*.cu compiled unchanged for sm_100a with its -use_fast_math,
oracle/_ref) against the same oracle, which measures how far the reference
itself lies from exact arithmetic under the same rule: the orientation genes
are the difference of two angles taken through a 1e-3 rad infinitesimal
rotation (cuda/calcMergeEneGra.cu:695-815), so one quantum of torque moves
them by far more than a quantum."""
import json

import numpy as np
import pytest
import torch

import helpers

pytestmark = pytest.mark.gpu
N = 10_000


@pytest.fixture(scope="module")
def cfg2(tmp_path_factory):
    d = tmp_path_factory.mktemp("contract")
    case = helpers.make_case(str(d / "cfg2"), 60, ["C", "A", "N", "OA", "HD"], 40, 10, 4, config_id=2)
    g = helpers.uniform_box_genotypes(case, N, seed=2024)
    e_or, g_or = case.host.score(g, True, nthreads=8)
    terms = np.array([case.host.score_terms(x)[2] for x in g])
    return case, g, e_or, g_or, terms


def _score_engine(case, g, tpp, monkeypatch):
    from adgpu_b200 import device
    monkeypatch.setenv("ADGPU_THREADS_PER_POSE", str(tpp))
    dj = device.DeviceJob(case.tables, case.dockpars, case.grid, case.runs, case.prng)
    dj.activate()
    e, gr = device.score(g, True)
    e_only = device.score(g, False)
    return e, gr, e_only


@pytest.mark.parametrize("tpp", [32, 64, 128])
def test_cfg2_energy_contract(cfg2, tpp, monkeypatch):
    case, g, e_or, g_or, terms = cfg2
    e, gr, e_only = _score_engine(case, g, tpp, monkeypatch)
    tol = helpers.energy_contract(e_or, terms)
    out = int(terms[:, 7].astype(bool).sum())
    assert out > N // 4, "the sample must put many poses partly outside the grid"
    assert np.all(np.abs(e - e_or) <= tol), np.abs(e - e_or).max()
    assert np.all(np.abs(e_only - e_or) <= tol)


@pytest.mark.parametrize("tpp", [32, 64])
def test_cfg2_gradient_contract(cfg2, tpp, monkeypatch):
    """Translation and torsion genes: every pose within the rule.
    Orientation genes: within the rule as often as the reference's own CUDA
    build (and never further out than it is at worst)."""
    from oracle import refpy
    case, g, e_or, g_or, terms = cfg2
    _, gr, _ = _score_engine(case, g, tpp, monkeypatch)
    ng = case.ngenes
    bound = helpers.gradient_contract(case, g_or)
    d = np.abs(gr[:, :ng] - g_or[:, :ng])
    assert np.all(d[:, :3] <= bound[:, :3]), (d[:, :3] / bound[:, :3]).max()
    assert np.all(d[:, 6:] <= bound[:, 6:]), (d[:, 6:] / bound[:, 6:]).max()
    frac_me = float((d[:, 3:6] > bound[:, 3:6]).mean())
    worst_me = float((d[:, 3:6] / bound[:, 3:6]).max())
    if not refpy.cuda_available():
        assert frac_me <= 0.01
        return
    import ctypes as C
    from adgpu_b200 import device
    rj = device.DeviceJob(case.tables, case.dockpars, case.grid, case.runs, case.prng)
    refpy.cuda_lib().adgpu_refcuda_set_gpudata(C.cast(C.pointer(rj.g), C.c_void_p))
    gt = torch.from_numpy(g).cuda()
    e_ref = torch.zeros(len(g), device="cuda")
    gr_ref = torch.zeros_like(gt)
    assert refpy.cuda_call("score", len(g), gt, e_ref, gr_ref) == 0
    d_ref = np.abs(gr_ref.cpu().numpy()[:, :ng] - g_or[:, :ng])
    frac_ref = float((d_ref[:, 3:6] > bound[:, 3:6]).mean())
    worst_ref = float((d_ref[:, 3:6] / bound[:, 3:6]).max())
    print(json.dumps({"tpp": tpp, "orientation_outside_rule": {"engine": frac_me, "reference_cuda": frac_ref},
                      "orientation_worst_ratio": {"engine": worst_me, "reference_cuda": worst_ref},
                      "translation_torsion_outside_rule_reference_cuda": float(
                          np.concatenate([(d_ref[:, :3] > bound[:, :3]).ravel(),
                                          (d_ref[:, 6:] > bound[:, 6:]).ravel()]).mean())}))
    assert frac_me <= max(frac_ref, 1e-3)
    assert worst_me <= max(worst_ref, 1.0)
