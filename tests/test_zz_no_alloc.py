"""adgpu_score_genotypes_noalloc: the scorer variant that allocates no device
memory.  Through the C ABI it must score as adgpu_score_genotypes does and
as the oracle does, on two calls in a row and after another ligand has used
its fixed scratch array, and reject ligands beyond that array's size before
touching the device.  The file is named to collect last, so it also runs after the rest
of the GPU suite in one process."""
import ctypes as C

import numpy as np
import pytest
import torch

import helpers
from adgpu_b200 import abi, lib


def _noalloc(job, g: torch.Tensor, grads: bool):
    n = g.shape[0]
    e = torch.full((n,), float("nan"), dtype=torch.float32, device=g.device)
    gr = torch.full((n, abi.GENOTYPE_STRIDE), float("nan"), dtype=torch.float32, device=g.device) if grads else None
    lib.call("adgpu_score_genotypes_noalloc", C.cast(C.pointer(job.g), C.c_void_p), n, g, e, gr)
    torch.cuda.synchronize()
    return (e.cpu().numpy(), gr.cpu().numpy()) if grads else e.cpu().numpy()


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    d = tmp_path_factory.mktemp("noalloc")
    return {
        "cfg2": helpers.make_case(str(d / "cfg2"), 60, ["C", "A", "N", "OA", "HD"], 40, 10, 4, config_id=2),
        "flex": helpers.make_case(str(d / "flex"), 60, ["C", "A", "N", "NA", "OA", "SA", "HD"], 30, 8, 2,
                                  config_id=4, flexres=2),
    }


@pytest.mark.gpu
def test_noalloc_matches_scorer_on_consecutive_calls(cases):
    from adgpu_b200 import device
    jobs = {}
    for name in ("cfg2", "flex", "cfg2"):
        case = cases[name]
        job = jobs.get(name) or device.DeviceJob(case.tables, case.dockpars, case.grid, case.runs, case.prng)
        jobs[name] = job
        job.activate()
        gh = helpers.in_box_genotypes(case, 1500, seed=11)
        e_ref, gr_ref = device.score(gh, True)
        e_ref_only = device.score(gh, False)
        g = torch.from_numpy(np.ascontiguousarray(gh, np.float32)).cuda()
        first = _noalloc(job, g, True)
        second = _noalloc(job, g, True)
        e_only = _noalloc(job, g, False)
        tol = helpers.energy_tolerance(e_ref)
        ng = case.ngenes
        for e, gr in (first, second):
            assert np.all(np.abs(e - e_ref) <= tol), np.abs(e - e_ref).max()
            diff = np.abs(gr[:, :ng] - gr_ref[:, :ng])
            assert np.all(diff <= helpers.gradient_bound(case, gr_ref)), diff.max(axis=0)
        assert np.array_equal(first[0], second[0]) and np.array_equal(first[1][:, :ng], second[1][:, :ng])
        assert np.all(np.abs(e_only - e_ref_only) <= helpers.energy_tolerance(e_ref_only))
        # and against the oracle directly (its own code path reads the
        # caller's reference-layout grid, which no other entry point does)
        e_or, gr_or = case.host.score(gh, True, nthreads=8)
        terms = np.array([case.host.score_terms(x)[2] for x in gh])
        assert np.all(np.abs(first[0] - e_or) <= helpers.energy_contract(e_or, terms)), np.abs(first[0] - e_or).max()
        d = np.abs(first[1][:, :ng] - gr_or[:, :ng])
        assert np.all(d <= helpers.gradient_bound(case, gr_or)), d.max(axis=0)


@pytest.mark.gpu
def test_noalloc_zero_poses_is_a_no_op(cases):
    from adgpu_b200 import device
    case = cases["cfg2"]
    job = device.DeviceJob(case.tables, case.dockpars, case.grid, case.runs, case.prng)
    g = torch.zeros((1, abi.GENOTYPE_STRIDE), dtype=torch.float32, device="cuda:0")
    e = torch.full((1,), 7.0, dtype=torch.float32, device="cuda:0")
    lib.call("adgpu_score_genotypes_noalloc", C.cast(C.pointer(job.g), C.c_void_p), 0, g, e, None)
    assert e.item() == 7.0


def test_noalloc_rejects_ligands_beyond_its_scratch():
    """Host-side checks only: the call returns before any device access."""
    L = lib.load()
    g = abi.GpuData()
    for f in ("pKerconst_interintra", "pKerconst_intracontrib", "pKerconst_intra", "pKerconst_rotlist",
              "pKerconst_conform", "pMem_fgrids", "pMem_rotbonds_const", "pMem_rotbonds_atoms_const",
              "pMem_num_rotating_atoms_per_rotbond_const"):
        setattr(g, f, 256)
    dp = g.dockpars
    dp.num_of_atoms, dp.true_ligand_atoms, dp.num_of_genes = 200, 200, 20
    dp.num_of_atypes, dp.num_of_map_atypes, dp.rotbondlist_length = 8, 8, 400
    dp.gridsize_x = dp.gridsize_y = dp.gridsize_z = 40
    dp.num_of_intraE_contributors = 40000          # 40000 pairs * 32 B > 1 MiB
    buf = C.c_void_p(256)
    st = L.adgpu_score_genotypes_noalloc(C.cast(C.pointer(g), C.c_void_p), 10, buf, buf, buf)
    assert st == 4, (st, L.adgpu_last_error())
    assert "1048576" in L.adgpu_last_error().decode()
    st = L.adgpu_score_genotypes_noalloc(None, 10, buf, buf, buf)
    assert st == 1, st
    # more map types than the reference's limit (the cell-record slot of an
    # atom is 8 bits wide)
    dp.num_of_intraE_contributors = 100
    dp.num_of_map_atypes = 40
    st = L.adgpu_score_genotypes_noalloc(C.cast(C.pointer(g), C.c_void_p), 10, buf, buf, buf)
    assert st == 4, (st, L.adgpu_last_error())


@pytest.mark.gpu
def test_noalloc_rejects_a_rotation_list_naming_no_atom(cases):
    """A rotation-list entry whose atom index is past the ligand's atoms is an
    error (the device repack checks every entry; no access depends on it)."""
    from adgpu_b200 import device
    case = cases["cfg2"]
    tables = dict(case.tables)
    rl = np.frombuffer(bytes(tables["rotlist"]), np.int32).copy()
    N = case.dockpars.num_of_atoms
    k = int(np.nonzero((rl[:case.dockpars.rotbondlist_length] & abi.RLIST_DUMMY_MASK) == 0)[0][0])
    rl[k] = (rl[k] & ~abi.RLIST_ATOMID_MASK) | N
    tables["rotlist"] = rl.view(np.uint8)
    job = device.DeviceJob(tables, case.dockpars, case.grid, case.runs, case.prng)
    g = torch.from_numpy(helpers.in_box_genotypes(case, 8, seed=1)).cuda()
    e = torch.zeros(8, dtype=torch.float32, device="cuda")
    st = lib.load().adgpu_score_genotypes_noalloc(C.cast(C.pointer(job.g), C.c_void_p), 8, C.c_void_p(g.data_ptr()),
                                                  C.c_void_p(e.data_ptr()), None)
    assert st == 1, st
    assert b"out of range" in lib.load().adgpu_last_error()
