"""Pins the C restatement (oracle/adgpu_oracle.c) to the reference's own
kernel sources, compiled for the CPU under the SIMT emulator (oracle/_ref):
same tables (prepared by the reference's own front end), same genotypes, same
PRNG states."""
import numpy as np
import pytest

import helpers
from adgpu_b200 import abi
from oracle import refpy

pytestmark = pytest.mark.skipif(not refpy.available(), reason="oracle/_ref not built (needs the reference checkout)")
T = 64


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    d = tmp_path_factory.mktemp("pins")
    return helpers.make_case(str(d / "cfg1"), 40, ["C", "A", "N", "OA", "HD"], 16, 4, 2, config_id=1)


@pytest.fixture(scope="module")
def flex_case(tmp_path_factory):
    d = tmp_path_factory.mktemp("pins_flex")
    return helpers.make_case(str(d / "flex"), 40, ["C", "A", "N", "NA", "OA", "SA", "HD"], 14, 3, 2,
                             config_id=4, flexres=2)


def _bind(case, dp=None):
    R, P = case.runs, case.dockpars.pop_size
    pr = case.prng.copy()
    po = case.prng.copy()
    enr, eno = np.zeros(R * P, np.int32), np.zeros(R * P, np.int32)
    err, ero = np.zeros(R, np.int32), np.zeros(R, np.int32)
    dp = dp or case.dockpars
    case.job.bind(pr, enr, err, dockpars=bytes(dp))
    case.host.g.dockpars = dp
    case.host.bind_state(po, eno, ero)
    return pr, po, enr, eno, err, ero


@pytest.mark.parametrize("which", ["case", "flex_case"])
def test_scorer_matches_reference_source(which, request):
    c = request.getfixturevalue(which)
    _bind(c)
    g = helpers.in_box_genotypes(c, 48, seed=11)
    e_ref, gr_ref = c.job.score(g, True)
    e_or, gr_or = c.host.score(g, True)
    assert np.all(np.abs(e_ref - e_or) <= 1e-5 * np.abs(e_ref) + 1e-4)
    ng = c.ngenes
    # fixed-point gradients: identical except for rare one-quantum flips
    q = np.ones(ng) / 1024.0
    q[3:] *= c.info.spacing ** 2 / 0.0174533 ** 2
    d = np.abs(gr_ref[:, :ng] - gr_or[:, :ng])
    assert (d > 2.5 * q + 1e-4 * np.abs(gr_ref[:, :ng])).mean() < 0.01
    assert np.array_equal(c.job.score(g, False), c.job.score(g, False))


def test_ga_generation_bit_exact(case):
    pr, po, enr, eno, err, ero = _bind(case)
    R, P = case.runs, case.dockpars.pop_size
    pop = case.initpop[:R * P].copy()
    e = case.host.score(pop, False)
    cn_r, en_r = np.zeros_like(pop), np.zeros_like(e)
    cn_o, en_o = np.zeros_like(pop), np.zeros_like(e)
    refpy.call("gen_and_eval_newpops", R * P, T, pop, e, cn_r, en_r)
    case.host.call("gen_and_eval_newpops", R * P, T, pop, e, cn_o, en_o, 2)
    assert np.array_equal(pr, po)
    assert np.array_equal(cn_r, cn_o)
    assert np.array_equal(enr, eno)
    assert np.all(np.abs(en_r - en_o) <= 1e-5 * np.abs(en_r) + 1e-4)


@pytest.mark.parametrize("method", ["perform_ls", "gradient_minad", "gradient_minadam"])
def test_local_search_short(case, method):
    dp = case.dockpars.copy()
    dp.max_num_of_iters = 4
    R, P = case.runs, dp.pop_size
    L = dp.num_of_lsentities
    nb = min(R * L, 60)
    pr, po, enr, eno, err, ero = _bind(case, dp)
    pop = case.initpop[:R * P].copy()
    e = case.host.score(pop, False)
    a_c, a_e, b_c, b_e = pop.copy(), e.copy(), pop.copy(), e.copy()
    refpy.call(method, nb, T, a_c, a_e)
    case.host.call(method, nb, T, b_c, b_e, 2)
    ng = case.ngenes
    close = np.abs(a_c[:, :ng] - b_c[:, :ng]).max(axis=1) <= 1e-2
    assert close.mean() >= 0.97
    if method != "perform_ls":
        assert np.array_equal(pr, po)
        assert np.array_equal(enr, eno)


def test_sum_evals_and_initpop(case):
    pr, po, enr, eno, err, ero = _bind(case)
    R, P = case.runs, case.dockpars.pop_size
    pop = case.initpop[:R * P].copy()
    e1, e2 = np.zeros(R * P, np.float32), np.zeros(R * P, np.float32)
    refpy.call("calc_initpop", R * P, T, pop.copy(), e1)
    case.host.call("calc_initpop", R * P, pop.copy(), e2, 2)
    refpy.call("sum_evals", R, T)
    case.host.call("sum_evals", R)
    assert np.all(np.abs(e1 - e2) <= 1e-5 * np.abs(e1) + 1e-4)
    assert np.array_equal(err, ero) and err.tolist() == [P] * R


@pytest.mark.parametrize("iters,min_close", [(1, 1.0), (4, 0.95)])
def test_fire_matches_reference_opencl_source(case, iters, min_close):
    """The oracle's FIRE against the reference's OpenCL FIRE kernel
    (device/kernel_fire.cl under the emulator), the reference's first
    gradient taken from its merged scorer: the same PRNG draws and evaluation
    counts, and genotypes that agree entity by entity (one step: all within
    1e-2; four steps: rounding can flip a step-size decision)."""
    dp = case.dockpars.copy()
    dp.max_num_of_iters = iters
    R, P = case.runs, dp.pop_size
    nb = min(R * dp.num_of_lsentities, 60)
    pr, po, enr, eno, err, ero = _bind(case, dp)
    pop = case.initpop[:R * P].copy()
    e = case.host.score(pop, False)
    a_c, a_e, b_c, b_e = pop.copy(), e.copy(), pop.copy(), e.copy()
    refpy.call("gradient_minfire", nb, T, a_c, a_e)
    case.host.call("gradient_minfire", nb, T, b_c, b_e, 2)
    assert np.array_equal(pr, po)
    assert np.array_equal(enr, eno)
    ng = case.ngenes
    close = np.abs(a_c[:nb, :ng] - b_c[:nb, :ng]).max(axis=1) <= 1e-2
    assert close.mean() >= min_close
    assert np.all(np.abs(a_e[:nb] - b_e[:nb]) <= 1e-3 * np.abs(a_e[:nb]) + 1e-2) or iters > 1


def test_reference_fire_first_gradient_reads_uninitialised_coordinates(case):
    """Why the engine takes FIRE's first gradient from the merged scorer: the
    reference's own first call (gpu_calc_gradient, kernel_fire.cl:318)
    rotates the kernel's __local calc_coords without loading the reference
    coordinates into them (calcgradient.cl:160-258), so its first step does
    not follow the entity's gradient: after one step its genotypes are far
    from those of a step along the merged scorer's gradient, which the oracle
    reproduces to rounding."""
    dp = case.dockpars.copy()
    dp.max_num_of_iters = 1
    R, P = case.runs, dp.pop_size
    nb = min(R * dp.num_of_lsentities, 60)
    pop = case.initpop[:R * P].copy()
    e = case.host.score(pop, False)
    out = {}
    for name in ("gradient_minfire_asis", "gradient_minfire"):
        _bind(case, dp)
        c, ee = pop.copy(), e.copy()
        refpy.call(name, nb, T, c, ee)
        out[name] = c[:nb, :case.ngenes]
    _bind(case, dp)
    c, ee = pop.copy(), e.copy()
    case.host.call("gradient_minfire", nb, T, c, ee, 2)
    ng = case.ngenes
    d_oracle = np.abs(c[:nb, :ng] - out["gradient_minfire"]).max(axis=1)
    d_asis = np.abs(out["gradient_minfire_asis"] - out["gradient_minfire"]).max(axis=1)
    assert np.median(d_oracle) < 1e-2
    assert np.median(d_asis) > 10 * max(np.median(d_oracle), 1e-3)


def test_reference_opencl_scorer_translation_gradient(case, flex_case):
    """The reference's two merged scorers agree on a rigid receptor, and with
    flexible residues its OpenCL one (used by its FIRE) sums the translation
    gradient over the residues' atoms as well (calcMergedEneGra.cl:635-649;
    the CUDA one, calcMergeEneGra.cu:616-640, over the ligand's atoms only):
    the oracle and the engine follow the CUDA scorer for every search."""
    for c, flex in ((case, False), (flex_case, True)):
        _bind(c)
        g = helpers.in_box_genotypes(c, 32, seed=11)
        e_cu, g_cu = c.job.score(g, True)
        e_cl, g_cl = refpy.ocl_score(g)
        assert np.all(np.abs(e_cu - e_cl) <= 1e-5 * np.abs(e_cu) + 1e-4)
        d = np.abs(g_cu[:, :3] - g_cl[:, :3])
        if flex:
            assert np.median(d) > 0.1
        else:
            assert d.max() <= 4.0 / 1024.0 + 1e-4 * np.abs(g_cu[:, :3]).max()
