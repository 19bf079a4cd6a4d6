"""CPU checks of the reference's result processing (oracle/_ref) that pin the
semantics the device restatement relies on: arrange_result's bubble sort
leaves NaN energies in place and sorts the segments between them stably, and
generate_output's clusters are founded by their lowest-energy member, with
every other member within the RMSD tolerance of it."""
import numpy as np
import pytest

import helpers
from adgpu_b200 import synth
from oracle import refpy

pytestmark = pytest.mark.skipif(not refpy.available(), reason="oracle/_ref not built (needs the reference checkout)")


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    d = tmp_path_factory.mktemp("result")
    return helpers.make_case(str(d), 40, synth.MAP_TYPES_5, 16, 4, 6, config_id=1, pop=20)


def segment_sort(e):
    """Stable ascending order inside the NaN-free segments; NaNs stay put."""
    out = np.array(e, copy=True)
    idx = np.arange(len(e))
    perm = idx.copy()
    nan = np.isnan(e)
    s = 0
    while s < len(e):
        if nan[s]:
            s += 1
            continue
        t = s
        while t < len(e) and not nan[t]:
            t += 1
        order = np.argsort(e[s:t], kind="stable")
        out[s:t] = e[s:t][order]
        perm[s:t] = idx[s:t][order]
        s = t
    return out, perm


def test_arrange_result_nan_segments_and_ties(case):
    R, P = case.runs, case.info.pop_size
    rng = np.random.default_rng(3)
    pops = helpers.in_box_genotypes(case, R * P, seed=5)
    pops[:, 63] = np.arange(R * P)                     # tag rows to follow the permutation
    en = rng.integers(-5, 5, R * P).astype(np.float32)  # many ties
    en[3] = np.nan
    en[P + 0] = np.nan
    en[2 * P + P - 1] = np.nan
    en[3 * P + 7] = en[3 * P + 8] = np.nan
    sp, se, runs, xyz, per = case.job.process_result(pops, en, clustering=False)
    for r in range(R):
        want_e, perm = segment_sort(en[r * P:(r + 1) * P])
        assert np.array_equal(se[r * P:(r + 1) * P], want_e, equal_nan=True)
        assert np.array_equal(sp[r * P:(r + 1) * P, 63], pops[r * P + perm, 63])


def test_clusters_founded_by_lowest_energy_member(case):
    R, P = case.runs, case.info.pop_size
    base = helpers.in_box_genotypes(case, 2, seed=11, spread=1.0)
    pops = np.repeat(base[np.arange(R) % 2], P, axis=0).copy()
    pops[:, :3] += np.random.default_rng(1).normal(0, 0.1, (R * P, 3)).astype(np.float32)
    en = np.random.default_rng(2).normal(-5, 1, R * P).astype(np.float32)
    sp, se, runs, xyz, per = case.job.process_result(pops, en, rmsd_tol=2.0)
    energy = np.array([r.inter_e + r.interflex_e for r in runs], np.float64)
    by_cluster = {}
    for i, r in enumerate(runs):
        by_cluster.setdefault(r.cluster_id, []).append(i)
    assert sorted(by_cluster) == list(range(1, len(by_cluster) + 1))
    for cid, members in by_cluster.items():
        members.sort(key=lambda i: runs[i].cluster_subrank)
        assert [runs[i].cluster_subrank for i in members] == list(range(1, len(members) + 1))
        centre = members[0]
        assert runs[centre].rmsd_from_cluster_center == 0.0
        assert all(energy[centre] <= energy[i] for i in members)
        assert all(runs[i].rmsd_from_cluster_center <= 2.0 for i in members)
