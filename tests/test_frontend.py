"""The engine's front end (grid reader, PDBQT ligand preparation, initial
population) against the reference's own host front end on the same files:
every table entry the kernels read must be identical."""
import numpy as np
import pytest

import helpers
from adgpu_b200 import abi, frontend, synth
from oracle import refpy

pytestmark = pytest.mark.skipif(not refpy.available(), reason="oracle/_ref not built (needs the reference checkout)")


def used_views(tables, dp, nrot):
    """The parts of the reference tables the kernels read (the rest is padding)."""
    N, NT, Q = dp.num_of_atoms, dp.num_of_atypes, dp.num_of_intraE_contributors
    ii = np.frombuffer(bytes(tables["interintra"]), np.uint8)
    q = ii[:1024].view(np.float32)[:N]
    t = ii[1024:2048].view(np.uint32)[:N]
    tm = ii[2048:3072].view(np.uint32)[:N]
    ig = ii[3072:3328][:N]
    pairs = np.frombuffer(bytes(tables["intracontrib"]), np.uint32)[:2 * Q]
    kin = abi.KcIntra.from_buffer_copy(bytes(tables["intra"]))
    n2 = NT * NT
    intra = dict(reqm=np.array(kin.atom_types_reqm_const[:NT]), exp=np.array(kin.VWpars_exp_const[:n2]),
                 reqmab=np.array(kin.reqm_AB_const[:n2]), ac=np.array(kin.VWpars_AC_const[:n2]),
                 bd=np.array(kin.VWpars_BD_const[:n2]), S=np.array(kin.dspars_S_const[:NT]),
                 V=np.array(kin.dspars_V_const[:NT]))
    rl = np.frombuffer(bytes(tables["rotlist"]), np.int32)[:dp.rotbondlist_length]
    cf = abi.KcConform.from_buffer_copy(bytes(tables["conform"]))
    conf = dict(xyz=np.array(cf.ref_coords_const[:3 * N]), mv=np.array(cf.rotbonds_moving_vectors_const[:3 * nrot]),
                uv=np.array(cf.rotbonds_unit_vectors_const[:3 * nrot]))
    gr = abi.KcGrads.from_buffer_copy(bytes(tables["grads"]))
    nr = np.array(gr.num_rotating_atoms_per_rotbond[:nrot])
    rba = np.array(gr.rotbonds_atoms).reshape(abi.MAX_ROTBONDS, abi.MAX_ATOMS)
    grads = dict(rb=np.array(gr.rotbonds[:2 * nrot]), nr=nr,
                 atoms=[rba[k, :nr[k]].tolist() for k in range(nrot)])
    return dict(q=q, t=t, tm=tm, ig=ig, pairs=pairs, rotlist=rl, **{f"intra_{k}": v for k, v in intra.items()},
                **{f"conf_{k}": v for k, v in conf.items()}, grads_rb=grads["rb"], grads_nr=grads["nr"],
                grads_atoms=grads["atoms"])


CASES = [
    ("cfg1", dict(npts=40, types=synth.MAP_TYPES_5, n_heavy=16, n_tors=4, config_id=1)),
    ("cfg2", dict(npts=60, types=synth.MAP_TYPES_5, n_heavy=40, n_tors=10, config_id=2)),
    ("big", dict(npts=40, types=synth.MAP_TYPES_5, n_heavy=64, n_tors=24, config_id=3)),
    ("rigid", dict(npts=40, types=synth.MAP_TYPES_5, n_heavy=12, n_tors=0, config_id=3)),
    ("flex", dict(npts=40, types=synth.MAP_TYPES_7, n_heavy=14, n_tors=3, config_id=4, flexres=2)),
]


@pytest.mark.parametrize("name,kw", CASES)
def test_front_end_matches_reference_front_end(tmp_path, name, kw):
    kw = dict(kw)
    case = helpers.make_case(str(tmp_path), kw.pop("npts"), kw.pop("types"), kw.pop("n_heavy"), kw.pop("n_tors"), 3,
                             **kw)
    g = frontend.Grid.read(str(tmp_path / "receptor.maps.fld"))
    assert np.array_equal(g.reference_layout(), case.grid)
    lig = (tmp_path / "ligand0.pdbqt").read_text()
    flex = (tmp_path / "flexres.pdbqt").read_text() if (tmp_path / "flexres.pdbqt").exists() else None
    seed = tuple(int(s) for s in helpers.SEEDS.split(","))
    L = frontend.Ligand(g, lig, flex, run=frontend.default_dockpars(g.spacing), seed=seed, num_runs=3)
    for f, _ in abi.Dockpars._fields_:
        assert getattr(L.dockpars, f) == getattr(case.dockpars, f), f
    nrot = case.info.num_of_rotbonds
    a = used_views(L.tables, L.dockpars, nrot)
    b = used_views(case.tables, case.dockpars, nrot)
    for k in a:
        if isinstance(a[k], list):
            assert a[k] == b[k], k
        else:
            assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(L.prng, case.prng)
    assert np.array_equal(L.initpop, case.initpop)
