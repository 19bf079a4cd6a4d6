"""The oracle (and, on a GPU, the engine) against the golden vectors that
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
    for meth in ("perform_ls", "gradient_minad", "gradient_minadam"):
        st[0][:] = f["ga_prng_after"]
        st[1][:] = 0
        c, ee = f["ga_next"].copy(), f["ga_next_energy"].copy()
        ht.call(meth, R * ldp.num_of_lsentities, T, c, ee, 1)
        close = np.abs(c[:, :ng] - f[f"{meth}_conf"][:, :ng]).max(axis=1) <= 1e-2
        assert close.mean() >= 0.95, meth
        if meth != "perform_ls":
            assert np.array_equal(st[0], f[f"{meth}_prng"])
            assert np.array_equal(st[1], f[f"{meth}_evals"])
