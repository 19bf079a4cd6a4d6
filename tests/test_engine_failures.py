"""Failure handling around the batch/serving engine, made on the host (no
GPU fault is involved anywhere): bad and oversized ligands are refused at
preparation and at submission, a request can be cancelled between ticks,
and a run whose tasks never complete (injected on the host) makes the tick
end with ADGPU_ERR_TIMEOUT after the engine's idle limit instead of hanging,
after which the rest of the batch docks as it would alone.  The reference's
convention for these is print-and-exit (cuda/GpuData.h:40-72) with per-job
error flags in its driver (host/src/main.cpp:333-352)."""
import time

import numpy as np
import pytest

from adgpu_b200 import frontend, lib, synth

SEED = (305419896, 2271560481, 3735928559)


@pytest.fixture(scope="module")
def grid():
    spec = synth.grid_spec(40, synth.MAP_TYPES_5, seed=12346)
    maps = synth.quantize_maps(synth.make_maps(spec))
    return frontend.Grid.from_maps(maps, synth.MAP_TYPES_5, spec.spacing, spec.origin)


def ligand_text(idx, n_heavy, n_tors):
    return "\n".join(synth.pdbqt_lines(synth.ligand_for(3, idx, n_heavy, n_tors))[0]) + "\n"


def prepare(grid, text, runs=2):
    return frontend.Ligand(grid, text, None, run=frontend.default_dockpars(grid.spacing, 150), seed=SEED,
                           num_runs=runs)


@pytest.mark.parametrize("text", [
    "not a pdbqt file\n",
    "ROOT\nENDROOT\nTORSDOF 0\n",                                                  # no atoms
    "ROOT\nATOM      1  C1  LIG A   1       0.000   0.000   0.000  0.00  0.00    +0.000 Qx\nENDROOT\nTORSDOF 0\n",
])
def test_bad_pdbqt_is_refused(grid, text):
    with pytest.raises(lib.AdgpuError):
        prepare(grid, text)


def test_oversized_ligands_are_refused(grid):
    """Past the reference's limits: more than 256 atoms, more than 57
    torsions (common/defines.h:83-95)."""
    with pytest.raises(lib.AdgpuError, match="LIMIT|limit|atoms|torsion"):
        prepare(grid, ligand_text(1, 270, 8))
    with pytest.raises(lib.AdgpuError, match="LIMIT|limit|atoms|torsion"):
        prepare(grid, ligand_text(2, 90, 60))


@pytest.mark.gpu
def test_cancel_between_ticks(grid):
    from adgpu_b200 import engine
    ligs = [prepare(grid, ligand_text(20 + i, 16 + 4 * i, 3 + i)) for i in range(3)]
    nev = 40_000
    alone = []
    for lg in ligs[:2]:
        en = engine.Engine(threads_per_pose=32)
        rec = en.add_receptor(grid)
        rid = en.submit(lg, rec, "ad", max_evals=nev)
        en.run()
        alone.append(en.result(rid))
        en.close()
    en = engine.Engine(threads_per_pose=32, gens_per_tick=1)
    rec = en.add_receptor(grid)
    ids = [en.submit(lg, rec, "ad", max_evals=nev) for lg in ligs]
    used = en.stats().bytes_used
    en.tick()
    en.cancel(ids[2])                           # mid-docking
    assert en.stats().bytes_used < used and en.stats().cancelled == 1
    with pytest.raises(lib.AdgpuError):
        en.done(ids[2])
    en.run()
    for k in range(2):
        r = en.result(ids[k])
        np.testing.assert_array_equal(r.best_energies, alone[k].best_energies)
        np.testing.assert_array_equal(r.evals, alone[k].evals)
    en.close()


@pytest.mark.gpu
def test_stalled_run_times_out_and_the_batch_recovers(grid):
    """The injected stall leaves the request's runs active with nothing to
    hand out: the pose groups' bounded wait (idle_timeout_ms) ends the tick
    with ADGPU_ERR_TIMEOUT; after cancelling that request the others finish
    with the results they have alone."""
    from adgpu_b200 import engine
    ligs = [prepare(grid, ligand_text(30 + i, 18 + 4 * i, 4)) for i in range(3)]
    nev = 40_000
    alone = []
    for lg in ligs[1:]:
        en = engine.Engine(threads_per_pose=32)
        rec = en.add_receptor(grid)
        rid = en.submit(lg, rec, "ad", max_evals=nev)
        en.run()
        alone.append(en.result(rid))
        en.close()
    en = engine.Engine(threads_per_pose=32, gens_per_tick=1, idle_timeout_ms=200.0)
    rec = en.add_receptor(grid)
    ids = [en.submit(lg, rec, "ad", max_evals=nev) for lg in ligs]
    en.tick()
    en.inject_stall(ids[0])
    t0 = time.perf_counter()
    with pytest.raises(lib.AdgpuError, match="timed out|TIMEOUT"):
        en.run()
    assert time.perf_counter() - t0 < 30.0
    en.cancel(ids[0])
    en.run()
    for k in range(2):
        r = en.result(ids[k + 1])
        np.testing.assert_array_equal(r.best_energies, alone[k].best_energies)
        np.testing.assert_array_equal(r.evals, alone[k].evals)
    en.close()


@pytest.mark.gpu
def test_engine_configuration_is_checked():
    """Out-of-range engine settings are refused at creation."""
    from adgpu_b200 import engine
    for kw in ({"priority": 2}, {"priority": -1}, {"threads_per_pose": 48}, {"tick_ms": -1.0},
               {"idle_timeout_ms": -5.0}):
        with pytest.raises(lib.AdgpuError):
            engine.Engine(**kw)
