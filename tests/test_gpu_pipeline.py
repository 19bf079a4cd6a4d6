"""The pipelined plain docking loop (adgpu_dock_resident without AutoStop):
runs advance independently, up to three generations ahead of the stop test,
and the generations run past a stop are discarded.  Its results must be
bit-identical to the reference's generation-synchronous host loop over the
same kernels (docking_with_gpu's loop, one kernel-API call per kernel per
generation): final populations, energies, per-run evaluation counts and the
generation count."""
import ctypes as C

import numpy as np
import pytest
import torch

import helpers
from adgpu_b200 import device, dock, lib

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    d = tmp_path_factory.mktemp("pipe")
    return helpers.make_case(str(d / "cfg1"), 40, ["C", "A", "N", "OA", "HD"], 16, 4, 12, config_id=1)


def _job(case, tpp, pipeline, monkeypatch):
    monkeypatch.setenv("ADGPU_THREADS_PER_POSE", str(tpp))
    monkeypatch.setenv("ADGPU_DOCK_PIPELINE", "1" if pipeline else "0")
    job = device.DeviceJob(case.tables, case.dockpars, case.grid, case.runs, case.prng)
    job.activate()
    return job


def _same(a: dock.DockResult, b: dock.DockResult):
    assert a.generations == b.generations
    np.testing.assert_array_equal(a.evals_per_run, b.evals_per_run)
    np.testing.assert_array_equal(a.energies.cpu().numpy(), b.energies.cpu().numpy())
    np.testing.assert_array_equal(a.conformations.cpu().numpy(), b.conformations.cpu().numpy())


@pytest.mark.parametrize("lsmet,tpp", [("ad", 32), ("ad", 64), ("sw", 32), ("adam", 32), ("fire", 32), ("ad", 128)])
def test_pipelined_matches_host_loop(case, lsmet, tpp, monkeypatch):
    # ADAM and FIRE searches run their full iteration count: more evaluations
    # per generation
    nev = 120_000 if lsmet in ("ad", "sw") else 400_000
    host = dock.dock_host_loop(_job(case, tpp, True, monkeypatch), case.initpop, lsmet, nev)
    pipe = dock.dock(_job(case, tpp, True, monkeypatch), case.initpop, lsmet, nev)
    assert host.generations > 3
    _same(host, pipe)
    # the generation-synchronous resident loop (CUDA graphs) gives the same
    sync = dock.dock(_job(case, tpp, False, monkeypatch), case.initpop, lsmet, nev)
    _same(host, sync)


@pytest.mark.parametrize("ngen", [1, 2, 3, 4, 5, 9])
def test_generation_budget(case, ngen, monkeypatch):
    """Stops on the generation count, also within the first look-ahead window."""
    host = dock.dock_host_loop(_job(case, 32, True, monkeypatch), case.initpop, "ad", 10**9, ngen)
    pipe = dock.dock(_job(case, 32, True, monkeypatch), case.initpop, "ad", 10**9, ngen)
    assert host.generations == ngen
    _same(host, pipe)


def test_no_generation_when_the_initial_population_suffices(case, monkeypatch):
    """Check 0 (initial evaluations only) already stops: the initial population
    is the result, in the first buffer."""
    P = case.dockpars.pop_size
    pipe = dock.dock(_job(case, 32, True, monkeypatch), case.initpop, "ad", P)
    assert pipe.generations == 0
    np.testing.assert_array_equal(pipe.evals_per_run, np.full(case.runs, P))


def test_repeated_calls_reuse_the_library_scratch(case, monkeypatch):
    """Two dockings in a row from the same PRNG states (the library keeps its
    buffers between calls) give the same results."""
    job = _job(case, 32, True, monkeypatch)
    prng0 = job.prng.clone()
    a = dock.dock(job, case.initpop, "ad", 60_000)
    a = dock.DockResult(a.conformations.clone(), a.energies.clone(), a.evals_per_run.copy(), a.generations)
    job.prng.copy_(prng0)
    b = dock.dock(job, case.initpop, "ad", 60_000)
    _same(a, b)
