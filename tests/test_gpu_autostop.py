"""Device-side AutoStop against the reference's own AutoStop class.

The resident loop runs the convergence test on the device
(adgpu_dock_resident_autostop); the reference host loop copies the energies
to the host every --asfreq generations and asks its AutoStop object
(host/inc/autostop.hpp, compiled from the reference checkout into
oracle/_ref).  Both drive the same kernels from the same states, so the
trajectories are identical and the test must stop at the same generation
with the same final population."""
import numpy as np
import pytest
import torch

import helpers
from adgpu_b200 import device, dock
from oracle import refpy

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not refpy.available(), reason="reference sources not built")]


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    d = tmp_path_factory.mktemp("autostop")
    return helpers.make_case(str(d / "cfg1"), 40, ["C", "A", "N", "OA", "HD"], 16, 4, 10, config_id=1)


def _run_both(case, monkeypatch, asfreq, stopstd, min_evals, nev=10**9, ngen=400):
    monkeypatch.setenv("ADGPU_THREADS_PER_POSE", "32")
    R, P = case.runs, case.dockpars.pop_size
    out = []
    for arm in ("host", "device"):
        job = device.DeviceJob(case.tables, case.dockpars, case.grid, R, case.prng)
        job.activate()
        if arm == "host":
            ref = refpy.RefAutoStop(P, R, stopstd, asfreq)
            res = dock.dock_host_loop(job, case.initpop, "ad", nev, ngen, autostop=(asfreq, min_evals, ref.check))
        else:
            res = dock.dock(job, case.initpop, "ad", nev, ngen,
                            autostop=dock.AutoStopParams(asfreq, stopstd, min_evals))
        torch.cuda.synchronize()
        out.append(res)
    return out


@pytest.mark.parametrize("asfreq,stopstd", [(5, 0.15), (2, 0.5)])
def test_autostop_matches_reference(case, monkeypatch, asfreq, stopstd):
    host, dev = _run_both(case, monkeypatch, asfreq, stopstd, 0)
    assert host.autostopped, "the reference's AutoStop did not trigger within the generation budget"
    assert dev.autostopped == host.autostopped
    assert dev.generations == host.generations
    np.testing.assert_array_equal(dev.evals_per_run, host.evals_per_run)
    assert torch.equal(dev.energies, host.energies)


def test_autostop_respects_minimum_evaluations(case, monkeypatch):
    """With a minimum above the budget the test never ends the loop early:
    the docking stops at the generation budget like one without AutoStop."""
    host, dev = _run_both(case, monkeypatch, 5, 0.5, 10**15, ngen=60)
    assert dev.generations == host.generations == 60
    assert torch.equal(dev.energies, host.energies)
