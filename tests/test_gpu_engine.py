"""The batch / serving engine: same results as the plain per-ligand path,
identical results alone and in a mix, continuous admission, memory budget."""
import numpy as np
import pytest
import torch

from adgpu_b200 import device, dock, engine, frontend, synth

pytestmark = pytest.mark.gpu
SEED = (305419896, 2271560481, 3735928559)


@pytest.fixture(scope="module")
def grid():
    spec = synth.grid_spec(40, synth.MAP_TYPES_5, seed=12346)
    maps = synth.quantize_maps(synth.make_maps(spec))
    return frontend.Grid.from_maps(maps, synth.MAP_TYPES_5, spec.spacing, spec.origin)


def ligand(grid, idx, n_heavy, n_tors, runs=4, pop=150):
    mol = synth.ligand_for(3, idx, n_heavy, n_tors)
    text = "\n".join(synth.pdbqt_lines(mol)[0]) + "\n"
    return frontend.Ligand(grid, text, None, run=frontend.default_dockpars(grid.spacing, pop), seed=SEED,
                           num_runs=runs)


@pytest.mark.parametrize("lsmet", ["ad", "sw", "adam", "fire"])
def test_engine_matches_plain_path(grid, lsmet, monkeypatch):
    """With a generation budget both paths stop at the same generation, so the
    run must come out identical (same kernels, same PRNG states).  One run:
    the engine gives local-search entity l of run r the PRNG states of GA
    block r*P + l (so that runs in different phases never share states), which
    for run 0 are the reference's own (block l)."""
    lig = ligand(grid, 0, 16, 4, runs=1)
    gens = 6
    # plain: reference kernel API, resident loop, with the engine's group size
    monkeypatch.setenv("ADGPU_THREADS_PER_POSE", "32")
    job = device.DeviceJob(lig.tables, lig.dockpars, grid.reference_layout(), 1, lig.prng)
    job.activate()
    res = dock.dock(job, lig.initpop, lsmet, nev=10**9, ngen=gens)
    assert res.generations == gens
    P = lig.dockpars.pop_size
    e_plain = res.energies.cpu().numpy().reshape(1, P)
    # engine
    en = engine.Engine(threads_per_pose=32)
    rec = en.add_receptor(grid)
    rid = en.submit(lig, rec, lsmet, max_evals=10**12, max_gens=gens)
    en.run()
    r = en.result(rid)
    assert np.all(r.generations == gens)
    np.testing.assert_array_equal(r.evals, res.evals_per_run)
    np.testing.assert_array_equal(r.best_energies, e_plain.min(axis=1))


@pytest.mark.parametrize("tpp", [32, 64])
def test_batch_uneven_ligands_and_mix_invariance(grid, tpp):
    sizes = [(12, 0), (16, 4), (24, 8), (30, 12), (20, 6), (40, 16)]
    ligs = [ligand(grid, i, a, t, runs=3) for i, (a, t) in enumerate(sizes)]
    nev = 40_000
    # alone
    alone = []
    for lg in ligs[:3]:
        en = engine.Engine(threads_per_pose=tpp)
        rec = en.add_receptor(grid)
        rid = en.submit(lg, rec, "ad", max_evals=nev)
        en.run()
        alone.append(en.result(rid))
        en.close()
    # all together in one batch
    en = engine.Engine(threads_per_pose=tpp)
    rec = en.add_receptor(grid)
    ids = [en.submit(lg, rec, "ad", max_evals=nev) for lg in ligs]
    en.run()
    mix = [en.result(i) for i in ids]
    for a, b in zip(alone, mix[:3]):
        np.testing.assert_array_equal(a.best_energies, b.best_energies)
        np.testing.assert_array_equal(a.best_genotypes, b.best_genotypes)
        np.testing.assert_array_equal(a.evals, b.evals)
    for lg, r in zip(ligs, mix):
        assert np.all(r.evals >= nev)
        e0 = np.array([lg.initpop.shape[0]])  # noqa: F841
        assert np.all(np.isfinite(r.best_energies))
        assert r.best_energies.max() < 1e6


def test_automatic_threads_per_pose(grid):
    """Tuned sizes (threads_per_pose -1): the size picked per ligand-size
    bucket, the same for every request of a bucket whatever its local
    search; the default is one warp per pose."""
    assert engine.Engine().submit is not None
    d = engine.Engine()
    drec = d.add_receptor(grid)
    assert d.info(d.submit(ligand(grid, 3, 20, 6, runs=2), drec, "ad", max_evals=5_000))[0] == 32
    d.close()
    en = engine.Engine(threads_per_pose=-1)
    rec = en.add_receptor(grid)
    lg = ligand(grid, 3, 20, 6, runs=2)
    got = {}
    for m in ("sw", "ad", "adam", "fire"):
        rid = en.submit(lg, rec, m, max_evals=5_000)
        got[m] = en.info(rid)[0]
    en.run()
    assert all(v in (32, 64, 128) for v in got.values())
    assert len(set(got.values())) == 1
    en.close()


def test_continuous_admission_and_budget(grid):
    ligs = [ligand(grid, 10 + i, 14 + 2 * i, 2 + i, runs=2) for i in range(5)]
    nev = 30_000
    ref = []
    for lg in ligs:
        en = engine.Engine(threads_per_pose=32)
        rec = en.add_receptor(grid)
        rid = en.submit(lg, rec, "ad", max_evals=nev)
        en.run()
        ref.append(en.result(rid))
        en.close()
    # serving: small ticks; requests arrive while others are in flight
    en = engine.Engine(threads_per_pose=32, gens_per_tick=2)
    rec = en.add_receptor(grid)
    pending = list(range(len(ligs)))
    live, out = {}, {}
    first = pending.pop(0)
    live[en.submit(ligs[first], rec, "ad", max_evals=nev)] = first
    ticks = 0
    while live or pending:
        en.tick()
        ticks += 1
        if pending and ticks % 2 == 1:
            k = pending.pop(0)
            live[en.submit(ligs[k], rec, "ad", max_evals=nev)] = k
        for rid in [r for r in live if en.done(r)]:
            out[live.pop(rid)] = en.result(rid)
    assert ticks > 2
    for k, r in out.items():
        np.testing.assert_array_equal(r.best_energies, ref[k].best_energies)
        np.testing.assert_array_equal(r.evals, ref[k].evals)
    # a budget too small for a second request is refused, and admitted after a result is taken
    small = engine.Engine(threads_per_pose=32, memory_budget_bytes=64 << 20)
    rec = small.add_receptor(grid)
    a = small.submit(ligs[0], rec, "ad", max_evals=nev)
    n = 1
    while small.submit(ligs[1], rec, "ad", max_evals=nev, raise_on_budget=False) is not None:
        n += 1
        assert n < 1000
    small.run()
    small.result(a)
    assert small.submit(ligs[1], rec, "ad", max_evals=nev, raise_on_budget=False) is not None
    torch.cuda.synchronize()


def test_ga_only_and_mixed_population_sizes(grid, monkeypatch):
    """Edge cases of the task queues: a request without local search (rate 0:
    only GA phases) next to requests of population 50 and 150 in one tick,
    each identical to its plain-path docking."""
    monkeypatch.setenv("ADGPU_THREADS_PER_POSE", "32")
    gens = 5
    specs = [(0, 150, 0.0), (1, 50, 100.0), (2, 150, 100.0)]
    ligs = []
    for idx, pop, rate in specs:
        run = frontend.default_dockpars(grid.spacing, pop)
        run.lsearch_rate = rate
        run.num_of_lsentities = int(rate / 100.0 * pop + 0.5)   # as the reference derives it
        mol = synth.ligand_for(3, 40 + idx, 14 + 3 * idx, 3)
        text = "\n".join(synth.pdbqt_lines(mol)[0]) + "\n"
        ligs.append(frontend.Ligand(grid, text, None, run=run, seed=SEED, num_runs=1))
    plain = []
    for lg in ligs:
        job = device.DeviceJob(lg.tables, lg.dockpars, grid.reference_layout(), 1, lg.prng)
        job.activate()
        res = dock.dock(job, lg.initpop, "ad", nev=10**9, ngen=gens)
        plain.append((res.evals_per_run.copy(), float(res.energies.min().item())))
    en = engine.Engine(threads_per_pose=32)
    rec = en.add_receptor(grid)
    ids = [en.submit(lg, rec, "ad", max_evals=10**12, max_gens=gens) for lg in ligs]
    en.run()
    for rid, (ev, best), (idx, pop, rate) in zip(ids, plain, specs):
        r = en.result(rid)
        assert np.all(r.generations == gens)
        np.testing.assert_array_equal(r.evals, ev)
        assert r.best_energies[0] == best
        if rate == 0.0:
            assert int(r.evals[0]) == pop * (gens + 1) - gens    # GA only: P per generation minus the elite


@pytest.mark.parametrize("priority", [0, 1])
def test_time_sliced_ticks_give_the_same_results(grid, priority):
    """Ticks that end on a wall-clock deadline (tick_ms) instead of a
    generation count cut runs at arbitrary generations; results must not
    depend on where the cuts fall, nor on which runs the pose groups serve
    first (priority 1: the oldest request's runs)."""
    ligs = [ligand(grid, 30 + i, 16 + 4 * i, 3 + i, runs=2) for i in range(3)]
    nev = 30_000
    ref = []
    for lg in ligs:
        en = engine.Engine(threads_per_pose=32)
        rec = en.add_receptor(grid)
        rid = en.submit(lg, rec, "ad", max_evals=nev)
        en.run()
        ref.append(en.result(rid))
        en.close()
    en = engine.Engine(threads_per_pose=32, tick_ms=2.0, priority=priority)
    rec = en.add_receptor(grid)
    ids = [en.submit(lg, rec, "ad", max_evals=nev) for lg in ligs]
    ticks = 0
    while not all(en.done(r) for r in ids):
        en.tick()
        ticks += 1
        assert ticks < 100000
    assert ticks > 1
    for rid, r0 in zip(ids, ref):
        r = en.result(rid)
        np.testing.assert_array_equal(r.best_energies, r0.best_energies)
        np.testing.assert_array_equal(r.evals, r0.evals)
