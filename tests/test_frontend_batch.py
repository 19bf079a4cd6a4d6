"""Front-end additions without a reference counterpart, on CPU: the binary
grid cache round-trips the parsed maps exactly, and batched ligand
preparation on several threads gives the same tables and populations as one
ligand at a time."""
import numpy as np
import pytest

from adgpu_b200 import frontend, lib, synth

TYPES = ["C", "A", "N", "OA", "HD"]


@pytest.fixture(scope="module")
def grid_dir(tmp_path_factory):
    d = tmp_path_factory.mktemp("maps")
    spec = synth.grid_spec(24, TYPES, seed=12345 + 9)
    synth.write_maps(spec, synth.make_maps(spec), str(d))
    return d


def test_grid_cache_round_trip(grid_dir, tmp_path):
    g = frontend.Grid.read(str(grid_dir / "receptor.maps.fld"))
    path = str(tmp_path / "receptor.grid")
    g.save(path)
    h = frontend.Grid.load(path)
    assert h.dims == g.dims and h.spacing == g.spacing and h.origin == g.origin
    assert h.num_map_atypes == g.num_map_atypes
    assert np.array_equal(h.reference_layout(), g.reference_layout())


def test_grid_cache_rejects_other_files(tmp_path):
    bad = tmp_path / "bad.grid"
    bad.write_bytes(b"not a grid cache at all")
    with pytest.raises(lib.AdgpuError):
        frontend.Grid.load(str(bad))


def test_prepare_batch_matches_single(grid_dir):
    g = frontend.Grid.read(str(grid_dir / "receptor.maps.fld"))
    texts = []
    for i in range(12):
        lines, _ = synth.pdbqt_lines(synth.ligand_for(3, i, 10 + 3 * i, i % 7))
        texts.append("\n".join(lines) + "\n")
    run = frontend.default_dockpars(g.spacing, 40)
    seeds = [(11 + i, 22 + i, 33 + i) for i in range(len(texts))]
    single = [frontend.Ligand(g, t, None, run=run, seed=s, num_runs=3) for t, s in zip(texts, seeds)]
    batch = frontend.Ligand.prepare_batch(g, texts, run=run, seeds=seeds, num_runs=3, nthreads=4)
    assert len(batch) == len(single)
    for a, b in zip(single, batch):
        assert bytes(a.dockpars) == bytes(b.dockpars)
        for k in a.tables:
            assert np.array_equal(a.tables[k], b.tables[k]), k
        assert np.array_equal(a.initpop, b.initpop) and np.array_equal(a.prng, b.prng)


def test_prepare_batch_reports_the_failing_ligand(grid_dir):
    g = frontend.Grid.read(str(grid_dir / "receptor.maps.fld"))
    lines, _ = synth.pdbqt_lines(synth.ligand_for(3, 0, 12, 2))
    good = "\n".join(lines) + "\n"
    with pytest.raises(lib.AdgpuError, match="ligand 1"):
        frontend.Ligand.prepare_batch(g, [good, "REMARK nothing here\n", good], num_runs=1)
