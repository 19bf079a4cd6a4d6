"""The drop-in, shown end to end: the reference's own host program
(host/src/*.cpp with performdocking.cpp.Cuda and main.cpp, built by
oracle/Makefile's `dropin` target as its Makefile.Cuda builds it) linked
against libadgpu_b200.so instead of its cuda/kernels.o, run through the
reference's command line on real .fld/.map/.pdbqt files.  It must write the
reference's .dlg and .xml, and its dockings must be statistically
indistinguishable from the same host program linked against the reference's
own CUDA kernels (oracle/_ref/autodock_gpu_ref): same evaluation budget,
run energies from the same distribution (two-sample Kolmogorov-Smirnov), and
the top-ranked binding modes within 2 A of each other's three best clusters."""
import os
import re
import subprocess

import numpy as np
import pytest

from adgpu_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(os.path.dirname(HERE), "oracle", "_ref")
B200_BIN = os.path.join(REF_DIR, "autodock_gpu_b200")
REF_BIN = os.path.join(REF_DIR, "autodock_gpu_ref")
SEED = "305419896,2271560481,3735928559"

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (os.path.exists(B200_BIN) and os.path.exists(REF_BIN)),
                                 reason="reference host program not built (make -C oracle dropin)")]


@pytest.fixture(scope="module")
def inputs(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("dropin"))
    spec = synth.grid_spec(40, ["C", "A", "N", "OA", "HD"], seed=12345 + 1)
    fld = synth.write_maps(spec, synth.make_maps(spec), d)
    lig = os.path.join(d, "ligand.pdbqt")
    synth.write_ligand(synth.ligand_for(1, 0, 16, 4), lig)
    return d, fld, lig


def run_cli(binary, d, fld, lig, name, lsmet, nrun, nev):
    args = [binary, "--ffile", fld, "--lfile", lig, "--nrun", str(nrun), "--lsmet", lsmet, "--heuristics", "0",
            "--autostop", "0", "--nev", str(nev), "--seed", SEED, "--resnam", os.path.join(d, name)]
    p = subprocess.run(args, capture_output=True, text=True, timeout=600, cwd=d)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return os.path.join(d, name + ".dlg"), os.path.join(d, name + ".xml"), p.stdout


def parse_dlg(path, natoms):
    """Run energies (Estimated Free Energy of Binding, in run order), the RMSD
    table (rank, sub-rank, run, energy) and each run's docked coordinates."""
    text = open(path).read()
    energies = [float(x) for x in re.findall(r"DOCKED: USER    Estimated Free Energy of Binding\s+=\s+([-+0-9.eE]+)", text)]
    table = []
    in_table = False
    for line in text.splitlines():
        if "RMSD TABLE" in line:
            in_table = True
            continue
        if in_table:
            m = re.match(r"\s*(\d+)\s+(\d+)\s+(\d+)\s+([-+0-9.]+)\s+([-+0-9.]+)\s+([-+0-9.]+)\s+RANKING", line)
            if m:
                table.append((int(m.group(1)), int(m.group(2)), int(m.group(3)), float(m.group(4))))
    coords = []
    for block in text.split("DOCKED: MODEL")[1:]:
        xyz = [(float(ln[38:46]), float(ln[46:54]), float(ln[54:62]))
               for ln in block.splitlines() if ln.startswith("DOCKED: ATOM") or ln.startswith("DOCKED: HETATM")]
        coords.append(np.array(xyz[:natoms]))
    return np.array(energies), table, coords


def cluster_tops(table, coords, k=3):
    tops = []
    for rank in range(1, k + 1):
        row = next((r for r in table if r[0] == rank and r[1] == 1), None)
        if row is not None:
            tops.append(coords[row[2] - 1])
    return tops


def rmsd(a, b):
    return float(np.sqrt(((a - b) ** 2).sum(axis=1).mean()))


@pytest.mark.parametrize("lsmet", ["ad", "sw"])
def test_reference_cli_on_the_engine(inputs, lsmet):
    from scipy import stats
    d, fld, lig = inputs
    nrun, nev = 24, 500_000
    dlg_b, xml_b, out_b = run_cli(B200_BIN, d, fld, lig, f"b200_{lsmet}", lsmet, nrun, nev)
    dlg_r, xml_r, out_r = run_cli(REF_BIN, d, fld, lig, f"ref_{lsmet}", lsmet, nrun, nev)
    for path in (dlg_b, xml_b):
        assert os.path.exists(path) and os.path.getsize(path) > 0, path
    xml = open(xml_b).read()
    assert xml.count("<run id=") == nrun
    natoms = sum(1 for ln in open(lig) if ln.startswith(("ATOM", "HETATM")))
    e_b, table_b, xyz_b = parse_dlg(dlg_b, natoms)
    e_r, table_r, xyz_r = parse_dlg(dlg_r, natoms)
    assert len(e_b) == nrun and len(e_r) == nrun
    assert len(table_b) == nrun and len(xyz_b) == nrun
    ks = stats.ks_2samp(e_b, e_r)
    tb, tr = cluster_tops(table_b, xyz_b), cluster_tops(table_r, xyz_r)
    b_in_r = min(rmsd(tb[0], t) for t in tr)
    r_in_b = min(rmsd(tr[0], t) for t in tb)
    print(lsmet, "median", np.median(e_b), np.median(e_r), "best", e_b.min(), e_r.min(), "ks", ks.pvalue,
          "top", b_in_r, r_in_b)
    assert ks.pvalue > 1e-3, ks
    assert b_in_r < 2.0 and r_in_b < 2.0, (b_in_r, r_in_b)
