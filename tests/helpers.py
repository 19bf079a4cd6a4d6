"""Shared test helpers: seeded synthetic inputs prepared by the reference's own
front end (oracle/_ref), and tolerance checks used by the parity tests."""
from __future__ import annotations

import os

import numpy as np

from adgpu_b200 import abi, synth
from oracle import oraclepy, refpy

SEEDS = "305419896,2271560481,3735928559"


class Case:
    """A prepared docking job: reference tables + oracle view of them."""

    def __init__(self, job: refpy.RefJob):
        self.job = job
        self.info = job.info
        self.tables = {k: job.blob(k) for k in ("interintra", "intracontrib", "intra", "rotlist", "conform", "grads")}
        self.dockpars = abi.Dockpars.from_bytes(job.blob("dockpars"))
        self.grid = job.blob("grid")
        self.initpop = job.blob("initpop").reshape(-1, abi.GENOTYPE_STRIDE)
        self.prng = job.blob("prng")
        self.host = oraclepy.tables_from_refjob(job)

    @property
    def runs(self):
        return self.info.num_of_runs

    @property
    def ngenes(self):
        return self.info.num_of_genes


def make_case(directory: str, npts: int, map_types, n_heavy: int, n_tors: int, nrun: int,
              config_id: int = 1, lig_index: int = 0, lsmet: str = "ad", flexres: int = 0,
              extra_args=(), pop: int = 150) -> Case:
    os.makedirs(directory, exist_ok=True)
    fld = os.path.join(directory, "receptor.maps.fld")
    if not os.path.exists(fld):
        spec = synth.grid_spec(npts, map_types, seed=12345 + config_id)
        synth.write_maps(spec, synth.make_maps(spec), directory)
    lig = os.path.join(directory, f"ligand{lig_index}.pdbqt")
    if not os.path.exists(lig):
        mol = synth.ligand_for(config_id, lig_index, n_heavy, n_tors)
        synth.write_ligand(mol, lig)
    args = ["--ffile", fld, "--lfile", lig, "--nrun", str(nrun), "--seed", SEEDS, "--lsmet", lsmet,
            "--heuristics", "0", "--autostop", "0", "--nev", "2500000", "--psize", str(pop)]
    if flexres:
        fr = os.path.join(directory, "flexres.pdbqt")
        if not os.path.exists(fr):
            rng = np.random.default_rng(77)
            res = [synth.make_flexres(100 + k, int(rng.integers(8, 11)), int(rng.integers(2, 5)),
                                      anchor=np.array([-3.0 + 6.0 * k, 4.0, 0.0])) for k in range(flexres)]
            synth.write_flexres(res, fr)
        args += ["--flexres", fr]
    args += list(extra_args)
    return Case(refpy.RefJob(args))


def in_box_genotypes(case: Case, n: int, seed: int = 0, spread: float = 2.5) -> np.ndarray:
    """Seeded genotypes: translations near the box centre, orientations uniform
    on SO(3) (Shoemake, as gen_initpop_and_reflig does), torsions uniform."""
    rng = np.random.default_rng(seed)
    g = np.zeros((n, abi.GENOTYPE_STRIDE), np.float32)
    gs = np.array(list(case.info.gridsize), np.float64)
    g[:, :3] = (gs / 2.0)[None, :] + rng.normal(0.0, spread, (n, 3))
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    qw = np.sqrt(1 - u1) * np.sin(2 * np.pi * u2)
    qx = np.sqrt(1 - u1) * np.cos(2 * np.pi * u2)
    qy = np.sqrt(u1) * np.sin(2 * np.pi * u3)
    qz = np.sqrt(u1) * np.cos(2 * np.pi * u3)
    rot = 2.0 * np.arccos(np.clip(qw, -1, 1))
    s = np.sqrt(np.maximum(1.0 - qw * qw, 1e-12))
    x, y, z = qx / s, qy / s, qz / s
    g[:, 3] = np.degrees(np.arctan2(y, x))
    g[:, 4] = np.degrees(np.arccos(np.clip(z, -1, 1)))
    g[:, 5] = np.degrees(rot)
    g[:, 6:case.ngenes] = rng.uniform(-180.0, 180.0, (n, case.ngenes - 6))
    return g


def uniform_box_genotypes(case: Case, n: int, seed: int = 0) -> np.ndarray:
    """The plain configuration's scorer sample: translations uniform over the
    grid box (grid units), orientations uniform on SO(3) (Shoemake, as
    gen_initpop_and_reflig draws them), torsions uniform in [-180, 180)."""
    g = in_box_genotypes(case, n, seed=seed)
    rng = np.random.default_rng(seed + 1)
    gs = np.array(list(case.info.gridsize), np.float64)
    g[:, :3] = rng.uniform(0.0, 1.0, (n, 3)) * (gs - 1.0)[None, :]
    g[:, 6:case.ngenes] = rng.uniform(-180.0, 180.0, (n, case.ngenes - 6))
    return g


def energy_contract(ref: np.ndarray, terms: np.ndarray) -> np.ndarray:
    """The energy rule for identical genotypes: |dE| <= 1e-4 |E| + 1e-6 * sum of
    |terms| (the seven energy terms and the out-of-grid penalties, 2^24 per
    atom outside), the floor covering cancellation between large terms."""
    mag = np.abs(terms[:, :7]).sum(axis=1) + 16777216.0 * terms[:, 7]
    return 1e-4 * np.abs(ref) + 1e-6 * mag


def gradient_contract(case: Case, ref: np.ndarray) -> np.ndarray:
    """The gradient rule for identical genotypes: |dg| <= 1e-4 |g| + n_terms /
    1024 in gene units, n_terms the quantised terms that feed a gene (every
    atom's intermolecular term and both ends of every intramolecular pair),
    genes >= 3 scaled by spacing^2 / DEG_TO_RAD^2."""
    ng = case.ngenes
    n_terms = case.info.num_of_atoms + 2 * case.info.num_of_intraE_contributors
    sp = case.info.spacing
    scale = np.ones(ng, np.float64)
    scale[3:] = sp * sp / (0.0174533 ** 2)
    return 1e-4 * np.abs(ref[..., :ng]) + scale * n_terms / 1024.0


def oracle_terms(case: Case, genotypes: np.ndarray) -> np.ndarray:
    """The oracle's eight energy terms per genotype (the seven energy terms
    and the number of atoms outside the grid), for energy_contract."""
    return np.array([case.host.score_terms(x)[2] for x in genotypes])


def energy_tolerance(ref: np.ndarray) -> np.ndarray:
    """|dE| <= 1e-4 |E| + 1e-6 * |E| floor -> effectively 1e-4 relative with a 1e-3 absolute floor."""
    return 1e-4 * np.abs(ref) + 1e-3


def gradient_tolerance(case: Case, ref: np.ndarray) -> np.ndarray:
    """Per-gene tolerance: 1e-4 relative plus a fixed-point floor.  The
    reference rounds every per-atom, per-pair and per-(torsion, atom) term to
    1/1024 before summing, so independent float rounding of one term can move
    the sum by one quantum per term (TERMSCALE, cuda/GpuData.h:31-35).  Genes
    >= 3 are then scaled by spacing^2 / DEG_TO_RAD^2."""
    ng = case.ngenes
    n_terms = case.info.num_of_atoms + 2 * case.info.num_of_intraE_contributors
    sp = case.info.spacing
    scale = np.ones(ng, np.float64)
    scale[3:] = sp * sp / (0.0174533 ** 2)
    quantum = scale / 1024.0
    floor = quantum * 8.0
    floor[3:6] = quantum[3:6] * 64.0        # orientation genes: difference of angles / 1e-3 rad
    floor[6:] = quantum[6:] * 16.0
    del n_terms
    return 1e-4 * np.abs(ref[..., :ng]) + floor


def gradient_bound(case: Case, ref: np.ndarray) -> np.ndarray:
    """Worst-case per-gene bound: 1e-4 relative plus one quantum (1/1024, in
    gene units) per quantised term that feeds the gene (every atom's inter
    term and both ends of every intramolecular pair); the orientation genes get
    the same bound amplified by the 1/INFINITESIMAL_RADIAN (1e3) step through
    which torques become angle differences (cuda/calcMergeEneGra.cu:701-815)."""
    ng = case.ngenes
    n_terms = case.info.num_of_atoms + 2 * case.info.num_of_intraE_contributors
    sp = case.info.spacing
    scale = np.ones(ng, np.float64)
    scale[3:] = sp * sp / (0.0174533 ** 2)
    bound = scale * n_terms / 1024.0
    bound[3:6] *= 1e3 / 1024.0 * 8.0
    return 1e-4 * np.abs(ref[..., :ng]) + bound


def generic_pairs(case: Case) -> int:
    """Intramolecular pairs whose vdW exponents are not the AD4 force field's
    12-6 / 12-10 (modified pair potentials)."""
    kin = abi.KcIntra.from_buffer_copy(bytes(case.tables["intra"]))
    ii = abi.KcInterintra.from_buffer_copy(bytes(case.tables["interintra"]))
    dp = case.dockpars
    nat, q = dp.num_of_atypes, dp.num_of_intraE_contributors
    ex = np.array(kin.VWpars_exp_const[:nat * nat], np.int64).reshape(nat, nat)
    pairs = np.frombuffer(bytes(case.tables["intracontrib"]), np.uint32)[:2 * q].reshape(-1, 2)
    t = np.array(ii.atom_types_const[:dp.num_of_atoms], np.int64)
    e = ex[t[pairs[:, 0]], t[pairs[:, 1]]]
    m, n = (e >> 8) & 0xFF, e & 0xFF
    return int(((m != 12) | ((n != 6) & (n != 10))).sum())
