"""Seeded synthetic docking inputs in AutoDock-4 file formats.

The workloads this engine is measured on have no public dataset here, so
receptors and ligands are generated from a seed and written in the formats
the reference's front end reads:

* grid maps: an AVS ``.maps.fld`` header plus one text ``.map`` per atom type
  and the ``e`` (electrostatics) and ``d`` (desolvation) maps, laid out as
  AutoGrid writes them (read by ``get_gridinfo``/``get_gridvalues``,
  host/src/processgrid.cpp:28-253); map values come from a field of
  pseudo-receptor atoms (12-6 type maps, a Coulomb-like e map with a
  distance-dependent dielectric, a Gaussian desolvation d map), clamped to
  [-2, 1e5] kcal/mol;
* ligands: a random tree of heavy atoms (1.5 A bonds, near-tetrahedral
  angles, every non-bonded heavy pair >= 2.3 A apart so distance-based bond
  perception (host/src/processligand.cpp:459) finds exactly the tree), polar
  hydrogens (HD) on N/O, Gaussian charges shifted to sum to zero, and a chosen
  number of rotatable bonds written as ROOT/BRANCH/ENDBRANCH records
  (parsed by parse_liganddata, host/src/processligand.cpp:1124);
* flexible residues: short chains written between BEGIN_RES/END_RES.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

# Per-type (R_ii [A], eps_ii [kcal/mol]) used only to shape the synthetic maps.
_MAP_TYPE_PARAMS = {
    "C": (4.00, 0.150), "A": (4.00, 0.150), "N": (3.50, 0.160), "NA": (3.50, 0.160),
    "OA": (3.20, 0.200), "SA": (4.00, 0.200), "S": (4.00, 0.200), "HD": (2.00, 0.020),
    "H": (2.00, 0.020), "F": (3.09, 0.080), "P": (4.20, 0.200), "OS": (3.20, 0.200),
}
_REC_R, _REC_EPS = 3.8, 0.15
_ELEC = 332.06363 * 0.1465


@dataclass
class GridSpec:
    npts: tuple            # even number of intervals per axis (grid has npts+1 points)
    spacing: float
    center: tuple
    types: list            # affinity map atom types, in .fld order
    seed: int = 12345
    n_rec_atoms: int = 300
    rec_box: float = 30.0

    @property
    def dims(self):
        return tuple(n + 1 for n in self.npts)

    @property
    def origin(self):
        return tuple(c - n * 0.5 * self.spacing for c, n in zip(self.center, self.npts))


def make_maps(spec: GridSpec) -> dict:
    """Returns {type: float32 array [z, y, x]} for every type plus 'e' and 'd'."""
    rng = np.random.default_rng(spec.seed)
    rec = (rng.random((spec.n_rec_atoms, 3)) - 0.5) * spec.rec_box + np.asarray(spec.center)
    rec_q = rng.normal(0.0, 0.3, spec.n_rec_atoms)
    nx, ny, nz = spec.dims
    ox, oy, oz = spec.origin
    xs = ox + spec.spacing * np.arange(nx)
    ys = oy + spec.spacing * np.arange(ny)
    zs = oz + spec.spacing * np.arange(nz)
    out = {t: np.empty((nz, ny, nx), np.float32) for t in list(spec.types) + ["e", "d"]}
    gy, gx = np.meshgrid(ys, xs, indexing="ij")
    plane = np.stack([gx.ravel(), gy.ravel()], axis=1)
    for iz, z in enumerate(zs):
        d2 = ((plane[:, None, 0] - rec[None, :, 0]) ** 2 + (plane[:, None, 1] - rec[None, :, 1]) ** 2
              + (z - rec[None, :, 2]) ** 2)
        r = np.sqrt(np.maximum(d2, 1e-4))
        for t in spec.types:
            rii, eii = _MAP_TYPE_PARAMS.get(t, (3.5, 0.15))
            rij = 0.5 * (rii + _REC_R)
            eij = math.sqrt(eii * _REC_EPS)
            x6 = (rij / r) ** 6
            v = (eij * (x6 * x6 - 2.0 * x6)).sum(axis=1)
            out[t][iz] = np.clip(v, -2.0, 1e5).reshape(ny, nx)
        e = (_ELEC * rec_q[None, :] / (4.0 * r * r)).sum(axis=1)
        out["e"][iz] = np.clip(e, -2.0, 1e5).reshape(ny, nx)
        dsol = (0.01097 * 12.0 * np.exp(-d2 / (2.0 * 3.6 * 3.6))).sum(axis=1)
        out["d"][iz] = np.clip(dsol, -2.0, 1e5).reshape(ny, nx)
    return out


def make_maps_fast(spec: GridSpec, device: str = "cuda") -> dict:
    """make_maps computed with torch on `device` (float64): the same field,
    seconds instead of minutes for 100^3 grids.  Values agree with make_maps
    to rounding, not bit for bit; benchmarks use it for large receptors."""
    import torch
    rng = np.random.default_rng(spec.seed)
    rec = (rng.random((spec.n_rec_atoms, 3)) - 0.5) * spec.rec_box + np.asarray(spec.center)
    rec_q = rng.normal(0.0, 0.3, spec.n_rec_atoms)
    nx, ny, nz = spec.dims
    ox, oy, oz = spec.origin
    dev = torch.device(device)
    rec_t = torch.tensor(rec, dtype=torch.float64, device=dev)
    q_t = torch.tensor(rec_q, dtype=torch.float64, device=dev)
    xs = ox + spec.spacing * torch.arange(nx, dtype=torch.float64, device=dev)
    ys = oy + spec.spacing * torch.arange(ny, dtype=torch.float64, device=dev)
    zs = oz + spec.spacing * torch.arange(nz, dtype=torch.float64, device=dev)
    out = {t: np.empty((nz, ny, nx), np.float32) for t in list(spec.types) + ["e", "d"]}
    gy, gx = torch.meshgrid(ys, xs, indexing="ij")
    px, py = gx.reshape(-1, 1), gy.reshape(-1, 1)
    for iz in range(nz):
        d2 = (px - rec_t[None, :, 0]) ** 2 + (py - rec_t[None, :, 1]) ** 2 + (zs[iz] - rec_t[None, :, 2]) ** 2
        r = torch.sqrt(torch.clamp(d2, min=1e-4))
        for t in spec.types:
            rii, eii = _MAP_TYPE_PARAMS.get(t, (3.5, 0.15))
            rij = 0.5 * (rii + _REC_R)
            eij = math.sqrt(eii * _REC_EPS)
            x6 = (rij / r) ** 6
            v = (eij * (x6 * x6 - 2.0 * x6)).sum(dim=1)
            out[t][iz] = torch.clamp(v, -2.0, 1e5).reshape(ny, nx).float().cpu().numpy()
        e = (_ELEC * q_t[None, :] / (4.0 * r * r)).sum(dim=1)
        out["e"][iz] = torch.clamp(e, -2.0, 1e5).reshape(ny, nx).float().cpu().numpy()
        dsol = (0.01097 * 12.0 * torch.exp(-d2 / (2.0 * 3.6 * 3.6))).sum(dim=1)
        out["d"][iz] = torch.clamp(dsol, -2.0, 1e5).reshape(ny, nx).float().cpu().numpy()
    return out


def write_maps(spec: GridSpec, maps: dict, directory: str, name: str = "receptor") -> str:
    """Writes name.maps.fld and name.<type>.map files; returns the .fld path."""
    os.makedirs(directory, exist_ok=True)
    nx, ny, nz = spec.dims
    labels = [(t, f"{t}-affinity", f"{name}.{t}.map") for t in spec.types]
    labels += [("e", "Electrostatics", f"{name}.e.map"), ("d", "Desolvation", f"{name}.d.map")]
    header = [
        f"GRID_PARAMETER_FILE {name}.gpf",
        f"GRID_DATA_FILE {name}.maps.fld",
        f"MACROMOLECULE {name}.pdbqt",
        f"SPACING {spec.spacing:.3f}",
        f"NELEMENTS {spec.npts[0]} {spec.npts[1]} {spec.npts[2]}",
        f"CENTER {spec.center[0]:.3f} {spec.center[1]:.3f} {spec.center[2]:.3f}",
    ]
    for key, _, fn in labels:
        vals = maps[key].ravel()  # z-major, then y, then x: x fastest as AutoGrid writes
        with open(os.path.join(directory, fn), "w") as f:
            f.write("\n".join(header) + "\n")
            f.write("\n".join(f"{v:.3f}" for v in vals.tolist()) + "\n")
    fld = os.path.join(directory, f"{name}.maps.fld")
    with open(fld, "w") as f:
        f.write("# AVS field file\n#\n# AutoDock Atomic Affinity and Electrostatic Grids\n#\n")
        f.write(f"#SPACING {spec.spacing:.3f}\n")
        f.write(f"#NELEMENTS {spec.npts[0]} {spec.npts[1]} {spec.npts[2]}\n")
        f.write(f"#CENTER {spec.center[0]:.3f} {spec.center[1]:.3f} {spec.center[2]:.3f}\n")
        f.write(f"#MACROMOLECULE {name}.pdbqt\n#GRID_PARAMETER_FILE {name}.gpf\n#\n")
        f.write(f"ndim=3\ndim1={nx}\ndim2={ny}\ndim3={nz}\nnspace=3\nveclen={len(labels)}\n")
        f.write("data=float\nfield=uniform\n")
        for k in range(3):
            f.write(f"coord {k+1} file={name}.maps.xyz filetype=ascii offset={2*k}\n")
        for i, (_, lab, _) in enumerate(labels):
            f.write(f"label={lab}\t# component label for variable {i+1}\n")
        f.write("#\n# location of affinity grid files and how to read them\n#\n")
        for i, (_, _, fn) in enumerate(labels):
            f.write(f"variable {i+1} file={fn} filetype=ascii skip=6\n")
    return fld


def quantize_maps(maps: dict) -> dict:
    """The values as the .map text stores them (3 decimals), i.e. what a reader gets back."""
    return {k: np.round(v.astype(np.float64), 3).astype(np.float32) for k, v in maps.items()}


# --------------------------------------------------------------------------
# ligands
# --------------------------------------------------------------------------

@dataclass
class Molecule:
    xyz: np.ndarray                 # [n, 3] Angstrom
    types: list                     # AD4 atom types
    charges: np.ndarray             # [n]
    bonds: list                     # (i, j) pairs
    rot_bonds: list = field(default_factory=list)   # (parent_atom, child_atom) rotatable
    names: list = field(default_factory=list)


def _unit(v):
    return v / np.linalg.norm(v)


def _place(rng, xyz, parent, grandparent, bond, existing, min_d):
    """Candidate position for a new atom bonded to `parent`, at a near-tetrahedral
    angle from `grandparent`, at least `min_d` from every atom in `existing`."""
    for _ in range(200):
        d = _unit(rng.normal(size=3))
        if grandparent is not None:
            back = _unit(xyz[grandparent] - xyz[parent])
            cosang = float(np.dot(d, back))
            if cosang > math.cos(math.radians(105.0)):   # angle < 105 deg: too tight
                continue
        p = xyz[parent] + bond * d
        if len(existing) == 0:
            return p
        dist = np.linalg.norm(xyz[existing] - p, axis=1)
        if dist.min() >= min_d:
            return p
    return None


def make_ligand(seed: int, n_heavy: int, n_torsions: int,
                type_probs=(("C", 0.60), ("A", 0.15), ("N", 0.10), ("OA", 0.15)),
                charge_sigma: float = 0.2, hydrogens: bool = True) -> Molecule:
    """Random tree ligand: n_heavy heavy atoms, HD on N/O, n_torsions rotatable bonds."""
    rng = np.random.default_rng(seed)
    for _attempt in range(500):
        xyz = np.zeros((n_heavy, 3))
        parent = [-1] * n_heavy
        deg = [0] * n_heavy
        ok = True
        for i in range(1, n_heavy):
            placed = False
            for _ in range(60):
                cand = [k for k in range(i) if deg[k] < 3]
                p = int(rng.choice(cand))
                gp = parent[p] if parent[p] >= 0 else None
                if gp is None and deg[p] > 0:
                    gp = next(k for k in range(i) if parent[k] == p)
                others = [k for k in range(i) if k != p]
                pos = _place(rng, xyz, p, gp, 1.5, others, 2.3)
                if pos is None:
                    continue
                # also keep >= 2.3 A from atoms bonded to p (1-3 pairs): enforced by the angle rule
                xyz[i] = pos
                parent[i] = p
                deg[p] += 1
                deg[i] += 1
                placed = True
                break
            if not placed:
                ok = False
                break
        if not ok:
            continue
        bonds = [(parent[i], i) for i in range(1, n_heavy)]
        internal = [(a, b) for (a, b) in bonds if deg[a] > 1 and deg[b] > 1]
        if len(internal) < n_torsions and _attempt < 50:
            continue
        n_torsions = min(n_torsions, len(internal))   # small trees cannot hold every requested torsion
        break
    else:
        raise RuntimeError("could not build ligand")
    names_t = [t for t, _ in type_probs]
    probs = np.array([p for _, p in type_probs], float)
    probs /= probs.sum()
    types = list(rng.choice(names_t, size=n_heavy, p=probs))
    heavy_xyz = xyz
    all_xyz = [p for p in heavy_xyz]
    all_types = list(types)
    all_bonds = list(bonds)
    if hydrogens:
        for i in range(n_heavy):
            if types[i] in ("N", "NA", "OA") and deg[i] < 3:
                nb = [b for (a, b) in bonds if a == i] + [a for (a, b) in bonds if b == i]
                arr = np.array(all_xyz)
                others = [k for k in range(len(all_xyz)) if k != i and k not in nb]
                pos = None
                for _ in range(100):
                    d = _unit(rng.normal(size=3))
                    if any(np.dot(d, _unit(arr[k] - arr[i])) > math.cos(math.radians(100.0)) for k in nb):
                        continue
                    cand = arr[i] + (1.01 if types[i].startswith("N") else 0.97) * d
                    if not others or np.linalg.norm(arr[others] - cand, axis=1).min() >= 2.0:
                        pos = cand
                        break
                if pos is not None:
                    all_bonds.append((i, len(all_xyz)))
                    all_xyz.append(pos)
                    all_types.append("HD")
    n = len(all_xyz)
    q = rng.normal(0.0, charge_sigma, n)
    q -= q.mean()
    rot = [internal[k] for k in rng.choice(len(internal), size=n_torsions, replace=False)] if n_torsions else []
    mol = Molecule(xyz=np.array(all_xyz), types=all_types, charges=q, bonds=all_bonds,
                   rot_bonds=[tuple(int(v) for v in r) for r in rot])
    mol.names = [f"{t[0]}{k+1}" for k, t in enumerate(all_types)]
    return mol


def _fragments(mol: Molecule):
    """Rigid fragments: components of the bond graph without the rotatable bonds."""
    n = len(mol.types)
    rot = set(tuple(sorted(r)) for r in mol.rot_bonds)
    adj = [[] for _ in range(n)]
    for a, b in mol.bonds:
        if tuple(sorted((a, b))) in rot:
            continue
        adj[a].append(b)
        adj[b].append(a)
    comp = [-1] * n
    nc = 0
    for s in range(n):
        if comp[s] >= 0:
            continue
        stack = [s]
        comp[s] = nc
        while stack:
            u = stack.pop()
            for v in adj[u]:
                if comp[v] < 0:
                    comp[v] = nc
                    stack.append(v)
        nc += 1
    return comp, nc


def _atom_line(serial, name, resname, chain, resseq, xyz, q, atype, record="ATOM"):
    nm = name if len(name) >= 4 else " " + name
    return (f"{record:<6s}{serial:5d} {nm:<4s} {resname:>3s} {chain:1s}{resseq:4d}    "
            f"{xyz[0]:8.3f}{xyz[1]:8.3f}{xyz[2]:8.3f}{1.0:6.2f}{0.0:6.2f}    {q:6.3f} {atype:<2s}")


def pdbqt_lines(mol: Molecule, root_atom: int = 0, resname="LIG", chain="A", resseq=1,
                flexres=False, first_serial=1):
    """PDBQT records of a molecule with its torsion tree rooted at `root_atom`'s fragment."""
    comp, nc = _fragments(mol)
    members = [[] for _ in range(nc)]
    for i, c in enumerate(comp):
        members[c].append(i)
    rot_adj = {}
    for a, b in mol.rot_bonds:
        rot_adj.setdefault(comp[a], []).append((a, b))
        rot_adj.setdefault(comp[b], []).append((b, a))
    order = []          # atom order in the file
    serial = {}
    lines = []

    def emit_atoms(c):
        for i in members[c]:
            serial[i] = first_serial + len(order)
            order.append(i)
            lines.append(_atom_line(serial[i], mol.names[i], resname, chain, resseq,
                                    mol.xyz[i], mol.charges[i], mol.types[i]))

    def emit_branch(parent_comp, via):
        a, b = via
        child = comp[b]
        lines.append(f"BRANCH {serial[a]:3d} {first_serial + len(order):3d}")
        # the child fragment's atoms start with b so that the BRANCH record names it
        mem = members[child]
        mem.remove(b)
        mem.insert(0, b)
        emit_atoms(child)
        for (x, y) in rot_adj.get(child, []):
            if comp[y] != parent_comp:
                emit_branch(child, (x, y))
        lines.append(f"ENDBRANCH {serial[a]:3d} {serial[b]:3d}")

    root = comp[root_atom]
    if flexres:
        members[root].remove(root_atom)
        members[root].insert(0, root_atom)
    lines.append("ROOT")
    emit_atoms(root)
    lines.append("ENDROOT")
    for (x, y) in rot_adj.get(root, []):
        emit_branch(root, (x, y))
    if not flexres:
        lines.append(f"TORSDOF {len(mol.rot_bonds)}")
    return lines, order


def write_ligand(mol: Molecule, path: str) -> list:
    """Writes a ligand .pdbqt; returns the file order of the atoms."""
    lines, order = pdbqt_lines(mol)
    with open(path, "w") as f:
        f.write("REMARK  synthetic ligand\n")
        f.write(f"REMARK  {len(mol.rot_bonds)} active torsions\n")
        f.write("\n".join(lines) + "\n")
    return order


def make_flexres(seed: int, n_atoms: int, n_torsions: int, anchor: np.ndarray) -> Molecule:
    """Short side chain: a bent chain of n_atoms starting at `anchor`."""
    rng = np.random.default_rng(seed)
    for _attempt in range(500):
        xyz = [np.asarray(anchor, float)]
        ok = True
        for i in range(1, n_atoms):
            gp = i - 2 if i >= 2 else None
            arr = np.array(xyz)
            pos = _place(rng, arr, i - 1, gp, 1.5, list(range(0, max(0, i - 1))), 2.3)
            if pos is None:
                ok = False
                break
            xyz.append(pos)
        if ok:
            break
    else:
        raise RuntimeError("could not build flexres")
    types = ["C"] * n_atoms
    types[-1] = "OA" if rng.random() < 0.5 else "N"
    bonds = [(i, i + 1) for i in range(n_atoms - 1)]
    # torsions on chain bonds after the first (the first two atoms are the residue's anchor)
    cand = [(i, i + 1) for i in range(1, n_atoms - 2)]
    sel = sorted(rng.choice(len(cand), size=min(n_torsions, len(cand)), replace=False).tolist())
    rot = [cand[k] for k in sel]
    q = rng.normal(0.0, 0.15, n_atoms)
    q -= q.mean()
    mol = Molecule(xyz=np.array(xyz), types=types, charges=q, bonds=bonds, rot_bonds=rot)
    mol.names = [f"C{k+1}" if t == "C" else f"{t[0]}{k+1}" for k, t in enumerate(types)]
    return mol


def write_flexres(residues: list, path: str) -> None:
    """Writes flexible residues (list of Molecule) in the AutoDock flexres format."""
    with open(path, "w") as f:
        f.write(flexres_text(residues))


def flexres_text(residues: list) -> str:
    """Flexible residues (list of Molecule) as AutoDock flexres PDBQT text."""
    out = []
    serial = 1
    for k, mol in enumerate(residues):
        resname, chain, resseq = "LYS", "A", 10 + k
        out.append(f"BEGIN_RES {resname} {chain}{resseq:4d}")
        out.append(f"REMARK  {len(mol.rot_bonds)} active torsions:")
        lines, order = pdbqt_lines(mol, root_atom=0, resname=resname, chain=chain, resseq=resseq,
                                   flexres=True, first_serial=serial)
        out.extend(lines)
        out.append(f"END_RES {resname} {chain}{resseq:4d}")
        serial += len(order)
    return "\n".join(out) + "\n"


# --------------------------------------------------------------------------
# named workloads (sizes follow the benchmark configurations)
# --------------------------------------------------------------------------

MAP_TYPES_5 = ["C", "A", "N", "OA", "HD"]
MAP_TYPES_7 = ["C", "A", "N", "NA", "OA", "SA", "HD"]


def grid_spec(npts: int, types, seed: int, spacing: float = 0.375) -> GridSpec:
    return GridSpec(npts=(npts, npts, npts), spacing=spacing, center=(0.0, 0.0, 0.0),
                    types=list(types), seed=seed)


def ligand_for(config_id: int, index: int, n_heavy: int, n_torsions: int, types=None) -> Molecule:
    kw = {}
    if types is not None:
        kw["type_probs"] = types
    return make_ligand(12345 + config_id + 1000 * (index + 1), n_heavy, n_torsions, **kw)
