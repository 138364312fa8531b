"""Seeded synthetic receptor/ligand systems written as AMBER prmtop + DCD.

The workloads this package is measured on have no public dataset: systems
are generated from a fixed recipe and seed so that every run (GPU kernels,
CPU restatement, benchmark) sees byte-identical inputs.

Recipe (per system):
  * receptor: ``n_rec`` atoms uniform in a sphere of volume n_rec / 0.12 A^3;
    ligand: ``n_lig`` atoms uniform in a sphere of the same density whose
    centre sits ``gap`` (3 A) beyond the receptor surface along +x;
  * elements H/C/N/O/S drawn with p = .50/.30/.09/.10/.01; mbondi2 radii
    1.2/1.7/1.55/1.5/1.8 A; GB screen 0.85/0.72/0.79/0.85/0.96;
  * charges U[-0.8, 0.8] e, shifted so each molecule is neutral, stored as
    q * 18.2223;
  * ``n_types`` Lennard-Jones types with sigma ~ U[1.0, 3.8] A and
    epsilon ~ U[0.01, 0.2] kcal/mol, Lorentz-Berthelot mixing,
    A = 4 eps sigma^12, B = 4 eps sigma^6; atoms draw a type uniformly;
  * receptor residues of ``res_size`` atoms, the ligand one residue;
  * no bonded terms; one placeholder exclusion (0) per atom;
  * frames: base coordinates + N(0, sigma^2) A per coordinate, float32 A,
    no unit cell.
Seeds: topology ``1000 + k``, frames ``2000 + k`` for workload k.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass

import numpy as np

ELEMENTS = ("H", "C", "N", "O", "S")
ELEMENT_P = (0.50, 0.30, 0.09, 0.10, 0.01)
RADII = {"H": 1.2, "C": 1.7, "N": 1.55, "O": 1.5, "S": 1.8}
SCREEN = {"H": 0.85, "C": 0.72, "N": 0.79, "O": 0.85, "S": 0.96}
MASS = {"H": 1.008, "C": 12.01, "N": 14.01, "O": 16.0, "S": 32.06}
ATOMIC_NUMBER = {"H": 1, "C": 6, "N": 7, "O": 8, "S": 16}
DENSITY = 0.12  # atoms / A^3
AMBER_CHARGE = 18.2223


@dataclass
class System:
    """A generated receptor + ligand complex (atom order: receptor, ligand)."""

    n_rec: int
    n_lig: int
    xyz: np.ndarray  # (N, 3) float64 base coordinates, A
    elements: list
    charges_e: np.ndarray
    type_idx: np.ndarray  # 0-based
    sigma: np.ndarray  # per type
    epsilon: np.ndarray  # per type
    residue_pointers: np.ndarray  # 0-based first atom of each residue
    residue_labels: list

    @property
    def n_atoms(self) -> int:
        return self.n_rec + self.n_lig

    @property
    def receptor_residues(self) -> list:
        return list(range(len(self.residue_labels) - 1))

    @property
    def ligand_residues(self) -> list:
        return [len(self.residue_labels) - 1]

    @property
    def radii(self) -> np.ndarray:
        return np.array([RADII[e] for e in self.elements])

    @property
    def screen(self) -> np.ndarray:
        return np.array([SCREEN[e] for e in self.elements])


def _ball(rng, n, radius):
    # uniform in a ball: direction from a normal draw, radius ~ U^(1/3)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    r = radius * rng.random(n) ** (1.0 / 3.0)
    return v * r[:, None]


def ball_radius(n: int) -> float:
    return (3.0 * n / (4.0 * math.pi * DENSITY)) ** (1.0 / 3.0)


def make_system(n_rec: int, n_lig: int, seed: int, res_size: int = 15, n_types: int = 64,
                gap: float = 3.0) -> System:
    rng = np.random.default_rng(seed)
    r_rec, r_lig = ball_radius(n_rec), ball_radius(n_lig)
    rec = _ball(rng, n_rec, r_rec)
    lig = _ball(rng, n_lig, r_lig) + np.array([r_rec + gap + r_lig, 0.0, 0.0])
    xyz = np.concatenate([rec, lig]).astype(np.float64)
    n = n_rec + n_lig
    elements = list(rng.choice(ELEMENTS, size=n, p=ELEMENT_P))
    q = rng.uniform(-0.8, 0.8, size=n)
    q[:n_rec] -= q[:n_rec].mean()
    q[n_rec:] -= q[n_rec:].mean()
    sigma = rng.uniform(1.0, 3.8, size=n_types)
    epsilon = rng.uniform(0.01, 0.2, size=n_types)
    type_idx = rng.integers(0, n_types, size=n)
    ptrs = list(range(0, n_rec, res_size)) + [n_rec]
    labels = ["RES"] * (len(ptrs) - 1) + ["LIG"]
    return System(n_rec, n_lig, xyz, elements, q, type_idx.astype(np.int64), sigma, epsilon,
                  np.array(ptrs, dtype=np.int64), labels)


def make_frames(system: System, n_frames: int, seed: int, sigma: float = 0.5) -> np.ndarray:
    """(F, N, 3) float32 Angstrom: base + N(0, sigma^2) per coordinate."""
    rng = np.random.default_rng(seed)
    out = np.empty((n_frames, system.n_atoms, 3), dtype=np.float32)
    for f in range(n_frames):
        out[f] = (system.xyz + rng.normal(0.0, sigma, size=system.xyz.shape)).astype(np.float32)
    return out


def lj_tables(system: System):
    """AMBER triangular LJ tables: (acoef, bcoef, nonbonded_parm_index)."""
    k = len(system.sigma)
    m = k * (k + 1) // 2
    a = np.zeros(m)
    b = np.zeros(m)
    nbi = np.zeros(k * k, dtype=np.int64)
    for i in range(k):
        for j in range(i, k):
            idx = i + j * (j + 1) // 2  # 0-based triangular index
            s = 0.5 * (system.sigma[i] + system.sigma[j])
            e = math.sqrt(system.epsilon[i] * system.epsilon[j])
            a[idx] = 4.0 * e * s ** 12
            b[idx] = 4.0 * e * s ** 6
            nbi[k * i + j] = idx + 1
            nbi[k * j + i] = idx + 1
    return a, b, nbi


def _fmt(values, per_line, fmt):
    lines = []
    for s in range(0, len(values), per_line):
        lines.append("".join(fmt % v for v in values[s:s + per_line]))
    return lines if lines else [""]


def write_prmtop(system: System, path: str, bonds=None) -> None:
    """AMBER prmtop of the system.  bonds: optional (i, j) atom pairs written
    as BONDS_WITHOUT_HYDROGEN with one bond type of zero force constant (they
    add no energy and no exclusion; they make molecules connected for
    periodic reimaging)."""
    n = system.n_atoms
    bonds = [] if bonds is None else [(int(i), int(j)) for i, j in bonds]
    nres = len(system.residue_labels)
    ntypes = len(system.sigma)
    a, b, nbi = lj_tables(system)
    pointers = [0] * 31
    pointers[0], pointers[1], pointers[11] = n, ntypes, nres
    pointers[10] = n  # NNB: one placeholder exclusion per atom
    if bonds:
        pointers[3] = pointers[12] = len(bonds)  # MBONA, NBONA
        pointers[15] = 1  # NUMBND
    out = ["%VERSION  VERSION_STAMP = V0001.000  synthetic", "%FLAG TITLE", "%FORMAT(20a4)", "synthetic"]

    def sec(flag, fmt_name, lines):
        out.append("%FLAG " + flag)
        out.append("%FORMAT(" + fmt_name + ")")
        out.extend(lines)

    names = [(e + str(i % 100)).ljust(4)[:4] for i, e in enumerate(system.elements)]
    sec("POINTERS", "10I8", _fmt(pointers, 10, "%8d"))
    sec("ATOM_NAME", "20a4", ["".join(names[s:s + 20]) for s in range(0, n, 20)])
    sec("CHARGE", "5E16.8", _fmt(list(system.charges_e * AMBER_CHARGE), 5, "%16.8E"))
    sec("ATOMIC_NUMBER", "10I8", _fmt([ATOMIC_NUMBER[e] for e in system.elements], 10, "%8d"))
    sec("MASS", "5E16.8", _fmt([MASS[e] for e in system.elements], 5, "%16.8E"))
    sec("ATOM_TYPE_INDEX", "10I8", _fmt(list(system.type_idx + 1), 10, "%8d"))
    sec("NUMBER_EXCLUDED_ATOMS", "10I8", _fmt([1] * n, 10, "%8d"))
    sec("NONBONDED_PARM_INDEX", "10I8", _fmt(list(nbi), 10, "%8d"))
    labels = [lab.ljust(4)[:4] for lab in system.residue_labels]
    sec("RESIDUE_LABEL", "20a4", ["".join(labels[s:s + 20]) for s in range(0, nres, 20)])
    sec("RESIDUE_POINTER", "10I8", _fmt(list(system.residue_pointers[:nres] + 1), 10, "%8d"))
    sec("BOND_FORCE_CONSTANT", "5E16.8", _fmt([0.0], 5, "%16.8E") if bonds else [""])
    sec("BOND_EQUIL_VALUE", "5E16.8", _fmt([1.0], 5, "%16.8E") if bonds else [""])
    for flag in ("ANGLE_FORCE_CONSTANT", "ANGLE_EQUIL_VALUE",
                 "DIHEDRAL_FORCE_CONSTANT", "DIHEDRAL_PERIODICITY", "DIHEDRAL_PHASE"):
        sec(flag, "5E16.8", [""])
    sec("SCEE_SCALE_FACTOR", "5E16.8", [""])
    sec("SCNB_SCALE_FACTOR", "5E16.8", [""])
    sec("LENNARD_JONES_ACOEF", "5E16.8", _fmt(list(a), 5, "%16.8E"))
    sec("LENNARD_JONES_BCOEF", "5E16.8", _fmt(list(b), 5, "%16.8E"))
    sec("BONDS_INC_HYDROGEN", "10I8", [""])
    sec("BONDS_WITHOUT_HYDROGEN", "10I8",
        _fmt([v for i, j in bonds for v in (3 * i, 3 * j, 1)], 10, "%8d") if bonds else [""])
    for flag in ("ANGLES_INC_HYDROGEN", "ANGLES_WITHOUT_HYDROGEN", "DIHEDRALS_INC_HYDROGEN",
                 "DIHEDRALS_WITHOUT_HYDROGEN"):
        sec(flag, "10I8", [""])
    sec("EXCLUDED_ATOMS_LIST", "10I8", _fmt([0] * n, 10, "%8d"))
    sec("RADIUS_SET", "1a80", ["modified Bondi radii (mbondi2)"])
    sec("RADII", "5E16.8", _fmt(list(system.radii), 5, "%16.8E"))
    sec("SCREEN", "5E16.8", _fmt(list(system.screen), 5, "%16.8E"))
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def write_dcd(frames_A: np.ndarray, path: str, cell=None) -> None:
    """CHARMM-layout little-endian DCD (float32 Angstrom).  cell: optional
    (a, b, c, alpha, beta, gamma) in Angstrom and degrees, written before
    every frame in CHARMM order (a, gamma, b, beta, alpha, c)."""
    frames_A = np.ascontiguousarray(frames_A, dtype=np.float32)
    nf, na, _ = frames_A.shape
    with open(path, "wb") as f:
        icntrl = [nf, 0, 1, nf, 0, 0, 0, 0, 0]
        hdr = b"CORD" + struct.pack("<9i", *icntrl) + struct.pack("<f", 1.0) + struct.pack("<i", 1 if cell else 0)
        hdr += b"\x00" * 32 + struct.pack("<i", 24)
        f.write(struct.pack("<i", len(hdr)) + hdr + struct.pack("<i", len(hdr)))
        title = b"synthetic MM-GBSA workload".ljust(80)
        blk = struct.pack("<i", 1) + title
        f.write(struct.pack("<i", len(blk)) + blk + struct.pack("<i", len(blk)))
        f.write(struct.pack("<iii", 4, na, 4))
        nb = struct.pack("<i", 4 * na)
        for fr in range(nf):
            if cell:
                a, b, c, al, be, ga = (float(v) for v in cell)
                f.write(struct.pack("<i", 48) + struct.pack("<6d", a, ga, b, be, al, c) + struct.pack("<i", 48))
            for d in range(3):
                f.write(nb + frames_A[fr, :, d].tobytes() + nb)


# Workloads the package is measured on (atom counts, frames, method).
WORKLOADS = {
    1: dict(n_rec=2000, n_lig=30, n_frames=10, method="gb"),
    2: dict(n_rec=5000, n_lig=50, n_frames=1000, method="gb", decompose=True),
    3: dict(n_rec=3000, n_lig=40, n_frames=100, method="pb"),
    5: dict(n_rec=25000, n_lig=80, n_frames=500, method="gb+pb"),
}


def workload(k: int, n_frames: int | None = None):
    """(system, frames_f32) for workload k with its fixed seeds."""
    w = WORKLOADS[k]
    s = make_system(w["n_rec"], w["n_lig"], seed=1000 + k)
    fr = make_frames(s, n_frames if n_frames is not None else w["n_frames"], seed=2000 + k)
    return s, fr
