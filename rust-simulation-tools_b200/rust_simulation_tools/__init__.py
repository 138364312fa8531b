"""MM-GBSA / MM-PBSA energies on B200 GPUs, with the Python API of the
MM-PBSA section of ``rust_simulation_tools`` (crates/bindings/src/lib.rs:1450-2280).

Function names, keyword arguments, defaults, units and raised exception
types follow the reference module: coordinates passed to the single-frame
functions are (N, 3) float64 arrays in **nanometres** (converted to Angstrom
as lib.rs:83-88 does), trajectory files are read in their own units.
Every computation runs in ``librstg.so`` on the GPU; there is no CPU path.

Beyond the reference API, :class:`BindingSystem` exposes the batched,
device-resident engine and :class:`Server` the continuous-batching loop.
"""
from __future__ import annotations

import ctypes as C
import enum
import math
from typing import List, Optional, Sequence

import numpy as np

from . import _native as N
from ._native import check

__all__ = [
    "AmberTopology", "read_prmtop", "DcdReader", "MdcrdReader", "GbModel", "GbParams", "PbParams", "SaParams",
    "MmEnergy", "GbEnergy", "SaEnergy", "PbEnergy", "FrameEnergy", "BindingResult", "ResidueContribution",
    "DecompositionResult", "EntropyEstimate", "compute_mm_energy", "compute_gb_energy", "compute_sa_energy",
    "compute_pb_energy", "compute_binding_energy", "compute_binding_energy_single_frame",
    "decompose_binding_energy", "interaction_entropy", "quasi_harmonic_entropy", "extract_subtopology",
    "BindingSystem", "Server", "device_count", "kernel_launches", "GbCache", "compute_gb_energy_cached",
]

USIZE_MAX = 2 ** 64 - 1


def device_count() -> int:
    return int(N.lib.rstg_device_count())


def kernel_launches() -> int:
    """Kernels this process has launched through the default context."""
    return int(N.lib.rstg_ctx_kernel_launches(N.ctx()))


def _i64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64).reshape(-1))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _coords_A(coords_nm) -> np.ndarray:
    a = np.asarray(coords_nm, dtype=np.float64)
    if a.ndim != 2 or a.shape[1] != 3:
        raise ValueError("coordinates must be an (N, 3) array")
    return np.ascontiguousarray(a * 10.0)


# ---------------------------------------------------------------------------
# topology
# ---------------------------------------------------------------------------
class AmberTopology:
    """AmberTopology (core/src/amber/prmtop.rs:34-105), held by librstg."""

    def __init__(self, handle):
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            N.lib.rstg_topology_free(h)
            self._h = None

    @classmethod
    def from_arrays(cls, charges_amber, radii, screen=None, atom_type_indices=None, n_types=1,
                    lj_acoef=(0.0,), lj_bcoef=(0.0,), nb_parm_index=(1,), residue_pointers=(0,), bonds=(),
                    bond_k=(), bond_req=(), angles=(), angle_k=(), angle_teq=(), dihedrals=(), dihedral_pk=(),
                    dihedral_pn=(), dihedral_phase=(), num_excluded=None, excluded_list=(), scee=1.2, scnb=2.0):
        """Build a topology from arrays (as the reference's unit tests build AmberTopology)."""
        n = len(charges_amber)
        keep = []

        def f(v):
            a = np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(-1))
            keep.append(a)
            return a.ctypes.data if a.size else None

        def i(v):
            a = np.ascontiguousarray(np.asarray(v, dtype=np.int64).reshape(-1))
            keep.append(a)
            return a.ctypes.data if a.size else None

        d = N.TopologyDesc()
        d.n_atoms, d.n_residues, d.n_types = n, len(residue_pointers), n_types
        d.atom_type_indices = i(atom_type_indices if atom_type_indices is not None else np.zeros(n))
        d.charges_amber, d.radii = f(charges_amber), f(radii)
        d.screen = f(screen if screen is not None else np.zeros(n))
        d.residue_pointers = i(residue_pointers)
        d.n_bonds, d.bonds = len(bonds), i(bonds)
        d.n_bond_types, d.bond_k, d.bond_req = len(bond_k), f(bond_k), f(bond_req)
        d.n_angles, d.angles = len(angles), i(angles)
        d.n_angle_types, d.angle_k, d.angle_teq = len(angle_k), f(angle_k), f(angle_teq)
        d.n_dihedrals, d.dihedrals = len(dihedrals), i(dihedrals)
        d.n_dihedral_types = len(dihedral_pk)
        d.dihedral_pk, d.dihedral_pn, d.dihedral_phase = f(dihedral_pk), f(dihedral_pn), f(dihedral_phase)
        d.num_excluded = i(num_excluded if num_excluded is not None else np.zeros(n))
        d.n_excluded, d.excluded_list = len(excluded_list), i(excluded_list)
        d.scee, d.scnb = scee, scnb
        d.n_lj, d.lj_acoef, d.lj_bcoef = len(lj_acoef), f(lj_acoef), f(lj_bcoef)
        d.nb_parm_index = i(nb_parm_index)
        h = N.vp()
        check(N.lib.rstg_topology_from_desc(C.byref(d), C.byref(h)))
        return cls(h)

    def _info(self):
        inf = N.TopologyInfo()
        check(N.lib.rstg_topology_info_get(self._h, C.byref(inf)))
        return inf

    @property
    def n_atoms(self) -> int:
        return int(self._info().n_atoms)

    @property
    def n_residues(self) -> int:
        return int(self._info().n_residues)

    def _names(self):
        n, r = self.n_atoms, self.n_residues
        a = C.create_string_buffer(max(4 * n, 1))
        b = C.create_string_buffer(max(4 * r, 1))
        check(N.lib.rstg_topology_names(self._h, a, b))
        dec = lambda buf, k: [buf.raw[4 * j:4 * j + 4].split(b"\0")[0].decode() for j in range(k)]
        return dec(a, n), dec(b, r)

    @property
    def atom_names(self) -> List[str]:
        return self._names()[0]

    @property
    def residue_labels(self) -> List[str]:
        return self._names()[1]

    def _atoms(self):
        n = self.n_atoms
        out = {k: np.zeros(n) for k in ("charges", "charges_amber", "radii", "screen", "masses")}
        ty = np.zeros(n, np.int64)
        res = np.zeros(n, np.int64)
        check(N.lib.rstg_topology_atoms(self._h, _dp(out["charges"]), _dp(out["charges_amber"]),
                                        _dp(out["radii"]), _dp(out["screen"]), _dp(out["masses"]), _ip(ty),
                                        _ip(res)))
        out["type_idx"], out["residue_index"] = ty, res
        return out

    def charges(self) -> np.ndarray:
        """Partial charges in elementary charge units."""
        return self._atoms()["charges"]

    def masses(self) -> np.ndarray:
        return self._atoms()["masses"]

    def radii(self) -> np.ndarray:
        return self._atoms()["radii"]

    def atom_residue_indices(self) -> np.ndarray:
        return self._atoms()["residue_index"]

    def residue_pointers(self) -> np.ndarray:
        out = np.zeros(self.n_residues, np.int64)
        check(N.lib.rstg_topology_residue_pointers(self._h, _ip(out)))
        return out

    def get_atom_indices(self, residue_indices) -> np.ndarray:
        r = _i64(residue_indices)
        n = C.c_int64()
        check(N.lib.rstg_topology_select(self._h, _ip(r), len(r), None, C.byref(n)))
        out = np.zeros(n.value, np.int64)
        check(N.lib.rstg_topology_select(self._h, _ip(r), len(r), _ip(out), C.byref(n)))
        return out

    def build_selection(self, residue_indices) -> dict:
        """prmtop.rs:165-204 as returned by lib.rs:864-889."""
        labels = self.residue_labels
        atoms, offsets = [], []
        for r in residue_indices:
            offsets.append(len(atoms))
            atoms.extend(self.get_atom_indices([r]).tolist())
        offsets.append(len(atoms))
        return {"atom_indices": np.array(atoms, np.int64), "residue_offsets": np.array(offsets, np.int64),
                "residue_labels": [labels[r] for r in residue_indices]}


def read_prmtop(path: str) -> AmberTopology:
    """parse_prmtop (core/src/amber/prmtop.rs:444-733); raises IOError."""
    h = N.vp()
    check(N.lib.rstg_topology_load_prmtop(str(path).encode(), C.byref(h)))
    return AmberTopology(h)


def extract_subtopology(topology: AmberTopology, atom_indices) -> AmberTopology:
    """crates/mmpbsa/src/subsystem.rs:22-169."""
    a = _i64(atom_indices)
    h = N.vp()
    check(N.lib.rstg_topology_extract(topology._h, _ip(a), len(a), C.byref(h)))
    return AmberTopology(h)


# ---------------------------------------------------------------------------
# trajectory readers
# ---------------------------------------------------------------------------
class DcdReader:
    """DcdReader (core/src/trajectory/dcd.rs): frames in nm."""

    def __init__(self, path: str):
        self.path = str(path)
        nf, na = C.c_int64(), C.c_int64()
        check(N.lib.rstg_dcd_read(self.path.encode(), None, 0, C.byref(nf), C.byref(na)))
        self._nf, self._na = nf.value, na.value
        self._data = None
        self._cur = 0

    @property
    def n_frames(self) -> int:
        return self._nf

    @property
    def n_atoms(self) -> int:
        return self._na

    @property
    def current_frame(self) -> int:
        return self._cur

    def _load(self):
        if self._data is None:
            out = np.zeros((self._nf, self._na, 3))
            nf, na = C.c_int64(), C.c_int64()
            check(N.lib.rstg_dcd_read(self.path.encode(), _dp(out), out.size, C.byref(nf), C.byref(na)))
            self._data = out
        return self._data

    def seek(self, frame: int) -> None:
        if frame >= self._nf:
            raise IOError(f"Frame {frame} out of range (0-{self._nf - 1})")
        self._cur = frame

    def read_frame(self):
        if self._cur >= self._nf:
            return None
        f = self._load()[self._cur].copy()
        self._cur += 1
        return f, None

    def read_frame_at(self, frame_index: int):
        self.seek(frame_index)
        return self.read_frame()

    def read_all(self):
        if self._nf == 0:
            raise ValueError("No frames to read")
        return self._load().copy(), None

    def read_all_f32_angstrom(self) -> np.ndarray:
        """Frames as stored (float32 Angstrom), the batched engine's input."""
        out = np.zeros((self._nf, self._na, 3), np.float32)
        nf, na = C.c_int64(), C.c_int64()
        check(N.lib.rstg_dcd_read_f32(self.path.encode(), out.ctypes.data_as(C.POINTER(C.c_float)), out.size,
                                      C.byref(nf), C.byref(na)))
        return out

    def __iter__(self):
        return self

    def __next__(self):
        r = self.read_frame()
        if r is None:
            raise StopIteration
        return r


class MdcrdReader:
    """MdcrdReader (crates/mmpbsa/src/mdcrd.rs): frames in Angstrom."""

    def __init__(self, path: str, n_atoms: int, has_box: bool):
        self.path, self.n_atoms, self.has_box = str(path), int(n_atoms), bool(has_box)
        nf = C.c_int64()
        check(N.lib.rstg_mdcrd_read(self.path.encode(), self.n_atoms, int(self.has_box), None, 0, C.byref(nf)))
        self._nf = nf.value
        self._data = None
        self._cur = 0

    @property
    def current_frame(self) -> int:
        return self._cur

    def read_frame(self):
        if self._data is None:
            out = np.zeros((self._nf, self.n_atoms, 3))
            nf = C.c_int64()
            check(N.lib.rstg_mdcrd_read(self.path.encode(), self.n_atoms, int(self.has_box), _dp(out), out.size,
                                        C.byref(nf)))
            self._data = out
        if self._cur >= self._nf:
            return None
        f = self._data[self._cur].copy()
        self._cur += 1
        return f

    def __iter__(self):
        return self

    def __next__(self):
        r = self.read_frame()
        if r is None:
            raise StopIteration
        return r


# ---------------------------------------------------------------------------
# parameters
# ---------------------------------------------------------------------------
class GbModel(enum.IntEnum):
    Hct = 0
    ObcI = 1
    ObcII = 2


class GbParams:
    """GbParams (gb_energy.rs:24-56); ``None`` keeps the reference default."""

    def __init__(self, model=None, solute_dielectric=None, solvent_dielectric=None, salt_concentration=None,
                 temperature=None, offset=None, rgbmax=None, cutoff=None):
        self._c = N.GbParams()
        N.lib.rstg_gb_params_default(C.byref(self._c))
        for k, v in (("model", None if model is None else int(model)), ("solute_dielectric", solute_dielectric),
                     ("solvent_dielectric", solvent_dielectric), ("salt_concentration", salt_concentration),
                     ("temperature", temperature), ("offset", offset), ("rgbmax", rgbmax), ("cutoff", cutoff)):
            if v is not None:
                setattr(self._c, k, v)

    model = property(lambda s: GbModel(s._c.model))
    solute_dielectric = property(lambda s: s._c.solute_dielectric)
    solvent_dielectric = property(lambda s: s._c.solvent_dielectric)
    salt_concentration = property(lambda s: s._c.salt_concentration)
    temperature = property(lambda s: s._c.temperature)
    offset = property(lambda s: s._c.offset)
    rgbmax = property(lambda s: s._c.rgbmax)
    cutoff = property(lambda s: s._c.cutoff)


class PbParams:
    """PbParams (pb_energy.rs:21-66)."""

    def __init__(self, grid_spacing=None, grid_buffer=None, solute_dielectric=None, solvent_dielectric=None,
                 salt_concentration=None, temperature=None, probe_radius=None, ion_radius=None, tolerance=None,
                 max_iterations=None, fillratio=None, fscale=None):
        self._c = N.PbParams()
        N.lib.rstg_pb_params_default(C.byref(self._c))
        for k, v in (("grid_spacing", grid_spacing), ("grid_buffer", grid_buffer),
                     ("solute_dielectric", solute_dielectric), ("solvent_dielectric", solvent_dielectric),
                     ("salt_concentration", salt_concentration), ("temperature", temperature),
                     ("probe_radius", probe_radius), ("ion_radius", ion_radius), ("tolerance", tolerance),
                     ("max_iterations", max_iterations), ("fillratio", fillratio), ("fscale", fscale)):
            if v is not None:
                setattr(self._c, k, v)

    grid_spacing = property(lambda s: s._c.grid_spacing)
    solute_dielectric = property(lambda s: s._c.solute_dielectric)
    solvent_dielectric = property(lambda s: s._c.solvent_dielectric)
    salt_concentration = property(lambda s: s._c.salt_concentration)
    temperature = property(lambda s: s._c.temperature)


class SaParams:
    """SaParams (sa_energy.rs:12-32)."""

    def __init__(self, surface_tension=None, offset=None, probe_radius=None, n_sphere_points=None):
        self._c = N.SaParams()
        N.lib.rstg_sa_params_default(C.byref(self._c))
        for k, v in (("surface_tension", surface_tension), ("offset", offset), ("probe_radius", probe_radius),
                     ("n_sphere_points", n_sphere_points)):
            if v is not None:
                setattr(self._c, k, v)

    surface_tension = property(lambda s: s._c.surface_tension)
    offset = property(lambda s: s._c.offset)
    probe_radius = property(lambda s: s._c.probe_radius)
    n_sphere_points = property(lambda s: s._c.n_sphere_points)


def _gb(p: Optional[GbParams]) -> N.GbParams:
    return (p or GbParams())._c


def _sa(p: Optional[SaParams]) -> N.SaParams:
    return (p or SaParams())._c


def _solvation(gb_params: Optional[GbParams], pb_params: Optional[PbParams]) -> N.Solvation:
    # build_solvation_method, lib.rs:2106-2115: pb_params wins over gb_params
    s = N.Solvation()
    s.gb = _gb(gb_params)
    s.pb = (pb_params or PbParams())._c
    s.method = 1 if pb_params is not None else 0
    return s


# ---------------------------------------------------------------------------
# results
# ---------------------------------------------------------------------------
class MmEnergy:
    def __init__(self, c: N.MmEnergy):
        for k, _ in N.MmEnergy._fields_:
            setattr(self, k, float(getattr(c, k)))

    def total(self) -> float:
        return self.bond + self.angle + self.dihedral + self.vdw + self.elec + self.vdw_14 + self.elec_14


class GbEnergy:
    def __init__(self, total: float, radii: np.ndarray):
        self.total = float(total)
        self._r = radii

    def born_radii(self) -> np.ndarray:
        return self._r.copy()


class SaEnergy:
    def __init__(self, total: float, total_sasa: float, per_atom: np.ndarray):
        self.total, self.total_sasa = float(total), float(total_sasa)
        self._p = per_atom

    def per_atom_sasa(self) -> np.ndarray:
        return self._p.copy()


class PbEnergy:
    def __init__(self, total: float, diag: N.PbDiag = None):
        self.total = float(total)
        self.diag = None if diag is None else {
            "iterations": list(diag.iterations), "residual": list(diag.residual),
            "converged": [bool(v) for v in diag.converged], "dims": list(diag.dims)}


class FrameEnergy:
    """FrameEnergy (binding.rs:48-56) with the getters of lib.rs:1767-1865."""

    def __init__(self, c: N.FrameEnergy):
        self.complex_mm, self.complex_polar, self.complex_sa = c.complex.mm, c.complex.polar, c.complex.sa
        self.receptor_mm, self.receptor_polar, self.receptor_sa = c.receptor.mm, c.receptor.polar, c.receptor.sa
        self.ligand_mm, self.ligand_polar, self.ligand_sa = c.ligand.mm, c.ligand.polar, c.ligand.sa
        self.delta_mm, self.delta_polar, self.delta_sa, self.delta_total = (
            c.delta_mm, c.delta_polar, c.delta_sa, c.delta_total)

    delta_gb = property(lambda s: s.delta_polar)
    complex_gb = property(lambda s: s.complex_polar)
    receptor_gb = property(lambda s: s.receptor_polar)
    ligand_gb = property(lambda s: s.ligand_polar)
    complex_total = property(lambda s: s.complex_mm + s.complex_polar + s.complex_sa)
    receptor_total = property(lambda s: s.receptor_mm + s.receptor_polar + s.receptor_sa)
    ligand_total = property(lambda s: s.ligand_mm + s.ligand_polar + s.ligand_sa)

    def as_array(self) -> np.ndarray:
        return np.array([self.complex_mm, self.complex_polar, self.complex_sa, self.receptor_mm,
                         self.receptor_polar, self.receptor_sa, self.ligand_mm, self.ligand_polar, self.ligand_sa,
                         self.delta_mm, self.delta_polar, self.delta_sa, self.delta_total])


FRAME_FIELDS = ("complex_mm", "complex_polar", "complex_sa", "receptor_mm", "receptor_polar", "receptor_sa",
                "ligand_mm", "ligand_polar", "ligand_sa", "delta_mm", "delta_polar", "delta_sa", "delta_total")


class BindingResult:
    """BindingResult (binding.rs:60-76) with the getters of lib.rs:1867-1933."""

    def __init__(self, frames: List[FrameEnergy], stats: np.ndarray, last: np.ndarray):
        self._frames = frames
        (self.mean_delta_mm, self.mean_delta_polar, self.mean_delta_sa, self.mean_delta_total,
         self.std_delta_total, self.std_delta_mm, self.std_delta_polar, self.std_delta_sa,
         self.sem_delta_total) = (float(v) for v in stats)
        self._last = last

    mean_delta_gb = property(lambda s: s.mean_delta_polar)
    std_delta_gb = property(lambda s: s.std_delta_polar)

    @property
    def frames(self) -> List[FrameEnergy]:
        return list(self._frames)

    def last_frame_coords(self) -> np.ndarray:
        return self._last.copy()


class ResidueContribution:
    def __init__(self, index: int, label: str, e: N.ResidueEnergy):
        self.residue_index, self.residue_label = int(index), label
        self.vdw, self.elec, self.polar, self.sa = e.vdw, e.elec, e.polar, e.sa

    gb = property(lambda s: s.polar)

    def total(self) -> float:
        return self.vdw + self.elec + self.polar + self.sa


class DecompositionResult:
    def __init__(self, rec: List[ResidueContribution], lig: List[ResidueContribution]):
        self._r, self._l = rec, lig

    @property
    def receptor_residues(self) -> List[ResidueContribution]:
        return list(self._r)

    @property
    def ligand_residues(self) -> List[ResidueContribution]:
        return list(self._l)


class EntropyEstimate:
    def __init__(self, minus_tds: float, method: str):
        self.minus_tds, self.method = float(minus_tds), method


# ---------------------------------------------------------------------------
# single-frame functions (coords in nm)
# ---------------------------------------------------------------------------
def compute_mm_energy(topology: AmberTopology, coords) -> MmEnergy:
    x = _coords_A(coords)
    out = N.MmEnergy()
    check(N.lib.rstg_mm_energy_compute(N.ctx(), topology._h, _dp(x), len(x), C.byref(out)))
    return MmEnergy(out)


def compute_gb_energy(topology: AmberTopology, coords, gb_params: GbParams = None) -> GbEnergy:
    x = _coords_A(coords)
    tot = C.c_double()
    R = np.zeros(len(x))
    check(N.lib.rstg_gb_energy_compute(N.ctx(), topology._h, _dp(x), len(x), C.byref(_gb(gb_params)),
                                       C.byref(tot), _dp(R)))
    return GbEnergy(tot.value, R)


class GbCache:
    """Born radii kept from a previous frame (gb_energy.rs:66-120): a frame
    whose RMSD to the cached coordinates is below ``rmsd_threshold`` (A)
    reuses them.  Rust-crate API; the reference's Python module does not
    expose it."""

    def __init__(self, rmsd_threshold: float = 0.5):
        h = N.vp()
        check(N.lib.rstg_gb_cache_create(float(rmsd_threshold), C.byref(h)))
        self._h = h
        self.last_reused = False

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            N.lib.rstg_gb_cache_destroy(h)
            self._h = None


def compute_gb_energy_cached(topology: AmberTopology, coords, gb_params: GbParams = None,
                             cache: GbCache = None) -> GbEnergy:
    """compute_gb_energy_cached (gb_energy.rs:372-387); coords in nm like the
    other calls.  ``cache.last_reused`` tells whether the radii were reused."""
    if cache is None:
        raise ValueError("cache must be a GbCache")
    x = _coords_A(coords)
    tot = C.c_double()
    R = np.zeros(len(x))
    hit = C.c_int32()
    check(N.lib.rstg_gb_energy_cached(N.ctx(), topology._h, _dp(x), len(x), C.byref(_gb(gb_params)), cache._h,
                                      C.byref(tot), _dp(R), C.byref(hit)))
    cache.last_reused = bool(hit.value)
    return GbEnergy(tot.value, R)


def compute_sa_energy(topology: AmberTopology, coords, sa_params: SaParams = None) -> SaEnergy:
    x = _coords_A(coords)
    tot, ts = C.c_double(), C.c_double()
    per = np.zeros(len(x))
    check(N.lib.rstg_sa_energy_compute(N.ctx(), topology._h, _dp(x), len(x), C.byref(_sa(sa_params)),
                                       C.byref(tot), C.byref(ts), _dp(per)))
    return SaEnergy(tot.value, ts.value, per)


def compute_pb_energy(topology: AmberTopology, coords, pb_params: PbParams = None,
                      solute_residues: Optional[Sequence[int]] = None) -> PbEnergy:
    x = _coords_A(coords)
    tot = C.c_double()
    d = N.PbDiag()
    sr = _i64(solute_residues) if solute_residues is not None else None
    check(N.lib.rstg_pb_energy_compute(N.ctx(), topology._h, _dp(x), len(x),
                                       C.byref((pb_params or PbParams())._c),
                                       _ip(sr) if sr is not None else None, len(sr) if sr is not None else 0,
                                       C.byref(tot), C.byref(d)))
    return PbEnergy(tot.value, d)


def compute_binding_energy_single_frame(topology: AmberTopology, coords, receptor_residues, ligand_residues,
                                        gb_params: GbParams = None, pb_params: PbParams = None,
                                        sa_params: SaParams = None) -> FrameEnergy:
    x = _coords_A(coords)
    rr, lr = _i64(receptor_residues), _i64(ligand_residues)
    out = N.FrameEnergy()
    check(N.lib.rstg_binding_frame(N.ctx(), topology._h, _dp(x), len(x), _ip(rr), len(rr), _ip(lr), len(lr),
                                   C.byref(_solvation(gb_params, pb_params)), C.byref(_sa(sa_params)),
                                   C.byref(out)))
    return FrameEnergy(out)


def decompose_binding_energy(topology: AmberTopology, coords, receptor_residues, ligand_residues,
                             gb_params: GbParams = None, sa_params: SaParams = None) -> DecompositionResult:
    x = _coords_A(coords)
    rr, lr = _i64(receptor_residues), _i64(ligand_residues)
    ro = (N.ResidueEnergy * max(len(rr), 1))()
    lo = (N.ResidueEnergy * max(len(lr), 1))()
    check(N.lib.rstg_decompose(N.ctx(), topology._h, _dp(x), len(x), _ip(rr), len(rr), _ip(lr), len(lr),
                               C.byref(_gb(gb_params)), C.byref(_sa(sa_params)), ro, lo))
    labels = topology.residue_labels
    return DecompositionResult([ResidueContribution(r, labels[r], ro[k]) for k, r in enumerate(rr)],
                               [ResidueContribution(r, labels[r], lo[k]) for k, r in enumerate(lr)])


def compute_binding_energy(topology, trajectory_path: str, receptor_residues, ligand_residues,
                           gb_params: GbParams = None, pb_params: PbParams = None, sa_params: SaParams = None,
                           trajectory_format: str = None, has_box: bool = False, stride: int = 1,
                           start_frame: int = 0, end_frame: int = USIZE_MAX, mode: str = "fused") -> BindingResult:
    """binding.rs:461-744 over a DCD (``trajectory_format="dcd"``) or mdcrd file.

    ``mode`` selects the batched fused engine (default) or ``"plain"``, the
    per-subsystem FP64 form."""
    if isinstance(topology, str):
        topology = read_prmtop(topology)
    if not isinstance(topology, AmberTopology):
        raise ValueError("topology must be an AmberTopology object or a path string")
    fmt = "dcd" if (trajectory_format or "mdcrd") == "dcd" else "mdcrd"
    rr, lr = _i64(receptor_residues), _i64(ligand_residues)
    n_frames = C.c_int64()
    stats = np.zeros(9)
    end = min(int(end_frame), 2 ** 63 - 1)
    # size pass: frames of the file bound the output
    cap = _trajectory_capacity(topology, trajectory_path, fmt, has_box)
    frames = (N.FrameEnergy * max(cap, 1))()
    last = np.zeros((topology.n_atoms, 3))
    check(N.lib.rstg_binding_trajectory(N.ctx(), topology._h, str(trajectory_path).encode(), fmt.encode(),
                                        int(has_box), _ip(rr), len(rr), _ip(lr), len(lr),
                                        C.byref(_solvation(gb_params, pb_params)), C.byref(_sa(sa_params)),
                                        int(stride), int(start_frame), end, 0 if mode == "plain" else 1,
                                        frames, cap, C.byref(n_frames), _dp(stats), _dp(last)))
    nf = n_frames.value
    n_complex = _complex_atoms(topology, rr, lr)
    return BindingResult([FrameEnergy(frames[k]) for k in range(nf)], stats, last[:n_complex])


def _trajectory_capacity(topology, path, fmt, has_box) -> int:
    if fmt == "dcd":
        return DcdReader(path).n_frames
    return MdcrdReader(path, topology.n_atoms, has_box)._nf


def _complex_atoms(topology, rr, lr) -> int:
    res = sorted(set(rr.tolist()) | set(lr.tolist()))
    return len(topology.get_atom_indices(res))


# ---------------------------------------------------------------------------
# entropy (crates/mmpbsa/src/entropy.rs), host-side post-processing
# ---------------------------------------------------------------------------
def interaction_entropy(frames: List[FrameEnergy], temperature: float = 298.15) -> Optional[EntropyEstimate]:
    """entropy.rs:53-95: -T dS = kT ln < exp(dE_int / kT) > (log-sum-exp)."""
    n = len(frames)
    if n < 2:
        return None
    kt = 0.00198688 * temperature
    de = np.array([f.delta_mm for f in frames])
    x = (de - de.sum() / n) / kt
    m = x.max()
    return EntropyEstimate(kt * (m + math.log(np.exp(x - m).sum() / n)), "interaction_entropy")


def quasi_harmonic_entropy(trajectory_3d, masses, temperature: float = 298.15) -> Optional[EntropyEstimate]:
    """entropy.rs:97-225: quantum harmonic-oscillator entropy of the
    mass-weighted covariance eigenvalues."""
    from ._entropy import quasi_harmonic

    v = quasi_harmonic(np.asarray(trajectory_3d, dtype=np.float64), np.asarray(masses, dtype=np.float64),
                       temperature)
    return None if v is None else EntropyEstimate(v, "quasi_harmonic")


# ---------------------------------------------------------------------------
# batched engine and serving loop (no reference counterpart)
# ---------------------------------------------------------------------------
class BindingSystem:
    """Device-resident binding problem: all frames x {complex, receptor,
    ligand} evaluated per batched launch sequence.

    ``mode``: ``"fused"`` (mixed precision, binding differences fused) or
    ``"plain"`` (FP64, one subsystem per launch sequence)."""

    def __init__(self, topology: AmberTopology, receptor_residues, ligand_residues, gb_params: GbParams = None,
                 pb_params: PbParams = None, sa_params: SaParams = None, mode: str = "fused",
                 batch_frames: int = 0, use_graphs: bool = True, autotune: bool = True, ctx=None):
        self.topology = topology
        self.ctx = ctx or N.ctx()
        rr, lr = _i64(receptor_residues), _i64(ligand_residues)
        o = N.SystemOpts()
        N.lib.rstg_system_opts_default(C.byref(o))
        o.mode = 0 if mode == "plain" else 1
        o.max_batch_frames = int(batch_frames)
        o.use_graphs = int(use_graphs)
        o.autotune = int(autotune)
        h = N.vp()
        check(N.lib.rstg_system_create(self.ctx, topology._h, _ip(rr), len(rr), _ip(lr), len(lr),
                                       C.byref(_solvation(gb_params, pb_params)), C.byref(_sa(sa_params)),
                                       C.byref(o), C.byref(h)))
        self._h = h
        sh = np.zeros(6, np.int64)
        check(N.lib.rstg_system_shape(h, _ip(sh)))
        (self.n_complex, self.n_receptor, self.n_ligand, self.n_receptor_residues, self.n_ligand_residues,
         self.n_atoms) = (int(v) for v in sh)
        self.receptor_residues, self.ligand_residues = rr, lr

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            N.lib.rstg_system_destroy(h)
            self._h = None

    @property
    def n_residues(self) -> int:
        return self.n_receptor_residues + self.n_ligand_residues

    def footprint(self, n_frames: int) -> int:
        return int(N.lib.rstg_system_footprint(self._h, n_frames))

    def run(self, frames_f32_A, decompose: bool = False):
        """frames: (F, n_atoms, 3) float32 Angstrom as stored in DCD.
        Returns (F, 13) energies in FRAME_FIELDS order and, if requested,
        (F, n_residues, 4) per-residue vdw/elec/polar/sa."""
        fr = np.ascontiguousarray(frames_f32_A, dtype=np.float32)
        if fr.ndim != 3 or fr.shape[1:] != (self.n_atoms, 3):
            raise ValueError(f"frames must have shape (F, {self.n_atoms}, 3)")
        F = fr.shape[0]
        out = np.zeros((F, 13))
        dec = np.zeros((F, self.n_residues, 4)) if decompose else None
        check(N.lib.rstg_system_run(self._h, fr.ctypes.data_as(C.POINTER(C.c_float)), F,
                                    out.ctypes.data_as(C.POINTER(N.FrameEnergy)),
                                    dec.ctypes.data_as(C.POINTER(N.ResidueEnergy)) if decompose else None))
        return (out, dec) if decompose else out

    def reimage(self, frames_A, boxes, on_device: bool = True) -> np.ndarray:
        """Periodic reimaging of the complex atoms of each frame
        (reimage_complex, binding.rs:234-308): frames (F, n_atoms, 3)
        float64 Angstrom in topology order, boxes (F, 3) edge lengths.
        Returns the reimaged frames (the other atoms as given)."""
        fr = np.ascontiguousarray(frames_A, dtype=np.float64)
        bx = np.ascontiguousarray(boxes, dtype=np.float64)
        if fr.ndim != 3 or fr.shape[1:] != (self.n_atoms, 3):
            raise ValueError(f"frames must have shape (F, {self.n_atoms}, 3)")
        if bx.shape != (fr.shape[0], 3):
            raise ValueError(f"boxes must have shape ({fr.shape[0]}, 3)")
        out = np.empty_like(fr)
        check(N.lib.rstg_system_reimage(self._h, fr.ctypes.data_as(N.dp), bx.ctypes.data_as(N.dp), fr.shape[0],
                                        int(bool(on_device)), out.ctypes.data_as(N.dp)))
        return out

    def run_device(self, d_frames: int, n_frames: int, d_out: int, d_decomp: int = 0) -> None:
        """Device pointers (e.g. torch ``data_ptr()``): frames float32
        [F][n_atoms][3], out float64 [F][13], decomp float64 [F][n_res][4]."""
        check(N.lib.rstg_system_run_device(self._h, N.vp(d_frames), int(n_frames), N.vp(d_out),
                                           N.vp(d_decomp) if d_decomp else None))

    def last_stats(self) -> dict:
        st = np.zeros(4, np.int64)
        check(N.lib.rstg_system_last_stats(self._h, _ip(st)))
        return {"launches": int(st[0]), "fp64_guard_pairs": int(st[1]), "sasa_rechecks": int(st[2]),
                "neighbour_overflow": int(st[3])}

    def tuning(self) -> dict:
        """Launch shapes of the fused engine (picked on the first run when
        autotuning) and the tuning pass's candidate times in ms."""
        sh = (C.c_int32 * 12)()
        ms = np.zeros(12)
        check(N.lib.rstg_system_tuning(self._h, sh, _dp(ms)))
        npair, nsasa, npsi = sh[6], sh[7], sh[10]
        return {"pairs_threads_per_row": sh[0], "pairs_min_blocks_per_sm": sh[1], "sasa_warps_per_block": sh[2],
                "batch_frames": sh[3], "tuned": bool(sh[4]), "tuning_frames": sh[5],
                "psi_threads_per_row": sh[8], "psi_min_blocks_per_sm": sh[9],
                "pairs_form": "warp items" if sh[11] else "block per tile",
                "pairs_candidates_ms": ms[:npair].tolist(), "sasa_candidates_ms": ms[npair:npair + nsasa].tolist(),
                "psi_candidates_ms": ms[npair + nsasa:npair + nsasa + npsi].tolist()}

    def pb_stats(self) -> dict:
        """Batched PB engine totals of a fused PB system (zeros otherwise)."""
        st = np.zeros(8)
        check(N.lib.rstg_system_pb_stats(self._h, _dp(st)))
        return {"grids": int(st[0]), "cycles": int(st[1]), "fp64_fallbacks": int(st[2]), "ms_setup": st[3],
                "ms_cycles": st[4], "ms_finish": st[5]}

    def set_pb_profile(self, on: bool = True) -> None:
        """Time the level-0 PB multigrid kernels with CUDA events on later runs
        (launches without graph capture while on)."""
        check(N.lib.rstg_system_set_pb_profile(self._h, int(bool(on))))

    def pb_profile(self) -> dict:
        """Per-kernel totals of the PB profile mode: ms, algorithmic DRAM bytes
        and launches of the finest-level full red-black sweep, FP32 residual
        and end-of-cycle update + FP64 residual ("residual64")."""
        st = np.zeros(12)
        check(N.lib.rstg_system_pb_profile(self._h, _dp(st)))
        names = ("sweep", "residual32", "residual64")
        return {n: {"ms": st[k], "bytes": st[4 + k], "launches": int(st[8 + k])} for k, n in enumerate(names)}

    def set_pb_convergence(self, rel_tol: float = 0.0) -> None:
        """PB stopping rule of later runs: 0 keeps the reference's schedule
        (absolute RMS below ``PbParams.tolerance`` or the 200-cycle cap);
        ``rel_tol`` > 0 solves every grid to that relative FP64 residual
        with FP32 V-cycles of a consistent multigrid under FP64 defect
        correction."""
        check(N.lib.rstg_system_set_pb_convergence(self._h, float(rel_tol)))

    def set_pb_batch(self, frames: int) -> None:
        """Frames per batched PB launch sequence (0: from the memory budget)."""
        check(N.lib.rstg_system_set_pb_batch(self._h, int(frames)))


class Server:
    """Continuous-batching request loop over :class:`BindingSystem` objects."""

    def __init__(self, memory_budget_bytes: int = 16 << 30, max_inflight: int = 4, ctx=None):
        o = N.ServerOpts()
        N.lib.rstg_server_opts_default(C.byref(o))
        o.memory_budget_bytes, o.max_inflight = int(memory_budget_bytes), int(max_inflight)
        h = N.vp()
        check(N.lib.rstg_server_create(ctx or N.ctx(), C.byref(o), C.byref(h)))
        self._h = h
        self._keep = {}

    def close(self):
        if getattr(self, "_h", None):
            N.lib.rstg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def submit(self, system: BindingSystem, frames_f32_A) -> int:
        fr = np.ascontiguousarray(frames_f32_A, dtype=np.float32)
        rid = C.c_int64()
        check(N.lib.rstg_server_submit(self._h, system._h, fr.ctypes.data_as(C.POINTER(C.c_float)), fr.shape[0],
                                       C.byref(rid)))
        self._keep[rid.value] = (system, fr.shape[0])
        return rid.value

    def wait(self, request_id: int, timeout_ms: int = -1) -> np.ndarray:
        F = self._keep[request_id][1]
        out = np.zeros((max(F, 1), 13))
        check(N.lib.rstg_server_wait(self._h, request_id, timeout_ms, out.ctypes.data_as(C.POINTER(N.FrameEnergy))))
        return out[:F]

    def poll(self, request_id: int):
        F = self._keep[request_id][1]
        out = np.zeros((max(F, 1), 13))
        rc = N.lib.rstg_server_poll(self._h, request_id, out.ctypes.data_as(C.POINTER(N.FrameEnergy)))
        if rc == N.ERR_NOT_READY:
            return None
        check(rc)
        return out[:F]

    def cancel(self, request_id: int) -> None:
        check(N.lib.rstg_server_cancel(self._h, request_id))

    def stats(self) -> dict:
        st = np.zeros(8)
        check(N.lib.rstg_server_stats(self._h, _dp(st)))
        keys = ("completed", "frames", "p50_ms", "p99_ms", "mean_ms", "peak_bytes", "wall_s", "frames_per_s")
        return dict(zip(keys, st.tolist()))
