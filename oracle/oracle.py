"""ctypes wrapper for the CPU restatement of the reference MM-PBSA/GBSA path.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()``
(as the checker) and by ``bench.py`` (the CPU baseline leg and the
``--impl reference`` arm).  The product package never imports this module.

The library is built by ``oracle/Makefile`` into ``oracle/_build/liborc.so``.
Parity pinning is described in ``oracle/oracle.hpp``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liborc.so")

GB_MODELS = {"hct": 0, "obc1": 1, "obc2": 2}


class GbP(C.Structure):
    _fields_ = [("model", C.c_int32), ("solute_dielectric", C.c_double), ("solvent_dielectric", C.c_double),
                ("salt", C.c_double), ("temperature", C.c_double), ("offset", C.c_double),
                ("rgbmax", C.c_double), ("cutoff", C.c_double)]


class SaP(C.Structure):
    _fields_ = [("surface_tension", C.c_double), ("offset", C.c_double), ("probe", C.c_double),
                ("n_points", C.c_int64)]


class PbP(C.Structure):
    _fields_ = [("grid_spacing", C.c_double), ("grid_buffer", C.c_double), ("solute_dielectric", C.c_double),
                ("solvent_dielectric", C.c_double), ("salt", C.c_double), ("temperature", C.c_double),
                ("probe", C.c_double), ("ion_radius", C.c_double), ("tolerance", C.c_double),
                ("max_iterations", C.c_int64), ("fillratio", C.c_double), ("fscale", C.c_int64),
                ("converged_rel_tol", C.c_double), ("converged_method", C.c_int64)]


class TopoDesc(C.Structure):
    _fields_ = [("n_atoms", C.c_int64), ("n_residues", C.c_int64), ("n_types", C.c_int64),
                ("type_idx", C.c_void_p), ("charges_amber", C.c_void_p), ("radii", C.c_void_p),
                ("screen", C.c_void_p), ("residue_pointers", C.c_void_p),
                ("n_bonds", C.c_int64), ("bonds", C.c_void_p), ("n_bond_types", C.c_int64),
                ("bond_k", C.c_void_p), ("bond_req", C.c_void_p),
                ("n_angles", C.c_int64), ("angles", C.c_void_p), ("n_angle_types", C.c_int64),
                ("angle_k", C.c_void_p), ("angle_teq", C.c_void_p),
                ("n_dihedrals", C.c_int64), ("dihedrals", C.c_void_p), ("n_dihedral_types", C.c_int64),
                ("dih_pk", C.c_void_p), ("dih_pn", C.c_void_p), ("dih_phase", C.c_void_p),
                ("num_excluded", C.c_void_p), ("n_excluded", C.c_int64), ("excluded_list", C.c_void_p),
                ("scee", C.c_double), ("scnb", C.c_double),
                ("n_lj", C.c_int64), ("lj_a", C.c_void_p), ("lj_b", C.c_void_p), ("nb_index", C.c_void_p)]


def build() -> str:
    """Compile the restatement (make) and return the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        vp, dp, ip, i64 = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.c_int64
        L.orc_topology_load.restype = vp
        L.orc_topology_load.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.orc_topology_from_desc.restype = vp
        L.orc_topology_from_desc.argtypes = [C.POINTER(TopoDesc)]
        L.orc_topology_free.argtypes = [vp]
        L.orc_topology_n_atoms.restype = i64
        L.orc_topology_n_atoms.argtypes = [vp]
        L.orc_topology_n_residues.restype = i64
        L.orc_topology_n_residues.argtypes = [vp]
        L.orc_topology_arrays.argtypes = [vp, dp, dp, dp, dp, ip, ip]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
        L.orc_kappa.restype = C.c_double
        L.orc_kappa.argtypes = [C.c_double] * 3
        L.orc_gb_energy.restype = C.c_double
        L.orc_gb_energy.argtypes = [vp, dp, C.POINTER(GbP), C.c_int, dp]
        L.orc_gb_energy_from_radii.restype = C.c_double
        L.orc_gb_energy_from_radii.argtypes = [vp, dp, C.POINTER(GbP), dp]
        L.orc_mm_energy.argtypes = [vp, dp, C.c_int, dp]
        L.orc_sa_energy.restype = C.c_double
        L.orc_sa_energy.argtypes = [vp, dp, C.POINTER(SaP), dp, dp]
        L.orc_sasa_raw.argtypes = [i64, dp, dp, C.c_double, i64, dp]
        L.orc_fibonacci.argtypes = [i64, dp]
        L.orc_pb_energy.restype = C.c_double
        L.orc_pb_energy.argtypes = [vp, dp, C.POINTER(PbP), ip, dp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.orc_pb_energy_raw.restype = C.c_double
        L.orc_pb_energy_raw.argtypes = [i64, dp, dp, dp, C.POINTER(PbP)]
        L.orc_pb_maps.restype = i64
        L.orc_pb_maps.argtypes = [i64, dp, dp, dp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                  C.c_double, C.c_double, C.c_double, C.c_int, ip, dp, dp,
                                  C.POINTER(C.c_uint8), dp, dp, dp, dp, dp]
        L.orc_pb_solve.restype = i64
        L.orc_pb_solve.argtypes = [i64, dp, dp, ip, dp, C.c_double, dp, dp, dp, dp, dp, C.c_double, C.c_double,
                                   C.c_double, i64, dp, dp, C.POINTER(C.c_int32), dp]
        L.orc_restrict_prolong_constant.argtypes = [C.c_double, dp, dp]
        L.orc_charge_total.restype = C.c_double
        L.orc_charge_total.argtypes = [i64, dp, dp, C.c_double, C.c_double]
        L.orc_binding_frame.restype = C.c_int
        L.orc_binding_frame.argtypes = [vp, dp, ip, i64, ip, i64, C.c_int, C.POINTER(GbP), C.POINTER(PbP),
                                        C.POINTER(SaP), C.c_int, dp, C.c_char_p, C.c_int]
        L.orc_binding_frames.restype = C.c_int
        L.orc_binding_frames.argtypes = [vp, dp, i64, ip, i64, ip, i64, C.c_int, C.POINTER(GbP), C.POINTER(PbP),
                                         C.POINTER(SaP), C.c_int, dp, C.c_char_p, C.c_int]
        L.orc_decompose.restype = C.c_int
        L.orc_decompose.argtypes = [vp, dp, ip, i64, ip, i64, C.POINTER(GbP), C.POINTER(SaP), C.c_int, dp, dp,
                                    C.c_char_p, C.c_int]
        L.orc_read_dcd.restype = i64
        L.orc_read_dcd.argtypes = [C.c_char_p, dp, i64, ip, C.c_char_p, C.c_int]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def gb_params(model="obc1", solute_dielectric=1.0, solvent_dielectric=78.3, salt=0.15, temperature=300.0,
              offset=0.09, rgbmax=25.0, cutoff=9999.0) -> GbP:
    """GbParams with the reference defaults (gb_energy.rs:43-56)."""
    return GbP(GB_MODELS.get(model, model) if isinstance(model, str) else model, solute_dielectric,
               solvent_dielectric, salt, temperature, offset, rgbmax, cutoff)


def sa_params(surface_tension=0.0072, offset=0.0, probe=1.4, n_points=480) -> SaP:
    """SaParams with the reference defaults (sa_energy.rs:23-32)."""
    return SaP(surface_tension, offset, probe, n_points)


def pb_params(grid_spacing=0.5, grid_buffer=10.0, solute_dielectric=1.0, solvent_dielectric=80.0, salt=0.15,
              temperature=300.0, probe=1.4, ion_radius=2.0, tolerance=1e-6, max_iterations=10000,
              fillratio=4.0, fscale=8, converged_rel_tol=0.0, converged_method=0) -> PbP:
    """PbParams with the reference defaults (pb_energy.rs:49-66).  With
    converged_rel_tol > 0 every grid is solved to that relative FP64
    residual instead of the reference's schedule: method 0 Jacobi-PCG,
    1 flexible CG preconditioned by a consistent V-cycle, 2 defect
    correction with that V-cycle."""
    return PbP(grid_spacing, grid_buffer, solute_dielectric, solvent_dielectric, salt, temperature, probe,
               ion_radius, tolerance, max_iterations, fillratio, fscale, converged_rel_tol, converged_method)


class Topology:
    """A parsed topology held by the restatement."""

    def __init__(self, handle):
        self.h = handle

    @classmethod
    def load(cls, path: str) -> "Topology":
        err = C.create_string_buffer(512)
        h = lib().orc_topology_load(path.encode(), err, 512)
        if not h:
            raise IOError(err.value.decode())
        return cls(h)

    @classmethod
    def from_arrays(cls, charges_amber, radii, screen=None, type_idx=None, n_types=1, lj_a=(0.0,), lj_b=(0.0,),
                    nb_index=(1,), residue_pointers=(0,), bonds=(), bond_k=(), bond_req=(), angles=(),
                    angle_k=(), angle_teq=(), dihedrals=(), dih_pk=(), dih_pn=(), dih_phase=(),
                    num_excluded=None, excluded_list=(), scee=1.2, scnb=2.0) -> "Topology":
        n = len(charges_amber)
        keep = []

        def f64(v):
            a = np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(-1))
            keep.append(a)
            return a.ctypes.data if a.size else None

        def i64(v):
            a = np.ascontiguousarray(np.asarray(v, dtype=np.int64).reshape(-1))
            keep.append(a)
            return a.ctypes.data if a.size else None

        d = TopoDesc()
        d.n_atoms, d.n_residues, d.n_types = n, len(residue_pointers), n_types
        d.type_idx = i64(type_idx if type_idx is not None else np.zeros(n))
        d.charges_amber, d.radii = f64(charges_amber), f64(radii)
        d.screen = f64(screen if screen is not None else np.zeros(n))
        d.residue_pointers = i64(residue_pointers)
        d.n_bonds, d.bonds = len(bonds), i64(bonds)
        d.n_bond_types, d.bond_k, d.bond_req = len(bond_k), f64(bond_k), f64(bond_req)
        d.n_angles, d.angles = len(angles), i64(angles)
        d.n_angle_types, d.angle_k, d.angle_teq = len(angle_k), f64(angle_k), f64(angle_teq)
        d.n_dihedrals, d.dihedrals = len(dihedrals), i64(dihedrals)
        d.n_dihedral_types, d.dih_pk, d.dih_pn, d.dih_phase = len(dih_pk), f64(dih_pk), f64(dih_pn), f64(dih_phase)
        d.num_excluded = i64(num_excluded if num_excluded is not None else np.zeros(n))
        d.n_excluded, d.excluded_list = len(excluded_list), i64(excluded_list)
        d.scee, d.scnb = scee, scnb
        d.n_lj, d.lj_a, d.lj_b = len(lj_a), f64(lj_a), f64(lj_b)
        d.nb_index = i64(nb_index)
        h = lib().orc_topology_from_desc(C.byref(d))
        return cls(h)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_topology_free(self.h)
            self.h = None

    @property
    def n_atoms(self) -> int:
        return int(lib().orc_topology_n_atoms(self.h))

    @property
    def n_residues(self) -> int:
        return int(lib().orc_topology_n_residues(self.h))

    def arrays(self) -> dict:
        n, r = self.n_atoms, self.n_residues
        out = {k: np.zeros(n) for k in ("charges", "charges_amber", "radii", "screen")}
        out["type_idx"] = np.zeros(n, np.int64)
        out["residue_pointers"] = np.zeros(r, np.int64)
        lib().orc_topology_arrays(self.h, _d(out["charges"]), _d(out["charges_amber"]), _d(out["radii"]),
                                  _d(out["screen"]), _i(out["type_idx"]), _i(out["residue_pointers"]))
        return out


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def threads() -> int:
    return int(lib().orc_get_threads())


def kappa(salt, eps, temperature) -> float:
    return lib().orc_kappa(salt, eps, temperature)


def gb_energy(top: Topology, xyz_A, params: GbP = None, accurate=False):
    x = np.ascontiguousarray(xyz_A, dtype=np.float64)
    R = np.zeros(top.n_atoms)
    e = lib().orc_gb_energy(top.h, _d(x), C.byref(params or gb_params()), int(accurate), _d(R))
    return e, R


def gb_energy_from_radii(top: Topology, xyz_A, params: GbP, radii) -> float:
    x = np.ascontiguousarray(xyz_A, dtype=np.float64)
    r = np.ascontiguousarray(radii, dtype=np.float64)
    return lib().orc_gb_energy_from_radii(top.h, _d(x), C.byref(params), _d(r))


def mm_energy(top: Topology, xyz_A, accurate=False) -> np.ndarray:
    """bond, angle, dihedral, vdw, elec, vdw_14, elec_14."""
    x = np.ascontiguousarray(xyz_A, dtype=np.float64)
    out = np.zeros(7)
    lib().orc_mm_energy(top.h, _d(x), int(accurate), _d(out))
    return out


def sa_energy(top: Topology, xyz_A, params: SaP = None):
    x = np.ascontiguousarray(xyz_A, dtype=np.float64)
    per = np.zeros(top.n_atoms)
    tot = C.c_double()
    e = lib().orc_sa_energy(top.h, _d(x), C.byref(params or sa_params()), C.byref(tot), _d(per))
    return e, tot.value, per


def sasa_raw(xyz, radii, probe=1.4, n_points=960) -> np.ndarray:
    x = np.ascontiguousarray(xyz, dtype=np.float64)
    r = np.ascontiguousarray(radii, dtype=np.float64)
    out = np.zeros(len(r))
    lib().orc_sasa_raw(len(r), _d(x), _d(r), probe, n_points, _d(out))
    return out


def fibonacci(n: int) -> np.ndarray:
    out = np.zeros((n, 3))
    lib().orc_fibonacci(n, _d(out))
    return out


def pb_energy(top: Topology, xyz_A, params: PbP = None):
    x = np.ascontiguousarray(xyz_A, dtype=np.float64)
    it = np.zeros(2, np.int64)
    res = np.zeros(2)
    conv = (C.c_int32 * 2)()
    dims = (C.c_int32 * 3)()
    e = lib().orc_pb_energy(top.h, _d(x), C.byref(params or pb_params()), _i(it), _d(res), conv, dims)
    return e, {"iterations": it.tolist(), "residual": res.tolist(), "converged": list(conv), "dims": list(dims)}


def pb_energy_raw(xyz, q_e, radii, params: PbP) -> float:
    x = np.ascontiguousarray(xyz, dtype=np.float64)
    q = np.ascontiguousarray(q_e, dtype=np.float64)
    r = np.ascontiguousarray(radii, dtype=np.float64)
    return lib().orc_pb_energy_raw(len(r), _d(x), _d(q), _d(r), C.byref(params))


def pb_maps(xyz, q_e, radii, h, buffer, probe, ion_radius, eps_in, eps_out, kappa_bulk, eps_solvent, use_ionic):
    """Grid set-up of one solve: dims, origin and every map (exact restatement)."""
    x = np.ascontiguousarray(xyz, dtype=np.float64)
    q = np.ascontiguousarray(q_e, dtype=np.float64)
    r = np.ascontiguousarray(radii, dtype=np.float64)
    dims = np.zeros(3, np.int64)
    org = np.zeros(3)
    L = lib()
    args = (len(r), _d(x), _d(q), _d(r), h, buffer, probe, ion_radius, eps_in, eps_out, kappa_bulk, eps_solvent,
            int(use_ionic), _i(dims), _d(org))
    n = L.orc_pb_maps(*args, None, None, None, None, None, None, None)
    m = {k: np.zeros(n) for k in ("charge", "ex", "ey", "ez", "k2", "boundary")}
    inside = np.zeros(n, np.uint8)
    L.orc_pb_maps(*args, _d(m["charge"]), inside.ctypes.data_as(C.POINTER(C.c_uint8)), _d(m["ex"]), _d(m["ey"]),
                  _d(m["ez"]), _d(m["k2"]), _d(m["boundary"]))
    m["inside"] = inside
    m["dims"] = dims
    m["origin"] = org
    return m


def pb_solve(xyz, q_e, dims, origin, h, maps, kappa_bc, eps_bc, tol, max_iter):
    x = np.ascontiguousarray(xyz, dtype=np.float64)
    q = np.ascontiguousarray(q_e, dtype=np.float64)
    dims = np.ascontiguousarray(dims, dtype=np.int64)
    org = np.ascontiguousarray(origin, dtype=np.float64)
    phi = np.zeros(int(np.prod(dims)))
    res = C.c_double()
    conv = C.c_int32()
    en = C.c_double()
    it = lib().orc_pb_solve(len(q), _d(x), _d(q), _i(dims), _d(org), h, _d(maps["charge"]), _d(maps["ex"]),
                            _d(maps["ey"]), _d(maps["ez"]), _d(maps["k2"]), kappa_bc, eps_bc, tol, max_iter,
                            _d(phi), C.byref(res), C.byref(conv), C.byref(en))
    return phi, {"iterations": int(it), "residual": res.value, "converged": bool(conv.value), "energy": en.value}


def restrict_prolong_constant(value=3.0):
    c = np.zeros(125)
    f = np.zeros(729)
    lib().orc_restrict_prolong_constant(value, _d(c), _d(f))
    return c, f


def charge_total(xyz, q_e, h, buffer) -> float:
    x = np.ascontiguousarray(xyz, dtype=np.float64)
    q = np.ascontiguousarray(q_e, dtype=np.float64)
    return lib().orc_charge_total(len(q), _d(x), _d(q), h, buffer)


FRAME_KEYS = ("complex_mm", "complex_polar", "complex_sa", "receptor_mm", "receptor_polar", "receptor_sa",
              "ligand_mm", "ligand_polar", "ligand_sa", "delta_mm", "delta_polar", "delta_sa", "delta_total")


def binding_frame(top: Topology, xyz_A, rec_res, lig_res, gb: GbP = None, pb: PbP = None, sa: SaP = None,
                  accurate=False) -> dict:
    x = np.ascontiguousarray(xyz_A, dtype=np.float64)
    rr = np.ascontiguousarray(rec_res, dtype=np.int64)
    lr = np.ascontiguousarray(lig_res, dtype=np.int64)
    out = np.zeros(13)
    err = C.create_string_buffer(512)
    rc = lib().orc_binding_frame(top.h, _d(x), _i(rr), len(rr), _i(lr), len(lr), 1 if pb is not None else 0,
                                 C.byref(gb or gb_params()), C.byref(pb or pb_params()), C.byref(sa or sa_params()),
                                 int(accurate), _d(out), err, 512)
    if rc:
        raise ValueError(err.value.decode())
    return dict(zip(FRAME_KEYS, out.tolist()))


def binding_frames(top: Topology, frames_A, rec_res, lig_res, gb: GbP = None, pb: PbP = None, sa: SaP = None,
                   accurate=False) -> np.ndarray:
    """(F, 13) array in FRAME_KEYS order; frames_A is (F, n_atoms, 3) in Angstrom."""
    x = np.ascontiguousarray(frames_A, dtype=np.float64)
    F = x.shape[0]
    rr = np.ascontiguousarray(rec_res, dtype=np.int64)
    lr = np.ascontiguousarray(lig_res, dtype=np.int64)
    out = np.zeros((F, 13))
    err = C.create_string_buffer(512)
    rc = lib().orc_binding_frames(top.h, _d(x), F, _i(rr), len(rr), _i(lr), len(lr), 1 if pb is not None else 0,
                                  C.byref(gb or gb_params()), C.byref(pb or pb_params()),
                                  C.byref(sa or sa_params()), int(accurate), _d(out), err, 512)
    if rc:
        raise ValueError(err.value.decode())
    return out


def decompose(top: Topology, xyz_A, rec_res, lig_res, gb: GbP = None, sa: SaP = None, accurate=False):
    """Per-residue (n, 4) arrays: vdw, elec, polar, sa for receptor and ligand residues."""
    x = np.ascontiguousarray(xyz_A, dtype=np.float64)
    rr = np.ascontiguousarray(rec_res, dtype=np.int64)
    lr = np.ascontiguousarray(lig_res, dtype=np.int64)
    ro = np.zeros((len(rr), 4))
    lo = np.zeros((len(lr), 4))
    err = C.create_string_buffer(512)
    rc = lib().orc_decompose(top.h, _d(x), _i(rr), len(rr), _i(lr), len(lr), C.byref(gb or gb_params()),
                             C.byref(sa or sa_params()), int(accurate), _d(ro), _d(lo), err, 512)
    if rc:
        raise ValueError(err.value.decode())
    return ro, lo


def read_dcd_nm(path: str) -> np.ndarray:
    err = C.create_string_buffer(512)
    na = C.c_int64()
    nf = lib().orc_read_dcd(path.encode(), None, 0, C.byref(na), err, 512)
    if nf < 0:
        raise IOError(err.value.decode())
    out = np.zeros((nf, na.value, 3))
    lib().orc_read_dcd(path.encode(), _d(out), out.size, C.byref(na), err, 512)
    return out


def reimage_complex(coords_A, bonds, box):
    """Restatement of reimage_complex (crates/mmpbsa/src/binding.rs:234-308)
    in plain Python floats, for small cases: unwrap every bonded component
    along a breadth-first walk (starts in atom order, neighbours in bond
    order; an atom found from `current` moves by one box edge where it sits
    more than half an edge from it), then move every component after the
    first by one box edge where its geometric centre (binding.rs:311-322, sum
    in visit order divided by the count) sits more than half an edge from the
    first one's.  coords_A: (n, 3); bonds: (a, b) pairs; box: 3 edges.
    Returns a new (n, 3) float64 array."""
    x = [[float(v) for v in row] for row in np.asarray(coords_A, dtype=np.float64)]
    box = [float(b) for b in box]
    n = len(x)
    if n == 0:
        return np.zeros((0, 3))
    adj = [[] for _ in range(n)]
    for a, b in bonds:
        if a < n and b < n:
            adj[a].append(b)
            adj[b].append(a)
    seen = [False] * n
    comps = []
    for s in range(n):
        if seen[s]:
            continue
        comp, queue, head = [], [s], 0
        seen[s] = True
        while head < len(queue):
            cur = queue[head]
            head += 1
            comp.append(cur)
            for nb in adj[cur]:
                if seen[nb]:
                    continue
                seen[nb] = True
                for d in range(3):
                    diff = x[nb][d] - x[cur][d]
                    if diff > box[d] * 0.5:
                        x[nb][d] -= box[d]
                    elif diff < -box[d] * 0.5:
                        x[nb][d] += box[d]
                queue.append(nb)
        comps.append(comp)

    def centre(c):
        m = [0.0, 0.0, 0.0]
        for a in c:
            for d in range(3):
                m[d] += x[a][d]
        return [v / float(len(c)) for v in m]

    if len(comps) > 1:
        ref = centre(comps[0])
        for c in comps[1:]:
            cc = centre(c)
            sh = [0.0, 0.0, 0.0]
            for d in range(3):
                diff = cc[d] - ref[d]
                if diff > box[d] * 0.5:
                    sh[d] = -box[d]
                elif diff < -box[d] * 0.5:
                    sh[d] = box[d]
            for a in c:
                for d in range(3):
                    x[a][d] += sh[d]
    return np.array(x, dtype=np.float64)
