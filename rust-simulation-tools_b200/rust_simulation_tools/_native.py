"""ctypes binding of librstg (include/rstg.h).

The library is the only compute path: if ``librstg.so`` cannot be loaded the
import fails, and if no CUDA device is present every compute call raises.
ctypes releases the GIL for the duration of each call.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("RSTG_LIB", os.path.join(_HERE, "librstg.so"))

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"librstg.so not found at {LIB_PATH}; build it with `make -C rust-simulation-tools_b200` "
        "(there is no CPU fallback)")

lib = C.CDLL(LIB_PATH)

OK, ERR_INVALID, ERR_IO, ERR_CUDA, ERR_NOMEM, ERR_TIMEOUT, ERR_CANCELLED, ERR_NOT_READY = range(8)

vp, dp, fp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int64)
i64, i32, dbl, cs = C.c_int64, C.c_int32, C.c_double, C.c_char_p


class GbParams(C.Structure):
    _fields_ = [("model", i32), ("solute_dielectric", dbl), ("solvent_dielectric", dbl),
                ("salt_concentration", dbl), ("temperature", dbl), ("offset", dbl), ("rgbmax", dbl),
                ("cutoff", dbl)]


class SaParams(C.Structure):
    _fields_ = [("surface_tension", dbl), ("offset", dbl), ("probe_radius", dbl), ("n_sphere_points", i64)]


class PbParams(C.Structure):
    _fields_ = [("grid_spacing", dbl), ("grid_buffer", dbl), ("solute_dielectric", dbl),
                ("solvent_dielectric", dbl), ("salt_concentration", dbl), ("temperature", dbl),
                ("probe_radius", dbl), ("ion_radius", dbl), ("tolerance", dbl), ("max_iterations", i64),
                ("fillratio", dbl), ("fscale", i64)]


class Solvation(C.Structure):
    _fields_ = [("method", i32), ("gb", GbParams), ("pb", PbParams)]


class MmEnergy(C.Structure):
    _fields_ = [(k, dbl) for k in ("bond", "angle", "dihedral", "vdw", "elec", "vdw_14", "elec_14")]


class SubsystemEnergy(C.Structure):
    _fields_ = [("mm", dbl), ("polar", dbl), ("sa", dbl)]


class FrameEnergy(C.Structure):
    _fields_ = [("complex", SubsystemEnergy), ("receptor", SubsystemEnergy), ("ligand", SubsystemEnergy),
                ("delta_mm", dbl), ("delta_polar", dbl), ("delta_sa", dbl), ("delta_total", dbl)]


class ResidueEnergy(C.Structure):
    _fields_ = [("vdw", dbl), ("elec", dbl), ("polar", dbl), ("sa", dbl)]


class PbDiag(C.Structure):
    _fields_ = [("iterations", i64 * 2), ("residual", dbl * 2), ("converged", i32 * 2), ("dims", i32 * 3)]


class TopologyDesc(C.Structure):
    _fields_ = [("n_atoms", i64), ("n_residues", i64), ("n_types", i64), ("atom_type_indices", vp),
                ("charges_amber", vp), ("radii", vp), ("screen", vp), ("residue_pointers", vp),
                ("n_bonds", i64), ("bonds", vp), ("n_bond_types", i64), ("bond_k", vp), ("bond_req", vp),
                ("n_angles", i64), ("angles", vp), ("n_angle_types", i64), ("angle_k", vp), ("angle_teq", vp),
                ("n_dihedrals", i64), ("dihedrals", vp), ("n_dihedral_types", i64), ("dihedral_pk", vp),
                ("dihedral_pn", vp), ("dihedral_phase", vp), ("num_excluded", vp), ("n_excluded", i64),
                ("excluded_list", vp), ("scee", dbl), ("scnb", dbl), ("n_lj", i64), ("lj_acoef", vp),
                ("lj_bcoef", vp), ("nb_parm_index", vp)]


class TopologyInfo(C.Structure):
    _fields_ = [("n_atoms", i64), ("n_residues", i64), ("n_types", i64), ("n_bonds", i64), ("n_angles", i64),
                ("n_dihedrals", i64), ("scee", dbl), ("scnb", dbl)]


class SystemOpts(C.Structure):
    _fields_ = [("mode", i32), ("decompose", i32), ("max_batch_frames", i64), ("use_graphs", i32),
                ("autotune", i32)]


class ServerOpts(C.Structure):
    _fields_ = [("memory_budget_bytes", i64), ("max_inflight", i32), ("chunk_frames", i64)]


def _sig(name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


P = C.POINTER
_sig("rstg_last_error", cs)
_sig("rstg_device_count", C.c_int)
_sig("rstg_version", cs)
_sig("rstg_ctx_create", C.c_int, C.c_int, vp, P(vp))
_sig("rstg_ctx_destroy", None, vp)
_sig("rstg_ctx_kernel_launches", i64, vp)
_sig("rstg_gb_params_default", None, P(GbParams))
_sig("rstg_sa_params_default", None, P(SaParams))
_sig("rstg_pb_params_default", None, P(PbParams))
_sig("rstg_topology_load_prmtop", C.c_int, cs, P(vp))
_sig("rstg_topology_from_desc", C.c_int, P(TopologyDesc), P(vp))
_sig("rstg_topology_extract", C.c_int, vp, ip, i64, P(vp))
_sig("rstg_topology_free", None, vp)
_sig("rstg_topology_info_get", C.c_int, vp, P(TopologyInfo))
_sig("rstg_topology_atoms", C.c_int, vp, dp, dp, dp, dp, dp, ip, ip)
_sig("rstg_topology_residue_pointers", C.c_int, vp, ip)
_sig("rstg_topology_names", C.c_int, vp, C.c_char_p, C.c_char_p)
_sig("rstg_topology_select", C.c_int, vp, ip, i64, ip, ip)
_sig("rstg_dcd_read", C.c_int, cs, dp, i64, ip, ip)
_sig("rstg_dcd_read_f32", C.c_int, cs, fp, i64, ip, ip)
_sig("rstg_mdcrd_read", C.c_int, cs, i64, i32, dp, i64, ip)
_sig("rstg_mm_energy_compute", C.c_int, vp, vp, dp, i64, P(MmEnergy))
_sig("rstg_gb_energy_compute", C.c_int, vp, vp, dp, i64, P(GbParams), dp, dp)
_sig("rstg_gb_cache_create", C.c_int, dbl, P(vp))
_sig("rstg_gb_cache_destroy", None, vp)
_sig("rstg_gb_energy_cached", C.c_int, vp, vp, dp, i64, P(GbParams), vp, dp, dp, P(i32))
_sig("rstg_sa_energy_compute", C.c_int, vp, vp, dp, i64, P(SaParams), dp, dp, dp)
_sig("rstg_pb_energy_compute", C.c_int, vp, vp, dp, i64, P(PbParams), ip, i64, dp, P(PbDiag))
_sig("rstg_pb_grid_maps", C.c_int, vp, dp, i64, dp, dp, P(PbParams), dbl, dbl, i32, ip, dp, dp, P(C.c_uint8), dp, dp,
     dp, dp, dp)
_sig("rstg_binding_frame", C.c_int, vp, vp, dp, i64, ip, i64, ip, i64, P(Solvation), P(SaParams), P(FrameEnergy))
_sig("rstg_decompose", C.c_int, vp, vp, dp, i64, ip, i64, ip, i64, P(GbParams), P(SaParams), P(ResidueEnergy),
     P(ResidueEnergy))
_sig("rstg_gb_energy_noalloc_async", C.c_int, vp, vp, vp, vp, i64, P(GbParams), vp, vp, vp)
_sig("rstg_qh_covariance", C.c_int, vp, dp, i64, i64, dp, dp)
_sig("rstg_system_opts_default", None, P(SystemOpts))
_sig("rstg_system_create", C.c_int, vp, vp, ip, i64, ip, i64, P(Solvation), P(SaParams), P(SystemOpts), P(vp))
_sig("rstg_system_destroy", None, vp)
_sig("rstg_system_shape", C.c_int, vp, ip)
_sig("rstg_system_footprint", i64, vp, i64)
_sig("rstg_system_run", C.c_int, vp, fp, i64, P(FrameEnergy), P(ResidueEnergy))
_sig("rstg_system_run_device", C.c_int, vp, vp, i64, vp, vp)
_sig("rstg_system_last_stats", C.c_int, vp, ip)
_sig("rstg_system_pb_stats", C.c_int, vp, dp)
_sig("rstg_system_tuning", C.c_int, vp, P(i32), dp)
_sig("rstg_system_set_pb_batch", C.c_int, vp, i64)
_sig("rstg_system_set_pb_profile", C.c_int, vp, i32)
_sig("rstg_system_set_pb_convergence", C.c_int, vp, dbl)
_sig("rstg_system_pb_profile", C.c_int, vp, dp)
_sig("rstg_system_profile", C.c_int, vp, vp, i64, P(i32), C.c_char_p, dp, dp, dp)
_sig("rstg_calibrate", C.c_int, C.c_int, dp)
_sig("rstg_system_reimage", C.c_int, vp, dp, dp, i64, i32, dp)
_sig("rstg_binding_trajectory", C.c_int, vp, vp, cs, cs, i32, ip, i64, ip, i64, P(Solvation), P(SaParams), i64,
     i64, i64, i32, P(FrameEnergy), i64, ip, dp, dp)
_sig("rstg_server_opts_default", None, P(ServerOpts))
_sig("rstg_server_create", C.c_int, vp, P(ServerOpts), P(vp))
_sig("rstg_server_destroy", None, vp)
_sig("rstg_server_submit", C.c_int, vp, vp, fp, i64, ip)
_sig("rstg_server_poll", C.c_int, vp, i64, P(FrameEnergy))
_sig("rstg_server_wait", C.c_int, vp, i64, i64, P(FrameEnergy))
_sig("rstg_server_cancel", C.c_int, vp, i64)
_sig("rstg_server_stats", C.c_int, vp, dp)


class CudaError(RuntimeError):
    pass


class RequestCancelled(RuntimeError):
    """A serving request was cancelled before its results were delivered."""


def check(rc: int) -> None:
    """Raise the Python exception the reference raises for this failure."""
    if rc == OK:
        return
    msg = lib.rstg_last_error().decode(errors="replace")
    if rc == ERR_IO:
        raise IOError(msg)
    if rc in (ERR_CUDA,):
        raise CudaError(msg)
    if rc == ERR_NOMEM:
        raise MemoryError(msg)
    if rc == ERR_TIMEOUT:
        raise TimeoutError(msg)
    if rc == ERR_CANCELLED:
        raise RequestCancelled(msg)
    raise ValueError(msg)


_ctx = None


def ctx():
    """The process-wide context on CUDA device 0 (created on first use)."""
    global _ctx
    if _ctx is None:
        h = vp()
        check(lib.rstg_ctx_create(int(os.environ.get("RSTG_DEVICE", "0")), None, C.byref(h)))
        _ctx = h
    return _ctx


def make_ctx(device: int = 0, stream_ptr: int | None = None):
    h = vp()
    check(lib.rstg_ctx_create(device, vp(stream_ptr) if stream_ptr else None, C.byref(h)))
    return h
