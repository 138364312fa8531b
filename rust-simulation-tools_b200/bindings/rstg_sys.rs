//! Raw Rust declarations of librstg's C ABI (include/rstg.h), for the
//! reference crate `crates/mmpbsa` to call the GPU engine in place of its
//! CPU functions.  Every struct is `#[repr(C)]` with the header's field order;
//! every function is the header's, with the same argument meaning.  A safe
//! layer (topology and context ownership, `Result<_, String>` from
//! `rstg_last_error`) is sketched at the end.  Link with `-lrstg` (the
//! library built by `make -C rust-simulation-tools_b200`) and the CUDA
//! runtime it was built against (static in librstg.so).
#![allow(non_camel_case_types, dead_code)]

use std::ffi::{c_char, c_int, c_void, CStr};

pub type rstg_status = c_int;
pub const RSTG_OK: rstg_status = 0;
pub const RSTG_ERR_INVALID: rstg_status = 1;
pub const RSTG_ERR_IO: rstg_status = 2;
pub const RSTG_ERR_CUDA: rstg_status = 3;
pub const RSTG_ERR_NOMEM: rstg_status = 4;
pub const RSTG_ERR_TIMEOUT: rstg_status = 5;
pub const RSTG_ERR_CANCELLED: rstg_status = 6;
pub const RSTG_ERR_NOT_READY: rstg_status = 7;

#[repr(C)]
pub struct rstg_ctx {
    _private: [u8; 0],
}
#[repr(C)]
pub struct rstg_topology {
    _private: [u8; 0],
}
#[repr(C)]
pub struct rstg_system {
    _private: [u8; 0],
}
#[repr(C)]
pub struct rstg_server {
    _private: [u8; 0],
}
#[repr(C)]
pub struct rstg_gb_cache {
    _private: [u8; 0],
}

pub const RSTG_GB_HCT: i32 = 0;
pub const RSTG_GB_OBC1: i32 = 1;
pub const RSTG_GB_OBC2: i32 = 2;

/// GbParams (gb_energy.rs:24-56)
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rstg_gb_params {
    pub model: i32,
    pub solute_dielectric: f64,
    pub solvent_dielectric: f64,
    pub salt_concentration: f64,
    pub temperature: f64,
    pub offset: f64,
    pub rgbmax: f64,
    pub cutoff: f64,
}

/// SaParams (sa_energy.rs:12-32)
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rstg_sa_params {
    pub surface_tension: f64,
    pub offset: f64,
    pub probe_radius: f64,
    pub n_sphere_points: i64,
}

/// PbParams (pb_energy.rs:21-66)
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rstg_pb_params {
    pub grid_spacing: f64,
    pub grid_buffer: f64,
    pub solute_dielectric: f64,
    pub solvent_dielectric: f64,
    pub salt_concentration: f64,
    pub temperature: f64,
    pub probe_radius: f64,
    pub ion_radius: f64,
    pub tolerance: f64,
    pub max_iterations: i64,
    pub fillratio: f64,
    pub fscale: i64,
}

/// SolvationMethod (binding.rs:23-30): method 0 GB, 1 PB
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rstg_solvation {
    pub method: i32,
    pub gb: rstg_gb_params,
    pub pb: rstg_pb_params,
}

/// MmEnergy (mm_energy.rs:43-58)
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rstg_mm_energy {
    pub bond: f64,
    pub angle: f64,
    pub dihedral: f64,
    pub vdw: f64,
    pub elec: f64,
    pub vdw_14: f64,
    pub elec_14: f64,
}

/// SubsystemEnergy (binding.rs:33-46)
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rstg_subsystem_energy {
    pub mm: f64,
    pub polar: f64,
    pub sa: f64,
}

/// FrameEnergy (binding.rs:48-56)
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rstg_frame_energy {
    pub complex: rstg_subsystem_energy,
    pub receptor: rstg_subsystem_energy,
    pub ligand: rstg_subsystem_energy,
    pub delta_mm: f64,
    pub delta_polar: f64,
    pub delta_sa: f64,
    pub delta_total: f64,
}

/// ResidueContribution numbers (decomposition.rs:30-43)
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rstg_residue_energy {
    pub vdw: f64,
    pub elec: f64,
    pub polar: f64,
    pub sa: f64,
}

/// PbSolveResult diagnostics of the solvated and reference solves (pb_solver.rs:143-152)
#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rstg_pb_diag {
    pub iterations: [i64; 2],
    pub residual: [f64; 2],
    pub converged: [i32; 2],
    pub dims: [i32; 3],
}

/// Flat AmberTopology (core/src/amber/prmtop.rs:34-105); arrays are copied by
/// rstg_topology_from_desc.  bonds [n][3] i, j, type; angles [n][4] i, j, k,
/// type; dihedrals [n][6] i, j, k, l, type, ignore_14; excluded_list uses -1
/// for AMBER's 0 placeholder; nb_parm_index holds 1-based entries.
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct rstg_topology_desc {
    pub n_atoms: i64,
    pub n_residues: i64,
    pub n_types: i64,
    pub atom_type_indices: *const i64,
    pub charges_amber: *const f64,
    pub radii: *const f64,
    pub screen: *const f64,
    pub residue_pointers: *const i64,
    pub n_bonds: i64,
    pub bonds: *const i64,
    pub n_bond_types: i64,
    pub bond_k: *const f64,
    pub bond_req: *const f64,
    pub n_angles: i64,
    pub angles: *const i64,
    pub n_angle_types: i64,
    pub angle_k: *const f64,
    pub angle_teq: *const f64,
    pub n_dihedrals: i64,
    pub dihedrals: *const i64,
    pub n_dihedral_types: i64,
    pub dihedral_pk: *const f64,
    pub dihedral_pn: *const f64,
    pub dihedral_phase: *const f64,
    pub num_excluded: *const i64,
    pub n_excluded: i64,
    pub excluded_list: *const i64,
    pub scee: f64,
    pub scnb: f64,
    pub n_lj: i64,
    pub lj_acoef: *const f64,
    pub lj_bcoef: *const f64,
    pub nb_parm_index: *const i64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rstg_topology_info {
    pub n_atoms: i64,
    pub n_residues: i64,
    pub n_types: i64,
    pub n_bonds: i64,
    pub n_angles: i64,
    pub n_dihedrals: i64,
    pub scee: f64,
    pub scnb: f64,
}

pub const RSTG_MODE_PLAIN: i32 = 0;
pub const RSTG_MODE_FUSED: i32 = 1;

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rstg_system_opts {
    pub mode: i32,
    pub decompose: i32,
    pub max_batch_frames: i64,
    pub use_graphs: i32,
    pub autotune: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct rstg_server_opts {
    pub memory_budget_bytes: i64,
    pub max_inflight: i32,
    pub chunk_frames: i64,
}

#[link(name = "rstg")]
extern "C" {
    pub fn rstg_last_error() -> *const c_char;
    pub fn rstg_device_count() -> c_int;
    pub fn rstg_version() -> *const c_char;
    pub fn rstg_ctx_create(device: c_int, stream: *mut c_void, out: *mut *mut rstg_ctx) -> rstg_status;
    pub fn rstg_ctx_destroy(ctx: *mut rstg_ctx);
    pub fn rstg_ctx_kernel_launches(ctx: *const rstg_ctx) -> i64;

    pub fn rstg_gb_params_default(p: *mut rstg_gb_params);
    pub fn rstg_sa_params_default(p: *mut rstg_sa_params);
    pub fn rstg_pb_params_default(p: *mut rstg_pb_params);

    pub fn rstg_topology_load_prmtop(path: *const c_char, out: *mut *mut rstg_topology) -> rstg_status;
    pub fn rstg_topology_from_desc(desc: *const rstg_topology_desc, out: *mut *mut rstg_topology) -> rstg_status;
    pub fn rstg_topology_extract(t: *const rstg_topology, atom_indices: *const i64, n: i64,
                                 out: *mut *mut rstg_topology) -> rstg_status;
    pub fn rstg_topology_free(t: *mut rstg_topology);
    pub fn rstg_topology_info_get(t: *const rstg_topology, out: *mut rstg_topology_info) -> rstg_status;
    pub fn rstg_topology_atoms(t: *const rstg_topology, charges_e: *mut f64, charges_amber: *mut f64,
                               radii: *mut f64, screen: *mut f64, masses: *mut f64, type_idx: *mut i64,
                               residue_index: *mut i64) -> rstg_status;
    pub fn rstg_topology_residue_pointers(t: *const rstg_topology, out: *mut i64) -> rstg_status;
    pub fn rstg_topology_names(t: *const rstg_topology, atom_names4: *mut c_char,
                               residue_labels4: *mut c_char) -> rstg_status;
    pub fn rstg_topology_select(t: *const rstg_topology, residues: *const i64, n_res: i64, atoms_out: *mut i64,
                                n_atoms_out: *mut i64) -> rstg_status;

    pub fn rstg_dcd_read(path: *const c_char, out_nm: *mut f64, capacity_values: i64, n_frames: *mut i64,
                         n_atoms: *mut i64) -> rstg_status;
    pub fn rstg_dcd_read_f32(path: *const c_char, out_a: *mut f32, capacity_values: i64, n_frames: *mut i64,
                             n_atoms: *mut i64) -> rstg_status;
    pub fn rstg_mdcrd_read(path: *const c_char, n_atoms: i64, has_box: i32, out_a: *mut f64,
                           capacity_values: i64, n_frames: *mut i64) -> rstg_status;

    pub fn rstg_mm_energy_compute(ctx: *mut rstg_ctx, t: *const rstg_topology, xyz: *const f64, n: i64,
                                  out: *mut rstg_mm_energy) -> rstg_status;
    pub fn rstg_gb_energy_compute(ctx: *mut rstg_ctx, t: *const rstg_topology, xyz: *const f64, n: i64,
                                  p: *const rstg_gb_params, total: *mut f64, born_radii: *mut f64) -> rstg_status;
    pub fn rstg_gb_cache_create(rmsd_threshold: f64, out: *mut *mut rstg_gb_cache) -> rstg_status;
    pub fn rstg_gb_cache_destroy(c: *mut rstg_gb_cache);
    pub fn rstg_gb_energy_cached(ctx: *mut rstg_ctx, t: *const rstg_topology, xyz: *const f64, n: i64,
                                 p: *const rstg_gb_params, cache: *mut rstg_gb_cache, total: *mut f64,
                                 born_radii: *mut f64, reused: *mut i32) -> rstg_status;
    pub fn rstg_sa_energy_compute(ctx: *mut rstg_ctx, t: *const rstg_topology, xyz: *const f64, n: i64,
                                  p: *const rstg_sa_params, total: *mut f64, total_sasa: *mut f64,
                                  per_atom: *mut f64) -> rstg_status;
    pub fn rstg_pb_energy_compute(ctx: *mut rstg_ctx, t: *const rstg_topology, xyz: *const f64, n: i64,
                                  p: *const rstg_pb_params, solute_residues: *const i64, n_solute: i64,
                                  total: *mut f64, diag: *mut rstg_pb_diag) -> rstg_status;
    pub fn rstg_pb_grid_maps(ctx: *mut rstg_ctx, xyz: *const f64, n: i64, charges_e: *const f64,
                             radii: *const f64, p: *const rstg_pb_params, eps_in: f64, eps_out: f64,
                             use_ionic: i32, dims3: *mut i64, origin3: *mut f64, charge: *mut f64,
                             inside: *mut u8, eps_x: *mut f64, eps_y: *mut f64, eps_z: *mut f64,
                             kappa_sq: *mut f64, boundary_phi: *mut f64) -> rstg_status;
    pub fn rstg_binding_frame(ctx: *mut rstg_ctx, t: *const rstg_topology, xyz: *const f64, n: i64,
                              receptor_residues: *const i64, n_rec: i64, ligand_residues: *const i64, n_lig: i64,
                              solv: *const rstg_solvation, sa: *const rstg_sa_params,
                              out: *mut rstg_frame_energy) -> rstg_status;
    pub fn rstg_decompose(ctx: *mut rstg_ctx, t: *const rstg_topology, xyz: *const f64, n: i64,
                          receptor_residues: *const i64, n_rec: i64, ligand_residues: *const i64, n_lig: i64,
                          gb: *const rstg_gb_params, sa: *const rstg_sa_params, rec_out: *mut rstg_residue_energy,
                          lig_out: *mut rstg_residue_energy) -> rstg_status;
    pub fn rstg_qh_covariance(ctx: *mut rstg_ctx, traj_a: *const f64, n_frames: i64, n_atoms: i64,
                              masses: *const f64, cov: *mut f64) -> rstg_status;
    pub fn rstg_gb_energy_noalloc_async(d_xyz: *const f64, d_charges_amber: *const f64, d_radii: *const f64,
                                        d_screen: *const f64, n_atoms: i64, params: *const rstg_gb_params,
                                        d_total: *mut f64, d_born_radii: *mut f64,
                                        stream: *mut c_void) -> rstg_status;

    pub fn rstg_system_opts_default(o: *mut rstg_system_opts);
    pub fn rstg_system_create(ctx: *mut rstg_ctx, t: *const rstg_topology, receptor_residues: *const i64,
                              n_rec: i64, ligand_residues: *const i64, n_lig: i64, solv: *const rstg_solvation,
                              sa: *const rstg_sa_params, opts: *const rstg_system_opts,
                              out: *mut *mut rstg_system) -> rstg_status;
    pub fn rstg_system_destroy(s: *mut rstg_system);
    pub fn rstg_system_shape(s: *const rstg_system, shape6: *mut i64) -> rstg_status;
    pub fn rstg_system_footprint(s: *const rstg_system, n_frames: i64) -> i64;
    pub fn rstg_system_run(s: *mut rstg_system, frames: *const f32, n_frames: i64, out: *mut rstg_frame_energy,
                           decomp: *mut rstg_residue_energy) -> rstg_status;
    pub fn rstg_system_run_device(s: *mut rstg_system, d_frames: *const f32, n_frames: i64,
                                  d_out: *mut rstg_frame_energy, d_decomp: *mut rstg_residue_energy) -> rstg_status;
    pub fn rstg_system_last_stats(s: *const rstg_system, stats4: *mut i64) -> rstg_status;
    pub fn rstg_system_tuning(s: *const rstg_system, shape12: *mut i32, ms12: *mut f64) -> rstg_status;
    pub fn rstg_system_pb_stats(s: *const rstg_system, stats8: *mut f64) -> rstg_status;
    pub fn rstg_system_set_pb_batch(s: *mut rstg_system, frames: i64) -> rstg_status;
    pub fn rstg_system_set_pb_convergence(s: *mut rstg_system, rel_tol: f64) -> rstg_status;
    pub fn rstg_system_set_pb_profile(s: *mut rstg_system, on: i32) -> rstg_status;
    pub fn rstg_system_pb_profile(s: *const rstg_system, out12: *mut f64) -> rstg_status;
    pub fn rstg_system_profile(s: *mut rstg_system, d_frames: *const f32, n_frames: i64, n: *mut i32,
                               names: *mut c_char, ms: *mut f64, flops: *mut f64, bytes: *mut f64) -> rstg_status;
    pub fn rstg_calibrate(device: c_int, out4: *mut f64) -> rstg_status;
    pub fn rstg_system_reimage(s: *mut rstg_system, frames: *const f64, boxes: *const f64, n_frames: i64,
                               on_device: i32, out: *mut f64) -> rstg_status;
    pub fn rstg_binding_trajectory(ctx: *mut rstg_ctx, t: *const rstg_topology, path: *const c_char,
                                   format: *const c_char, has_box: i32, receptor_residues: *const i64, n_rec: i64,
                                   ligand_residues: *const i64, n_lig: i64, solv: *const rstg_solvation,
                                   sa: *const rstg_sa_params, stride: i64, start_frame: i64, end_frame: i64,
                                   mode: i32, frames_out: *mut rstg_frame_energy, frames_capacity: i64,
                                   n_frames: *mut i64, stats9: *mut f64, last_frame_coords: *mut f64) -> rstg_status;

    pub fn rstg_server_opts_default(o: *mut rstg_server_opts);
    pub fn rstg_server_create(ctx: *mut rstg_ctx, opts: *const rstg_server_opts,
                              out: *mut *mut rstg_server) -> rstg_status;
    pub fn rstg_server_destroy(s: *mut rstg_server);
    pub fn rstg_server_submit(s: *mut rstg_server, sys: *mut rstg_system, frames: *const f32, n_frames: i64,
                              request_id: *mut i64) -> rstg_status;
    pub fn rstg_server_poll(s: *mut rstg_server, request_id: i64, out: *mut rstg_frame_energy) -> rstg_status;
    pub fn rstg_server_wait(s: *mut rstg_server, request_id: i64, timeout_ms: i64,
                            out: *mut rstg_frame_energy) -> rstg_status;
    pub fn rstg_server_cancel(s: *mut rstg_server, request_id: i64) -> rstg_status;
    pub fn rstg_server_stats(s: *const rstg_server, stats8: *mut f64) -> rstg_status;
}

/// The reference's error convention: a status other than RSTG_OK becomes the
/// `Err(String)` the crate's functions return (binding.rs, pb_energy.rs).
pub fn check(rc: rstg_status) -> Result<(), String> {
    if rc == RSTG_OK {
        return Ok(());
    }
    // SAFETY: rstg_last_error returns a NUL-terminated thread-local string.
    let msg = unsafe { CStr::from_ptr(rstg_last_error()) };
    Err(msg.to_string_lossy().into_owned())
}

/// Owning handle of a context (one per GPU and thread pool).
pub struct Context(*mut rstg_ctx);

impl Context {
    pub fn new(device: i32) -> Result<Self, String> {
        let mut h = std::ptr::null_mut();
        check(unsafe { rstg_ctx_create(device, std::ptr::null_mut(), &mut h) })?;
        Ok(Context(h))
    }
    pub fn as_ptr(&self) -> *mut rstg_ctx {
        self.0
    }
}

impl Drop for Context {
    fn drop(&mut self) {
        unsafe { rstg_ctx_destroy(self.0) };
    }
}

/// compute_gb_energy (gb_energy.rs:357-365) on the GPU: total and Born radii.
/// `topo` comes from rstg_topology_load_prmtop / rstg_topology_from_desc,
/// `coords` are Angstrom.
pub fn gb_energy(ctx: &Context, topo: *const rstg_topology, coords: &[[f64; 3]],
                 params: &rstg_gb_params) -> Result<(f64, Vec<f64>), String> {
    let mut total = 0.0;
    let mut radii = vec![0.0; coords.len()];
    check(unsafe {
        rstg_gb_energy_compute(ctx.as_ptr(), topo, coords.as_ptr() as *const f64, coords.len() as i64, params,
                               &mut total, radii.as_mut_ptr())
    })?;
    Ok((total, radii))
}
