/*
 * rstg.h - C ABI of librstg, a B200 (sm_100a) implementation of the per-frame
 * MM-GBSA / MM-PBSA energy evaluation of crates/mmpbsa in
 * msinclair-py/rust-simulation-tools.
 *
 * Conventions (identical to the reference crate):
 *   - coordinates are Angstrom, row-major [n_atoms][3] float64, in the atom
 *     order of the topology passed with them;
 *   - energies are kcal/mol; GB charges are AMBER units (q * 18.2223), PB
 *     charges are elementary charges;
 *   - residue indices are 0-based.
 * Every call is synchronous unless its name says otherwise.  Buffers passed in
 * are caller-owned host memory unless a parameter name starts with d_ (device
 * memory on the context's device).  Errors return a non-zero rstg_status and
 * leave a message readable with rstg_last_error() on the calling thread; the
 * message is the reference's Result<_, String> text where one exists.
 * A context is internally locked: calls on one context from several threads
 * are serialised.
 */
#ifndef RSTG_H
#define RSTG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rstg_status {
  RSTG_OK = 0,
  RSTG_ERR_INVALID = 1,   /* bad argument (maps to PyValueError)            */
  RSTG_ERR_IO = 2,        /* unreadable / malformed file (PyIOError)        */
  RSTG_ERR_CUDA = 3,      /* CUDA runtime failure                          */
  RSTG_ERR_NOMEM = 4,     /* request exceeds the device-memory budget       */
  RSTG_ERR_TIMEOUT = 5,   /* a bounded device wait expired                  */
  RSTG_ERR_CANCELLED = 6, /* a serving request was cancelled               */
  RSTG_ERR_NOT_READY = 7  /* a serving request has not finished yet        */
} rstg_status;

typedef struct rstg_ctx rstg_ctx;
typedef struct rstg_topology rstg_topology;
typedef struct rstg_system rstg_system;
typedef struct rstg_server rstg_server;

/* ---- parameters: same fields and defaults as the reference structs ------ */

typedef enum rstg_gb_model { RSTG_GB_HCT = 0, RSTG_GB_OBC1 = 1, RSTG_GB_OBC2 = 2 } rstg_gb_model;

/* GbParams, crates/mmpbsa/src/gb_energy.rs:24-56 */
typedef struct rstg_gb_params {
  int32_t model; /* rstg_gb_model; default OBC1 */
  double solute_dielectric, solvent_dielectric, salt_concentration, temperature;
  double offset, rgbmax, cutoff;
} rstg_gb_params;

/* SaParams, crates/mmpbsa/src/sa_energy.rs:12-32 */
typedef struct rstg_sa_params {
  double surface_tension, offset, probe_radius;
  int64_t n_sphere_points;
} rstg_sa_params;

/* PbParams, crates/mmpbsa/src/pb_energy.rs:21-66 */
typedef struct rstg_pb_params {
  double grid_spacing, grid_buffer, solute_dielectric, solvent_dielectric;
  double salt_concentration, temperature, probe_radius, ion_radius, tolerance;
  int64_t max_iterations;
  double fillratio;
  int64_t fscale;
} rstg_pb_params;

/* SolvationMethod, crates/mmpbsa/src/binding.rs:23-30 (method: 0 GB, 1 PB) */
typedef struct rstg_solvation {
  int32_t method;
  rstg_gb_params gb;
  rstg_pb_params pb;
} rstg_solvation;

void rstg_gb_params_default(rstg_gb_params* p);
void rstg_sa_params_default(rstg_sa_params* p);
void rstg_pb_params_default(rstg_pb_params* p);

/* ---- results ------------------------------------------------------------ */

/* MmEnergy, crates/mmpbsa/src/mm_energy.rs:43-58 */
typedef struct rstg_mm_energy {
  double bond, angle, dihedral, vdw, elec, vdw_14, elec_14;
} rstg_mm_energy;

/* SubsystemEnergy / FrameEnergy, crates/mmpbsa/src/binding.rs:33-56 */
typedef struct rstg_subsystem_energy {
  double mm, polar, sa;
} rstg_subsystem_energy;
typedef struct rstg_frame_energy {
  rstg_subsystem_energy complex, receptor, ligand;
  double delta_mm, delta_polar, delta_sa, delta_total;
} rstg_frame_energy;

/* ResidueContribution numbers, crates/mmpbsa/src/decomposition.rs:30-43 */
typedef struct rstg_residue_energy {
  double vdw, elec, polar, sa;
} rstg_residue_energy;

/* PbSolveResult diagnostics of the two solves (solvated, reference),
 * crates/mmpbsa/src/pb_solver.rs:143-152 */
typedef struct rstg_pb_diag {
  int64_t iterations[2];
  double residual[2];
  int32_t converged[2];
  int32_t dims[3];
} rstg_pb_diag;

/* ---- errors, devices, contexts ----------------------------------------- */

const char* rstg_last_error(void);
int rstg_device_count(void);
const char* rstg_version(void);

/* stream may be NULL (the context creates its own) or a cudaStream_t owned by
 * the caller; every kernel of the context is launched on it. */
rstg_status rstg_ctx_create(int device, void* stream, rstg_ctx** out);
void rstg_ctx_destroy(rstg_ctx* ctx);
/* Kernels launched by this context since creation (all of them are this
 * library's own kernels). */
int64_t rstg_ctx_kernel_launches(const rstg_ctx* ctx);

/* ---- topology (host side) ---------------------------------------------- */

/* Flat AmberTopology, core/src/amber/prmtop.rs:34-105.  Arrays are copied. */
typedef struct rstg_topology_desc {
  int64_t n_atoms, n_residues, n_types;
  const int64_t* atom_type_indices; /* [n_atoms] 0-based            */
  const double* charges_amber;      /* [n_atoms] q * 18.2223        */
  const double* radii;              /* [n_atoms] intrinsic Born radii */
  const double* screen;             /* [n_atoms] GB screening        */
  const int64_t* residue_pointers;  /* [n_residues] first atom       */
  int64_t n_bonds;
  const int64_t* bonds; /* [n_bonds][3] i, j, type            */
  int64_t n_bond_types;
  const double* bond_k;
  const double* bond_req;
  int64_t n_angles;
  const int64_t* angles; /* [n_angles][4] i, j, k, type       */
  int64_t n_angle_types;
  const double* angle_k;
  const double* angle_teq;
  int64_t n_dihedrals;
  const int64_t* dihedrals; /* [n][6] i, j, k, l, type, ignore_14 */
  int64_t n_dihedral_types;
  const double* dihedral_pk;
  const double* dihedral_pn;
  const double* dihedral_phase;
  const int64_t* num_excluded; /* [n_atoms]                          */
  int64_t n_excluded;
  const int64_t* excluded_list; /* -1 marks AMBER's 0 placeholder      */
  double scee, scnb;
  int64_t n_lj;
  const double* lj_acoef;
  const double* lj_bcoef;
  const int64_t* nb_parm_index; /* [n_types * n_types], 1-based entries */
} rstg_topology_desc;

typedef struct rstg_topology_info {
  int64_t n_atoms, n_residues, n_types, n_bonds, n_angles, n_dihedrals;
  double scee, scnb;
} rstg_topology_info;

/* parse_prmtop, core/src/amber/prmtop.rs:444-733 */
rstg_status rstg_topology_load_prmtop(const char* path, rstg_topology** out);
rstg_status rstg_topology_from_desc(const rstg_topology_desc* desc, rstg_topology** out);
/* extract_subtopology, crates/mmpbsa/src/subsystem.rs:22-169 */
rstg_status rstg_topology_extract(const rstg_topology* t, const int64_t* atom_indices, int64_t n,
                                  rstg_topology** out);
void rstg_topology_free(rstg_topology* t);
rstg_status rstg_topology_info_get(const rstg_topology* t, rstg_topology_info* out);
/* Copies per-atom arrays out; any pointer may be NULL. */
rstg_status rstg_topology_atoms(const rstg_topology* t, double* charges_e, double* charges_amber, double* radii,
                                double* screen, double* masses, int64_t* type_idx, int64_t* residue_index);
rstg_status rstg_topology_residue_pointers(const rstg_topology* t, int64_t* out);
/* Fixed-width names: atom names and residue labels as 4-char, NUL-padded. */
rstg_status rstg_topology_names(const rstg_topology* t, char* atom_names4, char* residue_labels4);
/* AmberTopology::build_selection, prmtop.rs:165-204: atoms of the given residues. */
rstg_status rstg_topology_select(const rstg_topology* t, const int64_t* residues, int64_t n_res, int64_t* atoms_out,
                                 int64_t* n_atoms_out);

/* ---- trajectories (host side) ------------------------------------------ */

/* DcdReader::read_all_frames, core/src/trajectory/dcd.rs:54-135: frames in nm
 * (float32 Angstrom * 0.1 in float64).  Call with out_nm == NULL to size. */
rstg_status rstg_dcd_read(const char* path, double* out_nm, int64_t capacity_values, int64_t* n_frames,
                          int64_t* n_atoms);
/* Raw float32 Angstrom frames as stored (the batched engine consumes these). */
rstg_status rstg_dcd_read_f32(const char* path, float* out_A, int64_t capacity_values, int64_t* n_frames,
                              int64_t* n_atoms);
/* MdcrdReader, crates/mmpbsa/src/mdcrd.rs:12-108 (Angstrom). */
rstg_status rstg_mdcrd_read(const char* path, int64_t n_atoms, int32_t has_box, double* out_A,
                            int64_t capacity_values, int64_t* n_frames);

/* ---- single-term entry points (plain FP64 GPU form) --------------------- */

/* compute_mm_energy, crates/mmpbsa/src/mm_energy.rs:168-172 */
rstg_status rstg_mm_energy_compute(rstg_ctx* ctx, const rstg_topology* t, const double* xyz, int64_t n,
                                   rstg_mm_energy* out);
/* compute_gb_energy, crates/mmpbsa/src/gb_energy.rs:357-365 */
rstg_status rstg_gb_energy_compute(rstg_ctx* ctx, const rstg_topology* t, const double* xyz, int64_t n,
                                   const rstg_gb_params* p, double* total, double* born_radii);
/* Born-radius cache across frames (gb_energy.rs:66-120): when the RMSD
 * between the coordinates and the cached ones is below rmsd_threshold (A),
 * compute_gb_energy_cached (gb_energy.rs:372-387) reuses the cached radii;
 * otherwise it recomputes them and refreshes the cache.  The cache is a host
 * object; reused (optional) receives 1 on a hit. */
typedef struct rstg_gb_cache rstg_gb_cache;
rstg_status rstg_gb_cache_create(double rmsd_threshold, rstg_gb_cache** out);
void rstg_gb_cache_destroy(rstg_gb_cache* c);
rstg_status rstg_gb_energy_cached(rstg_ctx* ctx, const rstg_topology* t, const double* xyz, int64_t n,
                                  const rstg_gb_params* p, rstg_gb_cache* cache, double* total, double* born_radii,
                                  int32_t* reused);
/* compute_sa_energy, crates/mmpbsa/src/sa_energy.rs:51-75 */
rstg_status rstg_sa_energy_compute(rstg_ctx* ctx, const rstg_topology* t, const double* xyz, int64_t n,
                                   const rstg_sa_params* p, double* total, double* total_sasa, double* per_atom);
/* compute_pb_energy / compute_pb_energy_solvated, crates/mmpbsa/src/pb_energy.rs:332-482;
 * solute_residues may be NULL (n_solute ignored). */
rstg_status rstg_pb_energy_compute(rstg_ctx* ctx, const rstg_topology* t, const double* xyz, int64_t n,
                                   const rstg_pb_params* p, const int64_t* solute_residues, int64_t n_solute,
                                   double* total, rstg_pb_diag* diag);
/* Grid set-up of one PB solve (pb_grid.rs:188-985, pb_solver.rs:68-93), for
 * inspection: auto_grid dims and origin always; when charge != NULL (arrays of
 * dims[0]*dims[1]*dims[2]) the charge density, SES inside flags (may be NULL),
 * face dielectrics, kappa-bar^2 map and a grid holding the Debye-Hueckel
 * boundary potential (zero inside).  eps_out and use_ionic select the
 * solvated (solvent dielectric, salt) or reference (solute dielectric, none)
 * solve. */
rstg_status rstg_pb_grid_maps(rstg_ctx* ctx, const double* xyz, int64_t n, const double* charges_e,
                              const double* radii, const rstg_pb_params* p, double eps_in, double eps_out,
                              int32_t use_ionic, int64_t* dims3, double* origin3, double* charge, uint8_t* inside,
                              double* eps_x, double* eps_y, double* eps_z, double* kappa_sq, double* boundary_phi);

/* compute_binding_energy_single_frame, crates/mmpbsa/src/binding.rs:749-786 */
rstg_status rstg_binding_frame(rstg_ctx* ctx, const rstg_topology* t, const double* xyz, int64_t n,
                               const int64_t* receptor_residues, int64_t n_rec, const int64_t* ligand_residues,
                               int64_t n_lig, const rstg_solvation* solv, const rstg_sa_params* sa,
                               rstg_frame_energy* out);
/* decompose_binding_energy, crates/mmpbsa/src/decomposition.rs:75-92;
 * outputs are in the order of the residue lists given. */
rstg_status rstg_decompose(rstg_ctx* ctx, const rstg_topology* t, const double* xyz, int64_t n,
                           const int64_t* receptor_residues, int64_t n_rec, const int64_t* ligand_residues,
                           int64_t n_lig, const rstg_gb_params* gb, const rstg_sa_params* sa,
                           rstg_residue_energy* rec_out, rstg_residue_energy* lig_out);

/* Mass-weighted coordinate covariance of quasi_harmonic_entropy,
 * crates/mmpbsa/src/entropy.rs:97-160, in FP64 on the GPU: traj_A host
 * [n_frames][n_atoms][3] Angstrom, masses [n_atoms] amu, cov host
 * [3 n_atoms][3 n_atoms] (full symmetric, row-major), equal bit for bit to
 * the reference's frame-ordered sums.  The eigenvalues and the entropy sum
 * stay on the host. */
rstg_status rstg_qh_covariance(rstg_ctx* ctx, const double* traj_A, int64_t n_frames, int64_t n_atoms,
                               const double* masses, double* cov);

/* GB energy (Born radii + pair sum, same kernels and results as
 * rstg_gb_energy_compute) that allocates no device memory.  No counterpart in
 * the reference.  For callers that cannot call cudaMalloc where they need the
 * energy (an allocator owned by a host framework, latency-critical loops that
 * must not enter the driver's allocator).  All pointers are device memory on
 * the calling thread's current device; d_born_radii may be NULL.  Work is
 * enqueued on `stream` (NULL: the legacy default stream) and the call returns
 * without synchronising.  Scratch lives in a 1.5 MiB file-scope device array
 * that every GPU loading the library holds until exit; n_atoms is limited to
 * 1..131072 (larger requests fail with RSTG_ERR_INVALID).  The first call on a
 * device resolves the array's address and should come before any stream
 * capture.  Calls share the array: calls that overlap on the GPU race. */
rstg_status rstg_gb_energy_noalloc_async(const double* d_xyz, const double* d_charges_amber, const double* d_radii,
                                         const double* d_screen, int64_t n_atoms, const rstg_gb_params* params,
                                         double* d_total, double* d_born_radii, void* stream);

/* ---- batched engine ------------------------------------------------------ */

typedef enum rstg_mode {
  RSTG_MODE_PLAIN = 0, /* FP64 kernels, one subsystem of one frame per launch  */
  RSTG_MODE_FUSED = 1  /* mixed precision, frames x {C,R,L} fused per launch   */
} rstg_mode;

typedef struct rstg_system_opts {
  int32_t mode;            /* rstg_mode, default FUSED                          */
  int32_t decompose;       /* also produce per-residue terms for every frame    */
  int64_t max_batch_frames; /* frames per device batch (0: as many as fit a
                              2 GB share of device memory, at most 256)      */
  int32_t use_graphs;      /* capture each batch's launch sequence (default 1) */
  int32_t autotune;        /* time the launch shapes of the pair and SASA
                              kernels on the first run and keep the fastest
                              (default 1; 0: fixed default shapes)          */
} rstg_system_opts;
void rstg_system_opts_default(rstg_system_opts* o);

/* A device-resident binding problem: complex = receptor U ligand residues of
 * the topology (binding.rs:142-211), parameters and work buffers resident. */
rstg_status rstg_system_create(rstg_ctx* ctx, const rstg_topology* t, const int64_t* receptor_residues,
                               int64_t n_rec, const int64_t* ligand_residues, int64_t n_lig,
                               const rstg_solvation* solv, const rstg_sa_params* sa, const rstg_system_opts* opts,
                               rstg_system** out);
void rstg_system_destroy(rstg_system* s);
/* n_complex_atoms, n_receptor_atoms, n_ligand_atoms, n_receptor_residues,
 * n_ligand_residues, n_topology_atoms */
rstg_status rstg_system_shape(const rstg_system* s, int64_t* shape6);
/* Device bytes held by the system for a batch of n_frames. */
int64_t rstg_system_footprint(const rstg_system* s, int64_t n_frames);

/* End-to-end: frames are host float32 Angstrom [F][n_topology_atoms][3] as
 * stored in DCD; they are read through the reference's DCD path
 * (float32 -> nm float64 -> Angstrom).  Results land in host memory.
 * decomp may be NULL; else [F][n_receptor_residues + n_ligand_residues]. */
rstg_status rstg_system_run(rstg_system* s, const float* frames, int64_t n_frames, rstg_frame_energy* out,
                            rstg_residue_energy* decomp);
/* Device-resident variant: d_frames [F][n_topology_atoms][3] float32 on the
 * device, d_out / d_decomp device memory.  Enqueued on the context stream;
 * returns without synchronising. */
rstg_status rstg_system_run_device(rstg_system* s, const float* d_frames, int64_t n_frames,
                                   rstg_frame_energy* d_out, rstg_residue_energy* d_decomp);
/* Kernel launches of the last run and its precision diagnostics:
 * [0] launches, [1] pairs sent to the FP64 guard path, [2] SASA point tests
 * re-checked in FP64, [3] neighbour-list overflows (must be 0). */
rstg_status rstg_system_last_stats(const rstg_system* s, int64_t* stats4);

/* Launch shapes of a fused system (no reference counterpart).  shape12 =
 * pair-kernel threads per tile row, its minimum resident blocks per SM
 * (register cap), SASA warps per block, frames per batch, tuned (1 once the
 * first run timed the candidates), frames of the tuning pass, number of
 * pair-kernel candidates, number of SASA candidates, Born-radius kernel
 * threads per row, its minimum resident blocks per SM, number of its
 * candidates, pair-kernel form (0 one block per 128 x 128 tile with
 * threads-per-row threads per row, 1 warp items with the tile's columns in
 * threads-per-row shares); ms12 = the tuning pass's best-of-two milliseconds per
 * candidate (pair-kernel shapes, then SASA shapes, then Born-radius shapes).
 * Systems of one process with the same device, atom counts and sphere
 * points share the tuned shapes, so equal inputs give equal results.  Either
 * pointer may be NULL; zeros for plain-mode systems. */
rstg_status rstg_system_tuning(const rstg_system* s, int32_t* shape12, double* ms12);

/* Batched Poisson-Boltzmann engine of a fused PB system (no reference
 * counterpart), accumulated over runs: grids solved, lock-step multigrid
 * cycles, grids solved by the FP64 path, then host milliseconds of the
 * set-up (maps, boundary values), the cycles and the finish (fallbacks,
 * energies).  Eight doubles; zeros for GB systems. */
rstg_status rstg_system_pb_stats(const rstg_system* s, double* stats8);
/* Frames per batched PB launch sequence (0: from the device memory budget,
 * at most 60 % of the free memory and 64 GB, about 140 bytes per grid point
 * of the complex, receptor and ligand grids of a frame). */
rstg_status rstg_system_set_pb_batch(rstg_system* s, int64_t frames);
/* Stopping rule of the batched PB engine (no reference counterpart).
 * rel_tol = 0 (default): the reference's schedule -- V-cycles until the
 * absolute RMS residual is below PbParams.tolerance, at most
 * clamp(max_iterations / 6, 1, 200) cycles, Chebyshev SOR after divergence
 * (pb_solver.rs:1015-1167) -- whose result on large solvated grids is the
 * iterate at the cycle cap.  rel_tol > 0: every grid (focusing coarse grids
 * included) is solved to ||f - A phi|| <= rel_tol ||f - A phi_0|| in FP64
 * by defect correction with FP32 V-cycles of a consistent multigrid
 * (Gauss-Seidel smoothing, full-weighting restriction, series/parallel
 * coarse dielectrics), which converges where the reference's V-cycle
 * stalls; the cycle cap stays.  Applies to later runs. */
rstg_status rstg_system_set_pb_convergence(rstg_system* s, double rel_tol);
/* Profile mode of the batched PB engine (no reference counterpart): when on,
 * later runs launch the multigrid cycles without graph capture and time the
 * finest-level kernels with CUDA events.  rstg_system_pb_profile returns
 * twelve doubles, for the full red-black sweep, FP32 residual, end-of-cycle
 * update + FP64 residual and a fourth slot that is no longer used (zero):
 * total milliseconds [0..3], algorithmic DRAM bytes of the timed launches
 * [4..7] and launch counts [8..11], accumulated since profiling began. */
rstg_status rstg_system_set_pb_profile(rstg_system* s, int32_t on);
rstg_status rstg_system_pb_profile(const rstg_system* s, double* out12);

/* Per-kernel device time of one pass of the fused engine over device frames
 * (no reference counterpart).  Each kernel is bracketed by CUDA events on the
 * system stream (direct launches).  Up to 8 kernels: names [8][32] NUL
 * terminated, ms[k] total milliseconds, flops[k] algorithmic FP operations
 * (pair counts times the per-pair operation counts of the reference
 * expressions; 0 where not defined), bytes[k] algorithmic DRAM bytes.
 * *n receives the kernel count. */
rstg_status rstg_system_profile(rstg_system* s, const float* d_frames, int64_t n_frames, int32_t* n, char* names,
                                double* ms, double* flops, double* bytes);

/* Measured peak rates of the non-tensor pipes on a device (no reference
 * counterpart): out4 = FP32 FMA TFLOP/s, FP64 FMA TFLOP/s, MUFU ex2 Gop/s,
 * nominal maximum SM clock in MHz. */
rstg_status rstg_calibrate(int device, double* out4);

/* Periodic reimaging of the system's complex, reimage_complex
 * (crates/mmpbsa/src/binding.rs:234-308): bonded components unwrapped along
 * a breadth-first walk of the bond graph, then each component after the
 * first moved to the minimum image of the first one's geometric centre.
 * frames: F frames in topology order [F][n_atoms][3] Angstrom, boxes [F][3]
 * edge lengths, both host memory; out (may equal frames) receives the frames
 * with the complex atoms reimaged and the other atoms as given.
 * on_device 1: one block per frame on the GPU; 0: on the host.  Both forms
 * use the reference's FP64 operations in its order and give the same bits.
 * The trajectory workflow below reimages boxed frames on the device. */
rstg_status rstg_system_reimage(rstg_system* s, const double* frames, const double* boxes, int64_t n_frames,
                                int32_t on_device, double* out);

/* compute_binding_energy over a trajectory file, crates/mmpbsa/src/binding.rs:461-744.
 * format: "dcd" or "mdcrd".  frames_out may be NULL; stats9 = mean_delta_mm,
 * mean_delta_polar, mean_delta_sa, mean_delta_total, std_delta_total,
 * std_delta_mm, std_delta_polar, std_delta_sa, sem_delta_total. */
rstg_status rstg_binding_trajectory(rstg_ctx* ctx, const rstg_topology* t, const char* path, const char* format,
                                    int32_t has_box, const int64_t* receptor_residues, int64_t n_rec,
                                    const int64_t* ligand_residues, int64_t n_lig, const rstg_solvation* solv,
                                    const rstg_sa_params* sa, int64_t stride, int64_t start_frame,
                                    int64_t end_frame, int32_t mode, rstg_frame_energy* frames_out,
                                    int64_t frames_capacity, int64_t* n_frames, double* stats9,
                                    double* last_frame_coords);

/* ---- serving loop -------------------------------------------------------- */

typedef struct rstg_server_opts {
  int64_t memory_budget_bytes; /* limit on the batch buffers systems keep resident
                                  between requests; idle systems are evicted,
                                  least recently used first, to admit a request */
  int32_t max_inflight;        /* worker threads: requests with a chunk in flight */
  int64_t chunk_frames;        /* frames per chunk (0: about 2.5e9 complex pair
                                  evaluations for GB systems, 16 frames for PB,
                                  8 in plain mode); chunks are dispatched oldest
                                  request first, each on a stream whose priority
                                  is its request's age rank among those in
                                  flight                                        */
} rstg_server_opts;
void rstg_server_opts_default(rstg_server_opts* o);

rstg_status rstg_server_create(rstg_ctx* ctx, const rstg_server_opts* opts, rstg_server** out);
void rstg_server_destroy(rstg_server* s);
/* Asynchronous: copies frames, returns a request id.  The system keeps its
 * batch buffers between requests (reused by its next request), so a system
 * submitted to a server must outlive the server. */
rstg_status rstg_server_submit(rstg_server* s, rstg_system* sys, const float* frames, int64_t n_frames,
                               int64_t* request_id);
/* RSTG_ERR_NOT_READY while running; RSTG_OK copies results (out [F]). */
rstg_status rstg_server_poll(rstg_server* s, int64_t request_id, rstg_frame_energy* out);
rstg_status rstg_server_wait(rstg_server* s, int64_t request_id, int64_t timeout_ms, rstg_frame_energy* out);
rstg_status rstg_server_cancel(rstg_server* s, int64_t request_id);
/* stats8 = completed, frames, p50_ms, p99_ms, mean_ms, peak_bytes, wall_s, frames_per_s */
rstg_status rstg_server_stats(const rstg_server* s, double* stats8);

#ifdef __cplusplus
}
#endif
#endif /* RSTG_H */
