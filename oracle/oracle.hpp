// CPU restatement of the reference MM-PBSA / MM-GBSA hot path.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library or the
// Python package) links, loads or calls this code.  It is used by tests/ as
// the parity checker, by __graft_entry__.smoke() as the checker, and by
// bench.py as the timed CPU baseline ("kind": "port").
//
// Two modes:
//   faithful  - the reference's arithmetic, operation order and iteration
//               schedule (crates/mmpbsa/src/*.rs), fixed-order reductions
//               where the reference uses rayon reductions.  This is the
//               parity target for the plain FP64 GPU form and the CPU
//               baseline.
//   accurate  - the same physics with long-double accumulation and the
//               exact binding-difference formulations (R x L pair sums for
//               the non-bonded difference, per-atom SASA differences), used
//               as the error reference for the mixed-precision GPU form.
//
// Parity pinning: the reference cannot be built here (Rust toolchain and
// crates absent).  The restatement is pinned against every known-answer
// test the reference holds for this path (kappa, single-ion GB, bond and
// angle energy, single-atom SASA, Fibonacci unit norm, charge conservation,
// restrict/prolong of a constant, the PB Born ion) -- see
// tests/test_oracle_pins.py.  The reference holds no real-system golden
// energies, so full-system values are pinned only through this restatement.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace orc {

struct V3 {
  double x, y, z;
};

// AmberTopology (core/src/amber/prmtop.rs:34-105), the fields the hot path uses.
struct Topology {
  size_t n_atoms = 0, n_residues = 0, n_types = 0;
  std::vector<std::string> atom_names;
  std::vector<size_t> type_idx;
  std::vector<double> charges, charges_amber;
  std::vector<std::string> residue_labels;
  std::vector<size_t> residue_pointers;
  std::vector<std::pair<size_t, size_t>> bonds;
  std::vector<size_t> bond_types;
  std::vector<double> masses, radii, screen;
  std::vector<double> bond_k, bond_req, angle_k, angle_teq, dih_pk, dih_pn, dih_phase;
  struct Angle {
    size_t i, j, k, t;
  };
  struct Dihedral {
    size_t i, j, k, l, t;
    bool ignore_14;
  };
  std::vector<Angle> angles;
  std::vector<Dihedral> dihedrals;
  std::vector<size_t> num_excluded;
  std::vector<size_t> excluded_list;  // SIZE_MAX marks the 0 placeholder
  double scee = 1.2, scnb = 2.0;
  std::vector<double> lj_a, lj_b;
  std::vector<int64_t> nb_index;

  std::vector<size_t> atom_residue_indices() const;
  // build_selection (prmtop.rs:165-204); returns false on out-of-range residue.
  bool build_selection(const std::vector<size_t>& residues, std::vector<size_t>& atoms,
                       std::string& err) const;
};

bool parse_prmtop(const std::string& path, Topology& out, std::string& err);
Topology extract_subtopology(const Topology& t, const std::vector<size_t>& atoms);

// DCD reader (core/src/trajectory/dcd.rs:217-444): frames in nm (f32 A * 0.1).
bool read_dcd(const std::string& path, std::vector<std::vector<V3>>& frames_nm, std::string& err);

struct GbParams {
  int model = 1;  // 0 HCT, 1 OBC-I, 2 OBC-II
  double solute_dielectric = 1.0, solvent_dielectric = 78.3, salt = 0.15, temperature = 300.0;
  double offset = 0.09, rgbmax = 25.0, cutoff = 9999.0;
};
struct SaParams {
  double surface_tension = 0.0072, offset = 0.0, probe = 1.4;
  size_t n_points = 480;
};
struct PbParams {
  double grid_spacing = 0.5, grid_buffer = 10.0, solute_dielectric = 1.0, solvent_dielectric = 80.0;
  double salt = 0.15, temperature = 300.0, probe = 1.4, ion_radius = 2.0, tolerance = 1e-6;
  size_t max_iterations = 10000;
  double fillratio = 4.0;
  size_t fscale = 8;
  // > 0: solve every grid to this relative FP64 residual instead of the
  // reference's schedule (the converged answer, not the reference's iterate)
  double converged_rel_tol = 0.0;
  size_t converged_max_iter = 20000;
  int converged_method = 0;  // 0 Jacobi-PCG, 1 flexible CG + V-cycle, 2 defect correction + V-cycle
};

struct MmEnergy {
  double bond = 0, angle = 0, dihedral = 0, vdw = 0, elec = 0, vdw_14 = 0, elec_14 = 0;
  double total() const { return bond + angle + dihedral + vdw + elec + vdw_14 + elec_14; }
};

double kappa(double salt, double eps, double temperature);
std::vector<double> born_radii(const Topology& t, const std::vector<V3>& x, const GbParams& p,
                               bool accurate);
double gb_energy_from_radii(const Topology& t, const std::vector<V3>& x, const GbParams& p,
                            const std::vector<double>& R, bool accurate);
MmEnergy mm_energy(const Topology& t, const std::vector<V3>& x, bool accurate);
std::vector<V3> fibonacci_sphere(size_t n);
std::vector<double> sasa_per_atom(const std::vector<V3>& x, const std::vector<double>& radii,
                                  double probe, size_t n_points);

struct PbDiag {
  size_t iterations[2] = {0, 0};
  double residual[2] = {0, 0};
  int converged[2] = {0, 0};
  int dims[3] = {0, 0, 0};
};
double pb_energy(const std::vector<V3>& x, const std::vector<double>& q_e,
                 const std::vector<double>& radii, const PbParams& p, PbDiag* diag);

struct SubsystemEnergy {
  double mm = 0, polar = 0, sa = 0;
  double total() const { return mm + polar + sa; }
};
struct FrameEnergy {
  SubsystemEnergy c, r, l;
  double d_mm = 0, d_polar = 0, d_sa = 0, d_total = 0;
};

struct Residue {
  size_t index;
  double vdw, elec, polar, sa;
};

}  // namespace orc
