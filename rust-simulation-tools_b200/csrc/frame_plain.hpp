// Plain FP64 evaluation of one binding frame: complex, receptor and ligand
// each evaluated with its own launch sequence (binding.rs:333-415).
#pragma once
#include <memory>

#include "plain.cuh"

namespace rstg {

// PB polar energy of one (sub)system (pb_energy.rs:332-438), pb.cu.  xyz_host
// is Angstrom [n][3]; charges in e.
double pb_energy_run(Ctx* c, const std::vector<double>& xyz_host, const std::vector<double>& q_e,
                     const std::vector<double>& radii, const rstg_pb_params& p, rstg_pb_diag* diag,
                     double rtol);

struct PlainSub {
  Topology top;
  PairClasses pc;
  DevTopo dev;
};

struct PlainFrameEval {
  Split split;
  PlainSub sub[3];  // complex, receptor, ligand
  rstg_solvation solv;
  rstg_sa_params sa;
  DevBuf sphere, xyz[3], born, per_atom, out, overflow, rec_idx, lig_idx;
  int64_t n_sphere = 0;
  Ctx* ctx = nullptr;
  double pb_rel_tol = 0.0;  // > 0: PB grids solved to this relative residual (not the reference's rule)

  PlainFrameEval(Ctx* c, const Topology& t, const std::vector<int64_t>& rres, const std::vector<int64_t>& lres,
                 const rstg_solvation& solv, const rstg_sa_params& sa);
  // xyz: host complex coordinates, Angstrom [n_complex][3]
  rstg_frame_energy run(const double* xyz_complex_host);
  // Per-residue decomposition (decomposition.rs:210-410), outputs in residue-list order.
  void decompose(const double* xyz_complex_host, const rstg_gb_params& gb, rstg_residue_energy* rec_out,
                 rstg_residue_energy* lig_out);
};

}  // namespace rstg
