// Plain FP64 form: one (sub)system of one frame per launch sequence, with the
// reference's arithmetic (crates/mmpbsa/src/{gb,mm,sa}_energy.rs,
// core/src/sasa.rs).  Compiled with -fmad=false.
#pragma once
#include "internal.hpp"

namespace rstg {

// FP64 parameters of one (sub)topology resident on the device.
struct DevTopo {
  int64_t n = 0, nt = 0, nb = 0, na = 0, nd = 0;
  double scee = 1.2, scnb = 2.0;
  double max_radius = 0.0;  // fold(0.0, max) over radii (core/src/sasa.rs:213-214)
  DevBuf q, rad, scr, type, ljA, ljB, excl, p14;
  DevBuf bidx, bpar, aidx, apar, didx, dpar;
  static DevTopo upload(const Topology& t, const PairClasses& pc, cudaStream_t s);
};

// Fibonacci sphere (core/src/sasa.rs:147-169) evaluated on the host with the
// platform libm, as the reference does, and uploaded.
std::vector<double> fibonacci_sphere(int64_t n);

void plain_born_radii(Ctx* c, const DevTopo& t, const double* d_xyz, const rstg_gb_params& p, double* d_R);
// d_out: [1] total GB energy
void plain_gb_energy(Ctx* c, const DevTopo& t, const double* d_xyz, const rstg_gb_params& p, const double* d_R,
                     double* d_out);
// d_out: [7] bond angle dihedral vdw elec vdw_14 elec_14
void plain_mm_energy(Ctx* c, const DevTopo& t, const double* d_xyz, double* d_out);
// d_per_atom [n], d_total [1] (sum of per-atom SASA), d_overflow [1] int
void plain_sasa(Ctx* c, const DevTopo& t, const double* d_xyz, double probe, int64_t n_points,
                const double* d_sphere, double* d_per_atom, double* d_total, int* d_overflow);
// Receptor x ligand pair energies of the complex (decomposition.rs:240-283):
// d_rows [nR][2] and d_cols [nL][2] hold (vdw, elec) sums per atom.
void plain_decomp_pairs(Ctx* c, const DevTopo& C, const double* d_xyz, const int* d_rec, int nR, const int* d_lig,
                        int nL, double* d_rows, double* d_cols);
// Deterministic column sums: in [rows][cols] -> out[cols] (fixed order).
void sum_columns(Ctx* c, const double* d_in, int64_t rows, int cols, double* d_out);

// GB constants of gb_energy.rs:290-306 and the plain kernels behind
// plain_born_radii / plain_gb_energy / sum_columns (8 warps per block for the
// first two; part[] holds one partial per warp of (n + 1) / 2 warps).
struct GbConst {
  double kappa, inv_ein, inv_eout, diel_ns, cut2;
  int no_salt;
};
GbConst gb_const(const rstg_gb_params& p);
__global__ void k_born_radii_plain(int n, const double* __restrict__ xyz, const double* __restrict__ rad,
                                   const double* __restrict__ scr, double offset, double cut2, int model,
                                   double rgbmax, double* __restrict__ R);
__global__ void k_gb_plain(int n, const double* __restrict__ xyz, const double* __restrict__ q,
                           const double* __restrict__ R, GbConst k, double* __restrict__ part);
__global__ void k_sum_columns(const double* __restrict__ in, long long rows, int cols, double* __restrict__ out);

}  // namespace rstg
