// Poisson-Boltzmann engine: grid set-up (pb_grid.rs), multigrid solver
// (pb_solver.rs) and the paired solves with optional focusing (pb_energy.rs).
#pragma once
#include <vector>

#include "internal.hpp"

namespace rstg {

// PbGrid geometry (pb_grid.rs:13-81): layout ix + nx*(iy + ny*iz).
struct PbGeom {
  int nx = 0, ny = 0, nz = 0;
  double h = 0.5, ox = 0, oy = 0, oz = 0;
  size_t n() const { return (size_t)nx * ny * nz; }
};

PbGeom pb_auto_grid(const std::vector<double>& xyz, double h, double buffer);              // pb_grid.rs:188-215
PbGeom pb_coarse_grid(const std::vector<double>& xyz, double h, double fill, int64_t fs);  // pb_energy.rs:92-125
double pb_omega(int nx, int ny, int nz);                                                    // pb_solver.rs:124-139

// Atom spatial hash (pb_grid.rs:319-385) as CSR, built on the host; queried
// on the device with the reference's cell arithmetic.
struct PbHash {
  double inv = 1.0, ox = 0, oy = 0, oz = 0;
  int gx = 0, gy = 0, gz = 0;
  std::vector<int32_t> start, atoms;  // start[cell .. cell+1) into atoms
};
PbHash pb_build_hash(const std::vector<double>& xyz, double max_eff);

// Stream of the PB engine on this thread: the context's unless a
// PbStreamScope is active.
cudaStream_t pb_stream(Ctx* c);
struct PbStreamScope {
  cudaStream_t prev;
  explicit PbStreamScope(cudaStream_t s);
  ~PbStreamScope();
};

// Atoms of one solve: device copies plus the host arrays that the host-side
// set-up (hash, charge spreading) reads.  xyz Angstrom, q in e.
struct AtomsDev {
  DevBuf xyz, q, r;
  int n = 0;
  std::vector<double> hx, hq, hr;
  double max_r = 0.0;
  AtomsDev(const std::vector<double>& x, const std::vector<double>& qe, const std::vector<double>& rad,
           cudaStream_t st)
      : hx(x), hq(qe), hr(rad) {
    n = (int)qe.size();
    xyz = DevBuf(std::max<size_t>(x.size(), 3) * 8, st);
    q = DevBuf(std::max<size_t>(qe.size(), 1) * 8, st);
    r = DevBuf(std::max<size_t>(rad.size(), 1) * 8, st);
    if (n) {
      RSTG_CUDA(cudaMemcpyAsync(xyz.p, x.data(), x.size() * 8, cudaMemcpyHostToDevice, st));
      RSTG_CUDA(cudaMemcpyAsync(q.p, qe.data(), qe.size() * 8, cudaMemcpyHostToDevice, st));
      RSTG_CUDA(cudaMemcpyAsync(r.p, rad.data(), rad.size() * 8, cudaMemcpyHostToDevice, st));
    }
    for (double v : rad) max_r = std::max(max_r, v);
  }
};

struct BcSpec {
  int kind = 1;  // 1 Debye-Hueckel, 2 interpolated from a coarse potential
  double kappa = 0.0, eout = 1.0;
  const PbGeom* cg = nullptr;
  const double* cphi = nullptr;
};

double pb_kappa(const rstg_pb_params& p);  // Debye-Hueckel kappa, pb_energy.rs:337-345

// Maps of one solve into caller-owned arrays of g.n() doubles: rho (charge
// density) when non-null; ex/ey/ez (face dielectrics) when ex is non-null;
// k2 (kappa-bar^2) when non-null.
void pb_maps_into(Ctx* c, const PbGeom& g, const AtomsDev& A, const rstg_pb_params& p, double ein, double eout,
                  double kap, bool ionic, double* rho, double* ex, double* ey, double* ez, double* k2);
// Boundary values of phi (Debye-Hueckel or interpolated from a coarse grid).
void pb_boundary(Ctx* c, const PbGeom& g, double* phi, const AtomsDev& A, const BcSpec& bc);

// FP64 solve of one grid with the reference's multigrid / SOR logic; null
// ex means uniform dielectric uniform_eps and k2 = 0.  phi_out: g.n() doubles.
struct PbSolveStats {
  int64_t iterations;
  double residual;
  bool converged;
};
PbSolveStats pb_solve_fp64(Ctx* c, const PbGeom& g, const double* rho, const double* ex, const double* ey,
                           const double* ez, const double* k2, double uniform_eps, const AtomsDev& A,
                           const BcSpec& bc, double tol, int64_t maxit, double* phi_out);

// One paired PB energy (solvated - reference) of one (sub)system.
double pb_energy_run(Ctx* c, const std::vector<double>& xyz_host, const std::vector<double>& q_e,
                     const std::vector<double>& radii, const rstg_pb_params& p, rstg_pb_diag* diag,
                     double rtol = 0.0);

// Grid set-up of one solve (for inspection and tests): dims/origin always;
// with charge != NULL every map of that solve and the boundary potential.
void pb_grid_maps(Ctx* c, const std::vector<double>& x, const std::vector<double>& q, const std::vector<double>& radii,
                  const rstg_pb_params& p, double ein, double eout, bool ionic, int64_t* dims, double* origin,
                  double* charge, uint8_t* inside, double* ex, double* ey, double* ez, double* k2, double* bphi);

}  // namespace rstg
