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

// Device state of one solve: maps on the fine grid plus multigrid levels.
struct PbProblem;

// One paired PB energy (solvated - reference) of one (sub)system.
double pb_energy_run(Ctx* c, const std::vector<double>& xyz_host, const std::vector<double>& q_e,
                     const std::vector<double>& radii, const rstg_pb_params& p, rstg_pb_diag* diag);

// Grid set-up of one solve (for inspection and tests): dims/origin always;
// with charge != NULL every map of that solve and the boundary potential.
void pb_grid_maps(Ctx* c, const std::vector<double>& x, const std::vector<double>& q, const std::vector<double>& radii,
                  const rstg_pb_params& p, double ein, double eout, bool ionic, int64_t* dims, double* origin,
                  double* charge, uint8_t* inside, double* ex, double* ey, double* ez, double* k2, double* bphi);

}  // namespace rstg
