// PB pieces of the CPU restatement (TEST INFRASTRUCTURE ONLY, see oracle.hpp).
#pragma once
#include <cstdint>
#include <vector>

#include "oracle.hpp"

namespace orc {

// PbGrid (pb_grid.rs:13-183): layout ix + nx*(iy + ny*iz).
struct Grid {
  size_t dims[3] = {0, 0, 0};
  double h[3] = {0, 0, 0};
  double origin[3] = {0, 0, 0};
  size_t len() const { return dims[0] * dims[1] * dims[2]; }
  size_t index(size_t ix, size_t iy, size_t iz) const { return ix + dims[0] * (iy + dims[1] * iz); }
  void point(size_t ix, size_t iy, size_t iz, double* p) const {
    p[0] = origin[0] + (double)ix * h[0];
    p[1] = origin[1] + (double)iy * h[1];
    p[2] = origin[2] + (double)iz * h[2];
  }
};

struct Diel {
  std::vector<double> ex, ey, ez;
};

struct BC {
  int kind = 0;  // 0 zero, 1 Debye-Hueckel, 2 interpolated
  std::vector<std::pair<size_t, double>> values;
};

struct SolveResult {
  std::vector<double> phi;
  size_t iterations = 0;
  double residual = 0;
  bool converged = false;
  bool diverged = false;
};

Grid auto_grid(const std::vector<V3>& x, double h, double buffer);
Grid coarse_grid(const std::vector<V3>& x, double fine_h, double fillratio, size_t fscale);
std::vector<double> map_charges(const Grid& g, const std::vector<V3>& x, const std::vector<double>& q);
double interpolate(const Grid& g, const double* p, const std::vector<double>& data);
std::vector<uint8_t> inside_ses(const Grid& g, const std::vector<V3>& x, const std::vector<double>& radii,
                                double probe);
double fraction_inside(double lo, double hi, double p1, double p2, int axis, const std::vector<V3>& x,
                       const std::vector<double>& radii, double probe);
Diel assign_dielectrics(const Grid& g, const std::vector<V3>& x, const std::vector<double>& radii, double probe,
                        double ein, double eout);
std::vector<double> assign_kappa(const Grid& g, const std::vector<V3>& x, const std::vector<double>& radii,
                                 double ion_radius, double kbulk, double eps_s);
void set_dh_boundary(std::vector<double>& phi, const Grid& g, const std::vector<V3>& x,
                     const std::vector<double>& q, double kap, double eout);
double estimate_omega(const size_t* d);
void restrict_into(const double* fine, const size_t* fd, double* coarse, const size_t* cd, double scale);
void prolongate_add(const double* coarse, const size_t* cd, double* fine, const size_t* fd);
SolveResult solve_multigrid(const Grid& g, const std::vector<double>& rho, const Diel& D,
                            const std::vector<double>& k2, const BC& bc, const std::vector<V3>& x,
                            const std::vector<double>& q, double kb, double eout, double tol, size_t maxit);
// Converged solve of the same discrete system to a relative residual
// (method 0 Jacobi-preconditioned CG, 1 flexible CG with a consistent
// V-cycle, 2 defect correction with that V-cycle); not the reference's
// schedule.
SolveResult solve_converged(const Grid& g, const std::vector<double>& rho, const Diel& D,
                            const std::vector<double>& k2, const BC& bc, const std::vector<V3>& x,
                            const std::vector<double>& q, double kb, double eout, double rel_tol, size_t maxit,
                            int method);
double elec_energy(const Grid& g, const std::vector<double>& phi, const std::vector<V3>& x,
                   const std::vector<double>& q);

}  // namespace orc
