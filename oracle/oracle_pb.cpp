// CPU restatement of the reference Poisson-Boltzmann path.
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).
//   crates/mmpbsa/src/pb_grid.rs   : grid, charge spreading, SES, dielectrics, kappa
//   crates/mmpbsa/src/pb_solver.rs : DH boundary, red-black SOR, multigrid V-cycle
//   crates/mmpbsa/src/pb_energy.rs : paired solves, focusing
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <limits>

#include "oracle.hpp"
#include "oracle_pb.hpp"

namespace orc {

static const double PI = 3.14159265358979323846;
static const double FOUR_PI_EC = 4.0 * PI * 332.0522;  // pb_solver.rs:155

// pb_grid.rs:188-215
Grid auto_grid(const std::vector<V3>& x, double h, double buffer) {
  double mn[3] = {std::numeric_limits<double>::max(), std::numeric_limits<double>::max(),
                  std::numeric_limits<double>::max()};
  double mx[3] = {std::numeric_limits<double>::lowest(), std::numeric_limits<double>::lowest(),
                  std::numeric_limits<double>::lowest()};
  for (auto& c : x) {
    double v[3] = {c.x, c.y, c.z};
    for (int d = 0; d < 3; d++) {
      if (v[d] < mn[d]) mn[d] = v[d];
      if (v[d] > mx[d]) mx[d] = v[d];
    }
  }
  Grid g;
  for (int d = 0; d < 3; d++) {
    double ext = mx[d] - mn[d] + 2.0 * buffer;
    size_t n = (size_t)std::ceil(ext / h) + 1;
    g.dims[d] = (n % 2 == 0) ? n + 1 : n;
    double gext = (double)(g.dims[d] - 1) * h;
    double c = 0.5 * (mn[d] + mx[d]);
    g.origin[d] = c - 0.5 * gext;
    g.h[d] = h;
  }
  return g;
}

// pb_energy.rs:92-125
Grid coarse_grid(const std::vector<V3>& x, double fine_h, double fillratio, size_t fscale) {
  double mn[3] = {std::numeric_limits<double>::max(), std::numeric_limits<double>::max(),
                  std::numeric_limits<double>::max()};
  double mx[3] = {std::numeric_limits<double>::lowest(), std::numeric_limits<double>::lowest(),
                  std::numeric_limits<double>::lowest()};
  for (auto& c : x) {
    double v[3] = {c.x, c.y, c.z};
    for (int d = 0; d < 3; d++) {
      if (v[d] < mn[d]) mn[d] = v[d];
      if (v[d] > mx[d]) mx[d] = v[d];
    }
  }
  Grid g;
  double ch = fine_h * (double)fscale;
  for (int d = 0; d < 3; d++) {
    double ext = (mx[d] - mn[d]) * fillratio;
    size_t n = (size_t)std::ceil(ext / ch) + 1;
    g.dims[d] = (n % 2 == 0) ? n + 1 : n;
    double aext = (double)(g.dims[d] - 1) * ch;
    double c = 0.5 * (mn[d] + mx[d]);
    g.origin[d] = c - 0.5 * aext;
    g.h[d] = ch;
  }
  return g;
}

// pb_grid.rs:220-292 (summed in atom order)
std::vector<double> map_charges(const Grid& g, const std::vector<V3>& x, const std::vector<double>& q) {
  std::vector<double> out(g.len(), 0.0);
  long nx = (long)g.dims[0], ny = (long)g.dims[1], nz = (long)g.dims[2];
  for (size_t a = 0; a < x.size(); a++) {
    double fc[3] = {(x[a].x - g.origin[0]) / g.h[0], (x[a].y - g.origin[1]) / g.h[1],
                    (x[a].z - g.origin[2]) / g.h[2]};
    long ix = (long)std::floor(fc[0]), iy = (long)std::floor(fc[1]), iz = (long)std::floor(fc[2]);
    if (ix < 0 || ix >= nx - 1 || iy < 0 || iy >= ny - 1 || iz < 0 || iz >= nz - 1) continue;
    double dx = fc[0] - (double)ix, dy = fc[1] - (double)iy, dz = fc[2] - (double)iz;
    double vol = g.h[0] * g.h[1] * g.h[2];
    double qd = q[a] / vol;
    double wx[2] = {1.0 - dx, dx}, wy[2] = {1.0 - dy, dy}, wz[2] = {1.0 - dz, dz};
    for (int a0 = 0; a0 < 2; a0++)
      for (int a1 = 0; a1 < 2; a1++)
        for (int a2 = 0; a2 < 2; a2++)
          out[g.index(ix + a0, iy + a1, iz + a2)] += qd * wx[a0] * wy[a1] * wz[a2];
  }
  return out;
}

// pb_grid.rs:142-182
double interpolate(const Grid& g, const double* p, const std::vector<double>& data) {
  double fc[3] = {(p[0] - g.origin[0]) / g.h[0], (p[1] - g.origin[1]) / g.h[1],
                  (p[2] - g.origin[2]) / g.h[2]};
  long ix = (long)std::floor(fc[0]), iy = (long)std::floor(fc[1]), iz = (long)std::floor(fc[2]);
  long nx = (long)g.dims[0], ny = (long)g.dims[1], nz = (long)g.dims[2];
  if (ix < 0 || ix >= nx - 1 || iy < 0 || iy >= ny - 1 || iz < 0 || iz >= nz - 1) return 0.0;
  double dx = fc[0] - (double)ix, dy = fc[1] - (double)iy, dz = fc[2] - (double)iz;
  double c000 = data[g.index(ix, iy, iz)], c100 = data[g.index(ix + 1, iy, iz)];
  double c010 = data[g.index(ix, iy + 1, iz)], c110 = data[g.index(ix + 1, iy + 1, iz)];
  double c001 = data[g.index(ix, iy, iz + 1)], c101 = data[g.index(ix + 1, iy, iz + 1)];
  double c011 = data[g.index(ix, iy + 1, iz + 1)], c111 = data[g.index(ix + 1, iy + 1, iz + 1)];
  double c00 = c000 * (1.0 - dx) + c100 * dx, c10 = c010 * (1.0 - dx) + c110 * dx;
  double c01 = c001 * (1.0 - dx) + c101 * dx, c11 = c011 * (1.0 - dx) + c111 * dx;
  double c0 = c00 * (1.0 - dy) + c10 * dy, c1 = c01 * (1.0 - dy) + c11 * dy;
  return c0 * (1.0 - dz) + c1 * dz;
}

// AtomSpatialHash, pb_grid.rs:319-442
struct SpatialHash {
  double inv = 1.0, origin[3] = {0, 0, 0};
  size_t gd[3] = {0, 0, 0};
  std::vector<std::vector<size_t>> cells;
  SpatialHash(const std::vector<V3>& x, double max_eff) {
    if (x.empty()) return;
    double cs = std::max(max_eff, 0.1);
    inv = 1.0 / cs;
    double mn[3] = {std::numeric_limits<double>::max(), std::numeric_limits<double>::max(),
                    std::numeric_limits<double>::max()};
    double mx[3] = {std::numeric_limits<double>::lowest(), std::numeric_limits<double>::lowest(),
                    std::numeric_limits<double>::lowest()};
    for (auto& c : x) {
      double v[3] = {c.x, c.y, c.z};
      for (int d = 0; d < 3; d++) {
        if (v[d] < mn[d]) mn[d] = v[d];
        if (v[d] > mx[d]) mx[d] = v[d];
      }
    }
    for (int d = 0; d < 3; d++) origin[d] = mn[d] - max_eff;
    for (int d = 0; d < 3; d++) gd[d] = (size_t)std::ceil((mx[d] - origin[d]) * inv) + 1;
    cells.assign(gd[0] * gd[1] * gd[2], {});
    for (size_t i = 0; i < x.size(); i++) {
      size_t cx = (size_t)((x[i].x - origin[0]) * inv);
      size_t cy = (size_t)((x[i].y - origin[1]) * inv);
      size_t cz = (size_t)((x[i].z - origin[2]) * inv);
      cells[cx + gd[0] * (cy + gd[1] * cz)].push_back(i);
    }
  }
  bool inside(const double* p, const std::vector<V3>& x, const std::vector<double>& radii,
              double probe) const {
    if (cells.empty()) return false;
    double fx = (p[0] - origin[0]) * inv, fy = (p[1] - origin[1]) * inv, fz = (p[2] - origin[2]) * inv;
    long cx = (long)fx, cy = (long)fy, cz = (long)fz;  // `as isize` truncates toward zero
    for (long dz = -1; dz <= 1; dz++) {
      long jz = cz + dz;
      if (jz < 0 || jz >= (long)gd[2]) continue;
      for (long dy = -1; dy <= 1; dy++) {
        long jy = cy + dy;
        if (jy < 0 || jy >= (long)gd[1]) continue;
        for (long dx = -1; dx <= 1; dx++) {
          long jx = cx + dx;
          if (jx < 0 || jx >= (long)gd[0]) continue;
          for (size_t a : cells[jx + gd[0] * (jy + gd[1] * jz)]) {
            double ddx = p[0] - x[a].x, ddy = p[1] - x[a].y, ddz = p[2] - x[a].z;
            double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
            double th = radii[a] + probe;
            if (d2 < th * th) return true;
          }
        }
      }
    }
    return false;
  }
};

// pb_grid.rs:450-498
static void edt_1d(double* f, size_t n, double* d, size_t* v, double* z) {
  if (n <= 1) return;
  size_t k = 0;
  v[0] = 0;
  z[0] = -std::numeric_limits<double>::infinity();
  z[1] = std::numeric_limits<double>::infinity();
  for (size_t q = 1; q < n; q++) {
    for (;;) {
      size_t vk = v[k];
      double s = (f[q] + (double)(q * q) - f[vk] - (double)(vk * vk)) / (double)(2 * (q - vk));
      if (s > z[k]) {
        k++;
        v[k] = q;
        z[k] = s;
        z[k + 1] = std::numeric_limits<double>::infinity();
        break;
      }
      if (k == 0) {
        v[0] = q;
        z[0] = -std::numeric_limits<double>::infinity();
        z[1] = std::numeric_limits<double>::infinity();
        break;
      }
      k--;
    }
  }
  k = 0;
  for (size_t q = 0; q < n; q++) {
    while (z[k + 1] < (double)q) k++;
    double diff = (double)q - (double)v[k];
    d[q] = diff * diff + f[v[k]];
  }
  memcpy(f, d, n * sizeof(double));
}

// pb_grid.rs:507-560
static void edt_3d(std::vector<double>& dist, const size_t* dims) {
  size_t nx = dims[0], ny = dims[1], nz = dims[2];
  size_t m = std::max(nx, std::max(ny, nz));
  std::vector<double> d(m), z(m + 1), col(m);
  std::vector<size_t> v(m);
  for (size_t iz = 0; iz < nz; iz++)
    for (size_t iy = 0; iy < ny; iy++) edt_1d(&dist[iy * nx + iz * nx * ny], nx, d.data(), v.data(), z.data());
  for (size_t iz = 0; iz < nz; iz++)
    for (size_t ix = 0; ix < nx; ix++) {
      for (size_t iy = 0; iy < ny; iy++) col[iy] = dist[ix + nx * (iy + ny * iz)];
      edt_1d(col.data(), ny, d.data(), v.data(), z.data());
      for (size_t iy = 0; iy < ny; iy++) dist[ix + nx * (iy + ny * iz)] = col[iy];
    }
  for (size_t iy = 0; iy < ny; iy++)
    for (size_t ix = 0; ix < nx; ix++) {
      size_t base = ix + nx * iy, st = nx * ny;
      for (size_t iz = 0; iz < nz; iz++) col[iz] = dist[base + st * iz];
      edt_1d(col.data(), nz, d.data(), v.data(), z.data());
      for (size_t iz = 0; iz < nz; iz++) dist[base + st * iz] = col[iz];
    }
}

// pb_grid.rs:576-708
std::vector<uint8_t> inside_ses(const Grid& g, const std::vector<V3>& x, const std::vector<double>& radii,
                                double probe) {
  size_t nx = g.dims[0], ny = g.dims[1], nz = g.dims[2], n = nx * ny * nz;
  double maxr = 0.0;
  for (double r : radii) maxr = std::max(maxr, r);
  double max_eff = maxr + std::max(probe, 0.0);
  SpatialHash hash(x, max_eff);
  std::vector<uint8_t> out(n);
  if (probe <= 0.0) {
#pragma omp parallel for
    for (long idx = 0; idx < (long)n; idx++) {
      size_t iz = idx / (nx * ny), iy = (idx % (nx * ny)) / nx, ix = idx % nx;
      double p[3];
      g.point(ix, iy, iz, p);
      out[idx] = hash.inside(p, x, radii, 0.0);
    }
    return out;
  }
  std::vector<uint8_t> sas(n);
#pragma omp parallel for
  for (long idx = 0; idx < (long)n; idx++) {
    size_t iz = idx / (nx * ny), iy = (idx % (nx * ny)) / nx, ix = idx % nx;
    double p[3];
    g.point(ix, iy, iz, p);
    sas[idx] = hash.inside(p, x, radii, probe);
  }
  std::vector<uint8_t> ext(n, 0);
  std::deque<size_t> qu;
  for (size_t iz = 0; iz < nz; iz++)
    for (size_t iy = 0; iy < ny; iy++)
      for (size_t ix = 0; ix < nx; ix++) {
        bool bd = ix == 0 || ix == nx - 1 || iy == 0 || iy == ny - 1 || iz == 0 || iz == nz - 1;
        if (bd) {
          size_t idx = g.index(ix, iy, iz);
          if (!sas[idx]) {
            ext[idx] = 1;
            qu.push_back(idx);
          }
        }
      }
  while (!qu.empty()) {
    size_t idx = qu.front();
    qu.pop_front();
    size_t iz = idx / (nx * ny), iy = (idx % (nx * ny)) / nx, ix = idx % nx;
    size_t nb[6];
    int c = 0;
    if (ix > 0) nb[c++] = g.index(ix - 1, iy, iz);
    if (ix + 1 < nx) nb[c++] = g.index(ix + 1, iy, iz);
    if (iy > 0) nb[c++] = g.index(ix, iy - 1, iz);
    if (iy + 1 < ny) nb[c++] = g.index(ix, iy + 1, iz);
    if (iz > 0) nb[c++] = g.index(ix, iy, iz - 1);
    if (iz + 1 < nz) nb[c++] = g.index(ix, iy, iz + 1);
    for (int k = 0; k < c; k++)
      if (!ext[nb[k]] && !sas[nb[k]]) {
        ext[nb[k]] = 1;
        qu.push_back(nb[k]);
      }
  }
  double h = g.h[0];
  double thr = (probe / h) * (probe / h);
  double big = (double)n * 2.0;
  std::vector<double> dist(n);
  for (size_t i = 0; i < n; i++) dist[i] = ext[i] ? 0.0 : big;
  edt_3d(dist, g.dims);
  for (size_t i = 0; i < n; i++) out[i] = dist[i] > thr;
  return out;
}

// pb_grid.rs:717-801
double fraction_inside(double lo, double hi, double p1, double p2, int axis, const std::vector<V3>& x,
                       const std::vector<double>& radii, double probe) {
  double len = hi - lo;
  if (len <= 0.0) return 0.0;
  int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
  std::vector<std::pair<double, double>> iv;
  for (size_t a = 0; a < x.size(); a++) {
    double c[3] = {x[a].x, x[a].y, x[a].z};
    double R = radii[a] + probe;
    double d1 = p1 - c[a1], d2 = p2 - c[a2];
    double rs = R * R - d1 * d1 - d2 * d2;
    if (rs <= 0.0) continue;
    double rho = std::sqrt(rs);
    double ilo = std::max(c[axis] - rho, lo), ihi = std::min(c[axis] + rho, hi);
    if (ilo < ihi) iv.push_back({ilo, ihi});
  }
  if (iv.empty()) return 0.0;
  std::sort(iv.begin(), iv.end(), [](const std::pair<double, double>& A, const std::pair<double, double>& B) {
    return A.first < B.first;
  });
  double total = 0.0, clo = iv[0].first, chi = iv[0].second;
  for (size_t k = 1; k < iv.size(); k++) {
    if (iv[k].first <= chi) {
      chi = std::max(chi, iv[k].second);
    } else {
      total += chi - clo;
      clo = iv[k].first;
      chi = iv[k].second;
    }
  }
  total += chi - clo;
  return std::min(1.0, std::max(0.0, total / len));
}

static inline double harmonic_eps(double f, double ein, double eout) {  // pb_grid.rs:809-817
  if (f <= 0.0) return eout;
  if (f >= 1.0) return ein;
  return 1.0 / (f / ein + (1.0 - f) / eout);
}

// pb_grid.rs:827-940
Diel assign_dielectrics(const Grid& g, const std::vector<V3>& x, const std::vector<double>& radii,
                        double probe, double ein, double eout) {
  size_t nx = g.dims[0], ny = g.dims[1], nz = g.dims[2], n = nx * ny * nz;
  Diel D;
  if (std::fabs(ein - eout) < std::numeric_limits<double>::epsilon()) {
    D.ex.assign(n, ein);
    D.ey.assign(n, ein);
    D.ez.assign(n, ein);
    return D;
  }
  std::vector<uint8_t> in = inside_ses(g, x, radii, probe);
  D.ex.assign(n, eout);
  D.ey.assign(n, eout);
  D.ez.assign(n, eout);
#pragma omp parallel for schedule(dynamic, 1)
  for (long izl = 0; izl < (long)nz; izl++) {
    size_t iz = (size_t)izl;
    for (size_t iy = 0; iy < ny; iy++)
      for (size_t ix = 0; ix < nx; ix++) {
        size_t idx = g.index(ix, iy, iz);
        bool a = in[idx];
        double p[3];
        g.point(ix, iy, iz, p);
        if (ix + 1 < nx) {
          bool b = in[g.index(ix + 1, iy, iz)];
          D.ex[idx] = a == b ? (a ? ein : eout)
                             : harmonic_eps(fraction_inside(p[0], p[0] + g.h[0], p[1], p[2], 0, x, radii, 0.0),
                                            ein, eout);
        }
        if (iy + 1 < ny) {
          bool b = in[g.index(ix, iy + 1, iz)];
          D.ey[idx] = a == b ? (a ? ein : eout)
                             : harmonic_eps(fraction_inside(p[1], p[1] + g.h[1], p[0], p[2], 1, x, radii, 0.0),
                                            ein, eout);
        }
        if (iz + 1 < nz) {
          bool b = in[g.index(ix, iy, iz + 1)];
          D.ez[idx] = a == b ? (a ? ein : eout)
                             : harmonic_eps(fraction_inside(p[2], p[2] + g.h[2], p[0], p[1], 2, x, radii, 0.0),
                                            ein, eout);
        }
      }
  }
  return D;
}

// pb_grid.rs:951-985
std::vector<double> assign_kappa(const Grid& g, const std::vector<V3>& x, const std::vector<double>& radii,
                                 double ion_radius, double kbulk, double eps_s) {
  size_t nx = g.dims[0], ny = g.dims[1], n = g.len();
  double kbs = eps_s * kbulk * kbulk;
  double maxr = 0.0;
  for (double r : radii) maxr = std::max(maxr, r);
  SpatialHash hash(x, maxr + ion_radius);
  std::vector<double> out(n);
#pragma omp parallel for
  for (long idx = 0; idx < (long)n; idx++) {
    size_t iz = idx / (nx * ny), iy = (idx % (nx * ny)) / nx, ix = idx % nx;
    double p[3];
    g.point(ix, iy, iz, p);
    out[idx] = hash.inside(p, x, radii, ion_radius) ? 0.0 : kbs;
  }
  return out;
}

// pb_solver.rs:31-60 (same visiting order)
template <class F>
static void for_each_boundary(const size_t* d, F f) {
  size_t nx = d[0], ny = d[1], nz = d[2];
  for (size_t iz : {(size_t)0, nz - 1})
    for (size_t iy = 0; iy < ny; iy++)
      for (size_t ix = 0; ix < nx; ix++) f(ix, iy, iz);
  for (size_t iz = 1; iz + 1 < nz; iz++)
    for (size_t iy : {(size_t)0, ny - 1})
      for (size_t ix = 0; ix < nx; ix++) f(ix, iy, iz);
  for (size_t iz = 1; iz + 1 < nz; iz++)
    for (size_t iy = 1; iy + 1 < ny; iy++)
      for (size_t ix : {(size_t)0, nx - 1}) f(ix, iy, iz);
}

// pb_solver.rs:68-93
void set_dh_boundary(std::vector<double>& phi, const Grid& g, const std::vector<V3>& x,
                     const std::vector<double>& q, double kap, double eout) {
  const double conv = 332.0522;
  std::vector<size_t> pts;
  for_each_boundary(g.dims, [&](size_t ix, size_t iy, size_t iz) { pts.push_back(g.index(ix, iy, iz)); });
  size_t nx = g.dims[0], ny = g.dims[1];
#pragma omp parallel for schedule(static)
  for (long k = 0; k < (long)pts.size(); k++) {
    size_t idx = pts[k];
    size_t iz = idx / (nx * ny), iy = (idx % (nx * ny)) / nx, ix = idx % nx;
    double p[3];
    g.point(ix, iy, iz, p);
    double s = 0.0;
    for (size_t a = 0; a < x.size(); a++) {
      double dx = p[0] - x[a].x, dy = p[1] - x[a].y, dz = p[2] - x[a].z;
      double r = std::sqrt(dx * dx + dy * dy + dz * dz);
      if (r > 1e-10) s += conv * q[a] * std::exp(-kap * r) / (eout * r);
    }
    phi[idx] = s;
  }
}

static double spectral_radius(const size_t* d) {  // pb_solver.rs:124-132
  return (std::cos(PI / (double)d[0]) + std::cos(PI / (double)d[1]) + std::cos(PI / (double)d[2])) / 3.0;
}
double estimate_omega(const size_t* d) {  // pb_solver.rs:135-139
  double r = spectral_radius(d);
  return 2.0 / (1.0 + std::sqrt(1.0 - r * r));
}

struct Op {
  size_t d[3];
  double h[3];
  const double *ex, *ey, *ez, *k2;
};

static inline void stencil(const Op& o, const double* phi, size_t idx, double ihx, double ihy, double ihz,
                           double& nsum, double& diag) {
  // pb_solver.rs:162-194
  size_t sy = o.d[0], sz = o.d[0] * o.d[1];
  double exp_ = o.ex[idx], exm = o.ex[idx - 1], eyp = o.ey[idx], eym = o.ey[idx - sy], ezp = o.ez[idx],
         ezm = o.ez[idx - sz];
  nsum = (exp_ * phi[idx + 1] + exm * phi[idx - 1]) * ihx + (eyp * phi[idx + sy] + eym * phi[idx - sy]) * ihy +
         (ezp * phi[idx + sz] + ezm * phi[idx - sz]) * ihz;
  diag = (exp_ + exm) * ihx + (eyp + eym) * ihy + (ezp + ezm) * ihz + o.k2[idx];
}

// pb_solver.rs:214-327.  Red-black update (order within a colour does not
// matter: each update reads only opposite-colour neighbours).
double sor_smooth(const Op& o, double* phi, const double* rho, double omega, size_t sweeps, double rhs_scale) {
  size_t nx = o.d[0], ny = o.d[1], nz = o.d[2];
  double ihx = 1.0 / (o.h[0] * o.h[0]), ihy = 1.0 / (o.h[1] * o.h[1]), ihz = 1.0 / (o.h[2] * o.h[2]);
  double last = 0.0;
  for (size_t s = 0; s < sweeps; s++) {
    double rms = 0.0;
    uint64_t cnt = 0;
    for (size_t color = 0; color < 2; color++) {
      std::vector<double> part(nz, 0.0);
      std::vector<uint64_t> pc(nz, 0);
#pragma omp parallel for schedule(static)
      for (long izl = 1; izl < (long)nz - 1; izl++) {
        size_t iz = (size_t)izl;
        double lr = 0.0;
        uint64_t lc = 0;
        for (size_t iy = 1; iy + 1 < ny; iy++) {
          size_t x0 = 1 + ((1 + iy + iz + color) % 2);
          for (size_t ix = x0; ix + 1 < nx; ix += 2) {
            size_t idx = ix + nx * iy + nx * ny * iz;
            double ns, dg;
            stencil(o, phi, idx, ihx, ihy, ihz, ns, dg);
            double rhs = rhs_scale * rho[idx];
            double gs = (ns + rhs) / dg;
            double nw = phi[idx] + omega * (gs - phi[idx]);
            double res = gs - phi[idx];
            lr += res * res;
            lc++;
            phi[idx] = nw;
          }
        }
        part[iz] = lr;
        pc[iz] = lc;
      }
      for (size_t iz = 0; iz < nz; iz++) {
        rms += part[iz];
        cnt += pc[iz];
      }
    }
    last = cnt > 0 ? std::sqrt(rms / (double)cnt) : 0.0;
  }
  return last;
}

// pb_solver.rs:453-509
static void residual_into(const Op& o, const double* phi, const double* rho, double rhs_scale, double* out) {
  size_t nx = o.d[0], ny = o.d[1], nz = o.d[2];
  double ihx = 1.0 / (o.h[0] * o.h[0]), ihy = 1.0 / (o.h[1] * o.h[1]), ihz = 1.0 / (o.h[2] * o.h[2]);
  memset(out, 0, sizeof(double) * nx * ny * nz);
#pragma omp parallel for schedule(static)
  for (long izl = 1; izl < (long)nz - 1; izl++) {
    size_t iz = (size_t)izl;
    for (size_t iy = 1; iy + 1 < ny; iy++)
      for (size_t ix = 1; ix + 1 < nx; ix++) {
        size_t idx = ix + nx * iy + nx * ny * iz;
        double ns, dg;
        stencil(o, phi, idx, ihx, ihy, ihz, ns, dg);
        out[idx] = rhs_scale * rho[idx] + ns - dg * phi[idx];
      }
  }
}

// pb_solver.rs:578-624
void restrict_into(const double* fine, const size_t* fd, double* coarse, const size_t* cd, double scale) {
  long fnx = (long)fd[0], fny = (long)fd[1], fnz = (long)fd[2];
#pragma omp parallel for schedule(static)
  for (long cz = 0; cz < (long)cd[2]; cz++)
    for (size_t cy = 0; cy < cd[1]; cy++)
      for (size_t cx = 0; cx < cd[0]; cx++) {
        long fx = 2 * (long)cx, fy = 2 * (long)cy, fz = 2 * cz;
        double sum = 0.0, ws = 0.0;
        for (int dz = -1; dz <= 1; dz++)
          for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
              long ix = fx + dx, iy = fy + dy, iz = fz + dz;
              if (ix < 0 || ix >= fnx || iy < 0 || iy >= fny || iz < 0 || iz >= fnz) continue;
              double w = (dx == 0 ? 2.0 : 1.0) * (dy == 0 ? 2.0 : 1.0) * (dz == 0 ? 2.0 : 1.0);
              sum += w * fine[ix + fnx * (iy + fny * iz)];
              ws += w;
            }
        coarse[cx + cd[0] * (cy + cd[1] * cz)] = scale * sum / ws;
      }
}

// pb_solver.rs:628-681
void prolongate_add(const double* coarse, const size_t* cd, double* fine, const size_t* fd) {
  size_t cnx = cd[0], cny = cd[1], cnz = cd[2];
  auto ci = [&](size_t x, size_t y, size_t z) { return x + cnx * (y + cny * z); };
  size_t mx = cnx >= 2 ? cnx - 2 : 0, my = cny >= 2 ? cny - 2 : 0, mz = cnz >= 2 ? cnz - 2 : 0;
#pragma omp parallel for schedule(static)
  for (long fzl = 0; fzl < (long)fd[2]; fzl++) {
    size_t fz = (size_t)fzl;
    for (size_t fy = 0; fy < fd[1]; fy++)
      for (size_t fx = 0; fx < fd[0]; fx++) {
        double cxf = (double)fx / 2.0, cyf = (double)fy / 2.0, czf = (double)fz / 2.0;
        size_t x0 = std::min((size_t)std::floor(cxf), mx), y0 = std::min((size_t)std::floor(cyf), my),
               z0 = std::min((size_t)std::floor(czf), mz);
        double dx = cxf - (double)x0, dy = cyf - (double)y0, dz = czf - (double)z0;
        double c000 = coarse[ci(x0, y0, z0)], c100 = coarse[ci(x0 + 1, y0, z0)];
        double c010 = coarse[ci(x0, y0 + 1, z0)], c110 = coarse[ci(x0 + 1, y0 + 1, z0)];
        double c001 = coarse[ci(x0, y0, z0 + 1)], c101 = coarse[ci(x0 + 1, y0, z0 + 1)];
        double c011 = coarse[ci(x0, y0 + 1, z0 + 1)], c111 = coarse[ci(x0 + 1, y0 + 1, z0 + 1)];
        double c00 = c000 * (1.0 - dx) + c100 * dx, c10 = c010 * (1.0 - dx) + c110 * dx;
        double c01 = c001 * (1.0 - dx) + c101 * dx, c11 = c011 * (1.0 - dx) + c111 * dx;
        double c0 = c00 * (1.0 - dy) + c10 * dy, c1 = c01 * (1.0 - dy) + c11 * dy;
        fine[fx + fd[0] * (fy + fd[1] * fz)] += c0 * (1.0 - dz) + c1 * dz;
      }
  }
}

// pb_solver.rs:684-748 (injection)
static void coarsen(const double* f, const size_t* fd, double* c, const size_t* cd) {
  for (size_t cz = 0; cz < cd[2]; cz++)
    for (size_t cy = 0; cy < cd[1]; cy++)
      for (size_t cx = 0; cx < cd[0]; cx++) {
        size_t fx = std::min(2 * cx, fd[0] - 1), fy = std::min(2 * cy, fd[1] - 1), fz = std::min(2 * cz, fd[2] - 1);
        c[cx + cd[0] * (cy + cd[1] * cz)] = f[fx + fd[0] * (fy + fd[1] * fz)];
      }
}

// Coarse face dielectrics of the converged solves' multigrid (the reference
// injects, pb_solver.rs:684-748): a coarse face spans two fine faces in
// series along its axis (harmonic mean; equal values are copied) and, across
// it, the fine faces of the 3 x 3 neighbouring lines in parallel (weights
// 1-2-1 in each transverse direction, renormalised at the grid edge).
static void coarsen_face(const double* f, const size_t* fd, double* c, const size_t* cd, int axis) {
  long n[3] = {(long)fd[0], (long)fd[1], (long)fd[2]};
  int t1 = (axis + 1) % 3, t2 = (axis + 2) % 3;
  for (size_t cz = 0; cz < cd[2]; cz++)
    for (size_t cy = 0; cy < cd[1]; cy++)
      for (size_t cx = 0; cx < cd[0]; cx++) {
        long b[3] = {std::min(2 * (long)cx, n[0] - 1), std::min(2 * (long)cy, n[1] - 1),
                     std::min(2 * (long)cz, n[2] - 1)};
        double sum = 0.0, ws = 0.0, first = 0.0;
        bool same = true, any = false;
        for (int u = -1; u <= 1; u++)
          for (int v = -1; v <= 1; v++) {
            long p[3] = {b[0], b[1], b[2]};
            p[t1] += u;
            p[t2] += v;
            if (p[t1] < 0 || p[t1] >= n[t1] || p[t2] < 0 || p[t2] >= n[t2]) continue;
            long q1[3] = {p[0], p[1], p[2]};
            q1[axis] = std::min(p[axis] + 1, n[axis] - 1);
            double e0 = f[p[0] + n[0] * (p[1] + n[1] * p[2])], e1 = f[q1[0] + n[0] * (q1[1] + n[1] * q1[2])];
            if (!any) first = e0;
            any = true;
            same = same && e0 == first && e1 == first;
            double w = (u == 0 ? 2.0 : 1.0) * (v == 0 ? 2.0 : 1.0);
            sum += w * (e0 == e1 ? e0 : 2.0 / (1.0 / e0 + 1.0 / e1));
            ws += w;
          }
        c[cx + cd[0] * (cy + cd[1] * cz)] = same ? first : sum / ws;
      }
}

struct Level {
  size_t cd[3], fd[3];
  double ch[3];
  std::vector<double> ex, ey, ez, k2, fres, crhs, ccorr;
  double omega;
};

// pb_solver.rs:776-836
static std::vector<Level> build_levels(const Op& top, size_t min_size, bool series_parallel = false) {
  std::vector<Level> L;
  size_t d[3] = {top.d[0], top.d[1], top.d[2]};
  double h[3] = {top.h[0], top.h[1], top.h[2]};
  const double *ex = top.ex, *ey = top.ey, *ez = top.ez, *k2 = top.k2;
  for (;;) {
    size_t md = std::min(d[0], std::min(d[1], d[2]));
    if (md <= min_size) break;
    Level lv;
    for (int k = 0; k < 3; k++) {
      lv.fd[k] = d[k];
      lv.cd[k] = (d[k] + 1) / 2;
      lv.ch[k] = h[k] * 2.0;
    }
    size_t cn = lv.cd[0] * lv.cd[1] * lv.cd[2], fn = d[0] * d[1] * d[2];
    lv.ex.resize(cn);
    lv.ey.resize(cn);
    lv.ez.resize(cn);
    lv.k2.resize(cn);
    if (series_parallel) {
      coarsen_face(ex, d, lv.ex.data(), lv.cd, 0);
      coarsen_face(ey, d, lv.ey.data(), lv.cd, 1);
      coarsen_face(ez, d, lv.ez.data(), lv.cd, 2);
    } else {
      coarsen(ex, d, lv.ex.data(), lv.cd);
      coarsen(ey, d, lv.ey.data(), lv.cd);
      coarsen(ez, d, lv.ez.data(), lv.cd);
    }
    coarsen(k2, d, lv.k2.data(), lv.cd);
    lv.omega = series_parallel ? 1.0 : estimate_omega(lv.cd);
    lv.fres.assign(fn, 0.0);
    lv.crhs.assign(cn, 0.0);
    lv.ccorr.assign(cn, 0.0);
    L.push_back(std::move(lv));
    Level& b = L.back();
    ex = b.ex.data();
    ey = b.ey.data();
    ez = b.ez.data();
    k2 = b.k2.data();
    for (int k = 0; k < 3; k++) {
      d[k] = b.cd[k];
      h[k] = b.ch[k];
    }
  }
  return L;
}

// pb_solver.rs:842-939
static void v_cycle(const Op& o, double* phi, const double* rho, double omega, Level* L, size_t nl, size_t pre,
                    size_t post, double rhs_scale, double rscale = 0.25) {
  if (nl == 0) {
    sor_smooth(o, phi, rho, omega, 50, rhs_scale);
    return;
  }
  Level& lv = L[0];
  sor_smooth(o, phi, rho, omega, pre, rhs_scale);
  residual_into(o, phi, rho, rhs_scale, lv.fres.data());
  restrict_into(lv.fres.data(), lv.fd, lv.crhs.data(), lv.cd, rscale);
  std::fill(lv.ccorr.begin(), lv.ccorr.end(), 0.0);
  Op co;
  for (int k = 0; k < 3; k++) {
    co.d[k] = lv.cd[k];
    co.h[k] = lv.ch[k];
  }
  co.ex = lv.ex.data();
  co.ey = lv.ey.data();
  co.ez = lv.ez.data();
  co.k2 = lv.k2.data();
  v_cycle(co, lv.ccorr.data(), lv.crhs.data(), lv.omega, L + 1, nl - 1, pre, post, 1.0, rscale);
  prolongate_add(lv.ccorr.data(), lv.cd, phi, o.d);
  sor_smooth(o, phi, rho, omega, post, rhs_scale);
}

// pb_solver.rs:946-1009
double rms_residual(const Op& o, const double* phi, const double* rho, double rhs_scale) {
  size_t nx = o.d[0], ny = o.d[1], nz = o.d[2];
  double ihx = 1.0 / (o.h[0] * o.h[0]), ihy = 1.0 / (o.h[1] * o.h[1]), ihz = 1.0 / (o.h[2] * o.h[2]);
  std::vector<double> part(nz, 0.0);
#pragma omp parallel for schedule(static)
  for (long izl = 1; izl < (long)nz - 1; izl++) {
    size_t iz = (size_t)izl;
    double s = 0.0;
    for (size_t iy = 1; iy + 1 < ny; iy++)
      for (size_t ix = 1; ix + 1 < nx; ix++) {
        size_t idx = ix + nx * iy + nx * ny * iz;
        double ns, dg;
        stencil(o, phi, idx, ihx, ihy, ihz, ns, dg);
        double r = rhs_scale * rho[idx] + ns - dg * phi[idx];
        s += r * r;
      }
    part[iz] = s;
  }
  double s = 0.0;
  for (double v : part) s += v;
  uint64_t cnt = (nx >= 2 && ny >= 2 && nz >= 2) ? (uint64_t)(nx - 2) * (ny - 2) * (nz - 2) : 0;
  return cnt > 0 ? std::sqrt(s / (double)cnt) : 0.0;
}

static void apply_bc(std::vector<double>& phi, const Grid& g, const BC& bc, const std::vector<V3>& x,
                     const std::vector<double>& q, double kb, double eout) {
  if (bc.kind == 1)
    set_dh_boundary(phi, g, x, q, kb, eout);
  else if (bc.kind == 2)
    for (auto& pv : bc.values) phi[pv.first] = pv.second;
}

// pb_solver.rs:373-447 (Chebyshev-ramped SOR)
static SolveResult solve_sor(const Grid& g, const Op& o, const double* rho, const BC& bc, const std::vector<V3>& x,
                             const std::vector<double>& q, double kb, double eout, double tol, size_t maxit,
                             std::vector<double>* init) {
  SolveResult R;
  R.phi = init ? std::move(*init) : std::vector<double>(g.len(), 0.0);
  apply_bc(R.phi, g, bc, x, q, kb, eout);
  double rj = spectral_radius(g.dims), rs = rj * rj, om = 1.0;
  R.residual = std::numeric_limits<double>::max();
  for (size_t it = 0; it < maxit; it++) {
    R.residual = sor_smooth(o, R.phi.data(), rho, om, 1, FOUR_PI_EC);
    R.iterations = it + 1;
    om = (it == 0) ? 1.0 / (1.0 - rs / 2.0) : 1.0 / (1.0 - rs * om / 4.0);
    if (R.residual < tol) {
      R.converged = true;
      return R;
    }
  }
  return R;
}

// pb_solver.rs:1015-1167
SolveResult solve_multigrid(const Grid& g, const std::vector<double>& rho, const Diel& D,
                            const std::vector<double>& k2, const BC& bc, const std::vector<V3>& x,
                            const std::vector<double>& q, double kb, double eout, double tol, size_t maxit) {
  Op o;
  for (int k = 0; k < 3; k++) {
    o.d[k] = g.dims[k];
    o.h[k] = g.h[k];
  }
  o.ex = D.ex.data();
  o.ey = D.ey.data();
  o.ez = D.ez.data();
  o.k2 = k2.data();
  SolveResult R;
  R.phi.assign(g.len(), 0.0);
  apply_bc(R.phi, g, bc, x, q, kb, eout);
  size_t md = std::min(g.dims[0], std::min(g.dims[1], g.dims[2]));
  if (md <= 8) return solve_sor(g, o, rho.data(), bc, x, q, kb, eout, tol, maxit, nullptr);
  size_t maxv = std::min<size_t>(std::max<size_t>(maxit / 6, 1), 200);
  std::vector<Level> L = build_levels(o, 5);
  double omega = estimate_omega(g.dims);
  double best = std::numeric_limits<double>::max(), prev = std::numeric_limits<double>::max();
  uint32_t growing = 0;
  for (size_t cyc = 0; cyc < maxv; cyc++) {
    v_cycle(o, R.phi.data(), rho.data(), omega, L.data(), L.size(), 3, 3, FOUR_PI_EC);
    double r = rms_residual(o, R.phi.data(), rho.data(), FOUR_PI_EC);
    if (r < best) {
      best = r;
      growing = 0;
    } else {
      growing++;
    }
    bool div = !std::isfinite(r) || r > best * 1e4 || (growing >= 5 && r > prev);
    if (div) {
      SolveResult S = solve_sor(g, o, rho.data(), bc, x, q, kb, eout, tol, maxit, &R.phi);
      S.diverged = true;
      return S;
    }
    prev = r;
    if (r < tol) {
      R.iterations = cyc + 1;
      R.residual = r;
      R.converged = true;
      return R;
    }
  }
  R.residual = rms_residual(o, R.phi.data(), rho.data(), FOUR_PI_EC);
  R.iterations = maxv;
  R.converged = false;
  return R;
}

// ---------------------------------------------------------------------------
// Converged solves (not part of the reference's schedule).  The reference
// stops its V-cycles on an absolute RMS residual or after at most 200 cycles
// (pb_solver.rs:1066, 1093-1141); on solvated grids of realistic size that
// cap is reached long before the discrete system is solved.  These solvers
// give the converged solution of the same discrete system (same maps, same
// boundary values, same 7-point operator), the error reference for solvers
// that stop on a relative residual.  The interior unknowns solve A phi = f,
// A = -div eps grad + kbar^2, symmetric positive definite (the face
// dielectric between two points is one value used by both rows); boundary
// values are fixed.  Relative residual = ||f - A phi||_2 / ||f - A phi_0||_2
// over interior points, phi_0 = the initial potential (zero inside,
// boundary values set).  The multigrid of methods 1 and 2 is a consistent
// one, unlike the reference's: red-black Gauss-Seidel smoothing (omega 1,
// 3 + 3 sweeps, 50 on the coarsest level), full-weighting restriction
// without the 0.25 factor, series/parallel coarse dielectrics, kbar^2
// injected, corrections zero on the boundary.
//   method 0: conjugate gradients, diagonal (Jacobi) preconditioner --
//             independent of any multigrid hierarchy;
//   method 1: flexible conjugate gradients (Polak-Ribiere form) with one
//             V-cycle on the residual equation as the preconditioner;
//   method 2: defect correction phi += V-cycle(f - A phi), the iteration
//             of the GPU engine's relative-residual mode, here in FP64.
static double dot_int(const Op& o, const double* a, const double* b) {
  size_t nx = o.d[0], ny = o.d[1], nz = o.d[2];
  std::vector<double> part(nz, 0.0);
#pragma omp parallel for schedule(static)
  for (long izl = 1; izl < (long)nz - 1; izl++) {
    size_t iz = (size_t)izl;
    double s = 0.0;
    for (size_t iy = 1; iy + 1 < ny; iy++)
      for (size_t ix = 1; ix + 1 < nx; ix++) {
        size_t idx = ix + nx * iy + nx * ny * iz;
        s += a[idx] * b[idx];
      }
    part[iz] = s;
  }
  double s = 0.0;
  for (double v : part) s += v;
  return s;
}

// q = A v at interior points, v taken as zero on the boundary
static void apply_op(const Op& o, const double* v, double* q) {
  size_t nx = o.d[0], ny = o.d[1], nz = o.d[2];
  double ihx = 1.0 / (o.h[0] * o.h[0]), ihy = 1.0 / (o.h[1] * o.h[1]), ihz = 1.0 / (o.h[2] * o.h[2]);
#pragma omp parallel for schedule(static)
  for (long izl = 1; izl < (long)nz - 1; izl++) {
    size_t iz = (size_t)izl;
    for (size_t iy = 1; iy + 1 < ny; iy++)
      for (size_t ix = 1; ix + 1 < nx; ix++) {
        size_t idx = ix + nx * iy + nx * ny * iz;
        double ns, dg;
        stencil(o, v, idx, ihx, ihy, ihz, ns, dg);
        q[idx] = dg * v[idx] - ns;
      }
  }
}

static void zero_boundary(const Op& o, double* v) {
  size_t nx = o.d[0], ny = o.d[1], nz = o.d[2];
  for (size_t iz = 0; iz < nz; iz++)
    for (size_t iy = 0; iy < ny; iy++)
      for (size_t ix = 0; ix < nx; ix++)
        if (ix == 0 || iy == 0 || iz == 0 || ix + 1 == nx || iy + 1 == ny || iz + 1 == nz)
          v[ix + nx * iy + nx * ny * iz] = 0.0;
}

SolveResult solve_converged(const Grid& g, const std::vector<double>& rho, const Diel& D,
                            const std::vector<double>& k2, const BC& bc, const std::vector<V3>& x,
                            const std::vector<double>& q, double kb, double eout, double rel_tol, size_t maxit,
                            int method) {
  Op o;
  for (int k = 0; k < 3; k++) {
    o.d[k] = g.dims[k];
    o.h[k] = g.h[k];
  }
  o.ex = D.ex.data();
  o.ey = D.ey.data();
  o.ez = D.ez.data();
  o.k2 = k2.data();
  SolveResult R;
  R.phi.assign(g.len(), 0.0);
  apply_bc(R.phi, g, bc, x, q, kb, eout);
  size_t n = g.len();
  std::vector<double> r(n, 0.0), z(n, 0.0), p(n, 0.0), Ap(n, 0.0), rold(n, 0.0), diag(n, 1.0);
  residual_into(o, R.phi.data(), rho.data(), FOUR_PI_EC, r.data());
  double r0 = std::sqrt(dot_int(o, r.data(), r.data()));
  R.residual = r0 > 0.0 ? 1.0 : 0.0;
  if (r0 == 0.0) {
    R.converged = true;
    return R;
  }
  size_t md = std::min(g.dims[0], std::min(g.dims[1], g.dims[2]));
  bool mg = method >= 1 && md > 8;
  std::vector<Level> L;
  if (mg) L = build_levels(o, 5, true);
  if (!mg) {
    size_t nx = o.d[0], ny = o.d[1];
    double ihx = 1.0 / (o.h[0] * o.h[0]), ihy = 1.0 / (o.h[1] * o.h[1]), ihz = 1.0 / (o.h[2] * o.h[2]);
    for (size_t iz = 1; iz + 1 < o.d[2]; iz++)
      for (size_t iy = 1; iy + 1 < ny; iy++)
        for (size_t ix = 1; ix + 1 < nx; ix++) {
          size_t idx = ix + nx * iy + nx * ny * iz;
          double ns, dg;
          stencil(o, R.phi.data(), idx, ihx, ihy, ihz, ns, dg);
          diag[idx] = dg;
        }
  }
  bool krylov = method != 2 || !mg;
  double rz_old = 0.0;
  for (size_t it = 0; it < maxit; it++) {
    if (mg) {
      std::fill(z.begin(), z.end(), 0.0);
      v_cycle(o, z.data(), r.data(), 1.0, L.data(), L.size(), 3, 3, 1.0, 1.0);
    } else {
      for (size_t i = 0; i < n; i++) z[i] = r[i] / diag[i];
    }
    zero_boundary(o, z.data());
    R.iterations = it + 1;
    if (!krylov) {
      for (size_t i = 0; i < n; i++) R.phi[i] += z[i];
      residual_into(o, R.phi.data(), rho.data(), FOUR_PI_EC, r.data());
    } else {
      double rz = dot_int(o, r.data(), z.data());
      if (it == 0) {
        p = z;
      } else {
        // Polak-Ribiere: CG for a fixed symmetric preconditioner, stable for a
        // variable or non-symmetric one (flexible CG)
        double beta = (rz - dot_int(o, rold.data(), z.data())) / rz_old;
        for (size_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
      }
      apply_op(o, p.data(), Ap.data());
      double alpha = rz / dot_int(o, p.data(), Ap.data());
      rold = r;
      for (size_t i = 0; i < n; i++) {
        R.phi[i] += alpha * p[i];
        r[i] -= alpha * Ap[i];
      }
      rz_old = rz;
    }
    double rel = std::sqrt(dot_int(o, r.data(), r.data())) / r0;
    if (krylov && (rel < rel_tol || (it + 1) % 50 == 0)) {  // the recurrence drifts: true residual
      residual_into(o, R.phi.data(), rho.data(), FOUR_PI_EC, r.data());
      rel = std::sqrt(dot_int(o, r.data(), r.data())) / r0;
    }
    R.residual = rel;
    if (!std::isfinite(rel)) break;
    if (rel < rel_tol) {
      R.converged = true;
      return R;
    }
  }
  return R;
}

// pb_solver.rs:1174-1186
double elec_energy(const Grid& g, const std::vector<double>& phi, const std::vector<V3>& x,
                   const std::vector<double>& q) {
  double e = 0.0;
  for (size_t a = 0; a < x.size(); a++) {
    double p[3] = {x[a].x, x[a].y, x[a].z};
    e += q[a] * interpolate(g, p, phi);
  }
  return 0.5 * e;
}

// pb_energy.rs:134-322
static double solve_focus(const Grid& fg, const std::vector<double>& fq, const Grid* cg, const std::vector<V3>& x,
                          const std::vector<double>& q, const std::vector<double>& radii, const PbParams& p,
                          double ein, double eout, double kap, bool ionic, SolveResult* out) {
  double bck = ionic ? kap : 0.0;
  BC dh;
  dh.kind = 1;
  auto fine_solve = [&](const Grid& g, const std::vector<double>& rho, const Diel& D, const std::vector<double>& K,
                        const BC& bc) {
    if (p.converged_rel_tol > 0.0)
      return solve_converged(g, rho, D, K, bc, x, q, bck, eout, p.converged_rel_tol, p.converged_max_iter,
                             p.converged_method);
    return solve_multigrid(g, rho, D, K, bc, x, q, bck, eout, p.tolerance, p.max_iterations);
  };
  auto fine_maps = [&](Diel& D, std::vector<double>& K) {
    D = assign_dielectrics(fg, x, radii, p.probe, ein, eout);
    if (ionic)
      K = assign_kappa(fg, x, radii, p.ion_radius, kap, p.solvent_dielectric);
    else
      K.assign(fg.len(), 0.0);
  };
  if (cg) {
    std::vector<double> cq = map_charges(*cg, x, q);
    Diel cD = assign_dielectrics(*cg, x, radii, p.probe, ein, eout);
    std::vector<double> cK =
        ionic ? assign_kappa(*cg, x, radii, p.ion_radius, kap, p.solvent_dielectric) : std::vector<double>(cg->len(), 0.0);
    SolveResult cr = p.converged_rel_tol > 0.0
                         ? solve_converged(*cg, cq, cD, cK, dh, x, q, bck, eout, p.converged_rel_tol,
                                           p.converged_max_iter, p.converged_method)
                         : solve_multigrid(*cg, cq, cD, cK, dh, x, q, bck, eout, p.tolerance * 10.0, p.max_iterations);
    double mp = 0.0;
    for (double v : cr.phi) mp = std::max(mp, std::fabs(v));
    bool ok = cr.converged && std::isfinite(mp) && mp < 1e10;
    Diel D;
    std::vector<double> K;
    fine_maps(D, K);
    if (!ok) {
      *out = fine_solve(fg, fq, D, K, dh);
      return elec_energy(fg, out->phi, x, q);
    }
    BC ib;
    ib.kind = 2;
    for_each_boundary(fg.dims, [&](size_t ix, size_t iy, size_t iz) {
      double pt[3];
      fg.point(ix, iy, iz, pt);
      ib.values.push_back({fg.index(ix, iy, iz), interpolate(*cg, pt, cr.phi)});
    });
    *out = fine_solve(fg, fq, D, K, ib);
    return elec_energy(fg, out->phi, x, q);
  }
  Diel D;
  std::vector<double> K;
  fine_maps(D, K);
  *out = fine_solve(fg, fq, D, K, dh);
  return elec_energy(fg, out->phi, x, q);
}

// pb_energy.rs:332-438
double pb_energy(const std::vector<V3>& x, const std::vector<double>& q, const std::vector<double>& radii,
                 const PbParams& p, PbDiag* diag) {
  double kap = kappa(p.salt, p.solvent_dielectric, p.temperature);
  Grid fg = auto_grid(x, p.grid_spacing, p.grid_buffer);
  Grid cg;
  bool focus = p.fillratio > 0.0 && p.fscale > 1;
  if (focus) cg = coarse_grid(x, p.grid_spacing, p.fillratio, p.fscale);
  std::vector<double> fq = map_charges(fg, x, q);
  SolveResult rs, rr;
  double es = solve_focus(fg, fq, focus ? &cg : nullptr, x, q, radii, p, p.solute_dielectric,
                          p.solvent_dielectric, kap, true, &rs);
  double er = solve_focus(fg, fq, focus ? &cg : nullptr, x, q, radii, p, p.solute_dielectric,
                          p.solute_dielectric, kap, false, &rr);
  if (diag) {
    diag->iterations[0] = rs.iterations;
    diag->iterations[1] = rr.iterations;
    diag->residual[0] = rs.residual;
    diag->residual[1] = rr.residual;
    diag->converged[0] = rs.converged;
    diag->converged[1] = rr.converged;
    for (int k = 0; k < 3; k++) diag->dims[k] = (int)fg.dims[k];
  }
  return es - er;
}

}  // namespace orc
