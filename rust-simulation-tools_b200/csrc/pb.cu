// Poisson-Boltzmann engine on the GPU, FP64 with unfused multiply-adds
// (built with -fmad=false) so every grid point follows the reference's
// arithmetic:
//   pb_grid.rs   auto_grid, map_charges, spatial hash, SAS test, flood fill
//                from the boundary, SES by distance threshold, face
//                dielectrics from exact chord intervals, kappa-bar^2 map
//   pb_solver.rs Debye-Hueckel boundary, red-black SOR, residual, full-
//                weighting restriction, trilinear prolongation, injection
//                coarsening, V-cycle, convergence / divergence logic, energy
//   pb_energy.rs solvated and reference solves, two-level focusing
//
// Set-up work that is O(atoms) -- the spatial hash and the trilinear charge
// spreading in atom order -- is done on the host; everything that touches
// the grid runs in the kernels below.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <unordered_map>

#include "common.cuh"
#include "frame_plain.hpp"
#include "pb.cuh"

namespace rstg {

static const double kFourPiEc = 4.0 * kPi * 332.0522;  // pb_solver.rs:155

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
static void bbox(const std::vector<double>& x, double* mn, double* mx) {
  for (int d = 0; d < 3; d++) {
    mn[d] = std::numeric_limits<double>::max();
    mx[d] = std::numeric_limits<double>::lowest();
  }
  for (size_t a = 0; a < x.size() / 3; a++)
    for (int d = 0; d < 3; d++) {
      if (x[3 * a + d] < mn[d]) mn[d] = x[3 * a + d];
      if (x[3 * a + d] > mx[d]) mx[d] = x[3 * a + d];
    }
}

PbGeom pb_auto_grid(const std::vector<double>& x, double h, double buffer) {
  double mn[3], mx[3];
  bbox(x, mn, mx);
  PbGeom g;
  int dims[3];
  double org[3];
  for (int d = 0; d < 3; d++) {
    double ext = mx[d] - mn[d] + 2.0 * buffer;
    size_t n = (size_t)std::ceil(ext / h) + 1;
    n = (n % 2 == 0) ? n + 1 : n;
    if (n > 4096) throw Error(RSTG_ERR_INVALID, "PB grid dimension exceeds 4096 points");
    dims[d] = (int)n;
    double gext = (double)(n - 1) * h;
    org[d] = 0.5 * (mn[d] + mx[d]) - 0.5 * gext;
  }
  g.nx = dims[0];
  g.ny = dims[1];
  g.nz = dims[2];
  g.ox = org[0];
  g.oy = org[1];
  g.oz = org[2];
  g.h = h;
  return g;
}

PbGeom pb_coarse_grid(const std::vector<double>& x, double h, double fill, int64_t fs) {
  double mn[3], mx[3];
  bbox(x, mn, mx);
  double ch = h * (double)fs;
  PbGeom g;
  int dims[3];
  double org[3];
  for (int d = 0; d < 3; d++) {
    double ext = (mx[d] - mn[d]) * fill;
    size_t n = (size_t)std::ceil(ext / ch) + 1;
    n = (n % 2 == 0) ? n + 1 : n;
    if (n > 4096) throw Error(RSTG_ERR_INVALID, "PB coarse grid dimension exceeds 4096 points");
    dims[d] = (int)n;
    org[d] = 0.5 * (mn[d] + mx[d]) - 0.5 * ((double)(n - 1) * ch);
  }
  g.nx = dims[0];
  g.ny = dims[1];
  g.nz = dims[2];
  g.ox = org[0];
  g.oy = org[1];
  g.oz = org[2];
  g.h = ch;
  return g;
}

double pb_omega(int nx, int ny, int nz) {
  double r = (std::cos(kPi / (double)nx) + std::cos(kPi / (double)ny) + std::cos(kPi / (double)nz)) / 3.0;
  return 2.0 / (1.0 + std::sqrt(1.0 - r * r));
}

static double spectral_radius(int nx, int ny, int nz) {
  return (std::cos(kPi / (double)nx) + std::cos(kPi / (double)ny) + std::cos(kPi / (double)nz)) / 3.0;
}

PbHash pb_build_hash(const std::vector<double>& x, double max_eff) {
  PbHash H;
  size_t n = x.size() / 3;
  if (n == 0) return H;
  double cs = std::max(max_eff, 0.1);
  H.inv = 1.0 / cs;
  double mn[3], mx[3];
  bbox(x, mn, mx);
  H.ox = mn[0] - max_eff;
  H.oy = mn[1] - max_eff;
  H.oz = mn[2] - max_eff;
  H.gx = (int)((size_t)std::ceil((mx[0] - H.ox) * H.inv) + 1);
  H.gy = (int)((size_t)std::ceil((mx[1] - H.oy) * H.inv) + 1);
  H.gz = (int)((size_t)std::ceil((mx[2] - H.oz) * H.inv) + 1);
  size_t nc = (size_t)H.gx * H.gy * H.gz;
  if (nc > (size_t)1 << 28) throw Error(RSTG_ERR_INVALID, "spatial hash too large");
  std::vector<int32_t> cell(n), cnt(nc + 1, 0);
  for (size_t a = 0; a < n; a++) {
    size_t cx = (size_t)((x[3 * a] - H.ox) * H.inv), cy = (size_t)((x[3 * a + 1] - H.oy) * H.inv),
           cz = (size_t)((x[3 * a + 2] - H.oz) * H.inv);
    cell[a] = (int32_t)(cx + (size_t)H.gx * (cy + (size_t)H.gy * cz));
    cnt[cell[a] + 1]++;
  }
  for (size_t c = 0; c < nc; c++) cnt[c + 1] += cnt[c];
  H.start = cnt;
  H.atoms.assign(n, 0);
  std::vector<int32_t> cur(cnt.begin(), cnt.end() - 1);
  for (size_t a = 0; a < n; a++) H.atoms[cur[cell[a]]++] = (int32_t)a;  // atom order within a cell
  return H;
}

// Trilinear charge spreading (pb_grid.rs:220-292) summed in atom order; the
// result is sparse (8 points per atom) and scattered on the device.
static void spread_charges(const PbGeom& g, const std::vector<double>& x, const std::vector<double>& q,
                           std::vector<int64_t>& idx, std::vector<double>& val) {
  idx.clear();
  val.clear();
  long nx = g.nx, ny = g.ny, nz = g.nz;
  double org[3] = {g.ox, g.oy, g.oz};
  // open-addressing table: grid index -> position in idx/val (first-touch order)
  size_t cap = 64;
  while (cap < 16 * q.size() + 16) cap <<= 1;
  std::vector<int64_t> key(cap, -1);
  std::vector<int32_t> pos(cap, 0);
  idx.reserve(8 * q.size());
  val.reserve(8 * q.size());
  for (size_t a = 0; a < q.size(); a++) {
    double fc[3];
    for (int d = 0; d < 3; d++) fc[d] = (x[3 * a + d] - org[d]) / g.h;
    long ix = (long)std::floor(fc[0]), iy = (long)std::floor(fc[1]), iz = (long)std::floor(fc[2]);
    if (ix < 0 || ix >= nx - 1 || iy < 0 || iy >= ny - 1 || iz < 0 || iz >= nz - 1) continue;
    double dx = fc[0] - (double)ix, dy = fc[1] - (double)iy, dz = fc[2] - (double)iz;
    double vol = g.h * g.h * g.h;
    double qd = q[a] / vol;
    double wx[2] = {1.0 - dx, dx}, wy[2] = {1.0 - dy, dy}, wz[2] = {1.0 - dz, dz};
    for (int a0 = 0; a0 < 2; a0++)
      for (int a1 = 0; a1 < 2; a1++)
        for (int a2 = 0; a2 < 2; a2++) {
          int64_t k = (ix + a0) + nx * ((iy + a1) + ny * (iz + a2));
          double v = qd * wx[a0] * wy[a1] * wz[a2];
          size_t h = (size_t)((uint64_t)k * 0x9E3779B97F4A7C15ull >> 20) & (cap - 1);
          while (key[h] != -1 && key[h] != k) h = (h + 1) & (cap - 1);
          if (key[h] == -1) {  // grid point first touched: 0.0 + v (pb_grid.rs:280-288)
            key[h] = k;
            pos[h] = (int32_t)val.size();
            idx.push_back(k);
            val.push_back(0.0 + v);
          } else {
            val[pos[h]] += v;
          }
        }
  }
}

// ---------------------------------------------------------------------------
// device: grid set-up
// ---------------------------------------------------------------------------
struct HashDev {
  double inv, ox, oy, oz;
  int gx, gy, gz;
  const int* start;
  const int* atoms;
};

struct GeomDev {
  int nx, ny, nz;
  double h, ox, oy, oz;
};

__device__ __forceinline__ void grid_point(const GeomDev& g, int ix, int iy, int iz, double* p) {
  p[0] = g.ox + (double)ix * g.h;
  p[1] = g.oy + (double)iy * g.h;
  p[2] = g.oz + (double)iz * g.h;
}

__device__ bool hash_inside(const HashDev& H, const double* p, const double* __restrict__ xyz,
                            const double* __restrict__ radii, double probe) {
  if (H.gx == 0) return false;
  long cx = (long)((p[0] - H.ox) * H.inv), cy = (long)((p[1] - H.oy) * H.inv), cz = (long)((p[2] - H.oz) * H.inv);
  for (long dz = -1; dz <= 1; dz++) {
    long jz = cz + dz;
    if (jz < 0 || jz >= H.gz) continue;
    for (long dy = -1; dy <= 1; dy++) {
      long jy = cy + dy;
      if (jy < 0 || jy >= H.gy) continue;
      for (long dx = -1; dx <= 1; dx++) {
        long jx = cx + dx;
        if (jx < 0 || jx >= H.gx) continue;
        long c = jx + (long)H.gx * (jy + (long)H.gy * jz);
        for (int k = H.start[c]; k < H.start[c + 1]; k++) {
          int a = H.atoms[k];
          double ddx = p[0] - xyz[3 * a], ddy = p[1] - xyz[3 * a + 1], ddz = p[2] - xyz[3 * a + 2];
          double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
          double th = radii[a] + probe;
          if (d2 < th * th) return true;
        }
      }
    }
  }
  return false;
}

__global__ void k_inside(GeomDev g, HashDev H, const double* __restrict__ xyz, const double* __restrict__ radii,
                         double probe, uint8_t* __restrict__ out) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)g.nx * g.ny * g.nz;
  if (idx >= n) return;
  int iz = (int)(idx / ((long long)g.nx * g.ny)), iy = (int)((idx / g.nx) % g.ny), ix = (int)(idx % g.nx);
  double p[3];
  grid_point(g, ix, iy, iz, p);
  out[idx] = hash_inside(H, p, xyz, radii, probe) ? 1 : 0;
}

__global__ void k_kappa(GeomDev g, HashDev H, const double* __restrict__ xyz, const double* __restrict__ radii,
                        double ion, double kbs, double* __restrict__ out) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)g.nx * g.ny * g.nz;
  if (idx >= n) return;
  int iz = (int)(idx / ((long long)g.nx * g.ny)), iy = (int)((idx / g.nx) % g.ny), ix = (int)(idx % g.nx);
  double p[3];
  grid_point(g, ix, iy, iz, p);
  out[idx] = hash_inside(H, p, xyz, radii, ion) ? 0.0 : kbs;
}

__global__ void k_flood_seed(GeomDev g, const uint8_t* __restrict__ sas, uint8_t* __restrict__ ext) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)g.nx * g.ny * g.nz;
  if (idx >= n) return;
  int iz = (int)(idx / ((long long)g.nx * g.ny)), iy = (int)((idx / g.nx) % g.ny), ix = (int)(idx % g.nx);
  bool bd = ix == 0 || ix == g.nx - 1 || iy == 0 || iy == g.ny - 1 || iz == 0 || iz == g.nz - 1;
  ext[idx] = (bd && !sas[idx]) ? 1 : 0;
}

// One propagation pass of the connected exterior (pb_grid.rs:621-686) over
// 8^3 tiles: inside a tile the front advances until it stops, across tiles
// through repeated launches until no point changes.  The fixed point is the
// set of outside-SAS points 6-connected to an outside-SAS boundary point,
// whatever the visiting order.  With act_in, only tiles marked there run; a
// tile that grew marks itself and its six face neighbours in act_out.
__global__ void k_flood(GeomDev g, const uint8_t* __restrict__ sas, uint8_t* __restrict__ ext, int* changed,
                        const uint8_t* __restrict__ act_in, uint8_t* __restrict__ act_out) {
  __shared__ uint8_t se[10][10][10], ss[10][10][10];
  int tile = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (act_in && !act_in[tile]) return;
  int tx = threadIdx.x, ty = threadIdx.y, tz = threadIdx.z;
  int bx = blockIdx.x * 8, by = blockIdx.y * 8, bz = blockIdx.z * 8;
  int t = tx + 8 * (ty + 8 * tz);
  for (int k = t; k < 1000; k += 512) {
    int hx = k % 10, hy = (k / 10) % 10, hz = k / 100;
    int gx = bx + hx - 1, gy = by + hy - 1, gz = bz + hz - 1;
    bool in = gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny && gz >= 0 && gz < g.nz;
    long long gi = in ? gx + (long long)g.nx * (gy + (long long)g.ny * gz) : 0;
    se[hz][hy][hx] = in ? ext[gi] : 0;
    ss[hz][hy][hx] = in ? sas[gi] : 1;
  }
  __syncthreads();
  int ix = bx + tx, iy = by + ty, iz = bz + tz;
  bool mine = ix < g.nx && iy < g.ny && iz < g.nz;
  bool grew = false;
  for (int it = 0; it < 512; it++) {
    int c = 0;
    if (mine && !ss[tz + 1][ty + 1][tx + 1] && !se[tz + 1][ty + 1][tx + 1]) {
      if (se[tz + 1][ty + 1][tx] | se[tz + 1][ty + 1][tx + 2] | se[tz + 1][ty][tx + 1] | se[tz + 1][ty + 2][tx + 1] |
          se[tz][ty + 1][tx + 1] | se[tz + 2][ty + 1][tx + 1])
        c = 1;
    }
    __syncthreads();
    if (c) {
      se[tz + 1][ty + 1][tx + 1] = 1;
      grew = true;
    }
    if (!__syncthreads_or(c)) break;
  }
  if (grew) ext[ix + (long long)g.nx * (iy + (long long)g.ny * iz)] = 1;
  if (__syncthreads_or(grew) && t == 0) {
    atomicExch(changed, 1);
    if (act_out) {
      int X = blockIdx.x, Y = blockIdx.y, Z = blockIdx.z, NX = gridDim.x, NY = gridDim.y, NZ = gridDim.z;
      act_out[tile] = 1;
      if (X > 0) act_out[tile - 1] = 1;
      if (X + 1 < NX) act_out[tile + 1] = 1;
      if (Y > 0) act_out[tile - NX] = 1;
      if (Y + 1 < NY) act_out[tile + NX] = 1;
      if (Z > 0) act_out[tile - NX * NY] = 1;
      if (Z + 1 < NZ) act_out[tile + NX * NY] = 1;
    }
  }
}

// SES classification (pb_grid.rs:688-707): a point is outside the SES when a
// connected-exterior point lies within squared index distance thr; the
// squared Euclidean distance transform there is an exact integer, so testing
// the integer offsets of the ball gives the same answer.
__global__ void k_ses(GeomDev g, const uint8_t* __restrict__ ext, const int4* __restrict__ offs, int noffs,
                      uint8_t* __restrict__ inside) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)g.nx * g.ny * g.nz;
  if (idx >= n) return;
  int iz = (int)(idx / ((long long)g.nx * g.ny)), iy = (int)((idx / g.nx) % g.ny), ix = (int)(idx % g.nx);
  bool out = false;
  for (int k = 0; k < noffs && !out; k++) {
    int4 o = offs[k];
    int x = ix + o.x, y = iy + o.y, z = iz + o.z;
    if (x < 0 || x >= g.nx || y < 0 || y >= g.ny || z < 0 || z >= g.nz) continue;
    out = ext[x + (long long)g.nx * (y + (long long)g.ny * z)] != 0;
  }
  inside[idx] = out ? 0 : 1;
}

constexpr int kMaxIntervals = 64;

// fraction_inside_along_axis (pb_grid.rs:717-801) with probe 0, candidate
// atoms from a hash whose cells are at least max radius + h wide.
__device__ double edge_fraction(const HashDev& H, const double* __restrict__ xyz, const double* __restrict__ radii,
                                double lo, double hi, double p1, double p2, int axis, const double* pt, int* ovf) {
  double len = hi - lo;
  if (len <= 0.0) return 0.0;
  int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
  double ilo_[kMaxIntervals], ihi_[kMaxIntervals];
  int m = 0;
  long cx = (long)((pt[0] - H.ox) * H.inv), cy = (long)((pt[1] - H.oy) * H.inv), cz = (long)((pt[2] - H.oz) * H.inv);
  for (long dz = -1; dz <= 1; dz++) {
    long jz = cz + dz;
    if (jz < 0 || jz >= H.gz) continue;
    for (long dy = -1; dy <= 1; dy++) {
      long jy = cy + dy;
      if (jy < 0 || jy >= H.gy) continue;
      for (long dx = -1; dx <= 1; dx++) {
        long jx = cx + dx;
        if (jx < 0 || jx >= H.gx) continue;
        long c = jx + (long)H.gx * (jy + (long)H.gy * jz);
        for (int k = H.start[c]; k < H.start[c + 1]; k++) {
          int a = H.atoms[k];
          double R = radii[a] + 0.0;
          double d1 = p1 - xyz[3 * a + a1], d2 = p2 - xyz[3 * a + a2];
          double rs = R * R - d1 * d1 - d2 * d2;
          if (rs <= 0.0) continue;
          double rho = sqrt(rs);
          double ca = xyz[3 * a + axis];
          double l = fmax(ca - rho, lo), u = fmin(ca + rho, hi);
          if (l < u) {
            if (m == kMaxIntervals) {
              atomicExch(ovf, 1);
              continue;
            }
            int p = m++;  // insertion by start
            while (p > 0 && ilo_[p - 1] > l) {
              ilo_[p] = ilo_[p - 1];
              ihi_[p] = ihi_[p - 1];
              p--;
            }
            ilo_[p] = l;
            ihi_[p] = u;
          }
        }
      }
    }
  }
  if (m == 0) return 0.0;
  double total = 0.0, clo = ilo_[0], chi = ihi_[0];
  for (int k = 1; k < m; k++) {
    if (ilo_[k] <= chi) {
      chi = fmax(chi, ihi_[k]);
    } else {
      total += chi - clo;
      clo = ilo_[k];
      chi = ihi_[k];
    }
  }
  total += chi - clo;
  return fmin(1.0, fmax(0.0, total / len));
}

__device__ __forceinline__ double harmonic(double f, double ein, double eout) {  // pb_grid.rs:809-817
  if (f <= 0.0) return eout;
  if (f >= 1.0) return ein;
  return 1.0 / (f / ein + (1.0 - f) / eout);
}

__global__ void k_eps(GeomDev g, const uint8_t* __restrict__ inside, HashDev H, const double* __restrict__ xyz,
                      const double* __restrict__ radii, double ein, double eout, double* __restrict__ ex,
                      double* __restrict__ ey, double* __restrict__ ez, int* ovf) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long n = (long long)g.nx * g.ny * g.nz;
  if (idx >= n) return;
  int iz = (int)(idx / ((long long)g.nx * g.ny)), iy = (int)((idx / g.nx) % g.ny), ix = (int)(idx % g.nx);
  bool a = inside[idx];
  double p[3];
  grid_point(g, ix, iy, iz, p);
  double vx = eout, vy = eout, vz = eout;
  if (ix + 1 < g.nx) {
    bool b = inside[idx + 1];
    vx = a == b ? (a ? ein : eout)
                : harmonic(edge_fraction(H, xyz, radii, p[0], p[0] + g.h, p[1], p[2], 0, p, ovf), ein, eout);
  }
  if (iy + 1 < g.ny) {
    bool b = inside[idx + g.nx];
    vy = a == b ? (a ? ein : eout)
                : harmonic(edge_fraction(H, xyz, radii, p[1], p[1] + g.h, p[0], p[2], 1, p, ovf), ein, eout);
  }
  if (iz + 1 < g.nz) {
    bool b = inside[idx + (long long)g.nx * g.ny];
    vz = a == b ? (a ? ein : eout)
                : harmonic(edge_fraction(H, xyz, radii, p[2], p[2] + g.h, p[0], p[1], 2, p, ovf), ein, eout);
  }
  ex[idx] = vx;
  ey[idx] = vy;
  ez[idx] = vz;
}

__global__ void k_fill(double* __restrict__ a, long long n, double v) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

__global__ void k_scatter(const long long* __restrict__ idx, const double* __restrict__ val, int m,
                          double* __restrict__ out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < m) out[idx[k]] = val[k];
}

// Boundary points of a grid enumerated face by face: the two z faces, the
// two y faces of the interior z planes, the two x faces of the interior
// rows.  Grids one or two points thick name some points twice (the same
// value is written twice).
__device__ __forceinline__ bool boundary_point(const GeomDev& g, long long k, int& ix, int& iy, int& iz) {
  long long nxy = (long long)g.nx * g.ny;
  int nzi = max(g.nz - 2, 0), nyi = max(g.ny - 2, 0);
  if (k < 2 * nxy) {
    iz = k < nxy ? 0 : g.nz - 1;
    long long r = k % nxy;
    ix = (int)(r % g.nx);
    iy = (int)(r / g.nx);
    return true;
  }
  k -= 2 * nxy;
  long long nyf = (long long)g.nx * nzi;
  if (k < 2 * nyf) {
    iy = k < nyf ? 0 : g.ny - 1;
    long long r = k % nyf;
    ix = (int)(r % g.nx);
    iz = 1 + (int)(r / g.nx);
    return true;
  }
  k -= 2 * nyf;
  long long nxf = (long long)nyi * nzi;
  if (k < 2 * nxf) {
    ix = k < nxf ? 0 : g.nx - 1;
    long long r = k % nxf;
    iy = 1 + (int)(r % nyi);
    iz = 1 + (int)(r / nyi);
    return true;
  }
  return false;
}

static long long boundary_count(const PbGeom& g) {
  long long nzi = std::max(g.nz - 2, 0), nyi = std::max(g.ny - 2, 0);
  return 2LL * g.nx * g.ny + 2LL * g.nx * nzi + 2LL * nyi * nzi;
}

// set_dh_boundary, pb_solver.rs:68-93: atoms summed in order per boundary
// point (pb_solver.rs:31-60 visits every point of a grid that is one or two
// points thick; those points are all boundary points).
__global__ void k_dh(GeomDev g, long long nbnd, const double* __restrict__ xyz, const double* __restrict__ q, int na,
                     double kap, double eout, double* __restrict__ phi) {
  __shared__ double sx[256], sy[256], sz[256], sq[256];
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int ix = 0, iy = 0, iz = 0;
  bool valid = k < nbnd && boundary_point(g, k, ix, iy, iz);
  double p[3];
  grid_point(g, ix, iy, iz, p);
  double s = 0.0;
  const double conv = 332.0522;
  for (int a0 = 0; a0 < na; a0 += 256) {
    int a = a0 + threadIdx.x;
    if (a < na) {
      sx[threadIdx.x] = xyz[3 * a];
      sy[threadIdx.x] = xyz[3 * a + 1];
      sz[threadIdx.x] = xyz[3 * a + 2];
      sq[threadIdx.x] = q[a];
    }
    __syncthreads();
    int m = min(256, na - a0);
    if (valid)
      for (int j = 0; j < m; j++) {
        double dx = p[0] - sx[j], dy = p[1] - sy[j], dz = p[2] - sz[j];
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        if (r > 1e-10) s += conv * sq[j] * exp(-kap * r) / (eout * r);
      }
    __syncthreads();
  }
  if (valid) phi[ix + (long long)g.nx * (iy + (long long)g.ny * iz)] = s;
}

// Focusing boundary: fine boundary values interpolated from the coarse
// potential (pb_solver.rs:100-114, pb_grid.rs:142-182).
__global__ void k_interp_boundary(GeomDev f, GeomDev c, const double* __restrict__ cphi, double* __restrict__ phi) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)f.nx * f.ny * f.nz) return;
  int iz = (int)(idx / ((long long)f.nx * f.ny)), iy = (int)((idx / f.nx) % f.ny), ix = (int)(idx % f.nx);
  if (!(ix == 0 || ix == f.nx - 1 || iy == 0 || iy == f.ny - 1 || iz == 0 || iz == f.nz - 1)) return;
  double p[3];
  grid_point(f, ix, iy, iz, p);
  double fc[3] = {(p[0] - c.ox) / c.h, (p[1] - c.oy) / c.h, (p[2] - c.oz) / c.h};
  long cx = (long)floor(fc[0]), cy = (long)floor(fc[1]), cz = (long)floor(fc[2]);
  double v = 0.0;
  if (!(cx < 0 || cx >= c.nx - 1 || cy < 0 || cy >= c.ny - 1 || cz < 0 || cz >= c.nz - 1)) {
    double dx = fc[0] - (double)cx, dy = fc[1] - (double)cy, dz = fc[2] - (double)cz;
    auto at = [&](long x, long y, long z) { return cphi[x + (long)c.nx * (y + (long)c.ny * z)]; };
    double c00 = at(cx, cy, cz) * (1.0 - dx) + at(cx + 1, cy, cz) * dx;
    double c10 = at(cx, cy + 1, cz) * (1.0 - dx) + at(cx + 1, cy + 1, cz) * dx;
    double c01 = at(cx, cy, cz + 1) * (1.0 - dx) + at(cx + 1, cy, cz + 1) * dx;
    double c11 = at(cx, cy + 1, cz + 1) * (1.0 - dx) + at(cx + 1, cy + 1, cz + 1) * dx;
    double c0 = c00 * (1.0 - dy) + c10 * dy, c1 = c01 * (1.0 - dy) + c11 * dy;
    v = c0 * (1.0 - dz) + c1 * dz;
  }
  phi[idx] = v;
}

// ---------------------------------------------------------------------------
// device: multigrid (pb_solver.rs)
// ---------------------------------------------------------------------------
struct LevelDev {
  int nx, ny, nz;
  double ihx, ihy, ihz;
  const double *ex, *ey, *ez, *k2;
};

__device__ __forceinline__ void stencil(const LevelDev& L, const double* __restrict__ phi, long long idx,
                                        double& ns, double& dg) {
  long long sy = L.nx, sz = (long long)L.nx * L.ny;
  double exp_ = L.ex[idx], exm = L.ex[idx - 1], eyp = L.ey[idx], eym = L.ey[idx - sy], ezp = L.ez[idx],
         ezm = L.ez[idx - sz];
  ns = (exp_ * phi[idx + 1] + exm * phi[idx - 1]) * L.ihx + (eyp * phi[idx + sy] + eym * phi[idx - sy]) * L.ihy +
       (ezp * phi[idx + sz] + ezm * phi[idx - sz]) * L.ihz;
  dg = (exp_ + exm) * L.ihx + (eyp + eym) * L.ihy + (ezp + ezm) * L.ihz + L.k2[idx];
}

// one colour of a red-black SOR sweep (pb_solver.rs:250-317); optional
// per-block sums of (phi_GS - phi)^2 for the plain-SOR convergence test
__global__ void k_rb(LevelDev L, double* __restrict__ phi, const double* __restrict__ rho, double omega,
                     double rhs_scale, int color, double* __restrict__ rms_part) {
  __shared__ double sh[32];
  int iy = blockIdx.y + 1, iz = blockIdx.z + 1;
  int x0 = 1 + ((1 + iy + iz + color) & 1);
  int ix = x0 + 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  double r2 = 0.0;
  if (ix < L.nx - 1) {
    long long idx = ix + (long long)L.nx * (iy + (long long)L.ny * iz);
    double ns, dg;
    stencil(L, phi, idx, ns, dg);
    double rhs = rhs_scale * rho[idx];
    double gs = (ns + rhs) / dg;
    double old = phi[idx];
    double res = gs - old;
    r2 = res * res;
    phi[idx] = old + omega * (gs - old);
  }
  if (rms_part) {
    double s = block_sum(r2, sh);
    if (threadIdx.x == 0)
      rms_part[blockIdx.x + gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z)] = s;
  }
}

__global__ void k_residual(LevelDev L, const double* __restrict__ phi, const double* __restrict__ rho,
                           double rhs_scale, double* __restrict__ out, double* __restrict__ sq_part) {
  __shared__ double sh[32];
  int ix = 1 + blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y + 1, iz = blockIdx.z + 1;
  double r2 = 0.0;
  if (ix < L.nx - 1) {
    long long idx = ix + (long long)L.nx * (iy + (long long)L.ny * iz);
    double ns, dg;
    stencil(L, phi, idx, ns, dg);
    double r = rhs_scale * rho[idx] + ns - dg * phi[idx];
    if (out) out[idx] = r;
    r2 = r * r;
  }
  if (sq_part) {
    double s = block_sum(r2, sh);
    if (threadIdx.x == 0) sq_part[blockIdx.x + gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z)] = s;
  }
}

__global__ void k_restrict(const double* __restrict__ f, int fnx, int fny, int fnz, double* __restrict__ c, int cnx,
                           int cny, int cnz, double scale) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)cnx * cny * cnz) return;
  int cz = (int)(i / ((long long)cnx * cny)), cy = (int)((i / cnx) % cny), cx = (int)(i % cnx);
  int fx = 2 * cx, fy = 2 * cy, fz = 2 * cz;
  double sum = 0.0, ws = 0.0;
  for (int dz = -1; dz <= 1; dz++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        int x = fx + dx, y = fy + dy, z = fz + dz;
        if (x < 0 || x >= fnx || y < 0 || y >= fny || z < 0 || z >= fnz) continue;
        double w = (dx == 0 ? 2.0 : 1.0) * (dy == 0 ? 2.0 : 1.0) * (dz == 0 ? 2.0 : 1.0);
        sum += w * f[x + (long long)fnx * (y + (long long)fny * z)];
        ws += w;
      }
  c[i] = scale * sum / ws;
}

// skipb (relative-residual mode): corrections vanish on the boundary, so
// boundary points are left alone
__global__ void k_prolong(const double* __restrict__ c, int cnx, int cny, int cnz, double* __restrict__ f, int fnx,
                          int fny, int fnz, int skipb) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)fnx * fny * fnz) return;
  int fz = (int)(i / ((long long)fnx * fny)), fy = (int)((i / fnx) % fny), fx = (int)(i % fnx);
  if (skipb && (fx == 0 || fy == 0 || fz == 0 || fx == fnx - 1 || fy == fny - 1 || fz == fnz - 1)) return;
  double cxf = (double)fx / 2.0, cyf = (double)fy / 2.0, czf = (double)fz / 2.0;
  int mx = cnx >= 2 ? cnx - 2 : 0, my = cny >= 2 ? cny - 2 : 0, mz = cnz >= 2 ? cnz - 2 : 0;
  int x0 = min((int)floor(cxf), mx), y0 = min((int)floor(cyf), my), z0 = min((int)floor(czf), mz);
  double dx = cxf - (double)x0, dy = cyf - (double)y0, dz = czf - (double)z0;
  auto at = [&](int x, int y, int z) { return c[x + (long long)cnx * (y + (long long)cny * z)]; };
  double c00 = at(x0, y0, z0) * (1.0 - dx) + at(x0 + 1, y0, z0) * dx;
  double c10 = at(x0, y0 + 1, z0) * (1.0 - dx) + at(x0 + 1, y0 + 1, z0) * dx;
  double c01 = at(x0, y0, z0 + 1) * (1.0 - dx) + at(x0 + 1, y0, z0 + 1) * dx;
  double c11 = at(x0, y0 + 1, z0 + 1) * (1.0 - dx) + at(x0 + 1, y0 + 1, z0 + 1) * dx;
  double c0 = c00 * (1.0 - dy) + c10 * dy, c1 = c01 * (1.0 - dy) + c11 * dy;
  f[i] += c0 * (1.0 - dz) + c1 * dz;
}

__global__ void k_coarsen(const double* __restrict__ f, int fnx, int fny, int fnz, double* __restrict__ c, int cnx,
                          int cny, int cnz) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)cnx * cny * cnz) return;
  int cz = (int)(i / ((long long)cnx * cny)), cy = (int)((i / cnx) % cny), cx = (int)(i % cnx);
  int fx = min(2 * cx, fnx - 1), fy = min(2 * cy, fny - 1), fz = min(2 * cz, fnz - 1);
  c[i] = f[fx + (long long)fnx * (fy + (long long)fny * fz)];
}

// Coarse face dielectric of the relative-residual mode: two fine faces in
// series along the face's axis (harmonic mean; equal values copied), the
// 3 x 3 neighbouring lines across it in parallel (weights 1-2-1 per
// transverse direction, renormalised at the grid edge).
__global__ void k_coarsen_face(const double* __restrict__ f, int fnx, int fny, int fnz, double* __restrict__ c,
                               int cnx, int cny, int cnz, int axis) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)cnx * cny * cnz) return;
  int cz = (int)(i / ((long long)cnx * cny)), cy = (int)((i / cnx) % cny), cx = (int)(i % cnx);
  const int n[3] = {fnx, fny, fnz};
  const int b[3] = {min(2 * cx, fnx - 1), min(2 * cy, fny - 1), min(2 * cz, fnz - 1)};
  const int t1 = axis == 0 ? 1 : 0, t2 = axis == 2 ? 1 : 2;
  double sum = 0.0, ws = 0.0, first = 0.0;
  bool same = true, any = false;
  for (int u = -1; u <= 1; u++)
    for (int v = -1; v <= 1; v++) {
      int p[3] = {b[0], b[1], b[2]};
      p[t1] += u;
      p[t2] += v;
      if (p[t1] < 0 || p[t1] >= n[t1] || p[t2] < 0 || p[t2] >= n[t2]) continue;
      int q[3] = {p[0], p[1], p[2]};
      q[axis] = min(p[axis] + 1, n[axis] - 1);
      const double e0 = f[p[0] + (long long)fnx * (p[1] + (long long)fny * p[2])];
      const double e1 = f[q[0] + (long long)fnx * (q[1] + (long long)fny * q[2])];
      if (!any) first = e0;
      any = true;
      same = same && e0 == first && e1 == first;
      const double w = (u == 0 ? 2.0 : 1.0) * (v == 0 ? 2.0 : 1.0);
      sum += w * (e0 == e1 ? e0 : 2.0 / (1.0 / e0 + 1.0 / e1));
      ws += w;
    }
  c[i] = same ? first : sum / ws;
}

// coarsest level: 50 red-black sweeps in one block (same arithmetic as k_rb)
__global__ void k_coarse_solve(LevelDev L, double* __restrict__ phi, const double* __restrict__ rho, double omega,
                               double rhs_scale, int sweeps) {
  long long ni = (long long)(L.nx - 2) * (L.ny - 2) * (L.nz - 2);
  for (int s = 0; s < sweeps; s++)
    for (int color = 0; color < 2; color++) {
      for (long long k = threadIdx.x; k < ni; k += blockDim.x) {
        int ix = 1 + (int)(k % (L.nx - 2)), iy = 1 + (int)((k / (L.nx - 2)) % (L.ny - 2)),
            iz = 1 + (int)(k / ((long long)(L.nx - 2) * (L.ny - 2)));
        if (((ix + iy + iz + color) & 1) != 0) continue;
        long long idx = ix + (long long)L.nx * (iy + (long long)L.ny * iz);
        double ns, dg;
        stencil(L, phi, idx, ns, dg);
        double gs = (ns + rhs_scale * rho[idx]) / dg;
        double old = phi[idx];
        phi[idx] = old + omega * (gs - old);
      }
      __syncthreads();
    }
}

__global__ void k_sum_fixed(const double* __restrict__ in, long long n, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) s += in[i];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) out[0] = s;
}

__global__ void k_maxabs(const double* __restrict__ in, long long n, double* __restrict__ out) {
  __shared__ double sh[1024];
  double m = 0.0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    double v = fabs(in[i]);
    m = (v > m || v != v) ? v : m;  // NaN propagates (pb_energy.rs:188-194 checks finiteness)
  }
  sh[threadIdx.x] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int k = 0; k < (int)blockDim.x; k++) r = (sh[k] > r || sh[k] != sh[k]) ? sh[k] : r;
    out[0] = r;
  }
}

// compute_elec_energy, pb_solver.rs:1174-1186: trilinear phi at each atom,
// then 0.5 * sum in atom order.
__global__ void k_atom_phi(GeomDev g, const double* __restrict__ phi, const double* __restrict__ xyz,
                           const double* __restrict__ q, int na, double* __restrict__ out) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= na) return;
  double fc[3] = {(xyz[3 * a] - g.ox) / g.h, (xyz[3 * a + 1] - g.oy) / g.h, (xyz[3 * a + 2] - g.oz) / g.h};
  long cx = (long)floor(fc[0]), cy = (long)floor(fc[1]), cz = (long)floor(fc[2]);
  double v = 0.0;
  if (!(cx < 0 || cx >= g.nx - 1 || cy < 0 || cy >= g.ny - 1 || cz < 0 || cz >= g.nz - 1)) {
    double dx = fc[0] - (double)cx, dy = fc[1] - (double)cy, dz = fc[2] - (double)cz;
    auto at = [&](long x, long y, long z) { return phi[x + (long)g.nx * (y + (long)g.ny * z)]; };
    double c00 = at(cx, cy, cz) * (1.0 - dx) + at(cx + 1, cy, cz) * dx;
    double c10 = at(cx, cy + 1, cz) * (1.0 - dx) + at(cx + 1, cy + 1, cz) * dx;
    double c01 = at(cx, cy, cz + 1) * (1.0 - dx) + at(cx + 1, cy, cz + 1) * dx;
    double c11 = at(cx, cy + 1, cz + 1) * (1.0 - dx) + at(cx + 1, cy + 1, cz + 1) * dx;
    double c0 = c00 * (1.0 - dy) + c10 * dy, c1 = c01 * (1.0 - dy) + c11 * dy;
    v = c0 * (1.0 - dz) + c1 * dz;
  }
  out[a] = q[a] * v;
}

__global__ void k_seq_sum(const double* __restrict__ in, int n, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double e = 0.0;
    for (int a = 0; a < n; a++) e += in[a];
    out[0] = 0.5 * e;
  }
}

// ===========================================================================
// host orchestration
// ===========================================================================
static GeomDev gdev(const PbGeom& g) { return GeomDev{g.nx, g.ny, g.nz, g.h, g.ox, g.oy, g.oz}; }

struct HashBuf {
  HashDev d{};
  DevBuf start, atoms;
  HashBuf(const PbHash& H, cudaStream_t st) {
    d.inv = H.inv;
    d.ox = H.ox;
    d.oy = H.oy;
    d.oz = H.oz;
    d.gx = H.gx;
    d.gy = H.gy;
    d.gz = H.gz;
    start = DevBuf(std::max<size_t>(H.start.size(), 1) * 4, st);
    atoms = DevBuf(std::max<size_t>(H.atoms.size(), 1) * 4, st);
    if (!H.start.empty())
      RSTG_CUDA(cudaMemcpyAsync(start.p, H.start.data(), H.start.size() * 4, cudaMemcpyHostToDevice, st));
    if (!H.atoms.empty())
      RSTG_CUDA(cudaMemcpyAsync(atoms.p, H.atoms.data(), H.atoms.size() * 4, cudaMemcpyHostToDevice, st));
    d.start = start.as<int>();
    d.atoms = atoms.as<int>();
  }
};

static unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// Device maps of one grid; MapsView is the non-owning form the solver reads.
struct MapsView {
  PbGeom g;
  const double *rho, *ex, *ey, *ez, *k2;
};

struct Maps {
  PbGeom g;
  DevBuf rho, ex, ey, ez, k2;
  MapsView view() const {
    return MapsView{g, rho.as<double>(), ex.as<double>(), ey.as<double>(), ez.as<double>(), k2.as<double>()};
  }
};

// Charge map of a grid (sparse host spreading, device scatter) into a
// caller-owned array of g.n() doubles.
static void charge_into(Ctx* c, const PbGeom& g, const AtomsDev& A, double* rho) {
  cudaStream_t st = pb_stream(c);
  RSTG_CUDA(cudaMemsetAsync(rho, 0, g.n() * 8, st));
  std::vector<int64_t> idx;
  std::vector<double> val;
  spread_charges(g, A.hx, A.hq, idx, val);
  if (idx.empty()) return;
  DevBuf di(idx.size() * 8, st), dv(val.size() * 8, st);
  RSTG_CUDA(cudaMemcpyAsync(di.p, idx.data(), idx.size() * 8, cudaMemcpyHostToDevice, st));
  RSTG_CUDA(cudaMemcpyAsync(dv.p, val.data(), val.size() * 8, cudaMemcpyHostToDevice, st));
  k_scatter<<<nblk((long long)idx.size(), 256), 256, 0, st>>>(di.as<long long>(), dv.as<double>(), (int)idx.size(),
                                                              rho);
  launched(c);
  // no synchronisation: copies from pageable host memory are staged before
  // cudaMemcpyAsync returns, and the device buffers are freed in stream order
}

static void charge_map(Ctx* c, const PbGeom& g, const AtomsDev& A, DevBuf& rho) {
  rho = DevBuf(g.n() * 8, pb_stream(c));
  charge_into(c, g, A, rho.as<double>());
}

// assign_dielectrics (pb_grid.rs:827-940) and assign_kappa (pb_grid.rs:951-985)
static void dielectric_into(Ctx* c, const PbGeom& g, const AtomsDev& A, double probe, double ein, double eout,
                            double* ex, double* ey, double* ez) {
  cudaStream_t st = pb_stream(c);
  long long n = (long long)g.n();
  GeomDev gd = gdev(g);
  if (std::fabs(ein - eout) < std::numeric_limits<double>::epsilon()) {
    for (double* b : {ex, ey, ez}) k_fill<<<nblk(n, 256), 256, 0, st>>>(b, n, ein);
    launched(c, 3);
    return;
  }
  double max_eff = A.max_r + std::max(probe, 0.0);
  HashBuf hs(pb_build_hash(A.hx, max_eff), st);
  DevBuf inside(n, st);
  if (probe <= 0.0) {
    k_inside<<<nblk(n, 256), 256, 0, st>>>(gd, hs.d, A.xyz.as<double>(), A.r.as<double>(), 0.0, inside.as<uint8_t>());
    launched(c);
  } else {
    DevBuf sas(n, st), ext(n, st), flag(8, st);
    k_inside<<<nblk(n, 256), 256, 0, st>>>(gd, hs.d, A.xyz.as<double>(), A.r.as<double>(), probe, sas.as<uint8_t>());
    k_flood_seed<<<nblk(n, 256), 256, 0, st>>>(gd, sas.as<uint8_t>(), ext.as<uint8_t>());
    launched(c, 2);
    dim3 fb(8, 8, 8), fg(nblk(g.nx, 8), nblk(g.ny, 8), nblk(g.nz, 8));
    size_t ntile = (size_t)fg.x * fg.y * fg.z;
    DevBuf act(2 * ntile, st);
    uint8_t* act_a = act.as<uint8_t>();
    uint8_t* act_b = act_a + ntile;
    long long limit = (long long)g.nx + g.ny + g.nz + 64;
    bool done = false;
    int pass = 0;
    for (long long it = 0; it < limit * 8 && !done; it += 8) {
      RSTG_CUDA(cudaMemsetAsync(flag.p, 0, 4, st));
      for (int k = 0; k < 8; k++, pass++) {  // pass 0 visits every tile, later passes the marked ones
        uint8_t* in = pass == 0 ? nullptr : ((pass & 1) ? act_a : act_b);
        uint8_t* out = (pass & 1) ? act_b : act_a;
        RSTG_CUDA(cudaMemsetAsync(out, 0, ntile, st));
        k_flood<<<fg, fb, 0, st>>>(gd, sas.as<uint8_t>(), ext.as<uint8_t>(), flag.as<int>(), in, out);
      }
      launched(c, 8);
      int h = 0;
      RSTG_CUDA(cudaMemcpyAsync(&h, flag.p, 4, cudaMemcpyDeviceToHost, st));
      RSTG_CUDA(cudaStreamSynchronize(st));
      done = h == 0;
    }
    if (!done) throw Error(RSTG_ERR_INVALID, "PB exterior flood fill did not settle");
    double thr = (probe / g.h) * (probe / g.h);
    int R = (int)std::floor(std::sqrt(thr)) + 1;
    std::vector<int4> offs;
    for (int z = -R; z <= R; z++)
      for (int y = -R; y <= R; y++)
        for (int x = -R; x <= R; x++)
          if ((double)(x * x + y * y + z * z) <= thr) offs.push_back(make_int4(x, y, z, x * x + y * y + z * z));
    std::sort(offs.begin(), offs.end(), [](const int4& a, const int4& b) { return a.w < b.w; });
    DevBuf doff(offs.size() * sizeof(int4), st);
    RSTG_CUDA(cudaMemcpyAsync(doff.p, offs.data(), offs.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
    k_ses<<<nblk(n, 256), 256, 0, st>>>(gd, ext.as<uint8_t>(), doff.as<int4>(), (int)offs.size(), inside.as<uint8_t>());
    launched(c);
  }
  HashBuf he(pb_build_hash(A.hx, A.max_r + g.h), st);
  DevBuf ovf(8, st);
  RSTG_CUDA(cudaMemsetAsync(ovf.p, 0, 4, st));
  k_eps<<<nblk(n, 128), 128, 0, st>>>(gd, inside.as<uint8_t>(), he.d, A.xyz.as<double>(), A.r.as<double>(), ein, eout,
                                      ex, ey, ez, ovf.as<int>());
  launched(c);
  int h = 0;
  RSTG_CUDA(cudaMemcpyAsync(&h, ovf.p, 4, cudaMemcpyDeviceToHost, st));
  RSTG_CUDA(cudaStreamSynchronize(st));
  if (h) throw Error(RSTG_ERR_INVALID, "more than 64 atom chords on one grid edge");
}

static void dielectric_maps(Ctx* c, Maps& M, const AtomsDev& A, double probe, double ein, double eout) {
  cudaStream_t st = pb_stream(c);
  long long n = (long long)M.g.n();
  M.ex = DevBuf(n * 8, st);
  M.ey = DevBuf(n * 8, st);
  M.ez = DevBuf(n * 8, st);
  dielectric_into(c, M.g, A, probe, ein, eout, M.ex.as<double>(), M.ey.as<double>(), M.ez.as<double>());
}

static void kappa_into(Ctx* c, const PbGeom& g, const AtomsDev& A, double ion, double kap, double eps_s, bool ionic,
                       double* k2) {
  cudaStream_t st = pb_stream(c);
  long long n = (long long)g.n();
  if (!ionic) {
    RSTG_CUDA(cudaMemsetAsync(k2, 0, n * 8, st));
    return;
  }
  double kbs = eps_s * kap * kap;
  HashBuf hk(pb_build_hash(A.hx, A.max_r + ion), st);
  k_kappa<<<nblk(n, 256), 256, 0, st>>>(gdev(g), hk.d, A.xyz.as<double>(), A.r.as<double>(), ion, kbs, k2);
  launched(c);
}

static void kappa_map(Ctx* c, Maps& M, const AtomsDev& A, double ion, double kap, double eps_s, bool ionic) {
  M.k2 = DevBuf(M.g.n() * 8, pb_stream(c));
  kappa_into(c, M.g, A, ion, kap, eps_s, ionic, M.k2.as<double>());
}

struct MgLevel {
  PbGeom g;
  DevBuf ex, ey, ez, k2, rhs, corr, res;  // res: residual buffer of the finer level
  double omega;
};

struct SolveOut {
  DevBuf phi;
  int64_t iterations = 0;
  double residual = 0.0;
  bool converged = false;
};

static LevelDev ldev(const PbGeom& g, const double* ex, const double* ey, const double* ez, const double* k2) {
  double ih = 1.0 / (g.h * g.h);
  return LevelDev{g.nx, g.ny, g.nz, ih, ih, ih, ex, ey, ez, k2};
}

// rel: the relative-residual mode's consistent multigrid (Gauss-Seidel
// smoothing, restriction without the 0.25 factor, series/parallel coarse
// dielectrics, corrections zero on the boundary) instead of the reference's.
struct Solver {
  Ctx* c;
  cudaStream_t st;
  MapsView M;
  std::vector<MgLevel> L;
  DevBuf part, scal;
  bool rel = false;
  Solver(Ctx* cc, const MapsView& m, bool relative = false) : c(cc), st(pb_stream(cc)), M(m), rel(relative) {
    size_t parts = (size_t)nblk(m.g.nx, 128) * std::max(m.g.ny - 2, 1) * std::max(m.g.nz - 2, 1);
    part = DevBuf(std::max<size_t>(parts, 1) * 8, st);
    scal = DevBuf(64, st);
  }

  void build_levels() {  // pb_solver.rs:776-836
    PbGeom g = M.g;
    const double *ex = M.ex, *ey = M.ey, *ez = M.ez, *k2 = M.k2;
    for (;;) {
      if (std::min(g.nx, std::min(g.ny, g.nz)) <= 5) break;
      MgLevel lv;
      lv.g.nx = (g.nx + 1) / 2;
      lv.g.ny = (g.ny + 1) / 2;
      lv.g.nz = (g.nz + 1) / 2;
      lv.g.h = g.h * 2.0;
      long long cn = (long long)lv.g.n(), fn = (long long)g.n();
      for (DevBuf* b : {&lv.ex, &lv.ey, &lv.ez, &lv.k2, &lv.rhs, &lv.corr}) *b = DevBuf(cn * 8, st);
      lv.res = DevBuf(fn * 8, st);
      const double* src[4] = {ex, ey, ez, k2};
      DevBuf* dst[4] = {&lv.ex, &lv.ey, &lv.ez, &lv.k2};
      for (int k = 0; k < 4; k++)
        if (rel && k < 3)
          k_coarsen_face<<<nblk(cn, 256), 256, 0, st>>>(src[k], g.nx, g.ny, g.nz, dst[k]->as<double>(), lv.g.nx,
                                                        lv.g.ny, lv.g.nz, k);
        else
          k_coarsen<<<nblk(cn, 256), 256, 0, st>>>(src[k], g.nx, g.ny, g.nz, dst[k]->as<double>(), lv.g.nx, lv.g.ny,
                                                   lv.g.nz);
      launched(c, 4);
      lv.omega = rel ? 1.0 : pb_omega(lv.g.nx, lv.g.ny, lv.g.nz);
      L.push_back(std::move(lv));
      MgLevel& b = L.back();
      ex = b.ex.as<double>();
      ey = b.ey.as<double>();
      ez = b.ez.as<double>();
      k2 = b.k2.as<double>();
      g = b.g;
    }
  }

  void smooth(const LevelDev& ld, double* phi, const double* rho, double omega, int sweeps, double rs, double* rms) {
    dim3 grid(nblk((ld.nx - 1) / 2, 64), std::max(ld.ny - 2, 1), std::max(ld.nz - 2, 1));
    if (ld.nx < 3 || ld.ny < 3 || ld.nz < 3) return;
    for (int s = 0; s < sweeps; s++) {
      for (int color = 0; color < 2; color++) {
        k_rb<<<grid, 64, 0, st>>>(ld, phi, rho, omega, rs, color, rms ? part.as<double>() + 0 : nullptr);
        launched(c);
        if (rms) {  // per-colour partial sums, accumulated in fixed order
          long long nb = (long long)grid.x * grid.y * grid.z;
          k_sum_fixed<<<1, 1024, 0, st>>>(part.as<double>(), nb, scal.as<double>() + 1 + color);
          launched(c);
        }
      }
    }
    if (rms) {
      double h[2];
      RSTG_CUDA(cudaMemcpyAsync(h, scal.as<double>() + 1, 16, cudaMemcpyDeviceToHost, st));
      RSTG_CUDA(cudaStreamSynchronize(st));
      long long cnt = 0;
      for (int color = 0; color < 2; color++)
        for (int iz = 1; iz < ld.nz - 1; iz++)
          for (int iy = 1; iy < ld.ny - 1; iy++) {
            int x0 = 1 + ((1 + iy + iz + color) & 1);
            if (x0 < ld.nx - 1) cnt += (ld.nx - 1 - x0 + 1) / 2;
          }
      *rms = cnt > 0 ? std::sqrt((h[0] + h[1]) / (double)cnt) : 0.0;
    }
  }

  void v_cycle(size_t lvl, const PbGeom& g, const LevelDev& ld, double* phi, const double* rho, double omega,
               double rs) {
    if (lvl == L.size()) {
      if (g.nx >= 3 && g.ny >= 3 && g.nz >= 3) {
        k_coarse_solve<<<1, 1024, 0, st>>>(ld, phi, rho, omega, rs, 50);
        launched(c);
      }
      return;
    }
    MgLevel& lv = L[lvl];
    smooth(ld, phi, rho, omega, 3, rs, nullptr);
    long long fn = (long long)g.n();
    RSTG_CUDA(cudaMemsetAsync(lv.res.p, 0, fn * 8, st));
    if (g.nx >= 3 && g.ny >= 3 && g.nz >= 3) {
      dim3 grid(nblk(g.nx - 2, 128), g.ny - 2, g.nz - 2);
      k_residual<<<grid, 128, 0, st>>>(ld, phi, rho, rs, lv.res.as<double>(), nullptr);
      launched(c);
    }
    long long cn = (long long)lv.g.n();
    k_restrict<<<nblk(cn, 256), 256, 0, st>>>(lv.res.as<double>(), g.nx, g.ny, g.nz, lv.rhs.as<double>(), lv.g.nx,
                                              lv.g.ny, lv.g.nz, rel ? 1.0 : 0.25);
    RSTG_CUDA(cudaMemsetAsync(lv.corr.p, 0, cn * 8, st));
    launched(c);
    LevelDev cl = ldev(lv.g, lv.ex.as<double>(), lv.ey.as<double>(), lv.ez.as<double>(), lv.k2.as<double>());
    v_cycle(lvl + 1, lv.g, cl, lv.corr.as<double>(), lv.rhs.as<double>(), lv.omega, 1.0);
    k_prolong<<<nblk(fn, 256), 256, 0, st>>>(lv.corr.as<double>(), lv.g.nx, lv.g.ny, lv.g.nz, phi, g.nx, g.ny, g.nz,
                                             rel ? 1 : 0);
    launched(c);
    smooth(ld, phi, rho, omega, 3, rs, nullptr);
  }

  double rms_residual(const LevelDev& ld, const double* phi, const double* rho, double rs) {
    const PbGeom& g = M.g;
    if (g.nx < 3 || g.ny < 3 || g.nz < 3) return 0.0;
    dim3 grid(nblk(g.nx - 2, 128), g.ny - 2, g.nz - 2);
    k_residual<<<grid, 128, 0, st>>>(ld, phi, rho, rs, nullptr, part.as<double>());
    long long nb = (long long)grid.x * grid.y * grid.z;
    k_sum_fixed<<<1, 1024, 0, st>>>(part.as<double>(), nb, scal.as<double>());
    launched(c, 2);
    double s = 0.0;
    RSTG_CUDA(cudaMemcpyAsync(&s, scal.p, 8, cudaMemcpyDeviceToHost, st));
    RSTG_CUDA(cudaStreamSynchronize(st));
    double cnt = (double)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
    return std::sqrt(s / cnt);
  }
};

static void apply_bc(Ctx* c, const PbGeom& g, double* phi, const AtomsDev& A, const BcSpec& bc) {
  cudaStream_t st = pb_stream(c);
  long long n = (long long)g.n();
  if (bc.kind == 1) {
    long long nbnd = boundary_count(g);
    k_dh<<<nblk(nbnd, 256), 256, 0, st>>>(gdev(g), nbnd, A.xyz.as<double>(), A.q.as<double>(), A.n, bc.kappa, bc.eout,
                                          phi);
  } else {
    k_interp_boundary<<<nblk(n, 256), 256, 0, st>>>(gdev(g), gdev(*bc.cg), bc.cphi, phi);
  }
  launched(c);
}

// solve_lpbe_multigrid (pb_solver.rs:1015-1167) with the plain SOR fallback
// (pb_solver.rs:373-447).  rtol > 0: the relative-residual mode -- the
// consistent multigrid, stopping when the RMS residual falls below rtol times
// its initial value (SOR grids: the residual after each sweep); the
// reference's cycle cap and divergence rule stay.
static SolveOut solve_mg(Ctx* c, const MapsView& M, const AtomsDev& A, const BcSpec& bc, double tol, int64_t maxit,
                         double rtol = 0.0) {
  cudaStream_t st = pb_stream(c);
  const PbGeom& g = M.g;
  long long n = (long long)g.n();
  SolveOut R;
  R.phi = DevBuf(n * 8, st);
  RSTG_CUDA(cudaMemsetAsync(R.phi.p, 0, n * 8, st));
  apply_bc(c, g, R.phi.as<double>(), A, bc);
  const bool rel = rtol > 0.0;
  Solver S(c, M, rel);
  LevelDev top = ldev(g, M.ex, M.ey, M.ez, M.k2);
  const double r0 = rel ? S.rms_residual(top, R.phi.as<double>(), M.rho, kFourPiEc) : 0.0;
  auto sor = [&](bool restart) {
    if (restart) RSTG_CUDA(cudaMemsetAsync(R.phi.p, 0, n * 8, st));
    apply_bc(c, g, R.phi.as<double>(), A, bc);
    double rj = spectral_radius(g.nx, g.ny, g.nz), rs2 = rj * rj, om = 1.0;
    R.residual = std::numeric_limits<double>::max();
    R.converged = false;
    for (int64_t it = 0; it < maxit; it++) {
      double rms = 0.0;
      S.smooth(top, R.phi.as<double>(), M.rho, om, 1, kFourPiEc, &rms);
      if (rel) rms = S.rms_residual(top, R.phi.as<double>(), M.rho, kFourPiEc) / std::max(r0, 1e-300);
      R.residual = rms;
      R.iterations = it + 1;
      om = it == 0 ? 1.0 / (1.0 - rs2 / 2.0) : 1.0 / (1.0 - rs2 * om / 4.0);
      if (rms < (rel ? rtol : tol)) {
        R.converged = true;
        return;
      }
    }
  };
  int md = std::min(g.nx, std::min(g.ny, g.nz));
  if (md <= 8) {
    sor(true);
    return R;
  }
  int64_t maxv = std::min<int64_t>(std::max<int64_t>(maxit / 6, 1), 200);
  S.build_levels();
  double omega = rel ? 1.0 : pb_omega(g.nx, g.ny, g.nz);
  double best = std::numeric_limits<double>::max(), prev = std::numeric_limits<double>::max();
  int growing = 0;
  for (int64_t cyc = 0; cyc < maxv; cyc++) {
    S.v_cycle(0, g, top, R.phi.as<double>(), M.rho, omega, kFourPiEc);
    double r = S.rms_residual(top, R.phi.as<double>(), M.rho, kFourPiEc);
    if (r < best) {
      best = r;
      growing = 0;
    } else {
      growing++;
    }
    bool div = !std::isfinite(r) || r > best * 1e4 || (growing >= 5 && r > prev);
    if (div) {
      sor(false);
      return R;
    }
    prev = r;
    if (rel ? r < rtol * r0 : r < tol) {
      R.iterations = cyc + 1;
      R.residual = rel ? r / std::max(r0, 1e-300) : r;
      R.converged = true;
      return R;
    }
  }
  R.residual = S.rms_residual(top, R.phi.as<double>(), M.rho, kFourPiEc) / (rel ? std::max(r0, 1e-300) : 1.0);
  R.iterations = maxv;
  R.converged = false;
  return R;
}

static double elec_energy(Ctx* c, const PbGeom& g, const double* phi, const AtomsDev& A) {
  cudaStream_t st = pb_stream(c);
  if (A.n == 0) return 0.0;
  DevBuf v(A.n * 8, st), e(8, st);
  k_atom_phi<<<nblk(A.n, 128), 128, 0, st>>>(gdev(g), phi, A.xyz.as<double>(), A.q.as<double>(), A.n, v.as<double>());
  k_seq_sum<<<1, 32, 0, st>>>(v.as<double>(), A.n, e.as<double>());
  launched(c, 2);
  double h = 0.0;
  RSTG_CUDA(cudaMemcpyAsync(&h, e.p, 8, cudaMemcpyDeviceToHost, st));
  RSTG_CUDA(cudaStreamSynchronize(st));
  return h;
}

static double maxabs(Ctx* c, const DevBuf& phi, long long n) {
  DevBuf o(8, pb_stream(c));
  k_maxabs<<<1, 1024, 0, pb_stream(c)>>>(phi.as<double>(), n, o.as<double>());
  launched(c);
  double h = 0.0;
  RSTG_CUDA(cudaMemcpyAsync(&h, o.p, 8, cudaMemcpyDeviceToHost, pb_stream(c)));
  RSTG_CUDA(cudaStreamSynchronize(pb_stream(c)));
  return h;
}

// pb_solve_with_focusing, pb_energy.rs:134-322
static double solve_focus(Ctx* c, const Maps& fine_rho, const PbGeom* cg, const AtomsDev& A, const rstg_pb_params& p,
                          double ein, double eout, double kap, bool ionic, SolveOut* out, double rtol) {
  double bck = ionic ? kap : 0.0;
  BcSpec dh;
  dh.kind = 1;
  dh.kappa = bck;
  dh.eout = eout;
  auto fine_maps = [&](Maps& M) {
    M.g = fine_rho.g;
    dielectric_maps(c, M, A, p.probe_radius, ein, eout);
    kappa_map(c, M, A, p.ion_radius, kap, p.solvent_dielectric, ionic);
  };
  Maps F;
  F.g = fine_rho.g;
  if (cg) {
    Maps C;
    C.g = *cg;
    charge_map(c, *cg, A, C.rho);
    dielectric_maps(c, C, A, p.probe_radius, ein, eout);
    kappa_map(c, C, A, p.ion_radius, kap, p.solvent_dielectric, ionic);
    SolveOut cr = solve_mg(c, C.view(), A, dh, p.tolerance * 10.0, p.max_iterations, rtol);
    double mp = maxabs(c, cr.phi, (long long)cg->n());
    bool ok = cr.converged && std::isfinite(mp) && mp < 1e10;
    fine_maps(F);
    F.rho = DevBuf(fine_rho.g.n() * 8, pb_stream(c));
    RSTG_CUDA(cudaMemcpyAsync(F.rho.p, fine_rho.rho.p, fine_rho.g.n() * 8, cudaMemcpyDeviceToDevice, pb_stream(c)));
    if (!ok) {
      *out = solve_mg(c, F.view(), A, dh, p.tolerance, p.max_iterations, rtol);
    } else {
      BcSpec ib;
      ib.kind = 2;
      ib.cg = cg;
      ib.cphi = cr.phi.as<double>();
      *out = solve_mg(c, F.view(), A, ib, p.tolerance, p.max_iterations, rtol);
      RSTG_CUDA(cudaStreamSynchronize(pb_stream(c)));
    }
    return elec_energy(c, F.g, out->phi.as<double>(), A);
  }
  fine_maps(F);
  F.rho = DevBuf(fine_rho.g.n() * 8, pb_stream(c));
  RSTG_CUDA(cudaMemcpyAsync(F.rho.p, fine_rho.rho.p, fine_rho.g.n() * 8, cudaMemcpyDeviceToDevice, pb_stream(c)));
  *out = solve_mg(c, F.view(), A, dh, p.tolerance, p.max_iterations, rtol);
  return elec_energy(c, F.g, out->phi.as<double>(), A);
}

void pb_grid_maps(Ctx* c, const std::vector<double>& x, const std::vector<double>& q, const std::vector<double>& radii,
                  const rstg_pb_params& p, double ein, double eout, bool ionic, int64_t* dims, double* origin,
                  double* charge, uint8_t* inside, double* ex, double* ey, double* ez, double* k2, double* bphi) {
  double s = p.salt_concentration;
  double kap = s <= 0.0 ? 0.0
                        : std::sqrt(8.0 * kPi * 332.0522 * 6.022e-4 * s / (p.solvent_dielectric * 0.00198688 * p.temperature));
  PbGeom g = pb_auto_grid(x, p.grid_spacing, p.grid_buffer);
  dims[0] = g.nx;
  dims[1] = g.ny;
  dims[2] = g.nz;
  origin[0] = g.ox;
  origin[1] = g.oy;
  origin[2] = g.oz;
  if (!charge) return;
  cudaStream_t st = pb_stream(c);
  AtomsDev A(x, q, radii, st);
  Maps M;
  M.g = g;
  charge_map(c, g, A, M.rho);
  dielectric_maps(c, M, A, p.probe_radius, ein, eout);
  kappa_map(c, M, A, p.ion_radius, kap, p.solvent_dielectric, ionic);
  long long n = (long long)g.n();
  DevBuf phi(n * 8, st), ins(n, st);
  RSTG_CUDA(cudaMemsetAsync(phi.p, 0, n * 8, st));
  BcSpec dh;
  dh.kappa = ionic ? kap : 0.0;
  dh.eout = eout;
  apply_bc(c, g, phi.as<double>(), A, dh);
  if (inside) {
    if (p.probe_radius > 0.0) {
      HashBuf hs(pb_build_hash(A.hx, A.max_r + p.probe_radius), st);
      DevBuf sas(n, st), ext(n, st), flag(8, st);
      GeomDev gd = gdev(g);
      k_inside<<<nblk(n, 256), 256, 0, st>>>(gd, hs.d, A.xyz.as<double>(), A.r.as<double>(), p.probe_radius,
                                             sas.as<uint8_t>());
      k_flood_seed<<<nblk(n, 256), 256, 0, st>>>(gd, sas.as<uint8_t>(), ext.as<uint8_t>());
      launched(c, 2);
      dim3 fb(8, 8, 8), fg(nblk(g.nx, 8), nblk(g.ny, 8), nblk(g.nz, 8));
      for (int guard = 0; guard < 100000; guard++) {
        RSTG_CUDA(cudaMemsetAsync(flag.p, 0, 4, st));
        k_flood<<<fg, fb, 0, st>>>(gd, sas.as<uint8_t>(), ext.as<uint8_t>(), flag.as<int>(), nullptr, nullptr);
        launched(c);
        int h = 0;
        RSTG_CUDA(cudaMemcpyAsync(&h, flag.p, 4, cudaMemcpyDeviceToHost, st));
        RSTG_CUDA(cudaStreamSynchronize(st));
        if (!h) break;
      }
      double thr = (p.probe_radius / g.h) * (p.probe_radius / g.h);
      int R = (int)std::floor(std::sqrt(thr)) + 1;
      std::vector<int4> offs;
      for (int z = -R; z <= R; z++)
        for (int y = -R; y <= R; y++)
          for (int xx = -R; xx <= R; xx++)
            if ((double)(xx * xx + y * y + z * z) <= thr) offs.push_back(make_int4(xx, y, z, 0));
      DevBuf doff(offs.size() * sizeof(int4), st);
      RSTG_CUDA(cudaMemcpyAsync(doff.p, offs.data(), offs.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
      k_ses<<<nblk(n, 256), 256, 0, st>>>(gd, ext.as<uint8_t>(), doff.as<int4>(), (int)offs.size(), ins.as<uint8_t>());
      launched(c);
      RSTG_CUDA(cudaStreamSynchronize(st));
    } else {
      HashBuf hs(pb_build_hash(A.hx, A.max_r), st);
      k_inside<<<nblk(n, 256), 256, 0, st>>>(gdev(g), hs.d, A.xyz.as<double>(), A.r.as<double>(), 0.0,
                                             ins.as<uint8_t>());
      launched(c);
      RSTG_CUDA(cudaStreamSynchronize(st));
    }
    RSTG_CUDA(cudaMemcpyAsync(inside, ins.p, n, cudaMemcpyDeviceToHost, st));
  }
  RSTG_CUDA(cudaMemcpyAsync(charge, M.rho.p, n * 8, cudaMemcpyDeviceToHost, st));
  RSTG_CUDA(cudaMemcpyAsync(ex, M.ex.p, n * 8, cudaMemcpyDeviceToHost, st));
  RSTG_CUDA(cudaMemcpyAsync(ey, M.ey.p, n * 8, cudaMemcpyDeviceToHost, st));
  RSTG_CUDA(cudaMemcpyAsync(ez, M.ez.p, n * 8, cudaMemcpyDeviceToHost, st));
  RSTG_CUDA(cudaMemcpyAsync(k2, M.k2.p, n * 8, cudaMemcpyDeviceToHost, st));
  RSTG_CUDA(cudaMemcpyAsync(bphi, phi.p, n * 8, cudaMemcpyDeviceToHost, st));
  RSTG_CUDA(cudaStreamSynchronize(st));
}

double pb_energy_run(Ctx* c, const std::vector<double>& x, const std::vector<double>& q,
                     const std::vector<double>& radii, const rstg_pb_params& p, rstg_pb_diag* diag, double rtol) {
  if (!(p.grid_spacing > 0.0)) throw Error(RSTG_ERR_INVALID, "grid_spacing must be positive");
  if (q.empty()) return 0.0;
  double s = p.salt_concentration;
  double kap = s <= 0.0 ? 0.0
                        : std::sqrt(8.0 * kPi * 332.0522 * 6.022e-4 * s / (p.solvent_dielectric * 0.00198688 * p.temperature));
  AtomsDev A(x, q, radii, pb_stream(c));
  Maps fine;
  fine.g = pb_auto_grid(x, p.grid_spacing, p.grid_buffer);
  if (fine.g.n() > (size_t)600 * 600 * 600) throw Error(RSTG_ERR_NOMEM, "PB grid exceeds 600^3 points");
  PbGeom cg;
  bool focus = p.fillratio > 0.0 && p.fscale > 1;
  if (focus) cg = pb_coarse_grid(x, p.grid_spacing, p.fillratio, p.fscale);
  charge_map(c, fine.g, A, fine.rho);
  SolveOut rs, rr;
  double es = solve_focus(c, fine, focus ? &cg : nullptr, A, p, p.solute_dielectric, p.solvent_dielectric, kap, true,
                          &rs, rtol);
  double er = solve_focus(c, fine, focus ? &cg : nullptr, A, p, p.solute_dielectric, p.solute_dielectric, kap, false,
                          &rr, rtol);
  if (diag) {
    diag->iterations[0] = rs.iterations;
    diag->iterations[1] = rr.iterations;
    diag->residual[0] = rs.residual;
    diag->residual[1] = rr.residual;
    diag->converged[0] = rs.converged;
    diag->converged[1] = rr.converged;
    diag->dims[0] = fine.g.nx;
    diag->dims[1] = fine.g.ny;
    diag->dims[2] = fine.g.nz;
  }
  return es - er;
}

// ---------------------------------------------------------------------------
// entry points of the batched engine (pb_batch.cu)
// ---------------------------------------------------------------------------
static thread_local cudaStream_t t_pb_stream = nullptr;
cudaStream_t pb_stream(Ctx* c) { return t_pb_stream ? t_pb_stream : c->stream; }
PbStreamScope::PbStreamScope(cudaStream_t s) : prev(t_pb_stream) { t_pb_stream = s; }
PbStreamScope::~PbStreamScope() { t_pb_stream = prev; }

double pb_kappa(const rstg_pb_params& p) {  // pb_energy.rs:337-345
  double s = p.salt_concentration;
  return s <= 0.0 ? 0.0
                  : std::sqrt(8.0 * kPi * 332.0522 * 6.022e-4 * s / (p.solvent_dielectric * 0.00198688 * p.temperature));
}

void pb_maps_into(Ctx* c, const PbGeom& g, const AtomsDev& A, const rstg_pb_params& p, double ein, double eout,
                  double kap, bool ionic, double* rho, double* ex, double* ey, double* ez, double* k2) {
  if (rho) charge_into(c, g, A, rho);
  if (ex) dielectric_into(c, g, A, p.probe_radius, ein, eout, ex, ey, ez);
  if (k2) kappa_into(c, g, A, p.ion_radius, kap, p.solvent_dielectric, ionic, k2);
}

void pb_boundary(Ctx* c, const PbGeom& g, double* phi, const AtomsDev& A, const BcSpec& bc) { apply_bc(c, g, phi, A, bc); }

PbSolveStats pb_solve_fp64(Ctx* c, const PbGeom& g, const double* rho, const double* ex, const double* ey,
                           const double* ez, const double* k2, double uniform_eps, const AtomsDev& A,
                           const BcSpec& bc, double tol, int64_t maxit, double* phi_out) {
  cudaStream_t st = pb_stream(c);
  long long n = (long long)g.n();
  DevBuf fx, fy, fz, fk;
  if (!ex) {
    fx = DevBuf(n * 8, st);
    fy = DevBuf(n * 8, st);
    fz = DevBuf(n * 8, st);
    fk = DevBuf(n * 8, st);
    for (DevBuf* b : {&fx, &fy, &fz}) k_fill<<<nblk(n, 256), 256, 0, st>>>(b->as<double>(), n, uniform_eps);
    RSTG_CUDA(cudaMemsetAsync(fk.p, 0, n * 8, st));
    launched(c, 3);
    ex = fx.as<double>();
    ey = fy.as<double>();
    ez = fz.as<double>();
    k2 = fk.as<double>();
  }
  MapsView M{g, rho, ex, ey, ez, k2};
  SolveOut R = solve_mg(c, M, A, bc, tol, maxit);
  RSTG_CUDA(cudaMemcpyAsync(phi_out, R.phi.p, n * 8, cudaMemcpyDeviceToDevice, st));
  RSTG_CUDA(cudaStreamSynchronize(st));
  return PbSolveStats{R.iterations, R.residual, R.converged};
}

}  // namespace rstg
