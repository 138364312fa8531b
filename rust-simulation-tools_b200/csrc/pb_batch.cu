// Batched mixed-precision Poisson-Boltzmann solves.
//
// Every grid of a batch (frames x {complex, receptor, ligand} x {solvated,
// reference}) advances in lock step: one launch per multigrid step covers all
// grids that are still iterating.  Each cycle is the reference's V-cycle
// (pb_solver.rs:838-1012) written as defect correction:
//     r   = 4 pi ec rho + (div eps grad - kbar^2) phi     FP64, exact maps
//     e   = V-cycle(r, e0 = 0)                            FP32
//     phi = phi + e                                       FP64
// The smoother, restriction and prolongation are linear, so the reference's
// V-cycle applied to phi equals phi + B r with B the V-cycle on the residual
// equation; evaluating B in FP32 perturbs each correction by a relative
// ~1e-7 and the FP64 residual keeps the iterates on the reference's
// sequence.  The convergence and divergence bookkeeping of
// solve_lpbe_multigrid (pb_solver.rs:1080-1160) runs per grid on the device.
// Grids too small for multigrid and grids whose V-cycles diverge continue
// with the reference's Chebyshev-accelerated red-black SOR
// (pb_solver.rs:373-447), also in defect-correction form: one SOR sweep on
// the residual equation from e = 0 equals one sweep on phi, and the sweep's
// update measure sum (gs - old)^2 is the same quantity.
//
// Launches are driven by work lists: for each launch the host lists the
// grids that take part and the first block of each, so no block is spent on
// a grid that has finished or is smaller than the largest one.  The lists
// (and the CUDA graph that holds a chunk of cycles) are rebuilt when a grid
// changes state; the host reads the per-grid states once per chunk.
//
// Layout in HBM: one FP64 pool (phi, rho and, for solvated grids, the four
// face-dielectric / kbar^2 maps, each g.n() doubles) and one FP32 pool (per
// multigrid level: correction, right-hand side, residual and the four maps
// of solvated grids).  Reference grids have a uniform dielectric and no
// salt term, so their stencil is the constant-coefficient Laplacian and they
// carry no maps.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>

#include "common.cuh"
#include "pb_batch.hpp"

namespace rstg {

namespace {

constexpr int kMaxLev = 16;
constexpr double kFourPiEcB = 4.0 * kPi * 332.0522;  // pb_solver.rs:155
constexpr int kT = 256;

// grid states
constexpr int kMg = 0, kConverged = 1, kDiverged = 2, kMgCap = 3, kSor = 5, kSorCap = 6;

struct JobD {
  double* phi;
  const double* rho;
  const double *ex, *ey, *ez, *k2;
  const double *axyz, *aq;
  int nx, ny, nz, uniform;
  int na, want_e, maxv, pad;
  double ih, eps, tol, rs2;
  double ox, oy, oz, h;
  long long maxit;
};

struct LvlD {
  float *e, *e2, *rhs, *res;  // correction (two buffers: a sweep reads one and writes the other)
  const float *ex, *ey, *ez, *k2;
  int nx, ny, nz, uniform;
  float ih, om, eps, pad;
};

struct JobState {
  double best, prev, rms, r0, om;
  int growing, cycles, status, pad;
  long long sor_it;
};

// Work list of one launch: job[k] owns blocks start[k] .. start[k+1]-1.
struct WL {
  const int* start;
  const int* job;
  int n;
};

__device__ __forceinline__ int wl_job(const WL& w, int b, int& lb) {
  int lo = 0, hi = w.n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (w.start[mid] <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  lb = b - w.start[lo];
  return w.job[lo];
}

// FP32 7-point stencil of pb_solver.rs:250-317: ns = sum of eps-weighted
// neighbours, dg = diagonal.
__device__ __forceinline__ void st32(const LvlD& d, const float* __restrict__ e, int i, int sy, int sz, float& ns,
                                     float& dg) {
  if (d.uniform) {
    float w = d.eps * d.ih;
    ns = w * ((e[i + 1] + e[i - 1]) + (e[i + sy] + e[i - sy]) + (e[i + sz] + e[i - sz]));
    dg = 6.0f * w;
  } else {
    float a = d.ex[i], b = d.ex[i - 1], c = d.ey[i], dd = d.ey[i - sy], f = d.ez[i], g = d.ez[i - sz];
    ns = ((a * e[i + 1] + b * e[i - 1]) + (c * e[i + sy] + dd * e[i - sy]) + (f * e[i + sz] + g * e[i - sz])) * d.ih;
    dg = ((a + b) + (c + dd) + (f + g)) * d.ih + d.k2[i];
  }
}

// FP64 residual r = 4 pi ec rho + ns - dg phi at the interior points; r is
// stored rounded to FP32 as the level-0 right-hand side and its squares are
// summed per block (fixed order) for the RMS test.
__global__ void k_res64(WL w, const JobD* __restrict__ J, const LvlD* __restrict__ L, const JobState* __restrict__ S,
                        int want, double* __restrict__ part, int nparts) {
  __shared__ double sh[32];
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != want) return;
  const JobD& d = J[j];
  float* rhs0 = L[j * kMaxLev].rhs;
  int nxi = d.nx - 2, nyi = d.ny - 2;
  int cnt = nxi * nyi * (d.nz - 2);
  int k = lb * blockDim.x + threadIdx.x;
  double acc = 0.0;
  if (k < cnt) {
    int ix = 1 + k % nxi, row = k / nxi;
    int iy = 1 + row % nyi, iz = 1 + row / nyi;
    int sy = d.nx, sz = d.nx * d.ny, i = ix + sy * iy + sz * iz;
    const double* p = d.phi;
    double ns, dg;
    if (d.uniform) {
      double wt = d.eps * d.ih;
      ns = wt * ((p[i + 1] + p[i - 1]) + (p[i + sy] + p[i - sy]) + (p[i + sz] + p[i - sz]));
      dg = 6.0 * wt;
    } else {
      double a = d.ex[i], b = d.ex[i - 1], c = d.ey[i], dd = d.ey[i - sy], f = d.ez[i], g = d.ez[i - sz];
      ns = (a * p[i + 1] + b * p[i - 1]) * d.ih + (c * p[i + sy] + dd * p[i - sy]) * d.ih +
           (f * p[i + sz] + g * p[i - sz]) * d.ih;
      dg = (a + b) * d.ih + (c + dd) * d.ih + (f + g) * d.ih + d.k2[i];
    }
    double r = kFourPiEcB * d.rho[i] + ns - dg * p[i];
    rhs0[i] = (float)r;
    acc = r * r;
  }
  double s = block_sum(acc, sh);
  if (threadIdx.x == 0) part[(long long)j * nparts + lb] = s;
}

// RMS of the residual and the reference's multigrid bookkeeping
// (pb_solver.rs:1080-1160); one block per listed grid.
__global__ void k_norm(WL w, const JobD* __restrict__ J, JobState* __restrict__ S, const double* __restrict__ part,
                       int nparts, int check) {
  __shared__ double sh[32];
  int j = w.job[blockIdx.x];
  if (S[j].status != kMg) return;
  const JobD& d = J[j];
  int used = (int)(((long long)(d.nx - 2) * (d.ny - 2) * (d.nz - 2) + kT - 1) / kT);
  double s = 0.0;
  for (int k = threadIdx.x; k < used; k += blockDim.x) s += part[(long long)j * nparts + k];
  s = block_sum(s, sh);
  if (threadIdx.x != 0) return;
  double cnt = (double)(d.nx - 2) * (double)(d.ny - 2) * (double)(d.nz - 2);
  double r = sqrt(s / cnt);
  JobState& t = S[j];
  t.rms = r;
  if (!check) {
    t.r0 = r;
    return;
  }
  t.cycles++;
  if (r < t.best) {
    t.best = r;
    t.growing = 0;
  } else {
    t.growing++;
  }
  bool div = !isfinite(r) || r > t.best * 1e4 || (t.growing >= 5 && r > t.prev);
  if (div) {
    t.status = kDiverged;
    return;
  }
  t.prev = r;
  if (r < d.tol) {
    t.status = kConverged;
  } else if (t.cycles >= d.maxv) {
    t.status = kMgCap;
  }
}

// phi += e over every point (the prolongation can reach boundary points of
// grids with even dimensions), then e = 0 for the next cycle.
__global__ void k_update64(WL w, const JobD* __restrict__ J, const LvlD* __restrict__ L,
                           const JobState* __restrict__ S, int want) {
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != want) return;
  const JobD& d = J[j];
  float* e0 = L[j * kMaxLev].e;
  int n = d.nx * d.ny * d.nz;
  int i = lb * blockDim.x + threadIdx.x;
  if (i >= n) return;
  d.phi[i] += (double)e0[i];
  e0[i] = 0.0f;
}

// One red-black SOR sweep (colour 0, then colour 1; pb_solver.rs:250-317) on
// a brick of 32 x 8 x 8 points of one level.  The brick's correction and a
// ring of two points around it are staged in shared memory; colour 0 is
// relaxed on the brick and the first ring, then colour 1 on the brick,
// whose colour-0 neighbours are then final.  Reading src and writing dst
// keeps the bricks independent, so the level's maps and right-hand side are
// read from DRAM once per sweep instead of once per colour (the overlapping
// rings are served by L2).  Boundary points are copied.
constexpr int kBX = 32, kBY = 8, kBZ = 8, kPX = kBX + 4, kPY = kBY + 4, kPZ = kBZ + 4;

// Relaxes point x of a row (smem index s, global index i) in place.
__device__ __forceinline__ void relax_pt(const LvlD& d, float* __restrict__ sm, int s, int i, int sy, int sz,
                                         bool uni, float w6, float ih, float om, const float* __restrict__ rhs) {
  constexpr int P = kPX * kPY;
  float ns, dg;
  if (uni) {
    ns = w6 * ((sm[s + 1] + sm[s - 1]) + (sm[s + kPX] + sm[s - kPX]) + (sm[s + P] + sm[s - P]));
    dg = 6.0f * w6;
  } else {
    float a = d.ex[i], b = d.ex[i - 1], c = d.ey[i], e = d.ey[i - sy], f = d.ez[i], g = d.ez[i - sz];
    ns = ((a * sm[s + 1] + b * sm[s - 1]) + (c * sm[s + kPX] + e * sm[s - kPX]) + (f * sm[s + P] + g * sm[s - P])) *
         ih;
    dg = ((a + b) + (c + e) + (f + g)) * ih + d.k2[i];
  }
  float old = sm[s];
  float gs = __fdividef(ns + rhs[i], dg);
  sm[s] = old + om * (gs - old);
}

__global__ void __launch_bounds__(256) k_sweep32(WL w, const LvlD* __restrict__ L, int lvl,
                                                 const JobState* __restrict__ S, int src) {
  __shared__ float sm[kPZ * kPY * kPX];
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != kMg) return;
  const LvlD& d = L[j * kMaxLev + lvl];
  const float* __restrict__ ein = src ? d.e2 : d.e;
  float* __restrict__ eout = src ? d.e : d.e2;
  const float* __restrict__ rhs = d.rhs;
  const int nx = d.nx, ny = d.ny, nz = d.nz, sy = nx, sz = nx * ny;
  const int ntx = (nx + kBX - 1) / kBX, nty = (ny + kBY - 1) / kBY;
  const int x0 = (lb % ntx) * kBX, y0 = ((lb / ntx) % nty) * kBY, z0 = (lb / (ntx * nty)) * kBZ;
  const float om = d.om, ih = d.ih, w6 = d.eps * d.ih;
  const bool uni = d.uniform;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  // stage the brick and a ring of two points: one warp per row of 36
  {
    constexpr int NR = kPY * kPZ / 8;  // rows per warp
    float v[NR], u[NR];
    const int xa = x0 - 2 + lane, xb = x0 + 30 + lane;
#pragma unroll
    for (int k = 0; k < NR; k++) {
      int r = wp + 8 * k;
      int y = y0 + r % kPY - 2, z = z0 + r / kPY - 2;
      bool rok = y >= 0 && y < ny && z >= 0 && z < nz;
      int base = sy * y + sz * z;
      v[k] = (rok && xa >= 0 && xa < nx) ? ein[base + xa] : 0.0f;
      u[k] = (rok && lane < 4 && xb < nx) ? ein[base + xb] : 0.0f;
    }
#pragma unroll
    for (int k = 0; k < NR; k++) {
      int r = wp + 8 * k;
      sm[r * kPX + lane] = v[k];
      if (lane < 4) sm[r * kPX + 32 + lane] = u[k];
    }
  }
  __syncthreads();
  // colour 0 ((x + y + z) even) on the brick and its first ring: rows of the
  // ring-1 cross-section, 16 points inside the brick per row (half a warp)
  {
    const int hl = lane & 15, half = lane >> 4;
#pragma unroll
    for (int r = 2 * wp + half; r < (kBY + 2) * (kBZ + 2); r += 16) {
      int ly = r % (kBY + 2) - 1, lz = r / (kBY + 2) - 1;
      int y = y0 + ly, z = z0 + lz;
      if (y < 1 || y > ny - 2 || z < 1 || z > nz - 2) continue;
      int x = x0 + ((x0 + y + z) & 1) + 2 * hl;
      if (x >= 1 && x <= nx - 2)
        relax_pt(d, sm, (x - x0 + 2) + kPX * ((ly + 2) + kPY * (lz + 2)), x + sy * y + sz * z, sy, sz, uni, w6, ih, om,
                 rhs);
    }
    // the colour-0 point of each row just outside the brick in x (x0 - 1 or x0 + 32)
    for (int r = threadIdx.x; r < (kBY + 2) * (kBZ + 2); r += 256) {
      int ly = r % (kBY + 2) - 1, lz = r / (kBY + 2) - 1;
      int y = y0 + ly, z = z0 + lz;
      if (y < 1 || y > ny - 2 || z < 1 || z > nz - 2) continue;
      int x = ((x0 - 1 + y + z) & 1) == 0 ? x0 - 1 : x0 + kBX;
      if (x >= 1 && x <= nx - 2)
        relax_pt(d, sm, (x - x0 + 2) + kPX * ((ly + 2) + kPY * (lz + 2)), x + sy * y + sz * z, sy, sz, uni, w6, ih, om,
                 rhs);
    }
  }
  __syncthreads();
  // colour 1 on the brick
  {
    const int hl = lane & 15, half = lane >> 4;
#pragma unroll
    for (int r = 2 * wp + half; r < kBY * kBZ; r += 16) {
      int ly = r % kBY, lz = r / kBY;
      int y = y0 + ly, z = z0 + lz;
      if (y < 1 || y > ny - 2 || z < 1 || z > nz - 2) continue;
      int x = x0 + ((x0 + y + z + 1) & 1) + 2 * hl;
      if (x >= 1 && x <= nx - 2)
        relax_pt(d, sm, (x - x0 + 2) + kPX * ((ly + 2) + kPY * (lz + 2)), x + sy * y + sz * z, sy, sz, uni, w6, ih, om,
                 rhs);
    }
  }
  __syncthreads();
  for (int r = wp; r < kBY * kBZ; r += 8) {
    int ly = r % kBY, lz = r / kBY;
    int x = x0 + lane, y = y0 + ly, z = z0 + lz;
    if (x < nx && y < ny && z < nz) eout[x + sy * y + sz * z] = sm[(lane + 2) + kPX * ((ly + 2) + kPY * (lz + 2))];
  }
}

// One colour of the plain SOR sweep (pb_solver.rs:373-447) on the level-0
// correction, from e = 0, with per-block sums of (gs - old)^2.
__global__ void k_sor32(WL w, const LvlD* __restrict__ L, const JobState* __restrict__ S, int colour,
                        double* __restrict__ part, int nparts) {
  __shared__ double sh[32];
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != kSor) return;
  const LvlD& d = L[j * kMaxLev];
  float om = (float)S[j].om;
  int hw = (d.nx - 1) >> 1, nyi = d.ny - 2;
  int cnt = hw * nyi * (d.nz - 2);
  int k = lb * blockDim.x + threadIdx.x;
  double acc = 0.0;
  if (k < cnt) {
    int t = k % hw, row = k / hw;
    int iy = 1 + row % nyi, iz = 1 + row / nyi;
    int ix = 1 + ((1 + iy + iz + colour) & 1) + 2 * t;
    if (ix < d.nx - 1) {
      int sy = d.nx, sz = d.nx * d.ny, i = ix + sy * iy + sz * iz;
      float ns, dg;
      st32(d, d.e, i, sy, sz, ns, dg);
      float old = d.e[i];
      float gs = (ns + d.rhs[i]) / dg;
      float dv = gs - old;
      acc = (double)dv * (double)dv;
      d.e[i] = old + om * dv;
    }
  }
  double s = block_sum(acc, sh);
  if (threadIdx.x == 0) part[((long long)j * 2 + colour) * nparts + lb] = s;
}

// SOR bookkeeping: rms of the sweep's updates, Chebyshev omega, convergence
// (pb_solver.rs:373-447).
__global__ void k_sor_norm(WL w, const JobD* __restrict__ J, JobState* __restrict__ S, const double* __restrict__ part,
                           int nparts) {
  __shared__ double sh[32];
  int j = w.job[blockIdx.x];
  if (S[j].status != kSor) return;
  const JobD& d = J[j];
  int used = (int)(((long long)((d.nx - 1) >> 1) * (d.ny - 2) * (d.nz - 2) + kT - 1) / kT);
  double s = 0.0;
  for (int c = 0; c < 2; c++) {  // per colour, then the two colour sums
    double sc = 0.0;
    for (int k = threadIdx.x; k < used; k += blockDim.x) sc += part[((long long)j * 2 + c) * nparts + k];
    sc = block_sum(sc, sh);
    s += sc;
  }
  if (threadIdx.x != 0) return;
  double cnt = (double)(d.nx - 2) * (double)(d.ny - 2) * (double)(d.nz - 2);
  JobState& t = S[j];
  double rms = cnt > 0.0 ? sqrt(s / cnt) : 0.0;
  long long it = t.sor_it;
  t.rms = rms;
  t.sor_it = it + 1;
  t.om = it == 0 ? 1.0 / (1.0 - d.rs2 / 2.0) : 1.0 / (1.0 - d.rs2 * t.om / 4.0);
  if (rms < d.tol)
    t.status = kConverged;
  else if (t.sor_it >= d.maxit)
    t.status = kSorCap;
}

__global__ void k_res32(WL w, const LvlD* __restrict__ L, int lvl, const JobState* __restrict__ S) {
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != kMg) return;
  const LvlD& d = L[j * kMaxLev + lvl];
  int nxi = d.nx - 2, nyi = d.ny - 2;
  int cnt = nxi * nyi * (d.nz - 2);
  int k = lb * blockDim.x + threadIdx.x;
  if (k >= cnt) return;
  int ix = 1 + k % nxi, row = k / nxi;
  int iy = 1 + row % nyi, iz = 1 + row / nyi;
  int sy = d.nx, sz = d.nx * d.ny, i = ix + sy * iy + sz * iz;
  float ns, dg;
  st32(d, d.e2, i, sy, sz, ns, dg);
  d.res[i] = d.rhs[i] + ns - dg * d.e2[i];
}

// Full-weighting restriction x 0.25 of the level-l residual into the
// level-(l+1) right-hand side (pb_solver.rs:459-520); the coarse correction
// starts from zero.
__global__ void k_restrict32(WL w, const LvlD* __restrict__ L, int lvl, const JobState* __restrict__ S) {
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != kMg) return;
  const LvlD& f = L[j * kMaxLev + lvl];
  const LvlD& c = L[j * kMaxLev + lvl + 1];
  int cn = c.nx * c.ny * c.nz;
  int i = lb * blockDim.x + threadIdx.x;
  if (i >= cn) return;
  int cx = i % c.nx, cy = (i / c.nx) % c.ny, cz = i / (c.nx * c.ny);
  int fx = 2 * cx, fy = 2 * cy, fz = 2 * cz;
  float sum = 0.0f, ws = 0.0f;
  for (int dz = -1; dz <= 1; dz++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        int x = fx + dx, y = fy + dy, z = fz + dz;
        if (x < 0 || x >= f.nx || y < 0 || y >= f.ny || z < 0 || z >= f.nz) continue;
        float wt = (dx == 0 ? 2.0f : 1.0f) * (dy == 0 ? 2.0f : 1.0f) * (dz == 0 ? 2.0f : 1.0f);
        sum += wt * f.res[x + f.nx * (y + f.ny * z)];
        ws += wt;
      }
  c.rhs[i] = 0.25f * sum / ws;
  c.e[i] = 0.0f;
}

// Trilinear prolongation of the level-(l+1) correction added at every
// level-l point (pb_solver.rs:522-578), into the pre-smoothed correction.
__global__ void k_prolong32(WL w, const LvlD* __restrict__ L, int lvl, const JobState* __restrict__ S) {
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != kMg) return;
  const LvlD& f = L[j * kMaxLev + lvl];
  const LvlD& c = L[j * kMaxLev + lvl + 1];
  int fn = f.nx * f.ny * f.nz;
  int i = lb * blockDim.x + threadIdx.x;
  if (i >= fn) return;
  int fx = i % f.nx, fy = (i / f.nx) % f.ny, fz = i / (f.nx * f.ny);
  float cxf = (float)fx * 0.5f, cyf = (float)fy * 0.5f, czf = (float)fz * 0.5f;
  int mx = c.nx >= 2 ? c.nx - 2 : 0, my = c.ny >= 2 ? c.ny - 2 : 0, mz = c.nz >= 2 ? c.nz - 2 : 0;
  int x0 = min(fx >> 1, mx), y0 = min(fy >> 1, my), z0 = min(fz >> 1, mz);
  float dx = cxf - (float)x0, dy = cyf - (float)y0, dz = czf - (float)z0;
  const float* ce = c.e;
  auto at = [&](int x, int y, int z) { return ce[x + c.nx * (y + c.ny * z)]; };
  float c00 = at(x0, y0, z0) * (1.0f - dx) + at(x0 + 1, y0, z0) * dx;
  float c10 = at(x0, y0 + 1, z0) * (1.0f - dx) + at(x0 + 1, y0 + 1, z0) * dx;
  float c01 = at(x0, y0, z0 + 1) * (1.0f - dx) + at(x0 + 1, y0, z0 + 1) * dx;
  float c11 = at(x0, y0 + 1, z0 + 1) * (1.0f - dx) + at(x0 + 1, y0 + 1, z0 + 1) * dx;
  float c0 = c00 * (1.0f - dy) + c10 * dy, c1 = c01 * (1.0f - dy) + c11 * dy;
  f.e2[i] += c0 * (1.0f - dz) + c1 * dz;
}

// Coarsest level: 50 red-black sweeps in one block per grid (pb_solver.rs:850-870).
__global__ void k_coarse32(WL w, const LvlD* __restrict__ L, int lvl, const JobState* __restrict__ S, int sweeps) {
  int j = w.job[blockIdx.x];
  if (S[j].status != kMg) return;
  const LvlD& d = L[j * kMaxLev + lvl];
  if (d.nx < 3 || d.ny < 3 || d.nz < 3) return;
  int nxi = d.nx - 2, nyi = d.ny - 2;
  int ni = nxi * nyi * (d.nz - 2);
  int sy = d.nx, sz = d.nx * d.ny;
  for (int s = 0; s < sweeps; s++)
    for (int colour = 0; colour < 2; colour++) {
      for (int k = threadIdx.x; k < ni; k += blockDim.x) {
        int ix = 1 + k % nxi, iy = 1 + (k / nxi) % nyi, iz = 1 + k / (nxi * nyi);
        if (((ix + iy + iz + colour) & 1) != 0) continue;
        int i = ix + sy * iy + sz * iz;
        float ns, dg;
        st32(d, d.e, i, sy, sz, ns, dg);
        float old = d.e[i];
        float gs = (ns + d.rhs[i]) / dg;
        d.e[i] = old + d.om * (gs - old);
      }
      __syncthreads();
    }
}

// Level-0 FP32 maps from the FP64 maps, then injection to coarser levels
// (pb_solver.rs:776-836).
__global__ void k_maps32(WL w, const JobD* __restrict__ J, const LvlD* __restrict__ L) {
  int lb, j = wl_job(w, blockIdx.x, lb);
  const JobD& d = J[j];
  const LvlD& l0 = L[j * kMaxLev];
  int n = d.nx * d.ny * d.nz;
  int i = lb * blockDim.x + threadIdx.x;
  if (i >= n) return;
  ((float*)l0.ex)[i] = (float)d.ex[i];
  ((float*)l0.ey)[i] = (float)d.ey[i];
  ((float*)l0.ez)[i] = (float)d.ez[i];
  ((float*)l0.k2)[i] = (float)d.k2[i];
}

__global__ void k_inject32(WL w, const LvlD* __restrict__ L, int lvl) {
  int lb, j = wl_job(w, blockIdx.x, lb);
  const LvlD& f = L[j * kMaxLev + lvl];
  const LvlD& c = L[j * kMaxLev + lvl + 1];
  int cn = c.nx * c.ny * c.nz;
  int i = lb * blockDim.x + threadIdx.x;
  if (i >= cn) return;
  int cx = i % c.nx, cy = (i / c.nx) % c.ny, cz = i / (c.nx * c.ny);
  int fi = min(2 * cx, f.nx - 1) + f.nx * (min(2 * cy, f.ny - 1) + f.ny * min(2 * cz, f.nz - 1));
  ((float*)c.ex)[i] = f.ex[fi];
  ((float*)c.ey)[i] = f.ey[fi];
  ((float*)c.ez)[i] = f.ez[fi];
  ((float*)c.k2)[i] = f.k2[fi];
}

// 0.5 sum_a q_a phi(x_a), trilinear phi (pb_solver.rs:1174-1186); one block per grid.
__global__ void k_energy64(const JobD* __restrict__ J, double* __restrict__ E) {
  __shared__ double sh[32];
  int j = blockIdx.x;
  const JobD& d = J[j];
  if (!d.want_e) return;
  double acc = 0.0;
  for (int a = threadIdx.x; a < d.na; a += blockDim.x) {
    double fc[3] = {(d.axyz[3 * a] - d.ox) / d.h, (d.axyz[3 * a + 1] - d.oy) / d.h, (d.axyz[3 * a + 2] - d.oz) / d.h};
    long cx = (long)floor(fc[0]), cy = (long)floor(fc[1]), cz = (long)floor(fc[2]);
    if (cx < 0 || cx >= d.nx - 1 || cy < 0 || cy >= d.ny - 1 || cz < 0 || cz >= d.nz - 1) continue;
    double dx = fc[0] - (double)cx, dy = fc[1] - (double)cy, dz = fc[2] - (double)cz;
    const double* p = d.phi;
    auto at = [&](long x, long y, long z) { return p[x + (long)d.nx * (y + (long)d.ny * z)]; };
    double c00 = at(cx, cy, cz) * (1.0 - dx) + at(cx + 1, cy, cz) * dx;
    double c10 = at(cx, cy + 1, cz) * (1.0 - dx) + at(cx + 1, cy + 1, cz) * dx;
    double c01 = at(cx, cy, cz + 1) * (1.0 - dx) + at(cx + 1, cy, cz + 1) * dx;
    double c11 = at(cx, cy + 1, cz + 1) * (1.0 - dx) + at(cx + 1, cy + 1, cz + 1) * dx;
    double c0 = c00 * (1.0 - dy) + c10 * dy, c1 = c01 * (1.0 - dy) + c11 * dy;
    acc += d.aq[a] * (c0 * (1.0 - dz) + c1 * dz);
  }
  double s = block_sum(acc, sh);
  if (threadIdx.x == 0) E[j] = 0.5 * s;
}

// max |phi| per grid, NaN propagating (pb_energy.rs:188-194).
__global__ void k_maxabs64(const JobD* __restrict__ J, double* __restrict__ M) {
  __shared__ double sh[1024];
  int j = blockIdx.x;
  const JobD& d = J[j];
  int n = d.nx * d.ny * d.nz;
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double v = fabs(d.phi[i]);
    m = (v > m || v != v) ? v : m;
  }
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      double a = sh[threadIdx.x], b = sh[threadIdx.x + s];
      sh[threadIdx.x] = (b > a || b != b) ? b : a;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) M[j] = sh[0];
}

long long cdiv(long long n, int t) { return (n + t - 1) / t; }

// Host-side work lists: per launch slot the listed grids and their first
// blocks, packed into one device buffer.
struct Lists {
  struct Slot {
    std::vector<int> start, job;
    int total = 0;
  };
  std::vector<Slot> slots;
  int add_slot() {
    slots.emplace_back();
    return (int)slots.size() - 1;
  }
  void add(int s, int j, long long blocks) {
    if (blocks <= 0) return;
    Slot& S = slots[s];
    S.start.push_back(S.total);
    S.job.push_back(j);
    S.total += (int)blocks;
  }
  // Uploads every slot; wl[s] receives the device view.
  void upload(DevBuf& buf, cudaStream_t st, std::vector<WL>& wl) {
    size_t n = 0;
    for (auto& S : slots) n += 2 * S.job.size();
    std::vector<int> h(std::max<size_t>(n, 1));
    std::vector<size_t> off(slots.size());
    size_t o = 0;
    for (size_t s = 0; s < slots.size(); s++) {
      off[s] = o;
      std::copy(slots[s].start.begin(), slots[s].start.end(), h.begin() + o);
      o += slots[s].start.size();
      std::copy(slots[s].job.begin(), slots[s].job.end(), h.begin() + o);
      o += slots[s].job.size();
    }
    if (buf.bytes < h.size() * 4) buf = DevBuf(h.size() * 4, st);
    RSTG_CUDA(cudaMemcpyAsync(buf.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice, st));
    RSTG_CUDA(cudaStreamSynchronize(st));  // h is pageable and goes out of scope
    wl.resize(slots.size());
    for (size_t s = 0; s < slots.size(); s++) {
      const int* b = buf.as<int>() + off[s];
      wl[s] = WL{b, b + slots[s].start.size(), (int)slots[s].job.size()};
    }
  }
};

}  // namespace

PbBatchEngine::~PbBatchEngine() {
  if (graph_) cudaGraphExecDestroy(graph_);
}

void PbBatchEngine::solve(std::vector<PbJob>& jobs, const rstg_pb_params& p, const std::vector<double*>* phi_out) {
  PbStreamScope scope(st_);
  cudaStream_t st = st_ ? st_ : c_->stream;
  int nj = (int)jobs.size();
  stats.jobs += nj;
  if (nj == 0) return;
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
  };
  auto t0 = now();

  // ---- layout -------------------------------------------------------------
  struct Lay {
    int nlev = 0;  // coarse multigrid levels; -1: plain SOR (minimum dimension <= 8)
    PbGeom lv[kMaxLev];
    size_t o64 = 0, o32[kMaxLev] = {};
  };
  std::vector<Lay> lay(nj);
  size_t n64 = 0, n32 = 0;
  for (int j = 0; j < nj; j++) {
    PbJob& J = jobs[j];
    Lay& Y = lay[j];
    size_t n = J.g.n();
    Y.o64 = n64;
    n64 += (J.uniform ? 2 : 6) * n;
    PbGeom g = J.g;
    Y.lv[0] = g;
    int nl = 0;
    if (std::min(g.nx, std::min(g.ny, g.nz)) <= 8) {  // pb_solver.rs:1044-1059
      nl = -1;
    } else {
      while (std::min(g.nx, std::min(g.ny, g.nz)) > 5) {  // pb_solver.rs:776-836
        if (nl + 1 >= kMaxLev) throw Error(RSTG_ERR_INVALID, "PB grid needs too many multigrid levels");
        PbGeom cg;
        cg.nx = (g.nx + 1) / 2;
        cg.ny = (g.ny + 1) / 2;
        cg.nz = (g.nz + 1) / 2;
        cg.h = g.h * 2.0;
        Y.lv[++nl] = cg;
        g = cg;
      }
    }
    Y.nlev = nl;
    for (int l = 0; l <= std::max(nl, 0); l++) {
      Y.o32[l] = n32;
      size_t m = Y.lv[l].n();
      n32 += (J.uniform ? 4 : 8) * m;
      n32 = (n32 + 63) & ~(size_t)63;
    }
  }
  size_t b64 = std::max<size_t>(n64, 1) * 8, b32 = std::max<size_t>(n32, 1) * 4;
  if (pool64_.bytes < b64) pool64_ = DevBuf(b64, st);
  if (pool32_.bytes < b32) pool32_ = DevBuf(b32, st);
  double* P64 = pool64_.as<double>();
  float* P32 = pool32_.as<float>();
  RSTG_CUDA(cudaMemsetAsync(P32, 0, b32, st));

  // ---- maps and boundary values (FP64, the reference's set-up) -------------
  for (int j = 0; j < nj; j++) {
    PbJob& J = jobs[j];
    size_t n = J.g.n();
    double* base = P64 + lay[j].o64;
    double *phi = base, *rho = base + n;
    double *ex = J.uniform ? nullptr : base + 2 * n, *ey = J.uniform ? nullptr : base + 3 * n,
           *ez = J.uniform ? nullptr : base + 4 * n, *k2 = J.uniform ? nullptr : base + 5 * n;
    pb_maps_into(c_, J.g, *J.atoms, p, J.ein, J.eout, J.kap, J.ionic, rho, ex, ey, ez, k2);
    RSTG_CUDA(cudaMemsetAsync(phi, 0, n * 8, st));
    pb_boundary(c_, J.g, phi, *J.atoms, J.bc);
  }

  // ---- descriptors ----------------------------------------------------------
  std::vector<JobD> hd(nj);
  std::vector<LvlD> hl((size_t)nj * kMaxLev);
  std::vector<JobState> hs(nj);
  long long max_res = 1, max_sor = 1;
  for (int j = 0; j < nj; j++) {
    PbJob& J = jobs[j];
    const Lay& Y = lay[j];
    size_t n = J.g.n();
    double* base = P64 + Y.o64;
    JobD& d = hd[j];
    std::memset(&d, 0, sizeof(d));
    d.phi = base;
    d.rho = base + n;
    if (!J.uniform) {
      d.ex = base + 2 * n;
      d.ey = base + 3 * n;
      d.ez = base + 4 * n;
      d.k2 = base + 5 * n;
    }
    d.nx = J.g.nx;
    d.ny = J.g.ny;
    d.nz = J.g.nz;
    d.uniform = J.uniform ? 1 : 0;
    d.ih = 1.0 / (J.g.h * J.g.h);
    d.eps = J.ein;
    d.tol = J.tol;
    d.maxv = (int)std::min<int64_t>(std::max<int64_t>(J.maxit / 6, 1), 200);
    d.maxit = J.maxit;
    double rj = (std::cos(kPi / (double)J.g.nx) + std::cos(kPi / (double)J.g.ny) + std::cos(kPi / (double)J.g.nz)) / 3.0;
    d.rs2 = rj * rj;  // spectral radius of Jacobi, squared (pb_solver.rs:387-392)
    d.axyz = J.atoms->xyz.as<double>();
    d.aq = J.atoms->q.as<double>();
    d.na = J.atoms->n;
    d.want_e = J.energy ? 1 : 0;
    d.ox = J.g.ox;
    d.oy = J.g.oy;
    d.oz = J.g.oz;
    d.h = J.g.h;
    JobState& s = hs[j];
    std::memset(&s, 0, sizeof(s));
    s.best = s.prev = DBL_MAX;
    s.om = 1.0;
    s.status = Y.nlev >= 0 ? kMg : kSor;
    max_res = std::max(max_res, cdiv((long long)(J.g.nx - 2) * (J.g.ny - 2) * (J.g.nz - 2), kT));
    max_sor = std::max(max_sor, cdiv((long long)((J.g.nx - 1) / 2) * (J.g.ny - 2) * (J.g.nz - 2), kT));
    for (int l = 0; l <= std::max(Y.nlev, 0); l++) {
      const PbGeom& g = Y.lv[l];
      size_t m = g.n();
      LvlD& L = hl[(size_t)j * kMaxLev + l];
      std::memset(&L, 0, sizeof(L));
      float* b = P32 + Y.o32[l];
      L.e = b;
      L.e2 = b + m;
      L.rhs = b + 2 * m;
      L.res = b + 3 * m;
      if (!J.uniform) {
        L.ex = b + 4 * m;
        L.ey = b + 5 * m;
        L.ez = b + 6 * m;
        L.k2 = b + 7 * m;
      }
      L.nx = g.nx;
      L.ny = g.ny;
      L.nz = g.nz;
      L.uniform = J.uniform ? 1 : 0;
      L.ih = (float)(1.0 / (g.h * g.h));
      L.om = (float)pb_omega(g.nx, g.ny, g.nz);
      L.eps = (float)J.ein;
    }
  }
  int nparts = (int)std::max(max_res, max_sor);
  size_t dbytes = sizeof(JobD) * nj + sizeof(LvlD) * hl.size() + sizeof(JobState) * nj;
  if (desc_.bytes < dbytes) desc_ = DevBuf(dbytes, st);
  JobD* dJ = (JobD*)desc_.p;
  LvlD* dL = (LvlD*)((char*)desc_.p + sizeof(JobD) * nj);
  JobState* dS = (JobState*)((char*)dL + sizeof(LvlD) * hl.size());
  RSTG_CUDA(cudaMemcpyAsync(dJ, hd.data(), sizeof(JobD) * nj, cudaMemcpyHostToDevice, st));
  RSTG_CUDA(cudaMemcpyAsync(dL, hl.data(), sizeof(LvlD) * hl.size(), cudaMemcpyHostToDevice, st));
  RSTG_CUDA(cudaMemcpyAsync(dS, hs.data(), sizeof(JobState) * nj, cudaMemcpyHostToDevice, st));
  size_t pbytes = (size_t)nparts * nj * 8 * 3;  // residual partials, then two colours of SOR partials
  if (part_.bytes < pbytes) part_ = DevBuf(pbytes, st);
  if (small_.bytes < (size_t)nj * 16) small_ = DevBuf((size_t)nj * 16, st);
  double* part = part_.as<double>();
  double* spart = part + (size_t)nparts * nj;

  // FP32 maps of the solvated grids
  {
    Lists setup;
    int s0 = setup.add_slot();
    std::vector<int> si(kMaxLev);
    for (int l = 0; l + 1 < kMaxLev; l++) si[l] = setup.add_slot();
    int maxl = 0;
    for (int j = 0; j < nj; j++) {
      if (jobs[j].uniform) continue;
      setup.add(s0, j, cdiv((long long)jobs[j].g.n(), kT));
      for (int l = 0; l < lay[j].nlev; l++) setup.add(si[l], j, cdiv((long long)lay[j].lv[l + 1].n(), kT));
      maxl = std::max(maxl, lay[j].nlev);
    }
    std::vector<WL> wl;
    setup.upload(lists_, st, wl);
    if (setup.slots[s0].total > 0) {
      k_maps32<<<setup.slots[s0].total, kT, 0, st>>>(wl[s0], dJ, dL);
      launched(c_);
    }
    for (int l = 0; l < maxl; l++)
      if (setup.slots[si[l]].total > 0) {
        k_inject32<<<setup.slots[si[l]].total, kT, 0, st>>>(wl[si[l]], dL, l);
        launched(c_);
      }
    RSTG_CUDA(cudaStreamSynchronize(st));
  }
  auto t1 = now();
  stats.ms_setup += ms(t0, t1);

  // ---- lock-step iterations ------------------------------------------------
  // Initial residuals of the multigrid grids (no convergence test: the
  // reference tests after each V-cycle).
  {
    Lists init;
    int s = init.add_slot(), sn = init.add_slot();
    for (int j = 0; j < nj; j++)
      if (hs[j].status == kMg) {
        init.add(s, j, cdiv((long long)(jobs[j].g.nx - 2) * (jobs[j].g.ny - 2) * (jobs[j].g.nz - 2), kT));
        init.add(sn, j, 1);
      }
    if (init.slots[s].total > 0) {
      std::vector<WL> wl;
      init.upload(lists_, st, wl);
      k_res64<<<init.slots[s].total, kT, 0, st>>>(wl[s], dJ, dL, dS, kMg, part, nparts);
      k_norm<<<init.slots[sn].total, 256, 0, st>>>(wl[sn], dJ, dS, part, nparts, 0);
      launched(c_, 2);
      RSTG_CUDA(cudaStreamSynchronize(st));
    }
  }
  const int K = std::max(1, chunk_cycles), KS = 4;  // cycles per chunk, SOR sweeps per cycle
  bool use_graph = st != nullptr && st != cudaStreamLegacy && st != cudaStreamPerThread;
  std::vector<int> key;  // (job, status) pairs of the current lists
  std::vector<WL> wl;
  Lists lists;
  int per_chunk = 0;
  cudaGraphExec_t exec = nullptr;
  struct LvSlots {
    int rb, res, restr, coarse, prol;
  };
  std::vector<LvSlots> ls(kMaxLev);
  int s_upd = 0, s_res = 0, s_norm = 0, s_sres = 0, s_sor = 0, s_supd = 0, s_snorm = 0, maxlev = 0;
  bool any_mg = false, any_sor = false;
  auto enqueue_chunk = [&]() {
    int n = 0;
    auto go = [&](int slot) { return lists.slots[slot].total; };
    for (int k = 0; k < K; k++) {
      if (any_mg) {
        for (int l = 0; l <= maxlev; l++) {
          if (go(ls[l].rb)) {
            for (int s = 0; s < 3; s++) {  // e -> e2 -> e -> e2
              k_sweep32<<<go(ls[l].rb), 256, 0, st>>>(wl[ls[l].rb], dL, l, dS, s & 1);
              n++;
            }
            k_res32<<<go(ls[l].res), kT, 0, st>>>(wl[ls[l].res], dL, l, dS);
            k_restrict32<<<go(ls[l].restr), kT, 0, st>>>(wl[ls[l].restr], dL, l, dS);
            n += 2;
          }
          if (go(ls[l].coarse)) {
            k_coarse32<<<go(ls[l].coarse), 256, 0, st>>>(wl[ls[l].coarse], dL, l, dS, 50);
            n++;
          }
        }
        for (int l = maxlev - 1; l >= 0; l--) {
          if (!go(ls[l].prol)) continue;
          k_prolong32<<<go(ls[l].prol), kT, 0, st>>>(wl[ls[l].prol], dL, l, dS);
          n++;
          for (int s = 0; s < 3; s++) {  // e2 -> e -> e2 -> e
            k_sweep32<<<go(ls[l].rb), 256, 0, st>>>(wl[ls[l].rb], dL, l, dS, 1 - (s & 1));
            n++;
          }
        }
        k_update64<<<go(s_upd), kT, 0, st>>>(wl[s_upd], dJ, dL, dS, kMg);
        k_res64<<<go(s_res), kT, 0, st>>>(wl[s_res], dJ, dL, dS, kMg, part, nparts);
        k_norm<<<go(s_norm), 256, 0, st>>>(wl[s_norm], dJ, dS, part, nparts, 1);
        n += 3;
      }
      if (any_sor)
        for (int q = 0; q < KS; q++) {
          k_res64<<<go(s_sres), kT, 0, st>>>(wl[s_sres], dJ, dL, dS, kSor, part, nparts);
          k_sor32<<<go(s_sor), kT, 0, st>>>(wl[s_sor], dL, dS, 0, spart, nparts);
          k_sor32<<<go(s_sor), kT, 0, st>>>(wl[s_sor], dL, dS, 1, spart, nparts);
          k_update64<<<go(s_supd), kT, 0, st>>>(wl[s_supd], dJ, dL, dS, kSor);
          k_sor_norm<<<go(s_snorm), 256, 0, st>>>(wl[s_snorm], dJ, dS, spart, nparts);
          n += 5;
        }
    }
    return n;
  };
  auto rebuild = [&]() {
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
      graph_ = nullptr;
    }
    lists = Lists();
    maxlev = 0;
    for (int l = 0; l < kMaxLev; l++)
      ls[l] = LvSlots{lists.add_slot(), lists.add_slot(), lists.add_slot(), lists.add_slot(), lists.add_slot()};
    s_upd = lists.add_slot();
    s_res = lists.add_slot();
    s_norm = lists.add_slot();
    s_sres = lists.add_slot();
    s_sor = lists.add_slot();
    s_supd = lists.add_slot();
    s_snorm = lists.add_slot();
    any_mg = any_sor = false;
    for (int j = 0; j < nj; j++) {
      const Lay& Y = lay[j];
      const PbGeom& g = jobs[j].g;
      long long nint = (long long)(g.nx - 2) * (g.ny - 2) * (g.nz - 2);
      if (hs[j].status == kMg) {
        any_mg = true;
        maxlev = std::max(maxlev, Y.nlev);
        for (int l = 0; l < Y.nlev; l++) {
          const PbGeom& a = Y.lv[l];
          lists.add(ls[l].rb, j,
                    (long long)((a.nx + kBX - 1) / kBX) * ((a.ny + kBY - 1) / kBY) * ((a.nz + kBZ - 1) / kBZ));
          lists.add(ls[l].res, j, cdiv((long long)(a.nx - 2) * (a.ny - 2) * (a.nz - 2), kT));
          lists.add(ls[l].restr, j, cdiv((long long)Y.lv[l + 1].n(), kT));
          lists.add(ls[l].prol, j, cdiv((long long)a.n(), kT));
        }
        lists.add(ls[Y.nlev].coarse, j, 1);
        lists.add(s_upd, j, cdiv((long long)g.n(), kT));
        lists.add(s_res, j, cdiv(nint, kT));
        lists.add(s_norm, j, 1);
      } else if (hs[j].status == kSor) {
        any_sor = true;
        lists.add(s_sres, j, cdiv(nint, kT));
        lists.add(s_sor, j, cdiv((long long)((g.nx - 1) / 2) * (g.ny - 2) * (g.nz - 2), kT));
        lists.add(s_supd, j, cdiv((long long)g.n(), kT));
        lists.add(s_snorm, j, 1);
      }
    }
    lists.upload(lists_, st, wl);
    if (use_graph && (any_mg || any_sor)) {
      cudaGraph_t g = nullptr;
      RSTG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      per_chunk = enqueue_chunk();
      cudaError_t ce = cudaStreamEndCapture(st, &g);
      if (ce != cudaSuccess) throw Error(RSTG_ERR_CUDA, std::string("PB graph capture: ") + cudaGetErrorString(ce));
      cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) throw Error(RSTG_ERR_CUDA, std::string("PB graph: ") + cudaGetErrorString(ie));
      graph_ = exec;
    }
  };
  long long guard_chunks = 0, max_chunks = 0;
  for (int j = 0; j < nj; j++) max_chunks = std::max<long long>(max_chunks, hd[j].maxv + hd[j].maxit / KS + 2);
  max_chunks = max_chunks / K + 4;
  for (;;) {
    // grids whose V-cycles diverged continue as SOR from their current
    // potential with the boundary values set again (pb_solver.rs:1118-1125)
    bool switched = false;
    for (int j = 0; j < nj; j++)
      if (hs[j].status == kDiverged) {
        pb_boundary(c_, jobs[j].g, hd[j].phi, *jobs[j].atoms, jobs[j].bc);
        hs[j].status = kSor;
        hs[j].om = 1.0;
        hs[j].sor_it = 0;
        hs[j].rms = DBL_MAX;
        switched = true;
      }
    if (switched) RSTG_CUDA(cudaMemcpyAsync(dS, hs.data(), sizeof(JobState) * nj, cudaMemcpyHostToDevice, st));
    std::vector<int> k2;
    for (int j = 0; j < nj; j++)
      if (hs[j].status == kMg || hs[j].status == kSor) {
        k2.push_back(j);
        k2.push_back(hs[j].status);
      }
    if (k2.empty()) break;
    if (k2 != key) {
      key = k2;
      rebuild();
    }
    if (++guard_chunks > max_chunks) throw Error(RSTG_ERR_INVALID, "PB batch did not finish within its iteration caps");
    if (use_graph) {
      RSTG_CUDA(cudaGraphLaunch(exec, st));
      c_->launches += per_chunk;
    } else {
      launched(c_, enqueue_chunk());
    }
    stats.cycles += K;
    RSTG_CUDA(cudaMemcpyAsync(hs.data(), dS, sizeof(JobState) * nj, cudaMemcpyDeviceToHost, st));
    RSTG_CUDA(cudaStreamSynchronize(st));
  }
  if (exec) {
    cudaGraphExecDestroy(exec);
    graph_ = nullptr;
  }

  // ---- results ----------------------------------------------------------------
  if (std::getenv("RSTG_PB_DEBUG"))
    for (int j = 0; j < nj; j++)
      std::fprintf(stderr, "pb grid %d: %dx%dx%d uniform %d status %d cycles %d sor %lld rms %.6e r0 %.6e\n", j,
                   jobs[j].g.nx, jobs[j].g.ny, jobs[j].g.nz, (int)jobs[j].uniform, hs[j].status, hs[j].cycles,
                   hs[j].sor_it, hs[j].rms, hs[j].r0);
  auto t2 = now();
  stats.ms_cycles += ms(t1, t2);
  for (int j = 0; j < nj; j++) {
    const JobState& s = hs[j];
    bool sor = s.status == kSorCap || s.sor_it > 0;
    jobs[j].fallback = sor;
    if (sor) stats.fallbacks++;
    jobs[j].stats = PbSolveStats{sor ? (int64_t)s.sor_it : (int64_t)s.cycles, s.rms, s.status == kConverged};
  }
  double* dE = small_.as<double>();
  double* dM = dE + nj;
  k_energy64<<<nj, 256, 0, st>>>(dJ, dE);
  k_maxabs64<<<nj, 1024, 0, st>>>(dJ, dM);
  launched(c_, 2);
  std::vector<double> he(2 * (size_t)nj);
  RSTG_CUDA(cudaMemcpyAsync(he.data(), dE, 16 * (size_t)nj, cudaMemcpyDeviceToHost, st));
  if (phi_out)
    for (int j = 0; j < nj; j++)
      if ((*phi_out)[j])
        RSTG_CUDA(cudaMemcpyAsync((*phi_out)[j], P64 + lay[j].o64, jobs[j].g.n() * 8, cudaMemcpyDeviceToDevice, st));
  RSTG_CUDA(cudaStreamSynchronize(st));
  for (int j = 0; j < nj; j++) {
    jobs[j].e = he[j];
    jobs[j].maxabs = he[nj + j];
  }
  stats.ms_finish += ms(t2, now());
}

void pb_polar_batch(Ctx* c, cudaStream_t st, PbBatchEngine& eng, const rstg_pb_params& p,
                    const std::vector<const std::vector<double>*>& xyz, const std::vector<const std::vector<double>*>& q,
                    const std::vector<const std::vector<double>*>& r, double* out, rstg_pb_diag* diag) {
  if (!(p.grid_spacing > 0.0)) throw Error(RSTG_ERR_INVALID, "grid_spacing must be positive");
  PbStreamScope scope(st);
  size_t n = xyz.size();
  double kap = pb_kappa(p);
  bool focus = p.fillratio > 0.0 && p.fscale > 1;
  std::vector<std::unique_ptr<AtomsDev>> A(n);
  std::vector<PbGeom> fine(n), coarse(n);
  for (size_t i = 0; i < n; i++) {
    out[i] = 0.0;
    if (diag) std::memset(&diag[i], 0, sizeof(rstg_pb_diag));
    if (q[i]->empty()) continue;  // pb_energy.rs:335
    A[i] = std::make_unique<AtomsDev>(*xyz[i], *q[i], *r[i], st);
    fine[i] = pb_auto_grid(*xyz[i], p.grid_spacing, p.grid_buffer);
    if (fine[i].n() > (size_t)600 * 600 * 600) throw Error(RSTG_ERR_NOMEM, "PB grid exceeds 600^3 points");
    if (focus) coarse[i] = pb_coarse_grid(*xyz[i], p.grid_spacing, p.fillratio, p.fscale);
  }
  auto make = [&](size_t i, int s, const PbGeom& g) {  // s 0 solvated, 1 reference (pb_energy.rs:380-420)
    PbJob J;
    J.g = g;
    J.atoms = A[i].get();
    J.uniform = s == 1;
    J.ionic = s == 0;
    J.ein = p.solute_dielectric;
    J.eout = s == 0 ? p.solvent_dielectric : p.solute_dielectric;
    J.kap = kap;
    J.bc.kind = 1;
    J.bc.kappa = s == 0 ? kap : 0.0;
    J.bc.eout = J.eout;
    J.tol = p.tolerance;
    J.maxit = p.max_iterations;
    return J;
  };
  std::vector<DevBuf> cphi(2 * n);
  std::vector<int> ok(2 * n, 0);
  if (focus) {  // pb_energy.rs:134-322: coarse solve, validity, interpolated boundary
    std::vector<PbJob> cj;
    std::vector<double*> outp;
    std::vector<size_t> who;
    for (size_t i = 0; i < n; i++) {
      if (!A[i]) continue;
      for (int s = 0; s < 2; s++) {
        PbJob J = make(i, s, coarse[i]);
        J.tol = p.tolerance * 10.0;
        J.energy = false;
        cphi[2 * i + s] = DevBuf(coarse[i].n() * 8, st);
        outp.push_back(cphi[2 * i + s].as<double>());
        cj.push_back(J);
        who.push_back(2 * i + s);
      }
    }
    eng.solve(cj, p, &outp);
    for (size_t k = 0; k < cj.size(); k++)
      ok[who[k]] = cj[k].stats.converged && std::isfinite(cj[k].maxabs) && cj[k].maxabs < 1e10;
  }
  std::vector<PbJob> fj;
  std::vector<size_t> who;
  for (size_t i = 0; i < n; i++) {
    if (!A[i]) continue;
    for (int s = 0; s < 2; s++) {
      PbJob J = make(i, s, fine[i]);
      if (focus && ok[2 * i + s]) {
        J.bc.kind = 2;
        J.bc.cg = &coarse[i];
        J.bc.cphi = cphi[2 * i + s].as<double>();
      }
      fj.push_back(J);
      who.push_back(2 * i + s);
    }
  }
  eng.solve(fj, p);
  std::vector<double> e(2 * n, 0.0);
  for (size_t k = 0; k < fj.size(); k++) {
    size_t i = who[k] / 2;
    int s = (int)(who[k] % 2);
    e[who[k]] = fj[k].e;
    if (diag) {
      diag[i].iterations[s] = fj[k].stats.iterations;
      diag[i].residual[s] = fj[k].stats.residual;
      diag[i].converged[s] = fj[k].stats.converged ? 1 : 0;
      diag[i].dims[0] = fine[i].nx;
      diag[i].dims[1] = fine[i].ny;
      diag[i].dims[2] = fine[i].nz;
    }
  }
  for (size_t i = 0; i < n; i++)
    if (A[i]) out[i] = e[2 * i] - e[2 * i + 1];
}

}  // namespace rstg
