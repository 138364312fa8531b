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
// Relative-residual mode (PbJob::rtol > 0; not the reference's schedule):
// the same FP64 defect correction, with a consistent multigrid as the FP32
// inner solver -- red-black Gauss-Seidel sweeps (omega 1), full-weighting
// restriction without the reference's 0.25 factor, series/parallel coarse
// face dielectrics (k_coarsen32), corrections kept zero on the boundary --
// and the stop when the FP64 residual norm falls below rtol times its
// initial value.  The reference's V-cycle stalls on solvated grids (its
// coarse correction is a quarter of the consistent one and its coarse
// dielectrics are injected); this one reaches a 1e-6 relative residual in
// about a dozen cycles on the 3,040-atom workload.
//
// Launches are driven by work lists: for each launch the host lists the
// grids that take part and the first block of each, so no block is spent on
// a grid that has finished or is smaller than the largest one.  The lists
// (and the CUDA graph that holds a chunk of cycles) are rebuilt when a grid
// changes state; the host reads the per-grid states once per chunk.
//
// Layout in HBM: one FP64 pool (phi, rho and, for solvated grids, the four
// face-dielectric / kbar^2 maps, each g.n() doubles), one FP32 pool (per
// multigrid level: correction, right-hand side, residual and the four maps
// of solvated grids) and one byte of stencil code per point and level.
// Reference grids have a uniform dielectric and no salt term, so their
// stencil is the constant-coefficient Laplacian and they carry no maps.
//
// Stencil codes: a face dielectric is eps_in on both sides of the molecular
// surface's interior, eps_out outside, and a harmonic mean only on the edges
// that cross the surface (pb_grid.rs:809-817); kbar^2 is 0 or one constant
// (assign_kappa, pb_grid.rs:951-985).  Per point one byte holds, for the
// x, y and z faces, 0 = eps_out, 1 = eps_in, 2 = read the map (bits 0-5),
// kbar^2 != 0 (bit 6) and, at level 0, rho != 0 (bit 7).  The kernels read
// the byte and touch a map or rho only where the code says so, with the
// same values and the same arithmetic as reading the maps everywhere: the
// results are bit-identical, and a solvated colour pass streams 11 bytes per
// point instead of 26.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <memory>
#include <thread>

#include "common.cuh"
#include "pb_batch.hpp"

namespace rstg {

namespace {

constexpr int kMaxLev = 16;
static_assert(kProfLevels >= kMaxLev, "profile table must cover every level");
constexpr double kFourPiEcB = 4.0 * kPi * 332.0522;  // pb_solver.rs:155
constexpr int kT = 256;

// grid states
constexpr int kMg = 0, kConverged = 1, kDiverged = 2, kMgCap = 3, kSor = 5, kSorCap = 6;

struct JobD {
  double *phi, *phi2;  // potential: two buffers, JobState::cur says which one is current
  const double* rho;
  const double *ex, *ey, *ez, *k2;
  const uint8_t* cd;      // level-0 stencil codes
  double din, dout, dkb;  // eps_in, eps_out, the non-zero kbar^2
  const double *axyz, *aq;
  int nx, ny, nz, uniform;
  int na, want_e, maxv, px;  // px: row pitch of the FP32 / code arrays
  double ih, eps, tol, rs2;
  double ox, oy, oz, h;
  long long maxit;
  double rtol;  // > 0: stop on the relative FP64 residual (consistent multigrid)
};

struct LvlD {
  float *e, *e2, *rhs, *res;  // correction (two buffers: a sweep reads one, writes the other), rhs, residual
  const float *ex, *ey, *ez, *k2;
  const uint8_t* cd;          // stencil codes
  int nx, ny, nz, uniform;
  int px, zc, skipb, pad2;    // row pitch (nx rounded up to 4: rows start on 16-byte boundaries), sweep z chunk,
                              // skipb: prolongation leaves boundary points alone (relative-residual mode)
  float ih, om, eps, rsc;     // rsc: restriction scale (0.25 the reference's, 1 relative-residual mode)
  float fin, fout, kb, pad3;
};

struct JobState {
  double best, prev, rms, r0, om;
  int growing, cycles, status, cur;  // cur: phi2 holds the current potential
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

// Level arrays and constants held in registers: reading them through a
// reference to the descriptor in global memory would make every global store
// force reloads of the pointers.
struct Lv {
  float *__restrict__ e, *__restrict__ e2, *__restrict__ rhs, *__restrict__ res;
  const float *__restrict__ ex, *__restrict__ ey, *__restrict__ ez, *__restrict__ k2;
  const uint8_t* __restrict__ cd;
  int nx, ny, nz, sy, sz, zc;
  bool uni;
  float ih, om, w6, fin, fout, kb;
};
__device__ __forceinline__ Lv lv_load(const LvlD* __restrict__ L, int j, int lvl) {
  const LvlD& d = L[j * kMaxLev + lvl];
  Lv v;
  v.e = d.e;
  v.e2 = d.e2;
  v.rhs = d.rhs;
  v.res = d.res;
  v.ex = d.ex;
  v.ey = d.ey;
  v.ez = d.ez;
  v.k2 = d.k2;
  v.cd = d.cd;
  v.nx = d.nx;
  v.ny = d.ny;
  v.nz = d.nz;
  v.sy = d.px;
  v.sz = d.px * d.ny;
  v.zc = d.zc;
  v.uni = d.uniform != 0;
  v.ih = d.ih;
  v.om = d.om;
  v.w6 = d.eps * d.ih;
  v.fin = d.fin;
  v.fout = d.fout;
  v.kb = d.kb;
  return v;
}

// Face dielectric from a 2-bit stencil code: 0 eps_out, 1 eps_in, 2 the map.
template <typename T>
__device__ __forceinline__ T face(unsigned c, const T* __restrict__ m, int i, T ein, T eout) {
  return c == 0u ? eout : (c == 1u ? ein : m[i]);
}

// Brick of 32 x 8 x 8 points for a 256-thread block: thread (lane, warp) owns
// the column (x, y) = (x0 + lane, y0 + warp) over the brick's 8 z planes, so
// the index arithmetic is done once per block and the 8 points of a column
// are independent loads in flight together.
__device__ __forceinline__ void brick_col(int lb, int nx, int ny, int& x, int& y, int& z0) {
  int ntx = (nx + 31) >> 5, nty = (ny + 7) >> 3;
  int bx = lb % ntx, t = lb / ntx, by = t % nty, bz = t / nty;
  x = (bx << 5) + (threadIdx.x & 31);
  y = (by << 3) + (threadIdx.x >> 5);
  z0 = bz << 3;
}

// FP32 7-point stencil of pb_solver.rs:250-317: ns = sum of eps-weighted
// neighbours, dg = diagonal.
__device__ __forceinline__ void st32(const Lv& d, const float* __restrict__ e, int i, float& ns, float& dg) {
  const int sy = d.sy, sz = d.sz;
  if (d.uni) {
    ns = d.w6 * ((e[i + 1] + e[i - 1]) + (e[i + sy] + e[i - sy]) + (e[i + sz] + e[i - sz]));
    dg = 6.0f * d.w6;
  } else {
    const unsigned c0 = d.cd[i];
    float a = face(c0 & 3u, d.ex, i, d.fin, d.fout), b = face(d.cd[i - 1] & 3u, d.ex, i - 1, d.fin, d.fout),
          c = face((c0 >> 2) & 3u, d.ey, i, d.fin, d.fout),
          dd = face((d.cd[i - sy] >> 2) & 3u, d.ey, i - sy, d.fin, d.fout),
          f = face((c0 >> 4) & 3u, d.ez, i, d.fin, d.fout),
          g = face((d.cd[i - sz] >> 4) & 3u, d.ez, i - sz, d.fin, d.fout);
    ns = ((a * e[i + 1] + b * e[i - 1]) + (c * e[i + sy] + dd * e[i - sy]) + (f * e[i + sz] + g * e[i - sz])) * d.ih;
    dg = ((a + b) + (c + dd) + (f + g)) * d.ih + ((c0 & 64u) ? d.kb : 0.0f);
  }
}

// FP64 residual r = 4 pi ec rho + ns - dg phi at the interior points; r is
// stored rounded to FP32 as the level-0 right-hand side and its squares are
// summed per brick (fixed order) for the RMS test.
__global__ void __launch_bounds__(256, 4) k_res64(WL w, const JobD* __restrict__ J, const LvlD* __restrict__ L,
                                               const JobState* __restrict__ S, int want, double* __restrict__ part,
                                               int nparts) {
  __shared__ double sh[32];
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != want) return;
  const JobD& d = J[j];
  float* __restrict__ rhs0 = L[j * kMaxLev].rhs;
  const double* __restrict__ p = S[j].cur ? d.phi2 : d.phi;
  const double* __restrict__ rho = d.rho;
  const double *__restrict__ ex = d.ex, *__restrict__ ey = d.ey, *__restrict__ ez = d.ez;
  const uint8_t* __restrict__ cd = d.cd;
  const double din = d.din, dout = d.dout, dkb = d.dkb;
  const bool uni = d.uniform != 0;
  const double ih = d.ih, wt = d.eps * d.ih;
  const int nx = d.nx, ny = d.ny, nz = d.nz, sy = nx, sz = nx * ny, cy = d.px, cz = d.px * ny;
  int x, y, z0;
  brick_col(lb, nx, ny, x, y, z0);
  double acc = 0.0;
  if (x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2) {
    int i = x + sy * y + sz * z0, ci = x + cy * y + cz * z0;  // FP64 and padded FP32 / code indices
#pragma unroll
    for (int k = 0; k < 8; k++, i += sz, ci += cz) {
      int z = z0 + k;
      if (z < 1 || z > nz - 2) continue;
      const unsigned c0 = cd[ci];
      double ns, dg;
      if (uni) {
        ns = wt * ((p[i + 1] + p[i - 1]) + (p[i + sy] + p[i - sy]) + (p[i + sz] + p[i - sz]));
        dg = 6.0 * wt;
      } else {
        double a = face(c0 & 3u, ex, i, din, dout), b = face(cd[ci - 1] & 3u, ex, i - 1, din, dout),
               c = face((c0 >> 2) & 3u, ey, i, din, dout), dd = face((cd[ci - cy] >> 2) & 3u, ey, i - sy, din, dout),
               f = face((c0 >> 4) & 3u, ez, i, din, dout), g = face((cd[ci - cz] >> 4) & 3u, ez, i - sz, din, dout);
        ns = (a * p[i + 1] + b * p[i - 1]) * ih + (c * p[i + sy] + dd * p[i - sy]) * ih +
             (f * p[i + sz] + g * p[i - sz]) * ih;
        dg = (a + b) * ih + (c + dd) * ih + (f + g) * ih + ((c0 & 64u) ? dkb : 0.0);
      }
      double q = (c0 & 128u) ? rho[i] : 0.0;
      double r = kFourPiEcB * q + ns - dg * p[i];
      rhs0[ci] = (float)r;
      acc += r * r;
    }
  }
  double t = block_sum(acc, sh);
  if (threadIdx.x == 0) part[(long long)j * nparts + lb] = t;
}

// End of a V-cycle (or of an SOR sweep): phi' = phi + e at every point (the prolongation can
// reach boundary points of grids with even dimensions) into the other
// potential buffer, and the FP64 residual of phi' at the interior points, from
// phi + e at the seven stencil points (the same values the separate update
// would store), rounded to FP32 as the next right-hand side, squares summed
// per brick.  The correction is not cleared: the next cycle's first sweep
// reads it as zero.
__global__ void __launch_bounds__(256, 4) k_upres64(WL w, const JobD* __restrict__ J, const LvlD* __restrict__ L,
                                                    const JobState* __restrict__ S, int want,
                                                    double* __restrict__ part, int nparts) {
  __shared__ double sh[32];
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != want) return;
  const JobD& d = J[j];
  const bool cur = S[j].cur != 0;
  const double* __restrict__ p = cur ? d.phi2 : d.phi;
  double* __restrict__ q = cur ? d.phi : d.phi2;
  const float* __restrict__ e0 = L[j * kMaxLev].e;
  float* __restrict__ rhs0 = L[j * kMaxLev].rhs;
  const double* __restrict__ rho = d.rho;
  const double *__restrict__ ex = d.ex, *__restrict__ ey = d.ey, *__restrict__ ez = d.ez;
  const uint8_t* __restrict__ cd = d.cd;
  const double din = d.din, dout = d.dout, dkb = d.dkb;
  const bool uni = d.uniform != 0;
  const double ih = d.ih, wt = d.eps * d.ih;
  const int nx = d.nx, ny = d.ny, nz = d.nz, sy = nx, sz = nx * ny, cy = d.px, cz = d.px * ny;
  int x, y, z0;
  brick_col(lb, nx, ny, x, y, z0);
  double acc = 0.0;
  if (x < nx && y < ny && z0 < nz) {
    const bool inxy = x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2;
    int i = x + sy * y + sz * z0, ci = x + cy * y + cz * z0;  // FP64 and padded FP32 / code indices
    // phi + e along the column in registers: the planes below, at and above
    // the current point (the z neighbours are not loaded again)
    double vm = (inxy && z0 >= 1) ? p[i - sz] + (double)e0[ci - cz] : 0.0;
    double vc = p[i] + (double)e0[ci];
#pragma unroll 1
    for (int k = 0; k < 8; k++, i += sz, ci += cz) {
      const int z = z0 + k;
      if (z >= nz) break;
      const double v = vc;
      const double vzp = z + 1 < nz ? p[i + sz] + (double)e0[ci + cz] : 0.0, vzm = vm;
      vm = vc;
      vc = vzp;
      q[i] = v;
      if (!inxy || z < 1 || z > nz - 2) continue;
      const double vxp = p[i + 1] + (double)e0[ci + 1], vxm = p[i - 1] + (double)e0[ci - 1],
                   vyp = p[i + sy] + (double)e0[ci + cy], vym = p[i - sy] + (double)e0[ci - cy];
      const unsigned c0 = cd[ci];
      double ns, dg;
      if (uni) {
        ns = wt * ((vxp + vxm) + (vyp + vym) + (vzp + vzm));
        dg = 6.0 * wt;
      } else {
        double a = face(c0 & 3u, ex, i, din, dout), b = face(cd[ci - 1] & 3u, ex, i - 1, din, dout),
               c = face((c0 >> 2) & 3u, ey, i, din, dout), dd = face((cd[ci - cy] >> 2) & 3u, ey, i - sy, din, dout),
               f = face((c0 >> 4) & 3u, ez, i, din, dout), g = face((cd[ci - cz] >> 4) & 3u, ez, i - sz, din, dout);
        ns = (a * vxp + b * vxm) * ih + (c * vyp + dd * vym) * ih + (f * vzp + g * vzm) * ih;
        dg = (a + b) * ih + (c + dd) * ih + (f + g) * ih + ((c0 & 64u) ? dkb : 0.0);
      }
      double rq = (c0 & 128u) ? rho[i] : 0.0;
      double r = kFourPiEcB * rq + ns - dg * v;
      rhs0[ci] = (float)r;
      acc += r * r;
    }
  }
  double t = block_sum(acc, sh);
  if (threadIdx.x == 0) part[(long long)j * nparts + lb] = t;
}

// RMS of the residual and the reference's multigrid bookkeeping
// (pb_solver.rs:1080-1160); one block per listed grid.
__global__ void k_norm(WL w, const JobD* __restrict__ J, JobState* __restrict__ S, const double* __restrict__ part,
                       int nparts, int check, int want) {
  __shared__ double sh[32];
  int j = w.job[blockIdx.x];
  if (S[j].status != want) return;
  const JobD& d = J[j];
  int used = ((d.nx + 31) >> 5) * ((d.ny + 7) >> 3) * ((d.nz + 7) >> 3);
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
  t.cur ^= 1;  // k_upres64 wrote the new potential into the other buffer
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
  if (d.rtol > 0.0 ? r < d.rtol * t.r0 : r < d.tol) {
    t.status = kConverged;
  } else if (t.cycles >= d.maxv) {
    t.status = kMgCap;
  }
}

// One full red-black sweep on one level (pb_solver.rs:250-317): every even
// point (x + y + z even) from its odd neighbours, then every odd point from
// the updated even ones, each point with the arithmetic of the
// single-colour update.  A block owns an x-y tile of kSwTX x kSwTY points and
// marches a chunk of z planes.  Planes of the correction (with a two-point
// halo), of the right-hand side and of the stencil codes stream into
// shared-memory rings with cp.async, two steps ahead of their use.  Step s
// updates, in one phase between barriers, the even points of plane s+2 over
// the tile and a one-point halo, the odd points of plane s (whose even
// neighbours in planes s-1 .. s+1 are already updated) and writes plane s-1
// out.  Halo values are recomputed by each tile that needs them, so the sweep
// reads `src` and writes the whole grid, boundary values copied, into `dst`:
// no block reads what another block writes.  Each thread's points, copy
// chunks and store are fixed for the whole march (only the colour parity
// alternates with the plane), so the per-step index work is a few adds; a
// half-warp covers 16 points of one colour in a row and the next half-warp
// the next row (opposite parity), so the shared loads are free of bank
// conflicts; ring depths are powers of two.
// z planes per block: long marches on the finest level, short ones on the
// coarse levels (few tiles per grid there, so more chunks keep the SMs busy)
constexpr int kSwTX = 32, kSwTY = 16, kSwThreads = 288, kSwZC0 = 48, kSwZC1 = 16;
int sweep_chunk(int lvl) { return lvl == 0 ? kSwZC0 : (lvl == 1 ? kSwZC1 : 8); }
constexpr int kSwW = kSwTX + 8;   // shared row: x in [xt-4, xt+TX+4), 16-byte chunks
constexpr int kSwEY = kSwTY + 4;  // correction rows: y in [yt-2, yt+TY+2)
constexpr int kSwRY = kSwTY + 2;  // right-hand-side rows: y in [yt-1, yt+TY+1)
constexpr int kSwCY = kSwTY + 3;  // code rows: y in [yt-2, yt+TY+1)
constexpr int kSwNE = 8, kSwNR = 8, kSwNC = 8;  // ring depths in planes (slot = plane & (depth - 1))
// first point of a thread: even points of plane s+2 inside the tile's x range, 16 per row, rows yt-1 .. yt+TY;
// second point: odd points of plane s (threads < TY*16), then the even points of plane s+2 on the
// x halo (one per row: x = xt-1 or xt+TX)
static_assert(kSwTX == 32 && (kSwTY + 2) * 16 == kSwThreads && kSwTY * 16 + kSwTY + 2 <= kSwThreads,
              "point assignment of the sweep");
static_assert(kSwEY * (kSwW / 4) <= kSwThreads && kSwRY * (kSwW / 4) <= kSwThreads &&
                  kSwCY * (kSwW / 4) <= kSwThreads && kSwTY * (kSwTX / 4) <= kSwThreads,
              "one copy chunk and one store per thread and plane");

struct SwSmem {
  float e[kSwNE][kSwEY * kSwW];
  float r[kSwNR][kSwRY * kSwW];
  uint8_t c[kSwNC][kSwCY * kSwW];
  // faces of every eps_in / eps_out pattern (bit k set: face k is eps_in;
  // faces x+, x-, y+, y-, z+, z-): [0] x+, x-, y+, y-; [1] z+, z-, their sum
  float4 tf[2][64];
};

__device__ __forceinline__ void cp_async16(void* s, const void* g) {
  unsigned a = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async4(void* s, const void* g) {
  unsigned a = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(a), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Update of one interior point: off is its offset in the shared planes (the
// right-hand-side planes start one row later), gi its padded global index
// (for the map values of faces that cross the surface).  Returns gs - old.
// Multigrid smoothing divides with the fast reciprocal; the SOR fallback
// (pb_solver.rs:373-447) with the exact division, as a plain sweep does.
template <bool kExact>
__device__ __forceinline__ float sw_update(const Lv& d, const float4 (*__restrict__ tf)[64], float om,
                                           float* __restrict__ E0, const float* __restrict__ Em,
                                           const float* __restrict__ Ep, const float* __restrict__ R,
                                           const uint8_t* __restrict__ C0, const uint8_t* __restrict__ Cm, int off,
                                           int gi) {
  float* ec = E0 + off;
  const float xm = ec[-1], xp = ec[1], ym = ec[-kSwW], yp = ec[kSwW], zm = Em[off], zp = Ep[off], old = ec[0];
  const float rhs = R[off - kSwW];
  float ns, dg;
  if (d.uni) {
    ns = d.w6 * ((xp + xm) + (yp + ym) + (zp + zm));
    dg = 6.0f * d.w6;
  } else {
    const unsigned c0 = C0[off], cxm = C0[off - 1], cym = C0[off - kSwW], czm = Cm[off];
    const float k2 = (c0 & 64u) ? d.kb : 0.0f;
    if (((c0 & 0x2Au) | (cxm & 0x2u) | (cym & 0x8u) | (czm & 0x20u)) == 0u) {  // no face crosses the surface
      const unsigned pat = (c0 & 0x15u) | ((cxm & 0x1u) << 1) | ((cym & 0x4u) << 1) | ((czm & 0x10u) << 1);
      const float4 u = tf[0][pat], v = tf[1][pat];
      ns = ((u.x * xp + u.y * xm) + (u.z * yp + u.w * ym) + (v.x * zp + v.y * zm)) * d.ih;
      dg = fmaf(v.z, d.ih, k2);
    } else {
      const float a = face(c0 & 3u, d.ex, gi, d.fin, d.fout), b = face(cxm & 3u, d.ex, gi - 1, d.fin, d.fout),
                  c = face((c0 >> 2) & 3u, d.ey, gi, d.fin, d.fout),
                  dd = face((cym >> 2) & 3u, d.ey, gi - d.sy, d.fin, d.fout),
                  f = face((c0 >> 4) & 3u, d.ez, gi, d.fin, d.fout),
                  g = face((czm >> 4) & 3u, d.ez, gi - d.sz, d.fin, d.fout);
      ns = ((a * xp + b * xm) + (c * yp + dd * ym) + (f * zp + g * zm)) * d.ih;
      dg = fmaf((a + b) + (c + dd) + (f + g), d.ih, k2);
    }
  }
  const float gs = kExact ? (ns + rhs) / dg : __fdividef(ns + rhs, dg);
  const float dv = gs - old;
  ec[0] = old + om * dv;
  return dv;
}

// kSorMode: one sweep of the SOR fallback on the finest level's correction
// equation from e = 0 (zero_src), with the grid's Chebyshev omega, and per
// block the sum of (gs - old)^2 over the block's own points into
// part[grid * nparts + block] (halo points are another block's).
template <bool kSorMode>
__global__ void __launch_bounds__(kSwThreads, 4) k_sweep_t(WL w, const LvlD* __restrict__ L, int lvl,
                                                        const JobState* __restrict__ S, int flip, int zero_src,
                                                        double* __restrict__ part, int nparts) {
  extern __shared__ __align__(16) unsigned char sw_raw[];  // sizeof(SwSmem), above the 48 KB static limit
  SwSmem& sm = *reinterpret_cast<SwSmem*>(sw_raw);
  __shared__ double red[32];
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != (kSorMode ? kSor : kMg)) return;
  const Lv d = lv_load(L, j, lvl);
  const float om = kSorMode ? (float)S[j].om : d.om;
  double acc = 0.0;
  const float* __restrict__ src = flip ? d.e2 : d.e;
  float* __restrict__ dst = flip ? d.e : d.e2;
  const int ntx = (d.nx + kSwTX - 1) / kSwTX, nty = (d.ny + kSwTY - 1) / kSwTY;
  const int bx = lb % ntx, q = lb / ntx, by = q % nty, bz = q / nty;
  const int xt = bx * kSwTX, yt = by * kSwTY;
  const int z0 = bz * d.zc, z1 = min(z0 + d.zc, d.nz);
  const int tid = threadIdx.x;

  // copy chunks of this thread (shared offset, global offset within a plane; -1: none)
  auto chunk = [&](int rows, int y0, int& so, int& go) {
    so = go = -1;
    if (tid >= rows * (kSwW / 4)) return;
    const int r = tid / (kSwW / 4), c = tid % (kSwW / 4), y = y0 + r, x = xt - 4 + 4 * c;
    if (y < 0 || y >= d.ny || x < 0 || x >= d.sy) return;
    so = r * kSwW + 4 * c;
    go = x + d.sy * y;
  };
  int eso, ego, rso, rgo, cso, cgo;
  chunk(kSwEY, yt - 2, eso, ego);
  chunk(kSwRY, yt - 1, rso, rgo);
  chunk(kSwCY, yt - 2, cso, cgo);
  if (d.uni) cso = -1;
  // ring slot of plane p (p >= -2; two's complement & keeps negatives in range)
  auto se_ = [](int p) { return p & (kSwNE - 1); };
  auto sr_ = [](int p) { return p & (kSwNR - 1); };
  auto sc_ = [](int p) { return p & (kSwNC - 1); };
  auto load_e = [&](int p) {  // zero_src: the correction is zero (first sweep of a cycle on the finest level)
    if (ego < 0 || p < 0 || p >= d.nz) return;
    if (zero_src)
      *(float4*)&sm.e[se_(p)][eso] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    else
      cp_async16(&sm.e[se_(p)][eso], src + ego + (long long)d.sz * p);
  };
  auto load_r = [&](int p) {
    if (rgo >= 0 && p >= 0 && p < d.nz) cp_async16(&sm.r[sr_(p)][rso], d.rhs + rgo + (long long)d.sz * p);
  };
  auto load_c = [&](int p) {
    if (cso >= 0 && p >= 0 && p < d.nz) cp_async4(&sm.c[sc_(p)][cso], d.cd + cgo + (long long)d.sz * p);
  };
  // this thread's points.  Main (first point): even point of row ym = yt-1+tid/16
  // at x = xt + 2(tid%16) + ((xt + ym + p) & 1).  Second point: odd point of row
  // yo = yt + tid/16 at x = xt + 2(tid%16) + ((xt + yo + p + 1) & 1), or for
  // threads TY*16 .. TY*16+TY+1 the halo even point of row yh = yt-1+(tid-TY*16)
  // at xt-1 or xt+TX, whichever has the even colour.
  const int cm = tid & 15;
  const int ym = yt - 1 + (tid >> 4);
  const bool m_ok = ym >= 1 && ym <= d.ny - 2;
  const int m_pb = (xt + ym) & 1, m_off = (ym - yt + 2) * kSwW + 4 + 2 * cm, m_g = xt + 2 * cm + d.sy * ym;
  int o_kind = 0, o_y = 0, o_pb = 0, o_off = 0, o_g = 0;  // 1 odd point, 2 halo even point
  if (tid < kSwTY * 16) {
    o_y = yt + (tid >> 4);
    o_kind = 1;
    o_pb = (xt + o_y + 1) & 1;
    o_off = (o_y - yt + 2) * kSwW + 4 + 2 * cm;
    o_g = xt + 2 * cm + d.sy * o_y;
  } else if (tid < kSwTY * 16 + kSwTY + 2) {
    o_y = yt - 1 + (tid - kSwTY * 16);
    o_kind = 2;
    o_pb = (xt - 1 + o_y) & 1;  // 0: x = xt-1 is even-coloured in even planes
    o_off = (o_y - yt + 2) * kSwW + 3;
    o_g = xt - 1 + d.sy * o_y;
  }
  if (o_y < 1 || o_y > d.ny - 2) o_kind = 0;
  // store of this thread: one aligned float4 of a tile row
  int sso = -1, sgo = 0;
  if (tid < kSwTY * (kSwTX / 4)) {
    const int r = tid / (kSwTX / 4), c = tid % (kSwTX / 4), y = yt + r, x = xt + 4 * c;
    if (y < d.ny && x < d.sy) {
      sso = (r + 2) * kSwW + 4 * c + 4;
      sgo = x + d.sy * y;
    }
  }
  struct Planes {
    float* E0;
    const float *Em, *Ep, *R;
    const uint8_t *C0, *Cm;
    int gp;
  };
  auto planes = [&](int p) {
    return Planes{sm.e[se_(p)], sm.e[se_(p - 1)], sm.e[se_(p + 1)], sm.r[sr_(p)],
                  sm.c[sc_(p)], sm.c[sc_(p - 1)], d.sz * p};
  };
  auto update = [&](const Planes& P, int x, int off, int g, bool own) {
    if (x < 1 || x > d.nx - 2) return;
    const float dv = sw_update<kSorMode>(d, sm.tf, om, P.E0, P.Em, P.Ep, P.R, P.C0, P.Cm, off, g + P.gp);
    if (kSorMode && own) acc += (double)dv * (double)dv;
  };
  const bool m_own = ym >= yt && ym < yt + kSwTY;  // first-point row inside the tile (not the y halo)
  // even points of plane p: first point and x-halo point
  auto even = [&](int p) {
    if (p < 1 || p > d.nz - 2) return;
    const Planes P = planes(p);
    const int par = m_pb ^ (p & 1);
    const bool own = p >= z0 && p < z1;
    if (m_ok) update(P, xt + 2 * cm + par, m_off + par, m_g + par, own && m_own);
    if (o_kind == 2) {
      const int h = (o_pb ^ (p & 1)) ? kSwTX + 1 : 0;  // xt-1 or xt+TX
      update(P, xt - 1 + h, o_off + h, o_g + h, false);
    }
  };
  auto odd = [&](int p) {
    if (o_kind != 1 || p < 1 || p > d.nz - 2) return;
    const Planes P = planes(p);
    const int par = o_pb ^ (p & 1);
    update(P, xt + 2 * cm + par, o_off + par, o_g + par, true);
  };
  auto store = [&](int p) {
    if (sso >= 0) *(float4*)(dst + sgo + (long long)d.sz * p) = *(const float4*)&sm.e[se_(p)][sso];
  };

  // prologue: what the even points of planes z0-1 .. z0+1 and step z0 read,
  // then the planes of step z0+1
  for (int p = z0 - 2; p <= z0 + 3; p++) load_e(p);
  for (int p = z0 - 1; p <= z0 + 2; p++) load_r(p);
  for (int p = z0 - 2; p <= z0 + 2; p++) load_c(p);
  cp_async_commit();
  if (!d.uni && tid < 64) {  // face table (read after the barrier below)
    const float a = (tid & 1) ? d.fin : d.fout, b = (tid & 2) ? d.fin : d.fout, c = (tid & 4) ? d.fin : d.fout,
                dd = (tid & 8) ? d.fin : d.fout, f = (tid & 16) ? d.fin : d.fout, g = (tid & 32) ? d.fin : d.fout;
    sm.tf[0][tid] = make_float4(a, b, c, dd);
    sm.tf[1][tid] = make_float4(f, g, (a + b) + (c + dd) + (f + g), 0.0f);
  }
  load_e(z0 + 4);
  load_r(z0 + 3);
  load_c(z0 + 3);
  cp_async_commit();
  cp_async_wait<1>();
  __syncthreads();
  even(z0 - 1);
  even(z0);
  even(z0 + 1);
  for (int s = z0; s < z1; s++) {
    cp_async_wait<1>();  // all groups but the newest: correction planes to s+3, rhs / codes to s+2
    __syncthreads();
    if (s + 5 <= z1 + 1) load_e(s + 5);  // the last step reads correction planes to z1+1, rhs / codes to z1
    if (s + 4 <= z1) {
      load_r(s + 4);
      load_c(s + 4);
    }
    cp_async_commit();
    if (s + 2 <= z1) even(s + 2);
    odd(s);
    if (s > z0) store(s - 1);
  }
  __syncthreads();
  store(z1 - 1);
  cp_async_wait<0>();
  if (kSorMode) {
    const double t = block_sum(acc, red);
    if (threadIdx.x == 0) part[(long long)j * nparts + lb] = t;
  }
}


// SOR bookkeeping after a sweep and its update (pb_solver.rs:373-447): rms
// of the sweep's updates from the sweep blocks' partial sums (fixed order),
// Chebyshev omega for the next sweep, convergence; k_upres64 wrote the new
// potential into the other buffer.
// In relative-residual mode the test is on the FP64 residual of the new
// potential (k_upres64's per-brick sums in rpart) against the initial one.
__global__ void k_sor_norm(WL w, const JobD* __restrict__ J, JobState* __restrict__ S, const double* __restrict__ part,
                           const double* __restrict__ rpart, int nparts) {
  __shared__ double sh[32];
  int j = w.job[blockIdx.x];
  if (S[j].status != kSor) return;
  const JobD& d = J[j];
  const bool rel = d.rtol > 0.0;
  const int used = rel ? ((d.nx + 31) >> 5) * ((d.ny + 7) >> 3) * ((d.nz + 7) >> 3)
                       : ((d.nx + kSwTX - 1) / kSwTX) * ((d.ny + kSwTY - 1) / kSwTY) * ((d.nz + kSwZC0 - 1) / kSwZC0);
  const double* src = rel ? rpart : part;
  double s = 0.0;
  for (int k = threadIdx.x; k < used; k += blockDim.x) s += src[(long long)j * nparts + k];
  s = block_sum(s, sh);
  if (threadIdx.x != 0) return;
  double cnt = (double)(d.nx - 2) * (double)(d.ny - 2) * (double)(d.nz - 2);
  JobState& t = S[j];
  t.cur ^= 1;
  double rms = cnt > 0.0 ? sqrt(s / cnt) : 0.0;
  long long it = t.sor_it;
  t.rms = rms;
  t.sor_it = it + 1;
  t.om = it == 0 ? 1.0 / (1.0 - d.rs2 / 2.0) : 1.0 / (1.0 - d.rs2 * t.om / 4.0);
  if (rel ? rms < d.rtol * t.r0 : rms < d.tol)
    t.status = kConverged;
  else if (t.sor_it >= d.maxit)
    t.status = kSorCap;
}

// FP32 residual of the level's correction, which is in e2 after the three
// pre-smoothing sweeps (e -> e2 -> e -> e2).
__global__ void __launch_bounds__(256) k_res32(WL w, const LvlD* __restrict__ L, int lvl,
                                               const JobState* __restrict__ S) {
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != kMg) return;
  const Lv d = lv_load(L, j, lvl);
  int x, y, z0;
  brick_col(lb, d.nx, d.ny, x, y, z0);
  if (x < 1 || x > d.nx - 2 || y < 1 || y > d.ny - 2) return;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    int z = z0 + k;
    if (z < 1 || z > d.nz - 2) continue;
    int i = x + d.sy * y + d.sz * z;
    float ns, dg;
    st32(d, d.e2, i, ns, dg);
    d.res[i] = d.rhs[i] + ns - dg * d.e2[i];
  }
}

// Full-weighting restriction (x 0.25 in the reference's schedule, x 1 in the
// relative-residual mode) of the level-l residual into the
// level-(l+1) right-hand side (pb_solver.rs:459-520); the coarse correction
// starts from zero.
__global__ void __launch_bounds__(256) k_restrict32(WL w, const LvlD* __restrict__ L, int lvl,
                                                    const JobState* __restrict__ S) {
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != kMg) return;
  const Lv f = lv_load(L, j, lvl), c = lv_load(L, j, lvl + 1);
  const float rsc = L[j * kMaxLev + lvl].rsc;
  int cx, cy, cz0;
  brick_col(lb, c.nx, c.ny, cx, cy, cz0);
  if (cx >= c.nx || cy >= c.ny) return;
  const float* __restrict__ res = f.res;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    int cz = cz0 + k;
    if (cz >= c.nz) continue;
    int fx = 2 * cx, fy = 2 * cy, fz = 2 * cz;
    float sum = 0.0f, ws = 0.0f;
    for (int dz = -1; dz <= 1; dz++) {
      int z = fz + dz;
      if (z < 0 || z >= f.nz) continue;
      float wz = dz == 0 ? 2.0f : 1.0f;
      for (int dy = -1; dy <= 1; dy++) {
        int y = fy + dy;
        if (y < 0 || y >= f.ny) continue;
        float wyz = wz * (dy == 0 ? 2.0f : 1.0f);
        for (int dx = -1; dx <= 1; dx++) {
          int x = fx + dx;
          if (x < 0 || x >= f.nx) continue;
          float wt = wyz * (dx == 0 ? 2.0f : 1.0f);
          sum += wt * res[x + f.sy * y + f.sz * z];
          ws += wt;
        }
      }
    }
    int i = cx + c.sy * cy + c.sz * cz;
    c.rhs[i] = rsc * sum / ws;
    c.e[i] = 0.0f;
  }
}

// Trilinear prolongation of the level-(l+1) correction added at every
// level-l point (pb_solver.rs:522-578; interior points only in the
// relative-residual mode, where corrections vanish on the boundary); the fine correction is in e2 between
// the pre- and post-smoothing sweeps, the coarse one in e.
__global__ void __launch_bounds__(256) k_prolong32(WL w, const LvlD* __restrict__ L, int lvl,
                                                   const JobState* __restrict__ S) {
  int lb, j = wl_job(w, blockIdx.x, lb);
  if (S[j].status != kMg) return;
  const Lv f = lv_load(L, j, lvl), c = lv_load(L, j, lvl + 1);
  const bool skipb = L[j * kMaxLev + lvl].skipb != 0;
  int fx, fy, fz0;
  brick_col(lb, f.nx, f.ny, fx, fy, fz0);
  if (fx >= f.nx || fy >= f.ny) return;
  if (skipb && (fx == 0 || fx == f.nx - 1 || fy == 0 || fy == f.ny - 1)) return;
  const float* __restrict__ ce = c.e;
  int mx = c.nx >= 2 ? c.nx - 2 : 0, my = c.ny >= 2 ? c.ny - 2 : 0, mz = c.nz >= 2 ? c.nz - 2 : 0;
  int x0 = min(fx >> 1, mx), y0 = min(fy >> 1, my);
  float dx = (float)fx * 0.5f - (float)x0, dy = (float)fy * 0.5f - (float)y0;
#pragma unroll
  for (int k = 0; k < 8; k++) {
    int fz = fz0 + k;
    if (fz >= f.nz || (skipb && (fz == 0 || fz == f.nz - 1))) continue;
    int z0 = min(fz >> 1, mz);
    float dz = (float)fz * 0.5f - (float)z0;
    const float* b = ce + x0 + c.sy * y0 + c.sz * z0;
    float c00 = b[0] * (1.0f - dx) + b[1] * dx;
    float c10 = b[c.sy] * (1.0f - dx) + b[c.sy + 1] * dx;
    float c01 = b[c.sz] * (1.0f - dx) + b[c.sz + 1] * dx;
    float c11 = b[c.sz + c.sy] * (1.0f - dx) + b[c.sz + c.sy + 1] * dx;
    float c0 = c00 * (1.0f - dy) + c10 * dy, c1 = c01 * (1.0f - dy) + c11 * dy;
    f.e2[fx + f.sy * fy + f.sz * fz] += c0 * (1.0f - dz) + c1 * dz;
  }
}

// Coarsest level: 50 red-black sweeps in one block per grid (pb_solver.rs:850-870).
__global__ void k_coarse32(WL w, const LvlD* __restrict__ L, int lvl, const JobState* __restrict__ S, int sweeps) {
  int j = w.job[blockIdx.x];
  if (S[j].status != kMg) return;
  const Lv d = lv_load(L, j, lvl);
  if (d.nx < 3 || d.ny < 3 || d.nz < 3) return;
  int nxi = d.nx - 2, nyi = d.ny - 2;
  int ni = nxi * nyi * (d.nz - 2);
  for (int s = 0; s < sweeps; s++)
    for (int colour = 0; colour < 2; colour++) {
      for (int k = threadIdx.x; k < ni; k += blockDim.x) {
        int ix = 1 + k % nxi, iy = 1 + (k / nxi) % nyi, iz = 1 + k / (nxi * nyi);
        if (((ix + iy + iz + colour) & 1) != 0) continue;
        int i = ix + d.sy * iy + d.sz * iz;
        float ns, dg;
        st32(d, d.e, i, ns, dg);
        float old = d.e[i];
        float gs = (ns + d.rhs[i]) / dg;
        d.e[i] = old + d.om * (gs - old);
      }
      __syncthreads();
    }
}

// Debye-Hueckel boundary values (set_dh_boundary, pb_solver.rs:68-93) of
// every grid of a batch in one launch: per boundary point the sum over atoms
// of 332.0522 q exp(-kappa r) / (eps_out r), pair terms in FP32 (coordinates
// relative to the grid origin), accumulated in FP64.  Reference grids
// (kappa = 0) skip the exponential.
// phi2 (may be null): a second grid of the same geometry and atoms whose
// boundary values take kappa kap2 and eout2 -- a solvated solve and its
// reference solve share the distance work.
struct DhD {
  double* phi;
  double* phi2;
  const double *xyz, *q;
  int nx, ny, nz, na;
  double ox, oy, oz, h, kap, eout, kap2, eout2;
};

// Boundary points enumerated face by face: the two z faces, the two y faces
// of the interior z planes, the two x faces of the interior rows.
__device__ __forceinline__ bool bnd_point(int nx, int ny, int nz, long long k, int& ix, int& iy, int& iz) {
  long long nxy = (long long)nx * ny;
  int nzi = max(nz - 2, 0), nyi = max(ny - 2, 0);
  if (k < 2 * nxy) {
    iz = k < nxy ? 0 : nz - 1;
    long long r = k % nxy;
    ix = (int)(r % nx);
    iy = (int)(r / nx);
    return true;
  }
  k -= 2 * nxy;
  long long nyf = (long long)nx * nzi;
  if (k < 2 * nyf) {
    iy = k < nyf ? 0 : ny - 1;
    long long r = k % nyf;
    ix = (int)(r % nx);
    iz = 1 + (int)(r / nx);
    return true;
  }
  k -= 2 * nyf;
  long long nxf = (long long)nyi * nzi;
  if (k < 2 * nxf) {
    ix = k < nxf ? 0 : nx - 1;
    long long r = k % nxf;
    iy = 1 + (int)(r % nyi);
    iz = 1 + (int)(r / nyi);
    return true;
  }
  return false;
}

long long bnd_count(const PbGeom& g) {
  long long nzi = std::max(g.nz - 2, 0), nyi = std::max(g.ny - 2, 0);
  return 2LL * g.nx * g.ny + 2LL * g.nx * nzi + 2LL * nyi * nzi;
}

__global__ void __launch_bounds__(256) k_dh32(WL w, const DhD* __restrict__ D) {
  __shared__ float4 sa[256];
  int lb, j = wl_job(w, blockIdx.x, lb);
  const DhD& d = D[j];
  long long nb = 2LL * d.nx * d.ny + 2LL * d.nx * max(d.nz - 2, 0) + 2LL * max(d.ny - 2, 0) * max(d.nz - 2, 0);
  long long k = (long long)lb * blockDim.x + threadIdx.x;
  int ix = 0, iy = 0, iz = 0;
  bool valid = k < nb && bnd_point(d.nx, d.ny, d.nz, k, ix, iy, iz);
  float px = (float)(ix * d.h), py = (float)(iy * d.h), pz = (float)(iz * d.h);
  const float kap = (float)d.kap, kap2 = (float)d.kap2;
  const bool ionic = d.kap != 0.0, ionic2 = d.kap2 != 0.0, two = d.phi2 != nullptr;
  double acc = 0.0, acc2 = 0.0;
  for (int a0 = 0; a0 < d.na; a0 += 256) {
    int a = a0 + threadIdx.x;
    if (a < d.na)
      sa[threadIdx.x] = make_float4((float)(d.xyz[3 * a] - d.ox), (float)(d.xyz[3 * a + 1] - d.oy),
                                    (float)(d.xyz[3 * a + 2] - d.oz), (float)d.q[a]);
    __syncthreads();
    int m = min(256, d.na - a0);
    if (valid) {
      for (int t = 0; t < m; t++) {
        float4 A = sa[t];
        float dx = px - A.x, dy = py - A.y, dz = pz - A.z;
        float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 <= 1e-20f) continue;
        float ir = rsqrtf(r2);
        float term = A.w * ir;
        const float r = r2 * ir;
        acc += (double)(ionic ? term * __expf(-kap * r) : term);
        if (two) acc2 += (double)(ionic2 ? term * __expf(-kap2 * r) : term);
      }
    }
    __syncthreads();
  }
  if (valid) {
    const long long o = ix + (long long)d.nx * (iy + (long long)d.ny * iz);
    d.phi[o] = 332.0522 * acc / d.eout;
    if (two) d.phi2[o] = 332.0522 * acc2 / d.eout2;
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
  const long long ci = i % d.nx + (long long)d.px * (i / d.nx);  // padded FP32 index
  ((float*)l0.ex)[ci] = (float)d.ex[i];
  ((float*)l0.ey)[ci] = (float)d.ey[i];
  ((float*)l0.ez)[ci] = (float)d.ez[i];
  ((float*)l0.k2)[ci] = (float)d.k2[i];
}

// Level-0 stencil codes of every grid from its FP64 maps (exact compares),
// with per-grid counts of map reads (edges that cross the surface) and of
// charged points for the traffic figures; bad is set if a kbar^2 value is
// neither 0 nor the grid's constant.
__device__ __forceinline__ unsigned fcode(double v, double ein, double eout) {
  return v == eout ? 0u : (v == ein ? 1u : 2u);
}
__global__ void k_codes(WL w, const JobD* __restrict__ J, const LvlD* __restrict__ L,
                        unsigned long long* __restrict__ counts, int* __restrict__ bad) {
  int lb, j = wl_job(w, blockIdx.x, lb);
  const JobD& d = J[j];
  int n = d.nx * d.ny * d.nz;
  int i = lb * blockDim.x + threadIdx.x;
  unsigned exc = 0, chg = 0;
  if (i < n) {
    const int x = i % d.nx, t = i / d.nx;
    const long long ci = x + (long long)d.px * t;  // t = y + ny z
    unsigned c = 0;
    if (!d.uniform) {
      unsigned a = fcode(d.ex[i], d.din, d.dout), b = fcode(d.ey[i], d.din, d.dout), e = fcode(d.ez[i], d.din, d.dout);
      c = a | (b << 2) | (e << 4);
      exc = (a == 2u) + (b == 2u) + (e == 2u);
      double k = d.k2[i];
      if (k != 0.0) {
        if (k == d.dkb)
          c |= 64u;
        else
          *bad = 1;
      }
    }
    if (d.rho[i] != 0.0) {
      c |= 128u;
      chg = 1;
    }
    ((uint8_t*)L[j * kMaxLev].cd)[ci] = (uint8_t)c;
  }
  exc = __reduce_add_sync(0xffffffffu, exc);
  chg = __reduce_add_sync(0xffffffffu, chg);
  if ((threadIdx.x & 31) == 0 && (exc | chg)) {
    atomicAdd(counts + 2 * j, (unsigned long long)exc);
    atomicAdd(counts + 2 * j + 1, (unsigned long long)chg);
  }
}

__global__ void k_inject32(WL w, const LvlD* __restrict__ L, int lvl) {
  int lb, j = wl_job(w, blockIdx.x, lb);
  const LvlD& f = L[j * kMaxLev + lvl];
  const LvlD& c = L[j * kMaxLev + lvl + 1];
  int cn = c.nx * c.ny * c.nz;
  int i = lb * blockDim.x + threadIdx.x;
  if (i >= cn) return;
  int cx = i % c.nx, cy = (i / c.nx) % c.ny, cz = i / (c.nx * c.ny);
  int fi = min(2 * cx, f.nx - 1) + f.px * (min(2 * cy, f.ny - 1) + f.ny * min(2 * cz, f.nz - 1));
  int ci = cx + c.px * (cy + c.ny * cz);
  ((float*)c.ex)[ci] = f.ex[fi];
  ((float*)c.ey)[ci] = f.ey[fi];
  ((float*)c.ez)[ci] = f.ez[fi];
  ((float*)c.k2)[ci] = f.k2[fi];
  ((uint8_t*)c.cd)[ci] = f.cd[fi] & 127u;  // maps are injected, so are their codes; no rho below level 0
}

// Coarse maps of the relative-residual mode: a coarse face spans two fine
// faces in series along its axis (harmonic mean, equal values copied) and
// the fine faces of the 3 x 3 neighbouring lines across it in parallel
// (weights 1-2-1 per transverse direction, renormalised at the grid edge);
// kbar^2 and its code bit are injected.  Face codes by exact compares, as at
// level 0 (a face whose lines are all eps_in is eps_in exactly).
__device__ __forceinline__ float coarse_face(const LvlD& f, const float* __restrict__ m, int axis, int bx, int by,
                                             int bz) {
  const int n[3] = {f.nx, f.ny, f.nz};
  const int t1 = axis == 0 ? 1 : 0, t2 = axis == 2 ? 1 : 2;
  float sum = 0.0f, ws = 0.0f, first = 0.0f;
  bool same = true, any = false;
  for (int u = -1; u <= 1; u++)
    for (int v = -1; v <= 1; v++) {
      int p[3] = {bx, by, bz};
      p[t1] += u;
      p[t2] += v;
      if (p[t1] < 0 || p[t1] >= n[t1] || p[t2] < 0 || p[t2] >= n[t2]) continue;
      int q[3] = {p[0], p[1], p[2]};
      q[axis] = min(p[axis] + 1, n[axis] - 1);
      const float e0 = m[p[0] + f.px * (p[1] + f.ny * p[2])], e1 = m[q[0] + f.px * (q[1] + f.ny * q[2])];
      if (!any) first = e0;
      any = true;
      same = same && e0 == first && e1 == first;
      const float w = (u == 0 ? 2.0f : 1.0f) * (v == 0 ? 2.0f : 1.0f);
      sum += w * (e0 == e1 ? e0 : 2.0f / (1.0f / e0 + 1.0f / e1));
      ws += w;
    }
  return same ? first : sum / ws;
}
__device__ __forceinline__ unsigned fcode32(float v, float ein, float eout) {
  return v == eout ? 0u : (v == ein ? 1u : 2u);
}
__global__ void k_coarsen32(WL w, const LvlD* __restrict__ L, int lvl) {
  int lb, j = wl_job(w, blockIdx.x, lb);
  const LvlD& f = L[j * kMaxLev + lvl];
  const LvlD& c = L[j * kMaxLev + lvl + 1];
  int cn = c.nx * c.ny * c.nz;
  int i = lb * blockDim.x + threadIdx.x;
  if (i >= cn) return;
  int cx = i % c.nx, cy = (i / c.nx) % c.ny, cz = i / (c.nx * c.ny);
  int bx = min(2 * cx, f.nx - 1), by = min(2 * cy, f.ny - 1), bz = min(2 * cz, f.nz - 1);
  int fi = bx + f.px * (by + f.ny * bz);
  int ci = cx + c.px * (cy + c.ny * cz);
  const float ex = coarse_face(f, f.ex, 0, bx, by, bz), ey = coarse_face(f, f.ey, 1, bx, by, bz),
              ez = coarse_face(f, f.ez, 2, bx, by, bz);
  ((float*)c.ex)[ci] = ex;
  ((float*)c.ey)[ci] = ey;
  ((float*)c.ez)[ci] = ez;
  ((float*)c.k2)[ci] = f.k2[fi];
  ((uint8_t*)c.cd)[ci] = (uint8_t)(fcode32(ex, c.fin, c.fout) | (fcode32(ey, c.fin, c.fout) << 2) |
                                   (fcode32(ez, c.fin, c.fout) << 4) | (f.cd[fi] & 64u));
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
// FP64 pool regions of a job, in units of g.n(): phi, phi2, rho (unless it
// uses another job's), then for solvated jobs ex, ey, ez, kbar^2
struct F64Lay {
  size_t rho, maps, total;
};
F64Lay f64_lay(const PbJob& J) {
  F64Lay f;
  f.rho = 2;
  f.maps = J.rho_of >= 0 ? 2 : 3;
  f.total = f.maps + (J.uniform ? 0 : 4);
  return f;
}
// FP32 and code arrays: rows padded to a multiple of 4 points (16 bytes of FP32)
int pitch(const PbGeom& g) { return (int)((g.nx + 3) & ~3); }
size_t padded_n(const PbGeom& g) { return (size_t)pitch(g) * g.ny * g.nz; }

long long nbricks(const PbGeom& g) { return cdiv(g.nx, 32) * cdiv(g.ny, 8) * cdiv(g.nz, 8); }

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
  void add(int s, long long j, long long blocks) {
    if (blocks <= 0) return;
    Slot& S = slots[s];
    S.start.push_back(S.total);
    S.job.push_back((int)j);
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

void PbBatchEngine::release() {
  if (graph_) cudaGraphExecDestroy(graph_);
  graph_ = nullptr;
  for (DevBuf* b : {&pool64_, &pool32_, &pool8_, &desc_, &part_, &small_, &lists_}) *b = DevBuf();
}

PbBatchEngine::~PbBatchEngine() {
  if (graph_) cudaGraphExecDestroy(graph_);
  for (cudaEvent_t e : prof_events_) cudaEventDestroy(e);
  for (cudaEvent_t e : setup_events_) cudaEventDestroy(e);
  if (start_event_) cudaEventDestroy(start_event_);
  for (cudaStream_t w : setup_streams_) {
    cudaStreamSynchronize(w);
    cudaStreamDestroy(w);
  }
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
    size_t o64 = 0, o32[kMaxLev] = {}, o8[kMaxLev] = {};
  };
  std::vector<Lay> lay(nj);
  size_t n64 = 0, n32 = 0, n8 = 0;
  for (int j = 0; j < nj; j++) {
    PbJob& J = jobs[j];
    Lay& Y = lay[j];
    size_t n = J.g.n();
    Y.o64 = n64;
    if (J.rho_of >= j || (J.rho_of >= 0 && (jobs[J.rho_of].atoms != J.atoms || jobs[J.rho_of].g.n() != J.g.n() ||
                                             jobs[J.rho_of].g.ox != J.g.ox || jobs[J.rho_of].g.oy != J.g.oy ||
                                             jobs[J.rho_of].g.oz != J.g.oz || jobs[J.rho_of].g.h != J.g.h ||
                                             jobs[J.rho_of].g.nx != J.g.nx || jobs[J.rho_of].g.ny != J.g.ny)))
      throw Error(RSTG_ERR_INVALID, "PB job shares the charge map of a job with another grid or atom set");
    n64 += f64_lay(J).total * n;
    n64 = (n64 + 63) & ~(size_t)63;
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
      size_t m = padded_n(Y.lv[l]);
      n32 += (J.uniform ? 4 : 8) * m;
      n32 = (n32 + 63) & ~(size_t)63;
      if (l == 0 || !J.uniform) {  // codes: rho bits of every level-0 grid, stencils of solvated grids
        Y.o8[l] = n8;
        n8 = (n8 + m + 255) & ~(size_t)255;
      }
    }
  }
  size_t b64 = std::max<size_t>(n64, 1) * 8, b32 = std::max<size_t>(n32, 1) * 4;
  if (pool64_.bytes < b64) pool64_ = DevBuf(b64, st);
  if (pool32_.bytes < b32) pool32_ = DevBuf(b32, st);
  size_t b8 = std::max<size_t>(n8, 1);
  if (pool8_.bytes < b8) pool8_ = DevBuf(b8, st);
  uint8_t* P8 = (uint8_t*)pool8_.p;
  double* P64 = pool64_.as<double>();
  float* P32 = pool32_.as<float>();
  RSTG_CUDA(cudaMemsetAsync(P32, 0, b32, st));

  // ---- maps and boundary values (FP64, the reference's set-up) -------------
  // One grid's set-up is a chain of small launches with host waits (the
  // exterior flood fill tests for its fixed point every eight passes), so the
  // grids are spread over worker threads, each on its own stream; the main
  // stream waits for all of them before the cycles start.
  {
    const int W = (int)std::min<size_t>(kSetupWorkers, (size_t)nj);
    int dev = 0;
    RSTG_CUDA(cudaGetDevice(&dev));
    while ((int)setup_streams_.size() < W) {
      cudaStream_t w;
      RSTG_CUDA(cudaStreamCreateWithFlags(&w, cudaStreamNonBlocking));
      setup_streams_.push_back(w);
      cudaEvent_t e;
      RSTG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      setup_events_.push_back(e);
    }
    if (!start_event_) RSTG_CUDA(cudaEventCreateWithFlags(&start_event_, cudaEventDisableTiming));
    RSTG_CUDA(cudaEventRecord(start_event_, st));  // the pools are allocated and cleared on st
    std::vector<std::exception_ptr> err(W);
    auto work = [&](int w) {
      try {
        cudaSetDevice(dev);
        cudaStream_t ws = setup_streams_[w];
        RSTG_CUDA(cudaStreamWaitEvent(ws, start_event_, 0));
        PbStreamScope sc(ws);
        for (int j = w; j < nj; j += W) {
          PbJob& J = jobs[j];
          size_t n = J.g.n();
          double* base = P64 + lay[j].o64;
          const F64Lay f = f64_lay(J);
          double *phi = base, *rho = J.rho_of >= 0 ? nullptr : base + f.rho * n;
          double* m = base + f.maps * n;
          double *ex = J.uniform ? nullptr : m, *ey = J.uniform ? nullptr : m + n,
                 *ez = J.uniform ? nullptr : m + 2 * n, *k2 = J.uniform ? nullptr : m + 3 * n;
          pb_maps_into(c_, J.g, *J.atoms, p, J.ein, J.eout, J.kap, J.ionic, rho, ex, ey, ez, k2);
          RSTG_CUDA(cudaMemsetAsync(phi, 0, n * 8, ws));
          if (J.bc.kind != 1) pb_boundary(c_, J.g, phi, *J.atoms, J.bc);
        }
        RSTG_CUDA(cudaEventRecord(setup_events_[w], ws));
      } catch (...) {
        err[w] = std::current_exception();
      }
    };
    std::vector<std::thread> th;
    for (int w = 1; w < W; w++) th.emplace_back(work, w);
    work(0);
    for (auto& t : th) t.join();
    for (auto& e : err)
      if (e) std::rethrow_exception(e);
    for (int w = 0; w < W; w++) RSTG_CUDA(cudaStreamWaitEvent(st, setup_events_[w], 0));
  }
  std::vector<double*> phi_now(nj);  // current potential buffer of each grid (host view)
  for (int j = 0; j < nj; j++) phi_now[j] = P64 + lay[j].o64;
  // Debye-Hueckel boundary values of the listed grids in one launch
  auto dh_launch = [&](const std::vector<int>& which) {
    std::vector<DhD> dd;
    Lists dl;
    int sd = dl.add_slot();
    std::vector<char> listed(nj, 0), merged(nj, 0);
    for (int j : which) listed[j] = 1;
    for (int j : which) {
      if (merged[j]) continue;
      const PbJob& J = jobs[j];
      DhD x;
      x.phi = phi_now[j];
      x.phi2 = nullptr;
      x.kap2 = 0.0;
      x.eout2 = 1.0;
      for (int k2 = j + 1; k2 < nj; k2++)  // the reference solve on the same grid and atoms
        if (listed[k2] && !merged[k2] && jobs[k2].rho_of == j) {
          x.phi2 = phi_now[k2];
          x.kap2 = jobs[k2].bc.kappa;
          x.eout2 = jobs[k2].bc.eout;
          merged[k2] = 1;
          break;
        }
      x.xyz = J.atoms->xyz.as<double>();
      x.q = J.atoms->q.as<double>();
      x.nx = J.g.nx;
      x.ny = J.g.ny;
      x.nz = J.g.nz;
      x.na = J.atoms->n;
      x.ox = J.g.ox;
      x.oy = J.g.oy;
      x.oz = J.g.oz;
      x.h = J.g.h;
      x.kap = J.bc.kappa;
      x.eout = J.bc.eout;
      dl.add(sd, (long long)dd.size(), cdiv(bnd_count(J.g), 256));
      dd.push_back(x);
    }
    if (dd.empty()) return;
    DevBuf dbuf(dd.size() * sizeof(DhD), st);
    RSTG_CUDA(cudaMemcpyAsync(dbuf.p, dd.data(), dd.size() * sizeof(DhD), cudaMemcpyHostToDevice, st));
    std::vector<WL> wl;
    dl.upload(lists_, st, wl);
    k_dh32<<<dl.slots[sd].total, 256, 0, st>>>(wl[sd], dbuf.as<DhD>());
    launched(c_);
    RSTG_CUDA(cudaStreamSynchronize(st));  // dd is pageable and goes out of scope
  };
  {
    std::vector<int> which;
    for (int j = 0; j < nj; j++)
      if (jobs[j].bc.kind == 1) which.push_back(j);
    dh_launch(which);
  }

  if (std::getenv("RSTG_PB_DEBUG")) {
    RSTG_CUDA(cudaStreamSynchronize(st));
    std::fprintf(stderr, "pb set-up: maps and boundary values of %d grids %.2f ms\n", nj, ms(t0, now()));
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
    const F64Lay f = f64_lay(J);
    d.phi = base;
    d.phi2 = base + n;
    d.rho = J.rho_of >= 0 ? hd[J.rho_of].rho : base + f.rho * n;
    if (!J.uniform) {
      d.ex = base + f.maps * n;
      d.ey = base + (f.maps + 1) * n;
      d.ez = base + (f.maps + 2) * n;
      d.k2 = base + (f.maps + 3) * n;
    }
    d.cd = P8 + Y.o8[0];
    d.px = pitch(J.g);
    d.din = J.ein;
    d.dout = J.eout;
    d.dkb = J.ionic ? p.solvent_dielectric * J.kap * J.kap : 0.0;  // assign_kappa, pb_grid.rs:964
    d.nx = J.g.nx;
    d.ny = J.g.ny;
    d.nz = J.g.nz;
    d.uniform = J.uniform ? 1 : 0;
    d.ih = 1.0 / (J.g.h * J.g.h);
    d.eps = J.ein;
    d.tol = J.tol;
    d.maxv = (int)std::min<int64_t>(std::max<int64_t>(J.maxit / 6, 1), 200);
    d.maxit = J.maxit;
    d.rtol = J.rtol > 0.0 ? J.rtol : 0.0;
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
    max_res = std::max(max_res, nbricks(J.g));
    max_sor = std::max(max_sor, cdiv(J.g.nx, kSwTX) * cdiv(J.g.ny, kSwTY) * cdiv(J.g.nz, kSwZC0));  // sweep blocks
    for (int l = 0; l <= std::max(Y.nlev, 0); l++) {
      const PbGeom& g = Y.lv[l];
      size_t m = padded_n(g);
      LvlD& L = hl[(size_t)j * kMaxLev + l];
      std::memset(&L, 0, sizeof(L));
      float* b = P32 + Y.o32[l];
      L.e = b;
      L.e2 = b + m;
      L.rhs = b + 2 * m;
      L.res = b + 3 * m;
      L.px = pitch(g);
      L.zc = sweep_chunk(l);
      if (!J.uniform) {
        L.ex = b + 4 * m;
        L.ey = b + 5 * m;
        L.ez = b + 6 * m;
        L.k2 = b + 7 * m;
        L.cd = P8 + Y.o8[l];
      } else if (l == 0) {
        L.cd = P8 + Y.o8[0];
      }
      L.fin = (float)J.ein;
      L.fout = (float)J.eout;
      L.kb = (float)d.dkb;
      L.rsc = J.rtol > 0.0 ? 1.0f : 0.25f;
      L.skipb = J.rtol > 0.0 ? 1 : 0;
      L.nx = g.nx;
      L.ny = g.ny;
      L.nz = g.nz;
      L.uniform = J.uniform ? 1 : 0;
      L.ih = (float)(1.0 / (g.h * g.h));
      L.om = J.rtol > 0.0 ? 1.0f : (float)pb_omega(g.nx, g.ny, g.nz);
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
  size_t pbytes = (size_t)nparts * nj * 8 * 2;  // residual partials, then SOR sweep partials
  if (part_.bytes < pbytes) part_ = DevBuf(pbytes, st);
  if (small_.bytes < (size_t)nj * 32 + 16) small_ = DevBuf((size_t)nj * 32 + 16, st);
  double* part = part_.as<double>();
  double* spart = part + (size_t)nparts * nj;

  // FP32 maps and stencil codes (level-0 codes of every grid: the rho bit)
  std::vector<unsigned long long> counts(2 * (size_t)nj);
  {
    Lists setup;
    int s0 = setup.add_slot(), sc = setup.add_slot();
    std::vector<int> si(kMaxLev), sv(kMaxLev);
    for (int l = 0; l + 1 < kMaxLev; l++) {
      si[l] = setup.add_slot();
      sv[l] = setup.add_slot();
    }
    int maxl = 0;
    for (int j = 0; j < nj; j++) {
      setup.add(sc, j, cdiv((long long)jobs[j].g.n(), kT));
      if (jobs[j].uniform) continue;
      setup.add(s0, j, cdiv((long long)jobs[j].g.n(), kT));
      for (int l = 0; l < lay[j].nlev; l++)
        setup.add(jobs[j].rtol > 0.0 ? sv[l] : si[l], j, cdiv((long long)lay[j].lv[l + 1].n(), kT));
      maxl = std::max(maxl, lay[j].nlev);
    }
    std::vector<WL> wl;
    setup.upload(lists_, st, wl);
    unsigned long long* dcnt = (unsigned long long*)small_.p;
    int* dbad = (int*)(dcnt + 2 * (size_t)nj);
    RSTG_CUDA(cudaMemsetAsync(dcnt, 0, 16 * (size_t)nj + 16, st));
    k_codes<<<setup.slots[sc].total, kT, 0, st>>>(wl[sc], dJ, dL, dcnt, dbad);
    launched(c_);
    if (setup.slots[s0].total > 0) {
      k_maps32<<<setup.slots[s0].total, kT, 0, st>>>(wl[s0], dJ, dL);
      launched(c_);
    }
    for (int l = 0; l < maxl; l++) {
      if (setup.slots[si[l]].total > 0) {
        k_inject32<<<setup.slots[si[l]].total, kT, 0, st>>>(wl[si[l]], dL, l);
        launched(c_);
      }
      if (setup.slots[sv[l]].total > 0) {
        k_coarsen32<<<setup.slots[sv[l]].total, kT, 0, st>>>(wl[sv[l]], dL, l);
        launched(c_);
      }
    }
    int bad = 0;
    RSTG_CUDA(cudaMemcpyAsync(counts.data(), dcnt, 16 * (size_t)nj, cudaMemcpyDeviceToHost, st));
    RSTG_CUDA(cudaMemcpyAsync(&bad, dbad, 4, cudaMemcpyDeviceToHost, st));
    RSTG_CUDA(cudaStreamSynchronize(st));
    if (bad) throw Error(RSTG_ERR_INVALID, "PB kbar^2 map holds a value other than 0 and eps_s kappa^2");
  }
  auto t1 = now();
  stats.ms_setup += ms(t0, t1);

  // ---- lock-step iterations ------------------------------------------------
  // Initial residuals of the multigrid grids (no convergence test: the
  // reference tests after each V-cycle).
  // SOR grids (too small for multigrid) start from the residual of their
  // initial potential as well.
  auto sor_residuals = [&](const std::vector<int>& which) {
    Lists rl;
    int s = rl.add_slot();
    for (int j : which) rl.add(s, j, nbricks(jobs[j].g));
    if (rl.slots[s].total == 0) return;
    std::vector<WL> wl;
    rl.upload(lists_, st, wl);
    k_res64<<<rl.slots[s].total, kT, 0, st>>>(wl[s], dJ, dL, dS, kSor, part, nparts);
    launched(c_);
  };
  {
    Lists init;
    int s = init.add_slot(), sn = init.add_slot();
    std::vector<int> sor0;
    for (int j = 0; j < nj; j++)
      if (hs[j].status == kMg) {
        init.add(s, j, nbricks(jobs[j].g));
        init.add(sn, j, 1);
      } else if (hs[j].status == kSor) {
        sor0.push_back(j);
      }
    if (init.slots[s].total > 0) {
      std::vector<WL> wl;
      init.upload(lists_, st, wl);
      k_res64<<<init.slots[s].total, kT, 0, st>>>(wl[s], dJ, dL, dS, kMg, part, nparts);
      k_norm<<<init.slots[sn].total, 256, 0, st>>>(wl[sn], dJ, dS, part, nparts, 0, kMg);
      launched(c_, 2);
    }
    sor_residuals(sor0);
    // relative-residual SOR grids keep their initial residual norm as r0
    Lists r0l;
    int s0 = r0l.add_slot();
    for (int j : sor0)
      if (jobs[j].rtol > 0.0) r0l.add(s0, j, 1);
    if (r0l.slots[s0].total > 0) {
      std::vector<WL> wl;
      r0l.upload(lists_, st, wl);
      k_norm<<<r0l.slots[s0].total, 256, 0, st>>>(wl[s0], dJ, dS, part, nparts, 0, kSor);
      launched(c_);
    }
    RSTG_CUDA(cudaStreamSynchronize(st));
  }
  const int K = std::max(1, chunk_cycles), KS = 4;  // cycles per chunk, SOR sweeps per cycle
  // the sweep's rings exceed the 48 KB default (set per call: the attribute is per device)
  RSTG_CUDA(cudaFuncSetAttribute(k_sweep_t<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SwSmem)));
  RSTG_CUDA(cudaFuncSetAttribute(k_sweep_t<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SwSmem)));
  bool use_graph = !profile && st != nullptr && st != cudaStreamLegacy && st != cudaStreamPerThread;
  std::vector<int> key;  // (job, status) pairs of the current lists
  std::vector<WL> wl;
  Lists lists;
  int per_chunk = 0;
  cudaGraphExec_t exec = nullptr;
  struct LvSlots {
    int rb, res, restr, coarse, prol;
  };
  std::vector<LvSlots> ls(kMaxLev);
  int s_res = 0, s_norm = 0, s_sres = 0, s_sor = 0, s_snorm = 0, maxlev = 0;
  bool any_mg = false, any_sor = false;
  // profile mode: events around every launch; the level-0 kernels also
  // carry their algorithmic bytes (compulsory DRAM traffic per launch) from
  // the current lists.  kind: roofline slot (-1 none); det: kernel family.
  double kbytes[kProfKernels] = {};
  struct Mark {
    int kind, det, lvl;
    cudaEvent_t a, b;
  };
  std::vector<Mark> marks;
  size_t next_ev = 0;
  auto mark = [&](int kind, int det, int lvl, auto&& launch) {
    if (!profile) {
      launch();
      return;
    }
    while (prof_events_.size() < 2 * (next_ev + 1)) {
      cudaEvent_t e;
      RSTG_CUDA(cudaEventCreate(&e));
      prof_events_.push_back(e);
    }
    cudaEvent_t a = prof_events_[2 * next_ev], b = prof_events_[2 * next_ev + 1];
    next_ev++;
    RSTG_CUDA(cudaEventRecord(a, st));
    launch();
    RSTG_CUDA(cudaEventRecord(b, st));
    marks.push_back({kind, det, lvl, a, b});
  };
  enum { dSweep, dRes32, dRestrict, dProlong, dCoarse, dRes64, dUpdate, dNorm, dSor };
  auto enqueue_chunk = [&]() {
    int n = 0;
    auto go = [&](int slot) { return lists.slots[slot].total; };
    // three sweeps: pre-smoothing e -> e2 -> e -> e2, post-smoothing back to e
    // (the finest level's correction is not cleared between cycles: its first sweep reads zeros)
    auto sweeps = [&](int l, int first) {
      for (int s = 0; s < 3; s++) {
        const int flip = first ^ (s & 1), zero = (l == 0 && first == 0 && s == 0) ? 1 : 0;
        mark(l == 0 ? 0 : -1, dSweep, l, [&] {
          k_sweep_t<false><<<go(ls[l].rb), kSwThreads, sizeof(SwSmem), st>>>(wl[ls[l].rb], dL, l, dS, flip, zero,
                                                                             nullptr, 0);
        });
        n++;
      }
    };
    for (int k = 0; k < K; k++) {
      if (any_mg) {
        for (int l = 0; l <= maxlev; l++) {
          if (go(ls[l].rb)) {
            sweeps(l, 0);
            mark(l == 0 ? 1 : -1, dRes32, l, [&] { k_res32<<<go(ls[l].res), kT, 0, st>>>(wl[ls[l].res], dL, l, dS); });
            mark(-1, dRestrict, l,
                 [&] { k_restrict32<<<go(ls[l].restr), kT, 0, st>>>(wl[ls[l].restr], dL, l, dS); });
            n += 2;
          }
          if (go(ls[l].coarse)) {
            mark(-1, dCoarse, l,
                 [&] { k_coarse32<<<go(ls[l].coarse), 256, 0, st>>>(wl[ls[l].coarse], dL, l, dS, 50); });
            n++;
          }
        }
        for (int l = maxlev - 1; l >= 0; l--) {
          if (!go(ls[l].prol)) continue;
          mark(-1, dProlong, l, [&] { k_prolong32<<<go(ls[l].prol), kT, 0, st>>>(wl[ls[l].prol], dL, l, dS); });
          n++;
          sweeps(l, 1);
        }
        mark(2, dRes64, 0, [&] { k_upres64<<<go(s_res), kT, 0, st>>>(wl[s_res], dJ, dL, dS, kMg, part, nparts); });
        mark(-1, dNorm, 0, [&] { k_norm<<<go(s_norm), 256, 0, st>>>(wl[s_norm], dJ, dS, part, nparts, 1, kMg); });
        n += 3;
      }
      if (any_sor)
        for (int q = 0; q < KS; q++) {
          // sweep from e = 0 into e (the residual of the current potential is in rhs),
          // phi' = phi + e with the next residual, bookkeeping
          mark(-1, dSor, 0, [&] {
            k_sweep_t<true><<<go(s_sor), kSwThreads, sizeof(SwSmem), st>>>(wl[s_sor], dL, 0, dS, 1, 1, spart, nparts);
            k_upres64<<<go(s_sres), kT, 0, st>>>(wl[s_sres], dJ, dL, dS, kSor, part, nparts);
            k_sor_norm<<<go(s_snorm), 256, 0, st>>>(wl[s_snorm], dJ, dS, spart, part, nparts);
          });
          n += 3;
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
    s_res = lists.add_slot();
    s_norm = lists.add_slot();
    s_sres = lists.add_slot();
    s_sor = lists.add_slot();
    s_snorm = lists.add_slot();
    any_mg = any_sor = false;
    for (int j = 0; j < nj; j++) {
      const Lay& Y = lay[j];
      const PbGeom& g = jobs[j].g;
      if (hs[j].status == kMg) {
        any_mg = true;
        maxlev = std::max(maxlev, Y.nlev);
        for (int l = 0; l < Y.nlev; l++) {
          const PbGeom& a = Y.lv[l];
          lists.add(ls[l].rb, j, cdiv(a.nx, kSwTX) * cdiv(a.ny, kSwTY) * cdiv(a.nz, sweep_chunk(l)));
          lists.add(ls[l].res, j, nbricks(a));
          lists.add(ls[l].restr, j, nbricks(Y.lv[l + 1]));
          lists.add(ls[l].prol, j, nbricks(a));
        }
        lists.add(ls[Y.nlev].coarse, j, 1);
        lists.add(s_res, j, nbricks(g));
        lists.add(s_norm, j, 1);
      } else if (hs[j].status == kSor) {
        any_sor = true;
        lists.add(s_sres, j, nbricks(g));
        lists.add(s_sor, j, cdiv(g.nx, kSwTX) * cdiv(g.ny, kSwTY) * cdiv(g.nz, kSwZC0));
        lists.add(s_snorm, j, 1);
      }
    }
    for (int k = 0; k < kProfKernels; k++) kbytes[k] = 0.0;
    for (int j = 0; j < nj; j++)
      if (hs[j].status == kMg) {
        double pts = (double)jobs[j].g.n(), exc = (double)counts[2 * j], chg = (double)counts[2 * j + 1];
        bool u = jobs[j].uniform;
        kbytes[0] += pts * (u ? 12.0 : 13.0) + 4.0 * exc;  // one sweep: e read and written, rhs, (codes); map reads
        kbytes[1] += pts * (u ? 12.0 : 13.0) + 4.0 * exc;  // e, rhs, (codes), res written; map reads
        kbytes[2] += pts * 25.0 + 8.0 * (exc + chg);  // phi and e read, phi' and rhs written, codes; map, rho reads
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
    std::vector<int> redo, now_sor;
    for (int j = 0; j < nj; j++)
      if (hs[j].status == kDiverged) {
        phi_now[j] = hs[j].cur ? hd[j].phi2 : hd[j].phi;
        if (jobs[j].bc.kind == 1)
          redo.push_back(j);
        else
          pb_boundary(c_, jobs[j].g, phi_now[j], *jobs[j].atoms, jobs[j].bc);
        now_sor.push_back(j);
        hs[j].status = kSor;
        hs[j].om = 1.0;
        hs[j].sor_it = 0;
        hs[j].rms = DBL_MAX;
        switched = true;
      }
    dh_launch(redo);
    if (switched) {
      RSTG_CUDA(cudaMemcpyAsync(dS, hs.data(), sizeof(JobState) * nj, cudaMemcpyHostToDevice, st));
      sor_residuals(now_sor);  // of the current potential with its boundary values set again
    }
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
    for (auto& m : marks) {
      float t = 0.0f;
      RSTG_CUDA(cudaEventElapsedTime(&t, m.a, m.b));
      if (m.kind >= 0) {
        prof.ms[m.kind] += t;
        prof.bytes[m.kind] += kbytes[m.kind];
        prof.launches[m.kind] += 1;
      }
      prof.detail_ms[m.det][m.lvl] += t;
      prof.detail_n[m.det][m.lvl] += 1;
    }
    marks.clear();
    next_ev = 0;
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
  if (profile && std::getenv("RSTG_PB_DEBUG")) {
    static const char* names[kProfDetail] = {"sweep", "res32", "restrict", "prolong", "coarse",
                                             "res64", "update", "norm",     "sor"};
    for (int d = 0; d < kProfDetail; d++)
      for (int l = 0; l < kProfLevels; l++)
        if (prof.detail_n[d][l])
          std::fprintf(stderr, "pb profile %-8s level %d: %8.2f ms over %lld launches\n", names[d], l,
                       prof.detail_ms[d][l], (long long)prof.detail_n[d][l]);
  }
  auto t2 = now();
  stats.ms_cycles += ms(t1, t2);
  for (int j = 0; j < nj; j++) {
    const JobState& s = hs[j];
    bool sor = s.status == kSorCap || s.sor_it > 0;
    jobs[j].fallback = sor;
    if (sor) stats.fallbacks++;
    double res = jobs[j].rtol > 0.0 ? (s.r0 > 0.0 ? s.rms / s.r0 : 0.0) : s.rms;  // relative in that mode
    jobs[j].stats = PbSolveStats{sor ? (int64_t)s.sor_it : (int64_t)s.cycles, res, s.status == kConverged};
  }
  for (int j = 0; j < nj; j++) {  // the energy kernels read JobD::phi: point it at the current buffer
    phi_now[j] = hs[j].cur ? hd[j].phi2 : hd[j].phi;
    hd[j].phi = phi_now[j];
  }
  RSTG_CUDA(cudaMemcpyAsync(dJ, hd.data(), sizeof(JobD) * nj, cudaMemcpyHostToDevice, st));
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
        RSTG_CUDA(cudaMemcpyAsync((*phi_out)[j], phi_now[j], jobs[j].g.n() * 8, cudaMemcpyDeviceToDevice, st));
  RSTG_CUDA(cudaStreamSynchronize(st));
  for (int j = 0; j < nj; j++) {
    jobs[j].e = he[j];
    jobs[j].maxabs = he[nj + j];
  }
  stats.ms_finish += ms(t2, now());
}

void pb_polar_batch(Ctx* c, cudaStream_t st, PbBatchEngine& eng, const rstg_pb_params& p,
                    const std::vector<const std::vector<double>*>& xyz, const std::vector<const std::vector<double>*>& q,
                    const std::vector<const std::vector<double>*>& r, double* out, rstg_pb_diag* diag, double rtol) {
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
    J.rtol = rtol;
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
        if (s == 1) J.rho_of = (int)cj.size() - 1;  // same grid and atoms as the solvated solve
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
      if (s == 1) J.rho_of = (int)fj.size() - 1;  // same grid and atoms as the solvated solve
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
