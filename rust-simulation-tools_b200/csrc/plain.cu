// Plain FP64 kernels.  Built with -fmad=false: every a*b+c is two rounded
// operations, as in the reference's Rust f64 code.
#include <cmath>

#include "common.cuh"
#include "plain.cuh"

namespace rstg {

static constexpr int kWarpsPerBlock = 8;
static constexpr int kSasaThreads = 128;
static constexpr int kSasaMaxNeighbors = 2048;

std::vector<double> fibonacci_sphere(int64_t n) {
  std::vector<double> v;
  if (n <= 0) return v;
  if (n == 1) return {0.0, 1.0, 0.0};
  double phi = kPi * (3.0 - std::sqrt(5.0));
  for (int64_t i = 0; i < n; i++) {
    double y = 1.0 - ((double)i / (double)(n - 1)) * 2.0;
    double r = std::sqrt(1.0 - y * y);
    double th = phi * (double)i;
    v.push_back(std::cos(th) * r);
    v.push_back(y);
    v.push_back(std::sin(th) * r);
  }
  return v;
}

DevTopo DevTopo::upload(const Topology& t, const PairClasses& pc, cudaStream_t s) {
  DevTopo d;
  d.n = t.n_atoms;
  d.nt = t.n_types;
  d.scee = t.scee;
  d.scnb = t.scnb;
  auto up = [&](DevBuf& b, const void* src, size_t bytes) {
    b = DevBuf(bytes ? bytes : 8, s);
    if (bytes) RSTG_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, s));
  };
  int64_t n = t.n_atoms;
  for (double r : t.radii) d.max_radius = std::max(d.max_radius, r);
  up(d.q, t.charges_amber.data(), n * 8);
  up(d.rad, t.radii.data(), n * 8);
  up(d.scr, t.screen.data(), n * 8);
  std::vector<int32_t> ty(t.type_idx.begin(), t.type_idx.end());
  up(d.type, ty.data(), n * 4);
  // dense LJ tables from NONBONDED_PARM_INDEX (lj_ab, mm_energy.rs:152-161)
  int64_t nt = std::max<int64_t>(t.n_types, 1);
  std::vector<double> A(nt * nt, 0.0), B(nt * nt, 0.0);
  for (int64_t a = 0; a < t.n_types; a++)
    for (int64_t b = 0; b < t.n_types; b++) {
      int64_t idx = t.nb_index[t.n_types * a + b];
      if (idx >= 1) {
        A[a * nt + b] = t.lj_a[idx - 1];
        B[a * nt + b] = t.lj_b[idx - 1];
      }
    }
  d.nt = nt;
  up(d.ljA, A.data(), A.size() * 8);
  up(d.ljB, B.data(), B.size() * 8);
  up(d.excl, pc.excl_bits.data(), pc.excl_bits.size() * 8);
  up(d.p14, pc.p14_bits.data(), pc.p14_bits.size() * 8);
  std::vector<int32_t> bi;
  std::vector<double> bp;
  for (size_t k = 0; k < t.bond_i.size(); k++) {
    bi.push_back((int32_t)t.bond_i[k]);
    bi.push_back((int32_t)t.bond_j[k]);
    bp.push_back(t.bond_k[t.bond_t[k]]);
    bp.push_back(t.bond_req[t.bond_t[k]]);
  }
  d.nb = t.bond_i.size();
  up(d.bidx, bi.data(), bi.size() * 4);
  up(d.bpar, bp.data(), bp.size() * 8);
  std::vector<int32_t> ai;
  std::vector<double> ap;
  for (size_t k = 0; k < t.ang_i.size(); k++) {
    ai.push_back((int32_t)t.ang_i[k]);
    ai.push_back((int32_t)t.ang_j[k]);
    ai.push_back((int32_t)t.ang_k[k]);
    ap.push_back(t.angle_k[t.ang_t[k]]);
    ap.push_back(t.angle_teq[t.ang_t[k]]);
  }
  d.na = t.ang_i.size();
  up(d.aidx, ai.data(), ai.size() * 4);
  up(d.apar, ap.data(), ap.size() * 8);
  std::vector<int32_t> di;
  std::vector<double> dp;
  for (size_t k = 0; k < t.dih_i.size(); k++) {
    di.push_back((int32_t)t.dih_i[k]);
    di.push_back((int32_t)t.dih_j[k]);
    di.push_back((int32_t)t.dih_k[k]);
    di.push_back((int32_t)t.dih_l[k]);
    dp.push_back(t.dih_pk[t.dih_t[k]]);
    dp.push_back(t.dih_pn[t.dih_t[k]]);
    dp.push_back(t.dih_phase[t.dih_t[k]]);
  }
  d.nd = t.dih_i.size();
  up(d.didx, di.data(), di.size() * 4);
  up(d.dpar, dp.data(), dp.size() * 8);
  return d;
}

// ---------------------------------------------------------------------------
// Born radii, gb_energy.rs:144-258: one warp per atom i, lanes stride j.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double hct_term64(double r2, double rho_i, double sj, bool& used) {
  double r = sqrt(r2);
  used = false;
  if (r == 0.0) return 0.0;
  if (rho_i >= r + sj) return 0.0;
  double u = r + sj;
  double l = (rho_i > fabs(r - sj)) ? rho_i : fabs(r - sj);
  double l_inv = 1.0 / l, u_inv = 1.0 / u;
  double contrib = 0.5 * (l_inv - u_inv + 0.25 * (u_inv * u_inv - l_inv * l_inv) * (r - sj * sj / r) +
                          log(l / u) / (2.0 * r));
  used = true;
  if (rho_i < sj - r) return contrib + 2.0 * (1.0 / rho_i - l_inv);
  return contrib;
}

__device__ __forceinline__ double radius_from_psi64(double psi, double rho_i, double radius_i, int model,
                                                    double rgbmax) {
  double alpha = 1.0, beta = 0.0, gamma = 0.0;
  if (model == 1) {
    alpha = 0.8;
    gamma = 2.909125;
  } else if (model == 2) {
    alpha = 1.0;
    beta = 0.8;
    gamma = 4.85;
  }
  double R;
  if (model == 0) {
    double inv_r = 1.0 / rho_i - psi;
    R = inv_r > 0.0 ? 1.0 / inv_r : rgbmax;
  } else {
    double pr = psi * rho_i, p2 = pr * pr, p3 = p2 * pr;
    double tv = tanh(alpha * pr - beta * p2 + gamma * p3);
    double inv_r = 1.0 / rho_i - tv / radius_i;
    R = inv_r > 0.0 ? 1.0 / inv_r : rgbmax;
  }
  if (R > rgbmax) R = rgbmax;
  return R;
}

__global__ void k_born_radii_plain(int n, const double* __restrict__ xyz, const double* __restrict__ rad,
                                   const double* __restrict__ scr, double offset, double cut2, int model,
                                   double rgbmax, double* __restrict__ R) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  int i = warp;
  double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2];
  double rho_i = rad[i] - offset, psi = 0.0;
  for (int j = lane; j < n; j += 32) {
    if (j == i) continue;
    double dx = xi - xyz[3 * j], dy = yi - xyz[3 * j + 1], dz = zi - xyz[3 * j + 2];
    double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 > cut2) continue;
    double sj = scr[j] * (rad[j] - offset);
    bool used;
    double t = hct_term64(r2, rho_i, sj, used);
    if (used) psi += t;
  }
  psi = warp_sum(psi);
  if (lane == 0) R[i] = radius_from_psi64(psi, rho_i, rad[i], model, rgbmax);
}

void plain_born_radii(Ctx* c, const DevTopo& t, const double* d_xyz, const rstg_gb_params& p, double* d_R) {
  if (t.n == 0) return;
  int threads = 32 * kWarpsPerBlock;
  int blocks = (int)((t.n + kWarpsPerBlock - 1) / kWarpsPerBlock);
  k_born_radii_plain<<<blocks, threads, 0, c->stream>>>((int)t.n, d_xyz, t.rad.as<double>(), t.scr.as<double>(),
                                                         p.offset, p.cutoff * p.cutoff, p.model, p.rgbmax, d_R);
  launched(c);
}

// ---------------------------------------------------------------------------
// GB energy from radii, gb_energy.rs:283-355.  Warp w handles rows w and
// n-1-w (balanced triangle); per-warp partials are summed in fixed order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double gb_pair64(double qi, double qj, double r2, double Ri, double Rj, const GbConst& k) {
  double rr = Ri * Rj;
  double f = sqrt(r2 + rr * exp(-r2 / (4.0 * rr)));
  if (k.no_salt) return k.diel_ns * qi * qj / f;
  return -0.5 * qi * qj * (k.inv_ein - exp(-kKScale * k.kappa * f) * k.inv_eout) / f;
}
__device__ __forceinline__ double gb_self64(double qi, double Ri, const GbConst& k) {
  if (k.no_salt) return k.diel_ns * qi * qi / Ri;
  return -0.5 * qi * qi * (k.inv_ein - exp(-kKScale * k.kappa * Ri) * k.inv_eout) / Ri;
}

__global__ void k_gb_plain(int n, const double* __restrict__ xyz, const double* __restrict__ q,
                           const double* __restrict__ R, GbConst k, double* __restrict__ part) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  int nw = (n + 1) / 2;
  if (warp >= nw) return;
  double acc = 0.0;
  for (int side = 0; side < 2; side++) {
    int i = side == 0 ? warp : n - 1 - warp;
    if (side == 1 && i == warp) break;
    double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2], qi = q[i], Ri = R[i];
    if (lane == 0) acc += gb_self64(qi, Ri, k);
    for (int j = i + 1 + lane; j < n; j += 32) {
      double dx = xi - xyz[3 * j], dy = yi - xyz[3 * j + 1], dz = zi - xyz[3 * j + 2];
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > k.cut2) continue;
      acc += 2.0 * gb_pair64(qi, q[j], r2, Ri, R[j], k);
    }
  }
  acc = warp_sum(acc);
  if (lane == 0) part[warp] = acc;
}

GbConst gb_const(const rstg_gb_params& p) {
  GbConst k;
  double s = p.salt_concentration;
  k.kappa = s <= 0.0 ? 0.0
                     : std::sqrt(8.0 * kPi * 332.0522 * 6.022e-4 * s / (p.solvent_dielectric * 0.00198688 * p.temperature));
  k.inv_ein = 1.0 / p.solute_dielectric;
  k.inv_eout = 1.0 / p.solvent_dielectric;
  k.diel_ns = -0.5 * (k.inv_ein - k.inv_eout);
  k.no_salt = k.kappa <= 0.0;
  k.cut2 = p.cutoff * p.cutoff;
  return k;
}

void plain_gb_energy(Ctx* c, const DevTopo& t, const double* d_xyz, const rstg_gb_params& p, const double* d_R,
                     double* d_out) {
  if (t.n == 0) {
    RSTG_CUDA(cudaMemsetAsync(d_out, 0, 8, c->stream));
    return;
  }
  int64_t nw = (t.n + 1) / 2;
  DevBuf part(nw * 8, c->stream);
  int threads = 32 * kWarpsPerBlock;
  int blocks = (int)((nw + kWarpsPerBlock - 1) / kWarpsPerBlock);
  k_gb_plain<<<blocks, threads, 0, c->stream>>>((int)t.n, d_xyz, t.q.as<double>(), d_R, gb_const(p),
                                                 part.as<double>());
  launched(c);
  sum_columns(c, part.as<double>(), nw, 1, d_out);
}

// ---------------------------------------------------------------------------
// MM energy, mm_energy.rs:179-267: bonded terms one thread each, non-bonded
// over i<j with the triangular 1-4 / exclusion bitmaps (1-4 tested first).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool bit_of(const unsigned long long* b, long long i, long long j) {
  unsigned long long k = (unsigned long long)j * (j - 1) / 2 + i;
  return (b[k >> 6] >> (k & 63)) & 1ull;
}

__global__ void k_nb_plain(int n, const double* __restrict__ xyz, const double* __restrict__ q,
                           const int* __restrict__ type, int nt, const double* __restrict__ A,
                           const double* __restrict__ B, const unsigned long long* __restrict__ excl,
                           const unsigned long long* __restrict__ p14, double scee, double scnb,
                           double* __restrict__ part) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  int nw = (n + 1) / 2;
  if (warp >= nw) return;
  double vdw = 0, elec = 0, v14 = 0, e14 = 0;
  for (int side = 0; side < 2; side++) {
    int i = side == 0 ? warp : n - 1 - warp;
    if (side == 1 && i == warp) break;
    double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2], qi = q[i];
    int ti = type[i];
    for (int j = i + 1 + lane; j < n; j += 32) {
      double dx = xi - xyz[3 * j], dy = yi - xyz[3 * j + 1], dz = zi - xyz[3 * j + 2];
      double r2 = dx * dx + dy * dy + dz * dz;
      bool is14 = bit_of(p14, i, j);
      if (!is14 && bit_of(excl, i, j)) continue;
      double r = sqrt(r2), r6 = r2 * r2 * r2, r12 = r6 * r6;
      int tj = type[j];
      double a = A[ti * nt + tj], b = B[ti * nt + tj];
      if (is14) {
        v14 += (a / r12 - b / r6) / scnb;
        e14 += qi * q[j] / r / scee;
      } else {
        vdw += a / r12 - b / r6;
        elec += qi * q[j] / r;
      }
    }
  }
  vdw = warp_sum(vdw);
  elec = warp_sum(elec);
  v14 = warp_sum(v14);
  e14 = warp_sum(e14);
  if (lane == 0) {
    part[4 * warp] = vdw;
    part[4 * warp + 1] = elec;
    part[4 * warp + 2] = v14;
    part[4 * warp + 3] = e14;
  }
}

__device__ __forceinline__ void cross3(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// Bonded terms, mm_energy.rs:97-149,187-212; part[blk][3].
__global__ void k_bonded_plain(const double* __restrict__ x, int nb, const int* __restrict__ bi,
                               const double* __restrict__ bp, int na, const int* __restrict__ ai,
                               const double* __restrict__ ap, int nd, const int* __restrict__ di,
                               const double* __restrict__ dp, double* __restrict__ part) {
  __shared__ double sh[32];
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  double eb = 0, ea = 0, ed = 0;
  if (t < nb) {
    int i = bi[2 * t], j = bi[2 * t + 1];
    double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1], dz = x[3 * i + 2] - x[3 * j + 2];
    double r = sqrt(dx * dx + dy * dy + dz * dz), k = bp[2 * t], req = bp[2 * t + 1];
    eb = k * (r - req) * (r - req);
  }
  if (t < na) {
    int i = ai[3 * t], j = ai[3 * t + 1], k = ai[3 * t + 2];
    double ba[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
    double bc[3] = {x[3 * k] - x[3 * j], x[3 * k + 1] - x[3 * j + 1], x[3 * k + 2] - x[3 * j + 2]};
    double dot = ba[0] * bc[0] + ba[1] * bc[1] + ba[2] * bc[2];
    double m1 = sqrt(ba[0] * ba[0] + ba[1] * ba[1] + ba[2] * ba[2]);
    double m2 = sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]);
    double cs = fmin(1.0, fmax(-1.0, dot / (m1 * m2)));
    double th = acos(cs), ka = ap[2 * t], teq = ap[2 * t + 1];
    ea = ka * (th - teq) * (th - teq);
  }
  if (t < nd) {
    int a = di[4 * t], b = di[4 * t + 1], c = di[4 * t + 2], d = di[4 * t + 3];
    double b1[3] = {x[3 * b] - x[3 * a], x[3 * b + 1] - x[3 * a + 1], x[3 * b + 2] - x[3 * a + 2]};
    double b2[3] = {x[3 * c] - x[3 * b], x[3 * c + 1] - x[3 * b + 1], x[3 * c + 2] - x[3 * b + 2]};
    double b3[3] = {x[3 * d] - x[3 * c], x[3 * d + 1] - x[3 * c + 1], x[3 * d + 2] - x[3 * c + 2]};
    double n1[3], n2[3], m1[3], u[3] = {0, 0, 0};
    cross3(b1, b2, n1);
    cross3(b2, b3, n2);
    double len = sqrt(b2[0] * b2[0] + b2[1] * b2[1] + b2[2] * b2[2]);
    if (!(len < 1e-20)) {
      u[0] = b2[0] / len;
      u[1] = b2[1] / len;
      u[2] = b2[2] / len;
    }
    cross3(n1, u, m1);
    double xx = n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2];
    double yy = m1[0] * n2[0] + m1[1] * n2[1] + m1[2] * n2[2];
    double phi = atan2(-yy, xx);
    ed = dp[3 * t] * (1.0 + cos(dp[3 * t + 1] * phi - dp[3 * t + 2]));
  }
  eb = block_sum(eb, sh);
  ea = block_sum(ea, sh);
  ed = block_sum(ed, sh);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x] = eb;
    part[3 * blockIdx.x + 1] = ea;
    part[3 * blockIdx.x + 2] = ed;
  }
}

void plain_mm_energy(Ctx* c, const DevTopo& t, const double* d_xyz, double* d_out) {
  RSTG_CUDA(cudaMemsetAsync(d_out, 0, 7 * 8, c->stream));
  int64_t m = std::max(t.nb, std::max(t.na, t.nd));
  if (m > 0) {
    int blocks = (int)((m + 255) / 256);
    DevBuf part(blocks * 3 * 8, c->stream);
    k_bonded_plain<<<blocks, 256, 0, c->stream>>>(d_xyz, (int)t.nb, t.bidx.as<int>(), t.bpar.as<double>(),
                                                   (int)t.na, t.aidx.as<int>(), t.apar.as<double>(), (int)t.nd,
                                                   t.didx.as<int>(), t.dpar.as<double>(), part.as<double>());
    launched(c);
    sum_columns(c, part.as<double>(), blocks, 3, d_out);
  }
  if (t.n >= 2) {
    int64_t nw = (t.n + 1) / 2;
    DevBuf part(nw * 4 * 8, c->stream);
    int threads = 32 * kWarpsPerBlock;
    int blocks = (int)((nw + kWarpsPerBlock - 1) / kWarpsPerBlock);
    k_nb_plain<<<blocks, threads, 0, c->stream>>>((int)t.n, d_xyz, t.q.as<double>(), t.type.as<int>(), (int)t.nt,
                                                   t.ljA.as<double>(), t.ljB.as<double>(),
                                                   t.excl.as<unsigned long long>(), t.p14.as<unsigned long long>(),
                                                   t.scee, t.scnb, part.as<double>());
    launched(c);
    sum_columns(c, part.as<double>(), nw, 4, d_out + 3);
  }
}

// ---------------------------------------------------------------------------
// SASA, core/src/sasa.rs:228-289: one block per atom.  Neighbours are the
// atoms within r_i + probe + max(r) + probe (the reference's KD-tree query
// radius, inclusive); the point test is the reference's exact FP64
// expression, so counts match bit for bit.
// ---------------------------------------------------------------------------
__global__ void k_sasa_plain(int n, const double* __restrict__ xyz, const double* __restrict__ rad, double probe,
                             double max_ext, int npts, const double* __restrict__ sphere,
                             double* __restrict__ per_atom, int* __restrict__ overflow) {
  __shared__ int nb[kSasaMaxNeighbors];
  __shared__ int cnt;
  __shared__ int wsum[kSasaThreads / 32];
  int i = blockIdx.x;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2];
  double er = rad[i] + probe, search = er + max_ext, s2 = search * search;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    if (j == i) continue;
    double dx = xyz[3 * j] - xi, dy = xyz[3 * j + 1] - yi, dz = xyz[3 * j + 2] - zi;
    if (dx * dx + dy * dy + dz * dz <= s2) {
      int k = atomicAdd(&cnt, 1);
      if (k < kSasaMaxNeighbors) nb[k] = j;
    }
  }
  __syncthreads();
  int m = cnt;
  if (m > kSasaMaxNeighbors) {
    if (threadIdx.x == 0) atomicExch(overflow, 1);
    m = kSasaMaxNeighbors;
  }
  int acc = 0;
  for (int p = threadIdx.x; p < npts; p += blockDim.x) {
    double tx = xi + sphere[3 * p] * er, ty = yi + sphere[3 * p + 1] * er, tz = zi + sphere[3 * p + 2] * er;
    bool ok = true;
    for (int k = 0; k < m && ok; k++) {
      int j = nb[k];
      double oer = rad[j] + probe;
      double dx = tx - xyz[3 * j], dy = ty - xyz[3 * j + 1], dz = tz - xyz[3 * j + 2];
      double d2 = dx * dx + dy * dy + dz * dz;
      ok = d2 > oer * oer;
    }
    acc += ok ? 1 : 0;
  }
  acc = warp_sumi(acc);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    int total = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) total += wsum[w];
    double frac = (double)total / (double)npts;
    double area = 4.0 * kPi * (er * er);
    per_atom[i] = frac * area;
  }
}

void plain_sasa(Ctx* c, const DevTopo& t, const double* d_xyz, double probe, int64_t n_points,
                const double* d_sphere, double* d_per_atom, double* d_total, int* d_overflow) {
  if (t.n == 0) {
    RSTG_CUDA(cudaMemsetAsync(d_total, 0, 8, c->stream));
    return;
  }
  k_sasa_plain<<<(unsigned)t.n, kSasaThreads, 0, c->stream>>>((int)t.n, d_xyz, t.rad.as<double>(), probe,
                                                               t.max_radius + probe, (int)n_points, d_sphere,
                                                               d_per_atom, d_overflow);
  launched(c);
  sum_columns(c, d_per_atom, t.n, 1, d_total);
}

// ---------------------------------------------------------------------------
// Decomposition pair loop, decomposition.rs:240-283 (note r2 = r*r there).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void decomp_pair64(const double* __restrict__ xyz, const double* __restrict__ q,
                                              const int* __restrict__ type, int nt, const double* __restrict__ A,
                                              const double* __restrict__ B, const unsigned long long* excl,
                                              const unsigned long long* p14, double scee, double scnb, int ri,
                                              int li, double& v, double& e) {
  v = 0.0;
  e = 0.0;
  int i = ri < li ? ri : li, j = ri < li ? li : ri;
  double dx = xyz[3 * ri] - xyz[3 * li], dy = xyz[3 * ri + 1] - xyz[3 * li + 1], dz = xyz[3 * ri + 2] - xyz[3 * li + 2];
  double r = sqrt(dx * dx + dy * dy + dz * dz);
  if (r < 1e-10) return;
  bool is14 = bit_of(p14, i, j);
  if (!is14 && bit_of(excl, i, j)) return;
  double r2 = r * r, r6 = r2 * r2 * r2, r12 = r6 * r6;
  int k = type[ri] * nt + type[li];
  double a = A[k], b = B[k];
  if (is14) {
    v = (a / r12 - b / r6) / scnb;
    e = q[ri] * q[li] / r / scee;
  } else {
    v = a / r12 - b / r6;
    e = q[ri] * q[li] / r;
  }
}

__global__ void k_decomp_rows(const double* __restrict__ xyz, const double* __restrict__ q, const int* __restrict__ type,
                              int nt, const double* __restrict__ A, const double* __restrict__ B,
                              const unsigned long long* __restrict__ excl, const unsigned long long* __restrict__ p14,
                              double scee, double scnb, const int* __restrict__ rec, int nR,
                              const int* __restrict__ lig, int nL, double* __restrict__ rows) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nR) return;
  double sv = 0.0, se = 0.0;
  for (int b = 0; b < nL; b++) {
    double v, e;
    decomp_pair64(xyz, q, type, nt, A, B, excl, p14, scee, scnb, rec[a], lig[b], v, e);
    sv += v;
    se += e;
  }
  rows[2 * a] = sv;
  rows[2 * a + 1] = se;
}

__global__ void k_decomp_cols(const double* __restrict__ xyz, const double* __restrict__ q, const int* __restrict__ type,
                              int nt, const double* __restrict__ A, const double* __restrict__ B,
                              const unsigned long long* __restrict__ excl, const unsigned long long* __restrict__ p14,
                              double scee, double scnb, const int* __restrict__ rec, int nR,
                              const int* __restrict__ lig, int nL, double* __restrict__ cols) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nL) return;
  double sv = 0.0, se = 0.0;
  for (int a = lane; a < nR; a += 32) {
    double v, e;
    decomp_pair64(xyz, q, type, nt, A, B, excl, p14, scee, scnb, rec[a], lig[warp], v, e);
    sv += v;
    se += e;
  }
  sv = warp_sum(sv);
  se = warp_sum(se);
  if (lane == 0) {
    cols[2 * warp] = sv;
    cols[2 * warp + 1] = se;
  }
}

void plain_decomp_pairs(Ctx* c, const DevTopo& C, const double* d_xyz, const int* d_rec, int nR, const int* d_lig,
                        int nL, double* d_rows, double* d_cols) {
  if (nR > 0) {
    k_decomp_rows<<<(nR + 127) / 128, 128, 0, c->stream>>>(d_xyz, C.q.as<double>(), C.type.as<int>(), (int)C.nt,
                                                           C.ljA.as<double>(), C.ljB.as<double>(),
                                                           C.excl.as<unsigned long long>(),
                                                           C.p14.as<unsigned long long>(), C.scee, C.scnb, d_rec, nR,
                                                           d_lig, nL, d_rows);
    launched(c);
  }
  if (nL > 0) {
    k_decomp_cols<<<(nL + 7) / 8, 256, 0, c->stream>>>(d_xyz, C.q.as<double>(), C.type.as<int>(), (int)C.nt,
                                                       C.ljA.as<double>(), C.ljB.as<double>(),
                                                       C.excl.as<unsigned long long>(), C.p14.as<unsigned long long>(),
                                                       C.scee, C.scnb, d_rec, nR, d_lig, nL, d_cols);
    launched(c);
  }
}

// ---------------------------------------------------------------------------
// Deterministic column sums (one block per column, fixed thread order).
// ---------------------------------------------------------------------------
__global__ void k_sum_columns(const double* __restrict__ in, long long rows, int cols, double* __restrict__ out) {
  __shared__ double sh[32];
  int c = blockIdx.x;
  double s = 0.0;
  for (long long r = threadIdx.x; r < rows; r += blockDim.x) s += in[r * cols + c];
  s = block_sum(s, sh);
  if (threadIdx.x == 0) out[c] = s;
}

void sum_columns(Ctx* c, const double* d_in, int64_t rows, int cols, double* d_out) {
  k_sum_columns<<<cols, 512, 0, c->stream>>>(d_in, rows, cols, d_out);
  launched(c);
}

}  // namespace rstg
