// Mass-weighted coordinate covariance of the quasi-harmonic entropy
// (crates/mmpbsa/src/entropy.rs:97-160) in FP64 on the GPU.
//
// With x_k the coordinates of one frame (k = 3 atom + axis) and w_k the
// square root of that atom's mass, the reference forms
//   mean_k = (sum over frames in order of x_k w_k) / F
//   d_k    = x_k w_k - mean_k
//   C_ij   = (sum over frames in order of d_i d_j) / F     (i <= j, mirrored)
// with unfused multiplies and adds.  k_qh_center computes mean and d with
// the same roundings (one thread per coordinate, frames in order);
// k_qh_syrk accumulates each C_ij over the frames in order with the same
// unfused operations, so C is bit-identical to the reference's.  C = D^T D
// is a symmetric rank-F update: 64 x 64 output tiles of the upper triangle,
// 16 frames of D staged in shared memory per step, 4 x 4 outputs per thread.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace rstg {

namespace {

constexpr int kQT = 64, kQF = 16;

// traj [F][dim] (dim = 3 n_atoms), w [dim] = sqrt(mass) per coordinate
__global__ void k_qh_center(const double* __restrict__ traj, const double* __restrict__ w, long long F, int dim,
                            double* __restrict__ D) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= dim) return;
  const double wk = w[k];
  double s = 0.0;
  for (long long f = 0; f < F; f++) s = __dadd_rn(s, __dmul_rn(traj[f * dim + k], wk));
  const double mean = __ddiv_rn(s, (double)F);
  for (long long f = 0; f < F; f++) D[f * dim + k] = __dsub_rn(__dmul_rn(traj[f * dim + k], wk), mean);
}

// C[i][j] (row-major dim x dim) for tiles bi <= bj; tile list in blockIdx.x
__global__ void __launch_bounds__(256) k_qh_syrk(const double* __restrict__ D, long long F, int dim,
                                                 const int2* __restrict__ tiles, double* __restrict__ C) {
  __shared__ double sa[kQF][kQT], sb[kQF][kQT];
  const int2 t = tiles[blockIdx.x];
  const int i0 = t.x * kQT, j0 = t.y * kQT;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
  for (long long f0 = 0; f0 < F; f0 += kQF) {
    for (int e = threadIdx.x; e < kQF * kQT; e += blockDim.x) {
      const int r = e / kQT, c = e % kQT;
      const long long f = f0 + r;
      sa[r][c] = (f < F && i0 + c < dim) ? D[f * dim + i0 + c] : 0.0;
      sb[r][c] = (f < F && j0 + c < dim) ? D[f * dim + j0 + c] : 0.0;
    }
    __syncthreads();
    const int nf = (int)min((long long)kQF, F - f0);
    for (int r = 0; r < nf; r++) {
      double a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        a[q] = sa[r][ty + 16 * q];
        b[q] = sb[r][tx + 16 * q];
      }
#pragma unroll
      for (int p = 0; p < 4; p++)
#pragma unroll
        for (int q = 0; q < 4; q++) acc[p][q] = __dadd_rn(acc[p][q], __dmul_rn(a[p], b[q]));
    }
    __syncthreads();
  }
  const double nf = (double)F;
#pragma unroll
  for (int p = 0; p < 4; p++)
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = i0 + ty + 16 * p, j = j0 + tx + 16 * q;
      if (i < dim && j < dim && i <= j) {
        const double v = __ddiv_rn(acc[p][q], nf);
        C[(long long)i * dim + j] = v;
        C[(long long)j * dim + i] = v;
      }
    }
}

}  // namespace

}  // namespace rstg

using namespace rstg;

extern "C" rstg_status rstg_qh_covariance(rstg_ctx* c, const double* traj, int64_t F, int64_t n_atoms,
                                          const double* masses, double* cov) {
  try {
    if (!c || !traj || !masses || !cov) throw Error(RSTG_ERR_INVALID, "ctx, trajectory, masses and out are required");
    if (F < 1 || n_atoms < 1) throw Error(RSTG_ERR_INVALID, "need at least one frame and one atom");
    if (n_atoms > 200000) throw Error(RSTG_ERR_INVALID, "quasi-harmonic covariance is limited to 200,000 atoms");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->bind();
    cudaStream_t st = c->stream;
    const int dim = (int)(3 * n_atoms);
    std::vector<double> w(dim);
    for (int64_t a = 0; a < n_atoms; a++) {
      if (!(masses[a] >= 0.0)) throw Error(RSTG_ERR_INVALID, "masses must be non-negative");
      for (int d = 0; d < 3; d++) w[3 * a + d] = std::sqrt(masses[a]);
    }
    const int nt = (dim + kQT - 1) / kQT;
    std::vector<int2> tiles;
    for (int bi = 0; bi < nt; bi++)
      for (int bj = bi; bj < nt; bj++) tiles.push_back(make_int2(bi, bj));
    DevBuf dT((size_t)F * dim * 8, st), dW((size_t)dim * 8, st), dD((size_t)F * dim * 8, st),
        dC((size_t)dim * dim * 8, st), dTl(tiles.size() * sizeof(int2), st);
    RSTG_CUDA(cudaMemcpyAsync(dT.p, traj, (size_t)F * dim * 8, cudaMemcpyHostToDevice, st));
    RSTG_CUDA(cudaMemcpyAsync(dW.p, w.data(), (size_t)dim * 8, cudaMemcpyHostToDevice, st));
    RSTG_CUDA(cudaMemcpyAsync(dTl.p, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
    k_qh_center<<<(dim + 255) / 256, 256, 0, st>>>(dT.as<double>(), dW.as<double>(), F, dim, dD.as<double>());
    k_qh_syrk<<<(unsigned)tiles.size(), 256, 0, st>>>(dD.as<double>(), F, dim, dTl.as<int2>(), dC.as<double>());
    launched(c, 2);
    RSTG_CUDA(cudaMemcpyAsync(cov, dC.p, (size_t)dim * dim * 8, cudaMemcpyDeviceToHost, st));
    RSTG_CUDA(cudaStreamSynchronize(st));
    return RSTG_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return RSTG_ERR_NOMEM;
  }
}
