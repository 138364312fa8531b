// Periodic reimaging of the complex of a boxed trajectory frame
// (reimage_complex, binding.rs:234-308): every bonded component is unwrapped
// by a breadth-first walk of the bond graph (an atom found from its parent
// moves by one box edge along each axis where it sits more than half an edge
// away from the parent's unwrapped position), then every component after the
// first moves by one box edge along each axis where its geometric centre sits
// more than half an edge from the first component's centre.
//
// The walk (visit order, parents, components) depends on the bonds only, so
// it is computed once on the host.  The device form runs one block per frame:
// the walk's levels in order (every atom of a level against its parent on the
// level before, a barrier between levels), then the centres, each summed by
// one thread in visit order as the reference sums them, then the shifts.  The
// FP64 operations and their order are the reference's, so both forms give the
// same bits.
#include <algorithm>
#include <deque>

#include "reimage.hpp"

namespace rstg {

namespace {

// Breadth-first forest of the bond graph, as the reference walks it: starts
// in atom order, neighbours in the order the bonds list them.
struct Forest {
  std::vector<int32_t> order;       // atoms in visit order, component by component
  std::vector<int32_t> parent;      // per atom: the atom it was found from (-1: a start)
  std::vector<int32_t> level;       // per atom: steps from its component's start
  std::vector<int32_t> comp_start;  // components' ranges in `order`
  std::vector<int32_t> comp_of;     // per atom: its component
};

Forest walk(int64_t n, const Topology& t) {
  std::vector<std::vector<int32_t>> adj(n);
  for (size_t b = 0; b < t.bond_i.size(); b++) {
    const int64_t a = t.bond_i[b], c = t.bond_j[b];
    if (a < n && c < n) {
      adj[a].push_back((int32_t)c);
      adj[c].push_back((int32_t)a);
    }
  }
  Forest w;
  w.parent.assign(n, -1);
  w.level.assign(n, 0);
  w.comp_of.assign(n, 0);
  std::vector<uint8_t> seen(n, 0);
  for (int64_t s = 0; s < n; s++) {
    if (seen[s]) continue;
    const int32_t comp = (int32_t)w.comp_start.size();
    w.comp_start.push_back((int32_t)w.order.size());
    std::deque<int32_t> q{(int32_t)s};
    seen[s] = 1;
    while (!q.empty()) {
      const int32_t cur = q.front();
      q.pop_front();
      w.order.push_back(cur);
      w.comp_of[cur] = comp;
      for (int32_t nb : adj[cur]) {
        if (seen[nb]) continue;
        seen[nb] = 1;
        w.parent[nb] = cur;
        w.level[nb] = w.level[cur] + 1;
        q.push_back(nb);
      }
    }
  }
  w.comp_start.push_back((int32_t)w.order.size());
  return w;
}

// One block per frame; x in topology order, top_of maps complex atoms to
// topology atoms; cen: [F][n_comp][3] scratch.
__global__ void __launch_bounds__(256) k_reimage(int n, long long n_top, const int* __restrict__ top_of,
                                                 const int* __restrict__ parent, const int* __restrict__ lvl_atoms,
                                                 const int* __restrict__ lvl_start, int n_lvl,
                                                 const int* __restrict__ order, const int* __restrict__ comp_start,
                                                 const int* __restrict__ comp_of, int n_comp,
                                                 const double* __restrict__ boxes, double* __restrict__ cen,
                                                 double* x) {
  const long long f = blockIdx.x;
  double* X = x + f * n_top * 3;
  const double b[3] = {boxes[3 * f], boxes[3 * f + 1], boxes[3 * f + 2]};
  const double h[3] = {b[0] * 0.5, b[1] * 0.5, b[2] * 0.5};
  for (int l = 1; l < n_lvl; l++) {  // level 0 holds the starts, which stay
    for (int k = lvl_start[l] + threadIdx.x; k < lvl_start[l + 1]; k += blockDim.x) {
      const int a = lvl_atoms[k];
      double* xa = X + 3LL * top_of[a];
      const double* xp = X + 3LL * top_of[parent[a]];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double diff = xa[d] - xp[d];
        if (diff > h[d])
          xa[d] -= b[d];
        else if (diff < -h[d])
          xa[d] += b[d];
      }
    }
    __syncthreads();  // the next level reads the positions this one wrote
  }
  if (n_comp <= 1) return;
  double* C = cen + f * n_comp * 3;
  for (int t = threadIdx.x; t < 3 * n_comp; t += blockDim.x) {  // geometric centres, visit order
    const int c = t / 3, d = t % 3;
    double s = 0.0;
    for (int k = comp_start[c]; k < comp_start[c + 1]; k++) s += X[3LL * top_of[order[k]] + d];
    C[t] = s / (double)(comp_start[c + 1] - comp_start[c]);
  }
  __syncthreads();
  for (int k = comp_start[1] + threadIdx.x; k < n; k += blockDim.x) {
    const int a = order[k], c = comp_of[a];
    double* xa = X + 3LL * top_of[a];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const double diff = C[3 * c + d] - C[d];
      const double sh = diff > h[d] ? -b[d] : (diff < -h[d] ? b[d] : 0.0);
      xa[d] += sh;
    }
  }
}

}  // namespace

void reimage_host(double* x, int64_t n, const Topology& t, const std::array<double, 3>& box) {
  if (n == 0) return;
  const Forest w = walk(n, t);
  for (int32_t a : w.order) {  // each atom after its parent
    const int32_t p = w.parent[a];
    if (p < 0) continue;
    for (int d = 0; d < 3; d++) {
      const double diff = x[3 * a + d] - x[3 * p + d];
      if (diff > box[d] * 0.5)
        x[3 * a + d] -= box[d];
      else if (diff < -box[d] * 0.5)
        x[3 * a + d] += box[d];
    }
  }
  const size_t nc = w.comp_start.size() - 1;
  if (nc <= 1) return;
  auto centre = [&](size_t c) {
    std::array<double, 3> m{0.0, 0.0, 0.0};
    for (int32_t k = w.comp_start[c]; k < w.comp_start[c + 1]; k++)
      for (int d = 0; d < 3; d++) m[d] += x[3 * w.order[k] + d];
    for (int d = 0; d < 3; d++) m[d] /= (double)(w.comp_start[c + 1] - w.comp_start[c]);
    return m;
  };
  const std::array<double, 3> ref = centre(0);
  for (size_t c = 1; c < nc; c++) {
    const std::array<double, 3> cc = centre(c);
    double sh[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < 3; d++) {
      const double diff = cc[d] - ref[d];
      if (diff > box[d] * 0.5)
        sh[d] = -box[d];
      else if (diff < -box[d] * 0.5)
        sh[d] = box[d];
    }
    for (int32_t k = w.comp_start[c]; k < w.comp_start[c + 1]; k++)
      for (int d = 0; d < 3; d++) x[3 * w.order[k] + d] += sh[d];
  }
}

void reimage_device(Ctx* ctx, cudaStream_t st, const Split& sp, int64_t n_top, double* d_frames,
                    const double* d_boxes, int64_t F) {
  const int64_t n = sp.complex.n_atoms;
  if (n == 0 || F <= 0) return;
  if (n > INT32_MAX / 3 || F > INT32_MAX) throw Error(RSTG_ERR_INVALID, "too many atoms or frames to reimage");
  const Forest w = walk(n, sp.complex);
  const int n_comp = (int)w.comp_start.size() - 1;
  int n_lvl = 0;
  for (int32_t l : w.level) n_lvl = std::max(n_lvl, l + 1);
  std::vector<int32_t> lvl_start(n_lvl + 1, 0), lvl_atoms(n);
  for (int32_t l : w.level) lvl_start[l + 1]++;
  for (int l = 0; l < n_lvl; l++) lvl_start[l + 1] += lvl_start[l];
  std::vector<int32_t> fill(lvl_start.begin(), lvl_start.end() - 1);
  for (int32_t a : w.order) lvl_atoms[fill[w.level[a]]++] = a;
  std::vector<int32_t> top_of(n);
  for (int64_t a = 0; a < n; a++) top_of[a] = (int32_t)(sp.complex_atoms.empty() ? a : sp.complex_atoms[a]);
  // one upload of the plan: top_of, parent, level lists, order, components
  std::vector<int32_t> plan;
  auto put = [&](const std::vector<int32_t>& v) {
    const size_t o = plan.size();
    plan.insert(plan.end(), v.begin(), v.end());
    return o;
  };
  const size_t o_top = put(top_of), o_par = put(w.parent), o_la = put(lvl_atoms), o_ls = put(lvl_start),
               o_ord = put(w.order), o_cs = put(w.comp_start), o_co = put(w.comp_of);
  DevBuf d_plan(plan.size() * sizeof(int32_t), st);
  RSTG_CUDA(cudaMemcpyAsync(d_plan.p, plan.data(), plan.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  DevBuf d_cen(n_comp > 1 ? (size_t)F * n_comp * 3 * sizeof(double) : 8, st);
  const int32_t* P = d_plan.as<int32_t>();
  k_reimage<<<(unsigned)F, 256, 0, st>>>((int)n, (long long)n_top, P + o_top, P + o_par, P + o_la, P + o_ls, n_lvl,
                                        P + o_ord, P + o_cs, P + o_co, n_comp, d_boxes, d_cen.as<double>(), d_frames);
  launched(ctx);
  // the plan's host vectors are read by the copy above before this returns
  RSTG_CUDA(cudaStreamSynchronize(st));
}

}  // namespace rstg
