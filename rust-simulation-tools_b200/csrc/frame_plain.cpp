// Plain FP64 binding frame and decomposition on the GPU.
#include "frame_plain.hpp"

#include <cmath>
#include <unordered_map>

namespace rstg {

PlainFrameEval::PlainFrameEval(Ctx* c, const Topology& t, const std::vector<int64_t>& rres,
                               const std::vector<int64_t>& lres, const rstg_solvation& sv, const rstg_sa_params& s)
    : split(Split::make(t, rres, lres)), solv(sv), sa(s), ctx(c) {
  if (sa.n_sphere_points < 1) throw Error(RSTG_ERR_INVALID, "n_sphere_points must be >= 1");
  sub[0].top = split.complex;
  sub[1].top = split.rec;
  sub[2].top = split.lig;
  cudaStream_t st = c->stream;
  for (int k = 0; k < 3; k++) {
    sub[k].pc = PairClasses::build(sub[k].top);
    sub[k].dev = DevTopo::upload(sub[k].top, sub[k].pc, st);
    xyz[k] = DevBuf(std::max<int64_t>(sub[k].top.n_atoms, 1) * 24, st);
  }
  auto sp = fibonacci_sphere(sa.n_sphere_points);
  n_sphere = sa.n_sphere_points;
  sphere = DevBuf(sp.size() * 8, st);
  RSTG_CUDA(cudaMemcpyAsync(sphere.p, sp.data(), sp.size() * 8, cudaMemcpyHostToDevice, st));
  int64_t nc = std::max<int64_t>(split.complex.n_atoms, 1);
  born = DevBuf(nc * 8, st);
  per_atom = DevBuf(nc * 8, st);
  out = DevBuf(3 * 12 * 8, st);
  overflow = DevBuf(8, st);
  std::vector<int32_t> ri(split.rec_atoms.begin(), split.rec_atoms.end()),
      li(split.lig_atoms.begin(), split.lig_atoms.end());
  rec_idx = DevBuf(std::max<size_t>(ri.size(), 1) * 4, st);
  lig_idx = DevBuf(std::max<size_t>(li.size(), 1) * 4, st);
  if (!ri.empty()) RSTG_CUDA(cudaMemcpyAsync(rec_idx.p, ri.data(), ri.size() * 4, cudaMemcpyHostToDevice, st));
  if (!li.empty()) RSTG_CUDA(cudaMemcpyAsync(lig_idx.p, li.data(), li.size() * 4, cudaMemcpyHostToDevice, st));
  RSTG_CUDA(cudaStreamSynchronize(st));
}

static std::vector<double> gather3(const double* x, const std::vector<int64_t>& idx) {
  std::vector<double> o(idx.size() * 3);
  for (size_t k = 0; k < idx.size(); k++)
    for (int d = 0; d < 3; d++) o[3 * k + d] = x[3 * idx[k] + d];
  return o;
}

rstg_frame_energy PlainFrameEval::run(const double* xc) {
  cudaStream_t st = ctx->stream;
  int64_t nc = split.complex.n_atoms;
  std::vector<double> hx[3];
  hx[0].assign(xc, xc + nc * 3);
  hx[1] = gather3(xc, split.rec_atoms);
  hx[2] = gather3(xc, split.lig_atoms);
  for (int k = 0; k < 3; k++)
    if (!hx[k].empty())
      RSTG_CUDA(cudaMemcpyAsync(xyz[k].p, hx[k].data(), hx[k].size() * 8, cudaMemcpyHostToDevice, st));
  RSTG_CUDA(cudaMemsetAsync(overflow.p, 0, 8, st));
  RSTG_CUDA(cudaMemsetAsync(out.p, 0, 36 * 8, st));
  double* o = out.as<double>();
  for (int k = 0; k < 3; k++) {
    const DevTopo& d = sub[k].dev;
    plain_mm_energy(ctx, d, xyz[k].as<double>(), o + 12 * k);
    if (solv.method == 0 && d.n > 0) {
      plain_born_radii(ctx, d, xyz[k].as<double>(), solv.gb, born.as<double>());
      plain_gb_energy(ctx, d, xyz[k].as<double>(), solv.gb, born.as<double>(), o + 12 * k + 7);
    }
    plain_sasa(ctx, d, xyz[k].as<double>(), sa.probe_radius, n_sphere, sphere.as<double>(), per_atom.as<double>(),
               o + 12 * k + 8, overflow.as<int>());
  }
  double h[36];
  int ov = 0;
  RSTG_CUDA(cudaMemcpyAsync(h, out.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  RSTG_CUDA(cudaMemcpyAsync(&ov, overflow.p, 4, cudaMemcpyDeviceToHost, st));
  RSTG_CUDA(cudaStreamSynchronize(st));
  if (ov) throw Error(RSTG_ERR_INVALID, "SASA neighbour list exceeded its capacity (2048)");
  rstg_subsystem_energy e[3];
  for (int k = 0; k < 3; k++) {
    const double* v = h + 12 * k;
    e[k].mm = v[0] + v[1] + v[2] + v[3] + v[4] + v[5] + v[6];
    if (solv.method == 0) {
      e[k].polar = v[7];
    } else {
      const Topology& t = sub[k].top;
      e[k].polar = t.n_atoms ? pb_energy_run(ctx, hx[k], t.charges, t.radii, solv.pb, nullptr, pb_rel_tol) : 0.0;
    }
    e[k].sa = sa.surface_tension * v[8] + sa.offset;
  }
  rstg_frame_energy f;
  f.complex = e[0];
  f.receptor = e[1];
  f.ligand = e[2];
  f.delta_mm = e[0].mm - e[1].mm - e[2].mm;
  f.delta_polar = e[0].polar - e[1].polar - e[2].polar;
  f.delta_sa = e[0].sa - e[1].sa - e[2].sa;
  f.delta_total = f.delta_mm + f.delta_polar + f.delta_sa;
  return f;
}

void PlainFrameEval::decompose(const double* xc, const rstg_gb_params& gb, rstg_residue_energy* rec_out,
                               rstg_residue_energy* lig_out) {
  cudaStream_t st = ctx->stream;
  int64_t nc = split.complex.n_atoms, nr = split.rec_atoms.size(), nl = split.lig_atoms.size();
  std::vector<double> hx[3];
  hx[0].assign(xc, xc + nc * 3);
  hx[1] = gather3(xc, split.rec_atoms);
  hx[2] = gather3(xc, split.lig_atoms);
  for (int k = 0; k < 3; k++)
    if (!hx[k].empty())
      RSTG_CUDA(cudaMemcpyAsync(xyz[k].p, hx[k].data(), hx[k].size() * 8, cudaMemcpyHostToDevice, st));
  DevBuf rows(std::max<int64_t>(nr, 1) * 16, st), cols(std::max<int64_t>(nl, 1) * 16, st);
  plain_decomp_pairs(ctx, sub[0].dev, xyz[0].as<double>(), rec_idx.as<int>(), (int)nr, lig_idx.as<int>(), (int)nl,
                     rows.as<double>(), cols.as<double>());
  // GB and SA of the three systems (decomposition.rs:295-307, 355-363)
  DevBuf R[3], S[3], tot(3 * 2 * 8, st);
  RSTG_CUDA(cudaMemsetAsync(tot.p, 0, 48, st));
  RSTG_CUDA(cudaMemsetAsync(overflow.p, 0, 8, st));
  for (int k = 0; k < 3; k++) {
    const DevTopo& d = sub[k].dev;
    R[k] = DevBuf(std::max<int64_t>(d.n, 1) * 8, st);
    S[k] = DevBuf(std::max<int64_t>(d.n, 1) * 8, st);
    if (d.n == 0) continue;
    plain_born_radii(ctx, d, xyz[k].as<double>(), gb, R[k].as<double>());
    plain_gb_energy(ctx, d, xyz[k].as<double>(), gb, R[k].as<double>(), tot.as<double>() + 2 * k);
    plain_sasa(ctx, d, xyz[k].as<double>(), sa.probe_radius, n_sphere, sphere.as<double>(), S[k].as<double>(),
               tot.as<double>() + 2 * k + 1, overflow.as<int>());
  }
  std::vector<double> hr(2 * nr), hc(2 * nl), ht(6), hR[3], hS[3];
  for (int k = 0; k < 3; k++) {
    int64_t n = sub[k].dev.n;
    hR[k].resize(n);
    hS[k].resize(n);
    if (n) {
      RSTG_CUDA(cudaMemcpyAsync(hR[k].data(), R[k].p, n * 8, cudaMemcpyDeviceToHost, st));
      RSTG_CUDA(cudaMemcpyAsync(hS[k].data(), S[k].p, n * 8, cudaMemcpyDeviceToHost, st));
    }
  }
  if (nr) RSTG_CUDA(cudaMemcpyAsync(hr.data(), rows.p, nr * 16, cudaMemcpyDeviceToHost, st));
  if (nl) RSTG_CUDA(cudaMemcpyAsync(hc.data(), cols.p, nl * 16, cudaMemcpyDeviceToHost, st));
  RSTG_CUDA(cudaMemcpyAsync(ht.data(), tot.p, 48, cudaMemcpyDeviceToHost, st));
  int ov = 0;
  RSTG_CUDA(cudaMemcpyAsync(&ov, overflow.p, 4, cudaMemcpyDeviceToHost, st));
  RSTG_CUDA(cudaStreamSynchronize(st));
  if (ov) throw Error(RSTG_ERR_INVALID, "SASA neighbour list exceeded its capacity (2048)");
  const Topology& C = split.complex;
  auto ar = C.atom_residue_indices();
  std::unordered_map<int64_t, rstg_residue_energy> res;
  auto at = [&](int64_t r) -> rstg_residue_energy& {
    auto it = res.find(r);
    if (it == res.end()) it = res.emplace(r, rstg_residue_energy{0, 0, 0, 0}).first;
    return it->second;
  };
  for (int64_t a = 0; a < nr; a++) {
    auto& e = at(ar[split.rec_atoms[a]]);
    e.vdw += hr[2 * a] * 0.5;
    e.elec += hr[2 * a + 1] * 0.5;
  }
  for (int64_t b = 0; b < nl; b++) {
    auto& e = at(ar[split.lig_atoms[b]]);
    e.vdw += hc[2 * b] * 0.5;
    e.elec += hc[2 * b + 1] * 0.5;
  }
  double dgb = ht[0] - ht[2] - ht[4];
  double f0 = -0.5 * (1.0 / gb.solute_dielectric - 1.0 / gb.solvent_dielectric);
  std::vector<double> w;
  double tw = 0.0;
  for (int side = 1; side <= 2; side++) {
    const auto& atoms = side == 1 ? split.rec_atoms : split.lig_atoms;
    for (size_t k = 0; k < atoms.size(); k++) {
      double q = C.charges_amber[atoms[k]];
      double a = f0 * q * q / hR[0][atoms[k]], b = f0 * q * q / hR[side][k];
      w.push_back(std::fabs(a - b));
      tw += w.back();
    }
  }
  if (tw > 1e-20) {
    size_t k = 0;
    for (int side = 1; side <= 2; side++)
      for (int64_t a : (side == 1 ? split.rec_atoms : split.lig_atoms)) at(ar[a]).polar += dgb * (w[k++] / tw);
  }
  for (int side = 1; side <= 2; side++) {
    const auto& atoms = side == 1 ? split.rec_atoms : split.lig_atoms;
    for (size_t k = 0; k < atoms.size(); k++)
      at(ar[atoms[k]]).sa += sa.surface_tension * (hS[0][atoms[k]] - hS[side][k]);
  }
  for (size_t k = 0; k < split.rec_res.size(); k++) rec_out[k] = at(split.rec_res[k]);
  for (size_t k = 0; k < split.lig_res.size(); k++) lig_out[k] = at(split.lig_res[k]);
}

}  // namespace rstg
