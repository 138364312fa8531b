// extern "C" surface: batched systems and the trajectory workflow.
#include <array>
#include <cmath>
#include <cstring>
#include <deque>
#include <memory>

#include "internal.hpp"
#include "system.hpp"
#include "reimage.hpp"
#include "trajectory.hpp"

namespace rstg {

template <class F>
static rstg_status guard(F&& f) {
  try {
    f();
    return RSTG_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return RSTG_ERR_NOMEM;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return RSTG_ERR_INVALID;
  }
}

static std::vector<int64_t> vec(const int64_t* p, int64_t n) {
  if (n < 0) throw Error(RSTG_ERR_INVALID, "negative length");
  if (n > 0 && !p) throw Error(RSTG_ERR_INVALID, "null array with non-zero length");
  return std::vector<int64_t>(p, p + n);
}

}  // namespace rstg

using namespace rstg;

extern "C" {

void rstg_system_opts_default(rstg_system_opts* o) {
  o->mode = RSTG_MODE_FUSED;
  o->decompose = 0;
  o->max_batch_frames = 0;
  o->use_graphs = 1;
  o->autotune = 1;
}

rstg_status rstg_system_create(rstg_ctx* c, const rstg_topology* t, const int64_t* rr, int64_t nr, const int64_t* lr,
                               int64_t nl, const rstg_solvation* solv, const rstg_sa_params* sa,
                               const rstg_system_opts* opts, rstg_system** out) {
  return guard([&] {
    if (!c || !t || !out) throw Error(RSTG_ERR_INVALID, "ctx, topology and out must not be NULL");
    rstg_solvation s;
    if (solv) {
      s = *solv;
    } else {
      s.method = 0;
      rstg_gb_params_default(&s.gb);
      rstg_pb_params_default(&s.pb);
    }
    if (s.method != 0 && s.method != 1) throw Error(RSTG_ERR_INVALID, "unknown solvation method");
    if (s.method == 0 && (s.gb.model < 0 || s.gb.model > 2)) throw Error(RSTG_ERR_INVALID, "unknown GB model");
    rstg_sa_params sp;
    if (sa)
      sp = *sa;
    else
      rstg_sa_params_default(&sp);
    rstg_system_opts o;
    if (opts)
      o = *opts;
    else
      rstg_system_opts_default(&o);
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->bind();
    *out = new rstg_system(c, *t, vec(rr, nr), vec(lr, nl), s, sp, o);
  });
}

void rstg_system_destroy(rstg_system* s) {
  if (!s) return;
  s->ctx->bind();
  cudaStreamSynchronize(s->stream());
  delete s;
}

rstg_status rstg_system_shape(const rstg_system* s, int64_t* sh) {
  return guard([&] {
    if (!s || !sh) throw Error(RSTG_ERR_INVALID, "system and out must not be NULL");
    sh[0] = s->nC;
    sh[1] = s->nR;
    sh[2] = s->nL;
    sh[3] = s->n_res_rec;
    sh[4] = s->n_res_lig;
    sh[5] = s->n_top;
  });
}

int64_t rstg_system_footprint(const rstg_system* s, int64_t n) { return s ? s->footprint(n) : 0; }

rstg_status rstg_system_run(rstg_system* s, const float* frames, int64_t F, rstg_frame_energy* out,
                            rstg_residue_energy* decomp) {
  return guard([&] {
    if (!s || !out || (F > 0 && !frames)) throw Error(RSTG_ERR_INVALID, "system, frames and out must not be NULL");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    s->ctx->bind();
    s->run(frames, false, true, F, out, true, decomp);
  });
}

rstg_status rstg_system_run_device(rstg_system* s, const float* d_frames, int64_t F, rstg_frame_energy* d_out,
                                   rstg_residue_energy* d_decomp) {
  return guard([&] {
    if (!s || !d_out || (F > 0 && !d_frames))
      throw Error(RSTG_ERR_INVALID, "system, frames and out must not be NULL");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    s->ctx->bind();
    s->run(d_frames, false, false, F, d_out, false, d_decomp);
  });
}

rstg_status rstg_system_last_stats(const rstg_system* s, int64_t* st) {
  return guard([&] {
    if (!s || !st) throw Error(RSTG_ERR_INVALID, "system and out must not be NULL");
    memcpy(st, s->last_stats, sizeof(s->last_stats));
  });
}

rstg_status rstg_system_tuning(const rstg_system* s, int32_t* shape12, double* ms12) {
  return guard([&] {
    if (!s) throw Error(RSTG_ERR_INVALID, "system must not be NULL");
    if (s->opts.mode != RSTG_MODE_FUSED || !s->fp) {
      if (shape12) memset(shape12, 0, 12 * sizeof(int32_t));
      if (ms12) memset(ms12, 0, 12 * sizeof(double));
      return;
    }
    s->tuning(shape12, ms12);
  });
}

rstg_status rstg_system_pb_stats(const rstg_system* s, double* o) {
  return guard([&] {
    if (!s || !o) throw Error(RSTG_ERR_INVALID, "system and out must not be NULL");
    for (int k = 0; k < 8; k++) o[k] = 0.0;
    if (!s->pbe) return;
    const rstg::PbBatchStats& t = s->pbe->stats;
    o[0] = (double)t.jobs;
    o[1] = (double)t.cycles;
    o[2] = (double)t.fallbacks;
    o[3] = t.ms_setup;
    o[4] = t.ms_cycles;
    o[5] = t.ms_finish;
  });
}

rstg_status rstg_system_set_pb_profile(rstg_system* s, int32_t on) {
  return guard([&] {
    if (!s) throw Error(RSTG_ERR_INVALID, "system must not be NULL");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    s->pb_profile = on != 0;
    if (s->pbe) {
      s->pbe->profile = on != 0;
      s->pbe->prof = rstg::PbProfile();
    }
  });
}

rstg_status rstg_system_pb_profile(const rstg_system* s, double* o) {
  return guard([&] {
    if (!s || !o) throw Error(RSTG_ERR_INVALID, "system and out must not be NULL");
    for (int k = 0; k < 12; k++) o[k] = 0.0;
    if (!s->pbe) return;
    const rstg::PbProfile& p = s->pbe->prof;
    for (int k = 0; k < rstg::kProfKernels; k++) {
      o[k] = p.ms[k];
      o[4 + k] = p.bytes[k];
      o[8 + k] = (double)p.launches[k];
    }
  });
}

rstg_status rstg_system_set_pb_batch(rstg_system* s, int64_t frames) {
  return guard([&] {
    if (!s) throw Error(RSTG_ERR_INVALID, "system must not be NULL");
    if (frames < 0) throw Error(RSTG_ERR_INVALID, "frames must be >= 0");
    s->pb_frames_per_batch = frames;
  });
}

rstg_status rstg_system_set_pb_convergence(rstg_system* s, double rel_tol) {
  return guard([&] {
    if (!s) throw Error(RSTG_ERR_INVALID, "system must not be NULL");
    if (!(rel_tol >= 0.0) || rel_tol >= 1.0) throw Error(RSTG_ERR_INVALID, "rel_tol must be in [0, 1)");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    s->pb_rel_tol = rel_tol;
  });
}

rstg_status rstg_system_profile(rstg_system* s, const float* d_frames, int64_t F, int32_t* n, char* names,
                                double* ms, double* flops, double* bytes) {
  return guard([&] {
    if (!s || !n || !d_frames || F <= 0) throw Error(RSTG_ERR_INVALID, "system, frames and n are required");
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    s->ctx->bind();
    s->profile(d_frames, F, n, names, ms, flops, bytes);
  });
}

rstg_status rstg_system_reimage(rstg_system* s, const double* frames, const double* boxes, int64_t F,
                                int32_t on_device, double* out) {
  return guard([&] {
    if (!s || (F > 0 && (!frames || !boxes || !out))) throw Error(RSTG_ERR_INVALID, "system, frames, boxes and out are required");
    if (F < 0) throw Error(RSTG_ERR_INVALID, "F must be >= 0");
    const int64_t n = s->n_top;
    const Split& sp = s->split;
    if (F == 0) return;
    if (out != frames) memcpy(out, frames, (size_t)F * n * 24);
    if (!on_device) {
      std::vector<double> cx(sp.complex.n_atoms * 3);
      for (int64_t f = 0; f < F; f++) {
        double* x = out + (size_t)f * n * 3;
        for (int64_t a = 0; a < sp.complex.n_atoms; a++) {
          const int64_t ta = sp.complex_atoms.empty() ? a : sp.complex_atoms[a];
          for (int d = 0; d < 3; d++) cx[3 * a + d] = x[3 * ta + d];
        }
        reimage_host(cx.data(), sp.complex.n_atoms, sp.complex, {boxes[3 * f], boxes[3 * f + 1], boxes[3 * f + 2]});
        for (int64_t a = 0; a < sp.complex.n_atoms; a++) {
          const int64_t ta = sp.complex_atoms.empty() ? a : sp.complex_atoms[a];
          for (int d = 0; d < 3; d++) x[3 * ta + d] = cx[3 * a + d];
        }
      }
      return;
    }
    std::lock_guard<std::recursive_mutex> lk(s->mu);
    Ctx* c = s->ctx;
    c->bind();
    DevBuf d_fr((size_t)F * n * 24, c->stream), d_bx((size_t)F * 24, c->stream);
    RSTG_CUDA(cudaMemcpyAsync(d_fr.p, out, (size_t)F * n * 24, cudaMemcpyHostToDevice, c->stream));
    RSTG_CUDA(cudaMemcpyAsync(d_bx.p, boxes, (size_t)F * 24, cudaMemcpyHostToDevice, c->stream));
    reimage_device(c, c->stream, sp, n, d_fr.as<double>(), d_bx.as<double>(), F);
    RSTG_CUDA(cudaMemcpyAsync(out, d_fr.p, (size_t)F * n * 24, cudaMemcpyDeviceToHost, c->stream));
    RSTG_CUDA(cudaStreamSynchronize(c->stream));
  });
}

rstg_status rstg_binding_trajectory(rstg_ctx* c, const rstg_topology* t, const char* path, const char* format,
                                    int32_t has_box, const int64_t* rr, int64_t nr, const int64_t* lr, int64_t nl,
                                    const rstg_solvation* solv, const rstg_sa_params* sa, int64_t stride,
                                    int64_t start, int64_t end, int32_t mode, rstg_frame_energy* frames_out,
                                    int64_t cap, int64_t* n_frames, double* stats9, double* last_coords) {
  return guard([&] {
    if (!c || !t || !path) throw Error(RSTG_ERR_INVALID, "ctx, topology and path must not be NULL");
    std::string fmt = format ? format : "mdcrd";
    int64_t n = t->n_atoms;
    std::vector<double> all;  // float64 Angstrom, topology order
    std::vector<std::array<double, 3>> boxes;
    int64_t nf = 0;
    if (fmt == "dcd") {
      DcdData d = read_dcd(path);
      if (d.n_atoms != n)
        throw Error(RSTG_ERR_INVALID, "DCD has " + std::to_string(d.n_atoms) + " atoms, topology has " +
                                          std::to_string(n));
      nf = d.n_frames;
      all.resize(d.xyz.size());
      for (size_t k = 0; k < d.xyz.size(); k++) all[k] = ((double)d.xyz[k] * 0.1) * 10.0;  // dcd.rs:429-437, binding.rs:630-633
      boxes = d.boxes;
    } else {
      all = read_mdcrd(path, n, has_box != 0, &boxes);
      nf = n > 0 ? (int64_t)all.size() / (n * 3) : 0;
    }
    int64_t st = std::max<int64_t>(stride, 1);
    std::vector<int64_t> sel;
    for (int64_t f = 0; f < nf && f < end; f++)
      if (f >= start && (f - start) % st == 0) sel.push_back(f);
    if (sel.empty()) throw Error(RSTG_ERR_INVALID, "No frames found in trajectory");
    rstg_system_opts o;
    rstg_system_opts_default(&o);
    o.mode = mode;
    rstg_system* sys = nullptr;
    rstg_status rc = rstg_system_create(c, t, rr, nr, lr, nl, solv, sa, &o, &sys);
    if (rc != RSTG_OK) throw Error(rc, rstg_last_error());
    std::unique_ptr<rstg_system, void (*)(rstg_system*)> hold(sys, rstg_system_destroy);
    std::vector<double> frames(sel.size() * n * 3);
    const Split& sp = sys->split;
    for (size_t k = 0; k < sel.size(); k++) memcpy(&frames[k * n * 3], &all[(size_t)sel[k] * n * 3], n * 24);
    if (!boxes.empty()) {  // reimaged on the device, in chunks of at most 512 MB of frames
      std::vector<double> bx(sel.size() * 3);
      for (size_t k = 0; k < sel.size(); k++)
        for (int d = 0; d < 3; d++) bx[3 * k + d] = boxes[sel[k]][d];
      c->bind();
      const int64_t per = std::max<int64_t>(1, (int64_t)(512ll << 20) / std::max<int64_t>(n * 24, 1));
      for (int64_t f0 = 0; f0 < (int64_t)sel.size(); f0 += per) {
        const int64_t F = std::min<int64_t>(per, (int64_t)sel.size() - f0);
        DevBuf d_fr((size_t)F * n * 24, c->stream), d_bx((size_t)F * 24, c->stream);
        RSTG_CUDA(cudaMemcpyAsync(d_fr.p, &frames[f0 * n * 3], (size_t)F * n * 24, cudaMemcpyHostToDevice, c->stream));
        RSTG_CUDA(cudaMemcpyAsync(d_bx.p, &bx[f0 * 3], (size_t)F * 24, cudaMemcpyHostToDevice, c->stream));
        reimage_device(c, c->stream, sp, n, d_fr.as<double>(), d_bx.as<double>(), F);
        RSTG_CUDA(cudaMemcpyAsync(&frames[f0 * n * 3], d_fr.p, (size_t)F * n * 24, cudaMemcpyDeviceToHost, c->stream));
        RSTG_CUDA(cudaStreamSynchronize(c->stream));
      }
    }
    std::vector<rstg_frame_energy> res(sel.size());
    {
      std::lock_guard<std::recursive_mutex> lk(sys->mu);
      c->bind();
      sys->run(frames.data(), true, true, (int64_t)sel.size(), res.data(), true, nullptr);
    }
    if (n_frames) *n_frames = (int64_t)sel.size();
    if (frames_out) memcpy(frames_out, res.data(), std::min<int64_t>(cap, (int64_t)res.size()) * sizeof(rstg_frame_energy));
    if (last_coords) {
      const double* lf = &frames[(sel.size() - 1) * n * 3];
      for (int64_t a = 0; a < sp.complex.n_atoms; a++) {
        int64_t ta = sp.complex_atoms.empty() ? a : sp.complex_atoms[a];
        for (int d = 0; d < 3; d++) last_coords[3 * a + d] = lf[3 * ta + d];
      }
    }
    if (stats9) {  // binding.rs:704-743
      double N = (double)res.size();
      double m[4] = {0, 0, 0, 0};
      for (auto& e : res) {
        m[0] += e.delta_mm;
        m[1] += e.delta_polar;
        m[2] += e.delta_sa;
        m[3] += e.delta_total;
      }
      for (double& v : m) v /= N;
      auto sd = [&](int which, double mean) {
        if (res.size() <= 1) return 0.0;
        double s = 0.0;
        for (auto& e : res) {
          double v = which == 0 ? e.delta_mm : which == 1 ? e.delta_polar : which == 2 ? e.delta_sa : e.delta_total;
          s += (v - mean) * (v - mean);
        }
        return std::sqrt(s / (double)(res.size() - 1));
      };
      double sdt = sd(3, m[3]);
      double v[9] = {m[0], m[1], m[2], m[3], sdt, sd(0, m[0]), sd(1, m[1]), sd(2, m[2]), sdt / std::sqrt(N)};
      memcpy(stats9, v, sizeof(v));
    }
  });
}

}  // extern "C"
