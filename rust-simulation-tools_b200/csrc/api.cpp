// extern "C" surface of librstg (include/rstg.h).
#include <cmath>
#include <cstring>
#include <memory>

#include "frame_plain.hpp"
#include "pb.cuh"
#include "internal.hpp"
#include "system.hpp"
#include "trajectory.hpp"

namespace rstg {

static thread_local std::string g_last_error;
void set_last_error(const std::string& m) { g_last_error = m; }

DevBuf::DevBuf(size_t n, cudaStream_t st) : bytes(n), s(st) {
  if (n == 0) return;
  cudaError_t e = cudaMallocAsync(&p, n, st);
  if (e != cudaSuccess) {
    p = nullptr;
    cudaGetLastError();
    throw Error(e == cudaErrorMemoryAllocation ? RSTG_ERR_NOMEM : RSTG_ERR_CUDA,
                std::string("device allocation of ") + std::to_string(n) + " bytes failed: " + cudaGetErrorString(e));
  }
}
DevBuf::~DevBuf() {
  if (p) cudaFreeAsync(p, s);
}
DevBuf& DevBuf::operator=(DevBuf&& o) noexcept {
  if (this != &o) {
    if (p) cudaFreeAsync(p, s);
    p = o.p;
    bytes = o.bytes;
    s = o.s;
    o.p = nullptr;
  }
  return *this;
}

void launched(Ctx* c, int n) {
  c->launches += n;
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(RSTG_ERR_CUDA, std::string("kernel launch failed: ") + cudaGetErrorString(e));
  }
}

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

static void need(const void* p, const char* what) {
  if (!p) throw Error(RSTG_ERR_INVALID, std::string(what) + " must not be NULL");
}

static void check_coords(const rstg_topology* t, const double* xyz, int64_t n) {
  need(t, "topology");
  if (n != t->n_atoms)
    throw Error(RSTG_ERR_INVALID, "coordinates have " + std::to_string(n) + " atoms, topology has " +
                                      std::to_string(t->n_atoms));
  if (n > 0) need(xyz, "coordinates");
}

static void check_gb(const rstg_gb_params& p) {
  if (p.model < 0 || p.model > 2) throw Error(RSTG_ERR_INVALID, "unknown GB model");
}

}  // namespace rstg

using namespace rstg;

extern "C" {

const char* rstg_last_error(void) { return g_last_error.c_str(); }
const char* rstg_version(void) { return "rstg 0.1.0 (sm_100a)"; }

int rstg_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

void rstg_gb_params_default(rstg_gb_params* p) {
  // gb_energy.rs:43-56
  p->model = RSTG_GB_OBC1;
  p->solute_dielectric = 1.0;
  p->solvent_dielectric = 78.3;
  p->salt_concentration = 0.15;
  p->temperature = 300.0;
  p->offset = 0.09;
  p->rgbmax = 25.0;
  p->cutoff = 9999.0;
}
void rstg_sa_params_default(rstg_sa_params* p) {
  // sa_energy.rs:23-32
  p->surface_tension = 0.0072;
  p->offset = 0.0;
  p->probe_radius = 1.4;
  p->n_sphere_points = 480;
}
void rstg_pb_params_default(rstg_pb_params* p) {
  // pb_energy.rs:49-66
  p->grid_spacing = 0.5;
  p->grid_buffer = 10.0;
  p->solute_dielectric = 1.0;
  p->solvent_dielectric = 80.0;
  p->salt_concentration = 0.15;
  p->temperature = 300.0;
  p->probe_radius = 1.4;
  p->ion_radius = 2.0;
  p->tolerance = 1e-6;
  p->max_iterations = 10000;
  p->fillratio = 4.0;
  p->fscale = 8;
}

rstg_status rstg_ctx_create(int device, void* stream, rstg_ctx** out) {
  return guard([&] {
    need(out, "out");
    int n = rstg_device_count();
    if (device < 0 || device >= n) throw Error(RSTG_ERR_CUDA, "no CUDA device " + std::to_string(device));
    auto c = std::make_unique<rstg_ctx>();
    c->device = device;
    RSTG_CUDA(cudaSetDevice(device));
    RSTG_CUDA(cudaGetDeviceProperties(&c->prop, device));
    if (stream) {
      c->stream = (cudaStream_t)stream;
    } else {
      RSTG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
      c->own_stream = true;
    }
    *out = c.release();
  });
}

void rstg_ctx_destroy(rstg_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  if (c->own_stream) cudaStreamDestroy(c->stream);
  delete c;
}

int64_t rstg_ctx_kernel_launches(const rstg_ctx* c) { return c ? c->launches.load() : 0; }

// ---- topology -------------------------------------------------------------

rstg_status rstg_topology_load_prmtop(const char* path, rstg_topology** out) {
  return guard([&] {
    need(path, "path");
    need(out, "out");
    auto t = std::make_unique<rstg_topology>();
    static_cast<Topology&>(*t) = parse_prmtop(path);
    *out = t.release();
  });
}

rstg_status rstg_topology_from_desc(const rstg_topology_desc* d, rstg_topology** out) {
  return guard([&] {
    need(d, "desc");
    need(out, "out");
    if (d->n_atoms < 0 || d->n_residues < 0 || d->n_types < 0) throw Error(RSTG_ERR_INVALID, "negative count");
    auto t = std::make_unique<rstg_topology>();
    int64_t n = d->n_atoms;
    t->n_atoms = n;
    t->n_residues = d->n_residues;
    t->n_types = d->n_types;
    for (int64_t i = 0; i < n; i++) {
      t->atom_names.push_back("");
      int64_t ty = d->atom_type_indices ? d->atom_type_indices[i] : 0;
      if (ty < 0 || (d->n_types > 0 && ty >= d->n_types)) throw Error(RSTG_ERR_INVALID, "atom type out of range");
      t->type_idx.push_back(ty);
      double qa = d->charges_amber ? d->charges_amber[i] : 0.0;
      t->charges_amber.push_back(qa);
      t->charges.push_back(qa / 18.2223);
      t->radii.push_back(d->radii ? d->radii[i] : 0.0);
      t->screen.push_back(d->screen ? d->screen[i] : 0.0);
      t->masses.push_back(0.0);
    }
    for (int64_t r = 0; r < d->n_residues; r++) {
      int64_t p = d->residue_pointers ? d->residue_pointers[r] : 0;
      if (p < 0 || p > n) throw Error(RSTG_ERR_INVALID, "residue pointer out of range");
      t->residue_pointers.push_back(p);
      t->residue_labels.push_back("");
    }
    auto chk = [&](int64_t a) {
      if (a < 0 || a >= n) throw Error(RSTG_ERR_INVALID, "bonded term references atom out of range");
    };
    for (int64_t b = 0; b < d->n_bonds; b++) {
      const int64_t* q = d->bonds + 3 * b;
      chk(q[0]);
      chk(q[1]);
      if (q[2] < 0 || q[2] >= d->n_bond_types) throw Error(RSTG_ERR_INVALID, "bond type out of range");
      t->bond_i.push_back(q[0]);
      t->bond_j.push_back(q[1]);
      t->bond_t.push_back(q[2]);
    }
    if (d->n_bond_types) {
      t->bond_k.assign(d->bond_k, d->bond_k + d->n_bond_types);
      t->bond_req.assign(d->bond_req, d->bond_req + d->n_bond_types);
    }
    for (int64_t a = 0; a < d->n_angles; a++) {
      const int64_t* q = d->angles + 4 * a;
      chk(q[0]);
      chk(q[1]);
      chk(q[2]);
      if (q[3] < 0 || q[3] >= d->n_angle_types) throw Error(RSTG_ERR_INVALID, "angle type out of range");
      t->ang_i.push_back(q[0]);
      t->ang_j.push_back(q[1]);
      t->ang_k.push_back(q[2]);
      t->ang_t.push_back(q[3]);
    }
    if (d->n_angle_types) {
      t->angle_k.assign(d->angle_k, d->angle_k + d->n_angle_types);
      t->angle_teq.assign(d->angle_teq, d->angle_teq + d->n_angle_types);
    }
    for (int64_t k = 0; k < d->n_dihedrals; k++) {
      const int64_t* q = d->dihedrals + 6 * k;
      for (int m = 0; m < 4; m++) chk(q[m]);
      if (q[4] < 0 || q[4] >= d->n_dihedral_types) throw Error(RSTG_ERR_INVALID, "dihedral type out of range");
      t->dih_i.push_back(q[0]);
      t->dih_j.push_back(q[1]);
      t->dih_k.push_back(q[2]);
      t->dih_l.push_back(q[3]);
      t->dih_t.push_back(q[4]);
      t->dih_ignore14.push_back(q[5] != 0);
    }
    if (d->n_dihedral_types) {
      t->dih_pk.assign(d->dihedral_pk, d->dihedral_pk + d->n_dihedral_types);
      t->dih_pn.assign(d->dihedral_pn, d->dihedral_pn + d->n_dihedral_types);
      t->dih_phase.assign(d->dihedral_phase, d->dihedral_phase + d->n_dihedral_types);
    }
    for (int64_t i = 0; i < n; i++) t->num_excluded.push_back(d->num_excluded ? d->num_excluded[i] : 0);
    for (int64_t k = 0; k < d->n_excluded; k++) t->excluded_list.push_back(d->excluded_list[k]);
    t->scee = d->scee;
    t->scnb = d->scnb;
    if (d->n_lj) {
      t->lj_a.assign(d->lj_acoef, d->lj_acoef + d->n_lj);
      t->lj_b.assign(d->lj_bcoef, d->lj_bcoef + d->n_lj);
    }
    t->nb_index.assign(d->nb_parm_index, d->nb_parm_index + d->n_types * d->n_types);
    for (auto v : t->nb_index)
      if (v > d->n_lj) throw Error(RSTG_ERR_INVALID, "nb_parm_index entry exceeds the LJ tables");
    *out = t.release();
  });
}

rstg_status rstg_topology_extract(const rstg_topology* t, const int64_t* atoms, int64_t n, rstg_topology** out) {
  return guard([&] {
    need(t, "topology");
    need(out, "out");
    auto s = std::make_unique<rstg_topology>();
    static_cast<Topology&>(*s) = extract_subtopology(*t, vec(atoms, n));
    *out = s.release();
  });
}

void rstg_topology_free(rstg_topology* t) { delete t; }

rstg_status rstg_topology_info_get(const rstg_topology* t, rstg_topology_info* o) {
  return guard([&] {
    need(t, "topology");
    need(o, "out");
    o->n_atoms = t->n_atoms;
    o->n_residues = t->n_residues;
    o->n_types = t->n_types;
    o->n_bonds = t->bond_i.size();
    o->n_angles = t->ang_i.size();
    o->n_dihedrals = t->dih_i.size();
    o->scee = t->scee;
    o->scnb = t->scnb;
  });
}

rstg_status rstg_topology_atoms(const rstg_topology* t, double* q, double* qa, double* r, double* s, double* m,
                                int64_t* ty, int64_t* res) {
  return guard([&] {
    need(t, "topology");
    size_t n = t->n_atoms;
    if (q) memcpy(q, t->charges.data(), n * 8);
    if (qa) memcpy(qa, t->charges_amber.data(), n * 8);
    if (r) memcpy(r, t->radii.data(), n * 8);
    if (s) memcpy(s, t->screen.data(), n * 8);
    if (m) memcpy(m, t->masses.data(), n * 8);
    if (ty) memcpy(ty, t->type_idx.data(), n * 8);
    if (res) {
      auto a = t->atom_residue_indices();
      memcpy(res, a.data(), n * 8);
    }
  });
}

rstg_status rstg_topology_residue_pointers(const rstg_topology* t, int64_t* out) {
  return guard([&] {
    need(t, "topology");
    need(out, "out");
    memcpy(out, t->residue_pointers.data(), t->residue_pointers.size() * 8);
  });
}

rstg_status rstg_topology_names(const rstg_topology* t, char* an, char* rl) {
  return guard([&] {
    need(t, "topology");
    if (an)
      for (int64_t i = 0; i < t->n_atoms; i++) {
        memset(an + 4 * i, 0, 4);
        memcpy(an + 4 * i, t->atom_names[i].c_str(), std::min<size_t>(4, t->atom_names[i].size()));
      }
    if (rl)
      for (int64_t i = 0; i < t->n_residues; i++) {
        memset(rl + 4 * i, 0, 4);
        memcpy(rl + 4 * i, t->residue_labels[i].c_str(), std::min<size_t>(4, t->residue_labels[i].size()));
      }
  });
}

rstg_status rstg_topology_select(const rstg_topology* t, const int64_t* residues, int64_t n_res, int64_t* atoms_out,
                                 int64_t* n_atoms_out) {
  return guard([&] {
    need(t, "topology");
    need(n_atoms_out, "n_atoms_out");
    auto a = t->select(vec(residues, n_res));
    *n_atoms_out = (int64_t)a.size();
    if (atoms_out) memcpy(atoms_out, a.data(), a.size() * 8);
  });
}

// ---- trajectories -----------------------------------------------------------

rstg_status rstg_dcd_read(const char* path, double* out_nm, int64_t cap, int64_t* nf, int64_t* na) {
  return guard([&] {
    need(path, "path");
    DcdData d = read_dcd(path);
    if (nf) *nf = d.n_frames;
    if (na) *na = d.n_atoms;
    if (out_nm) {
      int64_t m = std::min<int64_t>(cap, (int64_t)d.xyz.size());
      for (int64_t k = 0; k < m; k++) out_nm[k] = (double)d.xyz[k] * 0.1;  // dcd.rs:429-437
    }
  });
}

rstg_status rstg_dcd_read_f32(const char* path, float* out, int64_t cap, int64_t* nf, int64_t* na) {
  return guard([&] {
    need(path, "path");
    DcdData d = read_dcd(path);
    if (nf) *nf = d.n_frames;
    if (na) *na = d.n_atoms;
    if (out) memcpy(out, d.xyz.data(), std::min<int64_t>(cap, (int64_t)d.xyz.size()) * 4);
  });
}

rstg_status rstg_mdcrd_read(const char* path, int64_t n_atoms, int32_t has_box, double* out, int64_t cap,
                            int64_t* nf) {
  return guard([&] {
    need(path, "path");
    auto v = read_mdcrd(path, n_atoms, has_box != 0, nullptr);
    if (nf) *nf = n_atoms > 0 ? (int64_t)v.size() / (n_atoms * 3) : 0;
    if (out) memcpy(out, v.data(), std::min<int64_t>(cap, (int64_t)v.size()) * 8);
  });
}

// ---- single-term entry points ---------------------------------------------------

struct OneShot {
  Topology top;
  PairClasses pc;
  DevTopo dev;
  DevBuf xyz;
  OneShot(Ctx* c, const Topology& t, const double* x) : top(t) {
    pc = PairClasses::build(top);
    dev = DevTopo::upload(top, pc, c->stream);
    xyz = DevBuf(std::max<int64_t>(top.n_atoms, 1) * 24, c->stream);
    if (top.n_atoms)
      RSTG_CUDA(cudaMemcpyAsync(xyz.p, x, top.n_atoms * 24, cudaMemcpyHostToDevice, c->stream));
  }
};

rstg_status rstg_mm_energy_compute(rstg_ctx* c, const rstg_topology* t, const double* xyz, int64_t n,
                                   rstg_mm_energy* out) {
  return guard([&] {
    need(c, "ctx");
    need(out, "out");
    check_coords(t, xyz, n);
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->bind();
    OneShot o(c, *t, xyz);
    DevBuf r(7 * 8, c->stream);
    plain_mm_energy(c, o.dev, o.xyz.as<double>(), r.as<double>());
    double h[7];
    RSTG_CUDA(cudaMemcpyAsync(h, r.p, 56, cudaMemcpyDeviceToHost, c->stream));
    RSTG_CUDA(cudaStreamSynchronize(c->stream));
    *out = {h[0], h[1], h[2], h[3], h[4], h[5], h[6]};
  });
}

rstg_status rstg_gb_energy_compute(rstg_ctx* c, const rstg_topology* t, const double* xyz, int64_t n,
                                   const rstg_gb_params* p, double* total, double* born) {
  return guard([&] {
    need(c, "ctx");
    need(total, "total");
    check_coords(t, xyz, n);
    rstg_gb_params gp;
    if (p)
      gp = *p;
    else
      rstg_gb_params_default(&gp);
    check_gb(gp);
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->bind();
    OneShot o(c, *t, xyz);
    DevBuf R(std::max<int64_t>(n, 1) * 8, c->stream), e(8, c->stream);
    RSTG_CUDA(cudaMemsetAsync(e.p, 0, 8, c->stream));
    if (n) {
      plain_born_radii(c, o.dev, o.xyz.as<double>(), gp, R.as<double>());
      plain_gb_energy(c, o.dev, o.xyz.as<double>(), gp, R.as<double>(), e.as<double>());
    }
    RSTG_CUDA(cudaMemcpyAsync(total, e.p, 8, cudaMemcpyDeviceToHost, c->stream));
    if (born && n) RSTG_CUDA(cudaMemcpyAsync(born, R.p, n * 8, cudaMemcpyDeviceToHost, c->stream));
    RSTG_CUDA(cudaStreamSynchronize(c->stream));
  });
}

}  // extern "C"

struct rstg_gb_cache {
  std::vector<double> coords, radii;
  double threshold = 0.5;
};

extern "C" {

rstg_status rstg_gb_cache_create(double rmsd_threshold, rstg_gb_cache** out) {
  return guard([&] {
    need(out, "out");
    auto c = std::make_unique<rstg_gb_cache>();
    c->threshold = rmsd_threshold;
    *out = c.release();
  });
}

void rstg_gb_cache_destroy(rstg_gb_cache* c) { delete c; }

rstg_status rstg_gb_energy_cached(rstg_ctx* c, const rstg_topology* t, const double* xyz, int64_t n,
                                  const rstg_gb_params* p, rstg_gb_cache* cache, double* total, double* born,
                                  int32_t* reused) {
  return guard([&] {
    need(c, "ctx");
    need(cache, "cache");
    need(total, "total");
    check_coords(t, xyz, n);
    rstg_gb_params gp;
    if (p)
      gp = *p;
    else
      rstg_gb_params_default(&gp);
    check_gb(gp);
    // try_reuse (gb_energy.rs:88-110): same atom count, RMSD summed in atom order
    bool hit = false;
    if (n > 0 && (int64_t)cache->coords.size() == 3 * n) {
      double sum_sq = 0.0;
      for (int64_t a = 0; a < n; a++) {
        double dx = cache->coords[3 * a] - xyz[3 * a], dy = cache->coords[3 * a + 1] - xyz[3 * a + 1],
               dz = cache->coords[3 * a + 2] - xyz[3 * a + 2];
        sum_sq += dx * dx + dy * dy + dz * dz;
      }
      hit = std::sqrt(sum_sq / (double)n) < cache->threshold;
    }
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->bind();
    OneShot o(c, *t, xyz);
    DevBuf R(std::max<int64_t>(n, 1) * 8, c->stream), e(8, c->stream);
    RSTG_CUDA(cudaMemsetAsync(e.p, 0, 8, c->stream));
    if (n) {
      if (hit)
        RSTG_CUDA(cudaMemcpyAsync(R.p, cache->radii.data(), n * 8, cudaMemcpyHostToDevice, c->stream));
      else
        plain_born_radii(c, o.dev, o.xyz.as<double>(), gp, R.as<double>());
      plain_gb_energy(c, o.dev, o.xyz.as<double>(), gp, R.as<double>(), e.as<double>());
    }
    std::vector<double> hr(n);
    RSTG_CUDA(cudaMemcpyAsync(total, e.p, 8, cudaMemcpyDeviceToHost, c->stream));
    if (n) RSTG_CUDA(cudaMemcpyAsync(hr.data(), R.p, n * 8, cudaMemcpyDeviceToHost, c->stream));
    RSTG_CUDA(cudaStreamSynchronize(c->stream));
    if (!hit) {  // update (gb_energy.rs:112-119)
      cache->coords.assign(xyz, xyz + 3 * n);
      cache->radii = hr;
    }
    if (born && n) memcpy(born, hr.data(), n * 8);
    if (reused) *reused = hit ? 1 : 0;
  });
}

rstg_status rstg_sa_energy_compute(rstg_ctx* c, const rstg_topology* t, const double* xyz, int64_t n,
                                   const rstg_sa_params* p, double* total, double* total_sasa, double* per_atom) {
  return guard([&] {
    need(c, "ctx");
    check_coords(t, xyz, n);
    rstg_sa_params sp;
    if (p)
      sp = *p;
    else
      rstg_sa_params_default(&sp);
    if (sp.n_sphere_points < 1) throw Error(RSTG_ERR_INVALID, "n_sphere_points must be >= 1");
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->bind();
    OneShot o(c, *t, xyz);
    auto sph = fibonacci_sphere(sp.n_sphere_points);
    DevBuf ds(sph.size() * 8, c->stream), per(std::max<int64_t>(n, 1) * 8, c->stream), tot(8, c->stream),
        ov(8, c->stream);
    RSTG_CUDA(cudaMemcpyAsync(ds.p, sph.data(), sph.size() * 8, cudaMemcpyHostToDevice, c->stream));
    RSTG_CUDA(cudaMemsetAsync(ov.p, 0, 8, c->stream));
    plain_sasa(c, o.dev, o.xyz.as<double>(), sp.probe_radius, sp.n_sphere_points, ds.as<double>(), per.as<double>(),
               tot.as<double>(), ov.as<int>());
    double ts = 0.0;
    int ovf = 0;
    RSTG_CUDA(cudaMemcpyAsync(&ts, tot.p, 8, cudaMemcpyDeviceToHost, c->stream));
    RSTG_CUDA(cudaMemcpyAsync(&ovf, ov.p, 4, cudaMemcpyDeviceToHost, c->stream));
    if (per_atom && n) RSTG_CUDA(cudaMemcpyAsync(per_atom, per.p, n * 8, cudaMemcpyDeviceToHost, c->stream));
    RSTG_CUDA(cudaStreamSynchronize(c->stream));
    if (ovf) throw Error(RSTG_ERR_INVALID, "SASA neighbour list exceeded its capacity (2048)");
    if (total_sasa) *total_sasa = ts;
    if (total) *total = sp.surface_tension * ts + sp.offset;
  });
}

rstg_status rstg_pb_energy_compute(rstg_ctx* c, const rstg_topology* t, const double* xyz, int64_t n,
                                   const rstg_pb_params* p, const int64_t* solute, int64_t n_solute, double* total,
                                   rstg_pb_diag* diag) {
  return guard([&] {
    need(c, "ctx");
    need(total, "total");
    check_coords(t, xyz, n);
    rstg_pb_params pp;
    if (p)
      pp = *p;
    else
      rstg_pb_params_default(&pp);
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->bind();
    const Topology* top = t;
    Topology sub;
    std::vector<double> x(xyz, xyz + 3 * n);
    if (solute) {  // strip_to_solute, pb_energy.rs:442-457
      auto atoms = t->select(vec(solute, n_solute));
      sub = extract_subtopology(*t, atoms);
      std::vector<double> xs;
      for (int64_t a : atoms)
        for (int d = 0; d < 3; d++) xs.push_back(xyz[3 * a + d]);
      x.swap(xs);
      top = &sub;
    }
    if (diag) memset(diag, 0, sizeof(*diag));
    *total = top->n_atoms ? pb_energy_run(c, x, top->charges, top->radii, pp, diag) : 0.0;
  });
}

rstg_status rstg_pb_grid_maps(rstg_ctx* c, const double* xyz, int64_t n, const double* q, const double* r,
                              const rstg_pb_params* p, double ein, double eout, int32_t ionic, int64_t* dims,
                              double* origin, double* charge, uint8_t* inside, double* ex, double* ey, double* ez,
                              double* k2, double* bphi) {
  return guard([&] {
    need(c, "ctx");
    need(xyz, "xyz");
    need(q, "charges");
    need(r, "radii");
    need(dims, "dims3");
    need(origin, "origin3");
    if (n < 1) throw Error(RSTG_ERR_INVALID, "at least one atom is required");
    if (charge && !(ex && ey && ez && k2 && bphi)) throw Error(RSTG_ERR_INVALID, "all map outputs are required");
    rstg_pb_params pp;
    if (p)
      pp = *p;
    else
      rstg_pb_params_default(&pp);
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->bind();
    pb_grid_maps(c, std::vector<double>(xyz, xyz + 3 * n), std::vector<double>(q, q + n), std::vector<double>(r, r + n),
                 pp, ein, eout, ionic != 0, dims, origin, charge, inside, ex, ey, ez, k2, bphi);
  });
}

static rstg_solvation solv_or_default(const rstg_solvation* s) {
  rstg_solvation v;
  if (s) {
    v = *s;
  } else {
    v.method = 0;
    rstg_gb_params_default(&v.gb);
    rstg_pb_params_default(&v.pb);
  }
  if (v.method != 0 && v.method != 1) throw Error(RSTG_ERR_INVALID, "unknown solvation method");
  if (v.method == 0) check_gb(v.gb);
  return v;
}
static rstg_sa_params sa_or_default(const rstg_sa_params* s) {
  rstg_sa_params v;
  if (s)
    v = *s;
  else
    rstg_sa_params_default(&v);
  return v;
}

static std::vector<double> complex_coords(const Split& sp, const double* xyz) {
  if (sp.complex_atoms.empty()) return std::vector<double>(xyz, xyz + sp.complex.n_atoms * 3);
  std::vector<double> o;
  for (int64_t a : sp.complex_atoms)
    for (int d = 0; d < 3; d++) o.push_back(xyz[3 * a + d]);
  return o;
}

rstg_status rstg_binding_frame(rstg_ctx* c, const rstg_topology* t, const double* xyz, int64_t n,
                               const int64_t* rr, int64_t nr, const int64_t* lr, int64_t nl,
                               const rstg_solvation* solv, const rstg_sa_params* sa, rstg_frame_energy* out) {
  return guard([&] {
    need(c, "ctx");
    need(out, "out");
    check_coords(t, xyz, n);
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->bind();
    PlainFrameEval ev(c, *t, vec(rr, nr), vec(lr, nl), solv_or_default(solv), sa_or_default(sa));
    auto xc = complex_coords(ev.split, xyz);
    *out = ev.run(xc.data());
  });
}

rstg_status rstg_decompose(rstg_ctx* c, const rstg_topology* t, const double* xyz, int64_t n, const int64_t* rr,
                           int64_t nr, const int64_t* lr, int64_t nl, const rstg_gb_params* gb,
                           const rstg_sa_params* sa, rstg_residue_energy* ro, rstg_residue_energy* lo) {
  return guard([&] {
    need(c, "ctx");
    check_coords(t, xyz, n);
    if (nr > 0) need(ro, "rec_out");
    if (nl > 0) need(lo, "lig_out");
    rstg_solvation s;
    s.method = 0;
    if (gb)
      s.gb = *gb;
    else
      rstg_gb_params_default(&s.gb);
    check_gb(s.gb);
    rstg_pb_params_default(&s.pb);
    std::lock_guard<std::recursive_mutex> lk(c->mu);
    c->bind();
    PlainFrameEval ev(c, *t, vec(rr, nr), vec(lr, nl), s, sa_or_default(sa));
    auto xc = complex_coords(ev.split, xyz);
    ev.decompose(xc.data(), s.gb, ro, lo);
  });
}

}  // extern "C"
