// Binding workflow, decomposition and the extern "C" surface of the CPU
// restatement.  TEST INFRASTRUCTURE ONLY (see oracle.hpp): loaded by tests/
// through ctypes as the parity checker and by bench.py as the CPU baseline.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <set>
#include <unordered_map>
#include <unordered_set>

#include "oracle.hpp"
#include "oracle_pb.hpp"

namespace orc {

// binding.rs:142-211 (build_complex_subsystem) and
// decomposition.rs:125-208 (build_effective_complex): the same selection logic.
struct Split {
  Topology complex, rec, lig;
  std::vector<size_t> complex_atoms;  // empty: complex == whole topology
  std::vector<size_t> rec_atoms, lig_atoms;  // in complex numbering
  std::vector<size_t> rec_res_remapped, lig_res_remapped;
};

static bool make_split(const Topology& t, const std::vector<size_t>& rres, const std::vector<size_t>& lres,
                       Split& s, std::string& err) {
  std::set<size_t> cs(rres.begin(), rres.end());
  cs.insert(lres.begin(), lres.end());
  std::vector<size_t> cres(cs.begin(), cs.end()), catoms;
  if (!t.build_selection(cres, catoms, err)) return false;
  if (catoms.size() == t.n_atoms) {
    s.complex = t;
    s.rec_res_remapped = rres;
    s.lig_res_remapped = lres;
  } else {
    s.complex = extract_subtopology(t, catoms);
    s.complex_atoms = catoms;
    std::unordered_map<size_t, size_t> m;
    for (size_t k = 0; k < cres.size(); k++) m[cres[k]] = k;
    for (size_t r : rres) s.rec_res_remapped.push_back(m[r]);
    for (size_t r : lres) s.lig_res_remapped.push_back(m[r]);
  }
  if (!s.complex.build_selection(s.rec_res_remapped, s.rec_atoms, err)) return false;
  if (!s.complex.build_selection(s.lig_res_remapped, s.lig_atoms, err)) return false;
  s.rec = extract_subtopology(s.complex, s.rec_atoms);
  s.lig = extract_subtopology(s.complex, s.lig_atoms);
  return true;
}

static std::vector<V3> gather(const std::vector<V3>& x, const std::vector<size_t>& idx) {
  std::vector<V3> o;
  o.reserve(idx.size());
  for (size_t i : idx) o.push_back(x[i]);
  return o;
}

struct Method {
  int kind = 0;  // 0 GB, 1 PB
  GbParams gb;
  PbParams pb;
};

static double polar(const Topology& t, const std::vector<V3>& x, const Method& m, bool acc) {
  if (m.kind == 0) {
    auto R = born_radii(t, x, m.gb, acc);
    return gb_energy_from_radii(t, x, m.gb, R, acc);
  }
  PbParams p = m.pb;
  if (acc) p.tolerance = std::min(p.tolerance, 1e-10);
  return pb_energy(x, t.charges, t.radii, p, nullptr);
}

static SubsystemEnergy subsystem(const Topology& t, const std::vector<V3>& x, const Method& m,
                                 const SaParams& sa, bool acc) {
  SubsystemEnergy e;
  e.mm = mm_energy(t, x, acc).total();
  e.polar = polar(t, x, m, acc);
  auto s = sasa_per_atom(x, t.radii, sa.probe, sa.n_points);
  double tot = 0.0;
  long double tl = 0.0L;
  for (double v : s) {
    tot += v;
    tl += v;
  }
  e.sa = sa.surface_tension * (acc ? (double)tl : tot) + sa.offset;
  return e;
}

// ---- exact binding differences (accurate mode only) -----------------------
static bool is14(const Topology& t, size_t i, size_t j) {
  for (auto& d : t.dihedrals)
    if (!d.ignore_14 && ((d.i == i && d.l == j) || (d.i == j && d.l == i))) return true;
  return false;
}
static bool isexcl(const Topology& t, size_t i, size_t j) {
  size_t off = 0;
  for (size_t a = 0; a < t.n_atoms; a++) {
    size_t cnt = a < t.num_excluded.size() ? t.num_excluded[a] : 0;
    if (a == i || a == j)
      for (size_t k = 0; k < cnt; k++)
        if (off + k < t.excluded_list.size()) {
          size_t b = t.excluded_list[off + k];
          if ((a == i && b == j) || (a == j && b == i)) return true;
        }
    off += cnt;
  }
  return false;
}
static long double nb_pair(const Topology& t, const std::vector<V3>& x, size_t i, size_t j, int cls) {
  // cls 0 skip, 1 full, 2 scaled 1-4 (mm_energy.rs:230-252)
  if (cls == 0) return 0.0L;
  size_t a = std::min(i, j), b = std::max(i, j);
  double dx = x[a].x - x[b].x, dy = x[a].y - x[b].y, dz = x[a].z - x[b].z;
  double r2 = dx * dx + dy * dy + dz * dz, r = std::sqrt(r2), r6 = r2 * r2 * r2, r12 = r6 * r6;
  int64_t idx = t.nb_index[t.n_types * t.type_idx[a] + t.type_idx[b]];
  double A = idx < 1 ? 0.0 : t.lj_a[idx - 1], B = idx < 1 ? 0.0 : t.lj_b[idx - 1];
  double qq = t.charges_amber[a] * t.charges_amber[b];
  if (cls == 2) return (long double)((A / r12 - B / r6) / t.scnb) + (long double)(qq / r / t.scee);
  return (long double)(A / r12 - B / r6) + (long double)(qq / r);
}

static double delta_mm_exact(const Split& s, const std::vector<V3>& x) {
  const Topology& C = s.complex;
  // pair classes in the complex for R x L pairs; bitmap-free lookups via sets
  std::set<std::pair<size_t, size_t>> p14, ex;
  for (auto& d : C.dihedrals)
    if (!d.ignore_14) p14.insert({std::min(d.i, d.l), std::max(d.i, d.l)});
  size_t off = 0;
  for (size_t a = 0; a < C.n_atoms; a++) {
    size_t cnt = a < C.num_excluded.size() ? C.num_excluded[a] : 0;
    for (size_t k = 0; k < cnt; k++)
      if (off + k < C.excluded_list.size() && C.excluded_list[off + k] < C.n_atoms) {
        size_t b = C.excluded_list[off + k];
        ex.insert({std::min(a, b), std::max(a, b)});
      }
    off += cnt;
  }
  auto cls = [&](size_t i, size_t j) {
    auto k = std::make_pair(std::min(i, j), std::max(i, j));
    if (p14.count(k)) return 2;
    if (ex.count(k)) return 0;
    return 1;
  };
  long double d = 0.0L;
  std::vector<long double> part(s.rec_atoms.size(), 0.0L);
#pragma omp parallel for schedule(dynamic, 16)
  for (long a = 0; a < (long)s.rec_atoms.size(); a++) {
    long double acc = 0.0L;
    for (size_t j : s.lig_atoms) acc += nb_pair(C, x, s.rec_atoms[a], j, cls(s.rec_atoms[a], j));
    part[a] = acc;
  }
  for (auto v : part) d += v;
  // pairs inside one part whose 1-4 status comes from a dihedral that spans the parts
  for (int side = 0; side < 2; side++) {
    const std::vector<size_t>& at = side == 0 ? s.rec_atoms : s.lig_atoms;
    const Topology& sub = side == 0 ? s.rec : s.lig;
    std::unordered_map<size_t, size_t> loc;
    for (size_t k = 0; k < at.size(); k++) loc[at[k]] = k;
    std::set<std::pair<size_t, size_t>> seen;
    for (auto& dh : C.dihedrals) {
      if (dh.ignore_14) continue;
      auto li = loc.find(dh.i), ll = loc.find(dh.l);
      if (li == loc.end() || ll == loc.end()) continue;
      auto key = std::make_pair(std::min(dh.i, dh.l), std::max(dh.i, dh.l));
      if (seen.count(key)) continue;
      seen.insert(key);
      size_t a = li->second, b = ll->second;
      int cs = is14(sub, a, b) ? 2 : (isexcl(sub, a, b) ? 0 : 1);
      if (cs == 2) continue;
      d += nb_pair(C, x, dh.i, dh.l, 2) - nb_pair(C, x, dh.i, dh.l, cs);
    }
  }
  // bonded terms that span the parts
  MmEnergy ec = mm_energy(C, x, true);
  MmEnergy er = mm_energy(s.rec, gather(x, s.rec_atoms), true);
  MmEnergy el = mm_energy(s.lig, gather(x, s.lig_atoms), true);
  long double bonded = ((long double)ec.bond - er.bond - el.bond) + ((long double)ec.angle - er.angle - el.angle) +
                       ((long double)ec.dihedral - er.dihedral - el.dihedral);
  return (double)(d + bonded);
}

static double delta_gb_exact(const Split& s, const std::vector<V3>& x, const GbParams& p,
                             std::vector<double>* RC, std::vector<double>* Rsub) {
  const Topology& C = s.complex;
  auto rc = born_radii(C, x, p, true);
  auto xr = gather(x, s.rec_atoms), xl = gather(x, s.lig_atoms);
  auto rr = born_radii(s.rec, xr, p, true), rl = born_radii(s.lig, xl, p, true);
  size_t n = C.n_atoms;
  std::vector<int> side(n, -1);
  std::vector<double> rs(n, 0.0);
  for (size_t k = 0; k < s.rec_atoms.size(); k++) {
    side[s.rec_atoms[k]] = 0;
    rs[s.rec_atoms[k]] = rr[k];
  }
  for (size_t k = 0; k < s.lig_atoms.size(); k++) {
    side[s.lig_atoms[k]] = 1;
    rs[s.lig_atoms[k]] = rl[k];
  }
  double kap = kappa(p.salt, p.solvent_dielectric, p.temperature);
  double ie = 1.0 / p.solute_dielectric, io = 1.0 / p.solvent_dielectric, dn = -0.5 * (ie - io);
  bool ns = kap <= 0.0;
  double cut2 = p.cutoff * p.cutoff;
  const double KS = 0.73;
  auto pair = [&](double qi, double qj, double r2, double Ri, double Rj) {
    double rr2 = Ri * Rj, f = std::sqrt(r2 + rr2 * std::exp(-r2 / (4.0 * rr2)));
    return ns ? dn * qi * qj / f : -0.5 * qi * qj * (ie - std::exp(-KS * kap * f) * io) / f;
  };
  auto self = [&](double q, double R) {
    return ns ? dn * q * q / R : -0.5 * q * q * (ie - std::exp(-KS * kap * R) * io) / R;
  };
  long double d = 0.0L;
  for (size_t i = 0; i < n; i++) {
    if (side[i] < 0) continue;
    d += (long double)self(C.charges_amber[i], rc[i]) - (long double)self(C.charges_amber[i], rs[i]);
  }
  std::vector<long double> part(n, 0.0L);
#pragma omp parallel for schedule(dynamic, 16)
  for (long ii = 0; ii < (long)n; ii++) {
    size_t i = (size_t)ii;
    long double acc = 0.0L;
    for (size_t j = i + 1; j < n; j++) {
      double dx = x[i].x - x[j].x, dy = x[i].y - x[j].y, dz = x[i].z - x[j].z;
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > cut2) continue;
      double qi = C.charges_amber[i], qj = C.charges_amber[j];
      long double pc = pair(qi, qj, r2, rc[i], rc[j]);
      if (side[i] == side[j] && side[i] >= 0)
        acc += 2.0L * (pc - (long double)pair(qi, qj, r2, rs[i], rs[j]));
      else
        acc += 2.0L * pc;
    }
    part[i] = acc;
  }
  for (auto v : part) d += v;
  if (RC) *RC = rc;
  if (Rsub) *Rsub = rs;
  return (double)d;
}

static void frame_energy(const Split& s, const std::vector<V3>& x, const Method& m, const SaParams& sa, bool acc,
                         FrameEnergy& f) {
  auto xr = gather(x, s.rec_atoms), xl = gather(x, s.lig_atoms);
  f.c = subsystem(s.complex, x, m, sa, acc);
  f.r = subsystem(s.rec, xr, m, sa, acc);
  f.l = subsystem(s.lig, xl, m, sa, acc);
  if (!acc) {  // binding.rs:401-404
    f.d_mm = f.c.mm - f.r.mm - f.l.mm;
    f.d_polar = f.c.polar - f.r.polar - f.l.polar;
    f.d_sa = f.c.sa - f.r.sa - f.l.sa;
    f.d_total = f.d_mm + f.d_polar + f.d_sa;
    return;
  }
  f.d_mm = delta_mm_exact(s, x);
  if (m.kind == 0)
    f.d_polar = delta_gb_exact(s, x, m.gb, nullptr, nullptr);
  else
    f.d_polar = f.c.polar - f.r.polar - f.l.polar;
  auto sc = sasa_per_atom(x, s.complex.radii, sa.probe, sa.n_points);
  auto sr = sasa_per_atom(xr, s.rec.radii, sa.probe, sa.n_points);
  auto sl = sasa_per_atom(xl, s.lig.radii, sa.probe, sa.n_points);
  long double ds = 0.0L;
  for (size_t k = 0; k < s.rec_atoms.size(); k++) ds += (long double)sc[s.rec_atoms[k]] - sr[k];
  for (size_t k = 0; k < s.lig_atoms.size(); k++) ds += (long double)sc[s.lig_atoms[k]] - sl[k];
  f.d_sa = (double)((long double)sa.surface_tension * ds - sa.offset);
  f.d_total = f.d_mm + f.d_polar + f.d_sa;
}

// decomposition.rs:210-410
static void decompose(const Split& s, const std::vector<V3>& x, const GbParams& gb, const SaParams& sa, bool acc,
                      std::vector<Residue>& rec_out, std::vector<Residue>& lig_out) {
  const Topology& C = s.complex;
  auto ar = C.atom_residue_indices();
  std::set<std::pair<size_t, size_t>> p14, ex;
  for (auto& d : C.dihedrals)
    if (!d.ignore_14) p14.insert({std::min(d.i, d.l), std::max(d.i, d.l)});
  size_t off = 0;
  for (size_t a = 0; a < C.n_atoms; a++) {
    size_t cnt = a < C.num_excluded.size() ? C.num_excluded[a] : 0;
    for (size_t k = 0; k < cnt; k++)
      if (off + k < C.excluded_list.size() && C.excluded_list[off + k] < C.n_atoms) {
        size_t b = C.excluded_list[off + k];
        ex.insert({std::min(a, b), std::max(a, b)});
      }
    off += cnt;
  }
  std::unordered_map<size_t, long double> rv, re, rg, rsa;
  std::unordered_map<size_t, double> fv, fe, fg, fsa;
  for (size_t ri : s.rec_atoms)
    for (size_t li : s.lig_atoms) {
      size_t i = std::min(ri, li), j = std::max(ri, li);
      double dx = x[ri].x - x[li].x, dy = x[ri].y - x[li].y, dz = x[ri].z - x[li].z;
      double r = std::sqrt(dx * dx + dy * dy + dz * dz);
      if (r < 1e-10) continue;
      int64_t idx = C.nb_index[C.n_types * C.type_idx[ri] + C.type_idx[li]];
      double A = idx < 1 ? 0.0 : C.lj_a[idx - 1], B = idx < 1 ? 0.0 : C.lj_b[idx - 1];
      double qi = C.charges_amber[ri], qj = C.charges_amber[li];
      double v, e;
      double r2 = r * r, r6 = r2 * r2 * r2, r12 = r6 * r6;
      if (p14.count({i, j})) {
        v = (A / r12 - B / r6) / C.scnb;
        e = qi * qj / r / C.scee;
      } else if (!ex.count({i, j})) {
        v = A / r12 - B / r6;
        e = qi * qj / r;
      } else {
        continue;
      }
      size_t a = ar[ri], b = ar[li];
      fv[a] += v * 0.5;
      fv[b] += v * 0.5;
      fe[a] += e * 0.5;
      fe[b] += e * 0.5;
      rv[a] += (long double)v * 0.5L;
      rv[b] += (long double)v * 0.5L;
      re[a] += (long double)e * 0.5L;
      re[b] += (long double)e * 0.5L;
    }
  auto xr = gather(x, s.rec_atoms), xl = gather(x, s.lig_atoms);
  std::vector<double> Rc = born_radii(C, x, gb, acc), Rr = born_radii(s.rec, xr, gb, acc),
                      Rl = born_radii(s.lig, xl, gb, acc);
  double total_dgb;
  if (acc) {
    total_dgb = delta_gb_exact(s, x, gb, nullptr, nullptr);
  } else {
    double ec = gb_energy_from_radii(C, x, gb, Rc, false), er = gb_energy_from_radii(s.rec, xr, gb, Rr, false),
           el = gb_energy_from_radii(s.lig, xl, gb, Rl, false);
    total_dgb = ec - er - el;
  }
  double f0 = -0.5 * (1.0 / gb.solute_dielectric - 1.0 / gb.solvent_dielectric);
  std::vector<double> w;
  double tw = 0.0;
  long double twl = 0.0L;
  for (size_t k = 0; k < s.rec_atoms.size(); k++) {
    double q = C.charges_amber[s.rec_atoms[k]];
    double a = f0 * q * q / Rc[s.rec_atoms[k]], b = f0 * q * q / Rr[k];
    w.push_back(std::fabs(a - b));
    tw += w.back();
    twl += w.back();
  }
  for (size_t k = 0; k < s.lig_atoms.size(); k++) {
    double q = C.charges_amber[s.lig_atoms[k]];
    double a = f0 * q * q / Rc[s.lig_atoms[k]], b = f0 * q * q / Rl[k];
    w.push_back(std::fabs(a - b));
    tw += w.back();
    twl += w.back();
  }
  if (tw > 1e-20) {
    std::vector<size_t> all = s.rec_atoms;
    all.insert(all.end(), s.lig_atoms.begin(), s.lig_atoms.end());
    for (size_t k = 0; k < all.size(); k++) {
      size_t r = ar[all[k]];
      fg[r] += total_dgb * (w[k] / tw);
      rg[r] += (long double)total_dgb * ((long double)w[k] / twl);
    }
  }
  auto sc = sasa_per_atom(x, C.radii, sa.probe, sa.n_points);
  auto sr = sasa_per_atom(xr, s.rec.radii, sa.probe, sa.n_points);
  auto sl = sasa_per_atom(xl, s.lig.radii, sa.probe, sa.n_points);
  for (size_t k = 0; k < s.rec_atoms.size(); k++) {
    size_t r = ar[s.rec_atoms[k]];
    double d = sc[s.rec_atoms[k]] - sr[k];
    fsa[r] += sa.surface_tension * d;
    rsa[r] += (long double)sa.surface_tension * d;
  }
  for (size_t k = 0; k < s.lig_atoms.size(); k++) {
    size_t r = ar[s.lig_atoms[k]];
    double d = sc[s.lig_atoms[k]] - sl[k];
    fsa[r] += sa.surface_tension * d;
    rsa[r] += (long double)sa.surface_tension * d;
  }
  auto get = [&](std::unordered_map<size_t, double>& F, std::unordered_map<size_t, long double>& L, size_t r) {
    if (acc) {
      auto it = L.find(r);
      return it == L.end() ? 0.0 : (double)it->second;
    }
    auto it = F.find(r);
    return it == F.end() ? 0.0 : it->second;
  };
  rec_out.clear();
  lig_out.clear();
  for (size_t r : s.rec_res_remapped)
    rec_out.push_back({r, get(fv, rv, r), get(fe, re, r), get(fg, rg, r), get(fsa, rsa, r)});
  for (size_t r : s.lig_res_remapped)
    lig_out.push_back({r, get(fv, rv, r), get(fe, re, r), get(fg, rg, r), get(fsa, rsa, r)});
}

}  // namespace orc

// ===========================================================================
// extern "C" surface (ctypes)
// ===========================================================================
using namespace orc;

extern "C" {

struct orc_gb_params {
  int32_t model;
  double solute_dielectric, solvent_dielectric, salt, temperature, offset, rgbmax, cutoff;
};
struct orc_sa_params {
  double surface_tension, offset, probe;
  int64_t n_points;
};
struct orc_pb_params {
  double grid_spacing, grid_buffer, solute_dielectric, solvent_dielectric, salt, temperature, probe, ion_radius,
      tolerance;
  int64_t max_iterations;
  double fillratio;
  int64_t fscale;
  double converged_rel_tol;  // > 0: converged solves (not the reference's schedule)
  int64_t converged_method;
};
// Flat topology description for hand-built topologies (the reference's
// unit tests build AmberTopology structs directly).
struct orc_topo_desc {
  int64_t n_atoms, n_residues, n_types;
  const int64_t* type_idx;
  const double* charges_amber;
  const double* radii;
  const double* screen;
  const int64_t* residue_pointers;
  int64_t n_bonds;
  const int64_t* bonds;  // i, j, type
  int64_t n_bond_types;
  const double* bond_k;
  const double* bond_req;
  int64_t n_angles;
  const int64_t* angles;  // i, j, k, type
  int64_t n_angle_types;
  const double* angle_k;
  const double* angle_teq;
  int64_t n_dihedrals;
  const int64_t* dihedrals;  // i, j, k, l, type, ignore_14
  int64_t n_dihedral_types;
  const double* dih_pk;
  const double* dih_pn;
  const double* dih_phase;
  const int64_t* num_excluded;
  int64_t n_excluded;
  const int64_t* excluded_list;  // -1 = placeholder
  double scee, scnb;
  int64_t n_lj;
  const double* lj_a;
  const double* lj_b;
  const int64_t* nb_index;  // n_types * n_types
};

static void seterr(char* buf, int len, const std::string& s) {
  if (buf && len > 0) {
    strncpy(buf, s.c_str(), len - 1);
    buf[len - 1] = 0;
  }
}
static GbParams gbp(const orc_gb_params* p) {
  GbParams g;
  if (!p) return g;
  g.model = p->model;
  g.solute_dielectric = p->solute_dielectric;
  g.solvent_dielectric = p->solvent_dielectric;
  g.salt = p->salt;
  g.temperature = p->temperature;
  g.offset = p->offset;
  g.rgbmax = p->rgbmax;
  g.cutoff = p->cutoff;
  return g;
}
static SaParams sap(const orc_sa_params* p) {
  SaParams s;
  if (!p) return s;
  s.surface_tension = p->surface_tension;
  s.offset = p->offset;
  s.probe = p->probe;
  s.n_points = (size_t)p->n_points;
  return s;
}
static PbParams pbp(const orc_pb_params* p) {
  PbParams b;
  if (!p) return b;
  b.grid_spacing = p->grid_spacing;
  b.grid_buffer = p->grid_buffer;
  b.solute_dielectric = p->solute_dielectric;
  b.solvent_dielectric = p->solvent_dielectric;
  b.salt = p->salt;
  b.temperature = p->temperature;
  b.probe = p->probe;
  b.ion_radius = p->ion_radius;
  b.tolerance = p->tolerance;
  b.max_iterations = (size_t)p->max_iterations;
  b.fillratio = p->fillratio;
  b.fscale = (size_t)p->fscale;
  b.converged_rel_tol = p->converged_rel_tol;
  b.converged_method = (int)p->converged_method;
  return b;
}
static std::vector<V3> coords(const double* xyz, size_t n) {
  std::vector<V3> v(n);
  for (size_t i = 0; i < n; i++) v[i] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
  return v;
}
static Topology* T(void* h) { return (Topology*)h; }

void* orc_topology_load(const char* path, char* err, int errlen) {
  Topology* t = new Topology();
  std::string e;
  if (!parse_prmtop(path, *t, e)) {
    seterr(err, errlen, e);
    delete t;
    return nullptr;
  }
  return t;
}

void* orc_topology_from_desc(const orc_topo_desc* d) {
  Topology* t = new Topology();
  t->n_atoms = d->n_atoms;
  t->n_residues = d->n_residues;
  t->n_types = d->n_types;
  for (int64_t i = 0; i < d->n_atoms; i++) {
    t->atom_names.push_back("X");
    t->type_idx.push_back(d->type_idx ? d->type_idx[i] : 0);
    double qa = d->charges_amber ? d->charges_amber[i] : 0.0;
    t->charges_amber.push_back(qa);
    t->charges.push_back(qa / 18.2223);
    t->radii.push_back(d->radii ? d->radii[i] : 0.0);
    t->screen.push_back(d->screen ? d->screen[i] : 0.0);
    t->masses.push_back(0.0);
  }
  for (int64_t r = 0; r < d->n_residues; r++) {
    t->residue_pointers.push_back(d->residue_pointers ? d->residue_pointers[r] : 0);
    t->residue_labels.push_back("RES");
  }
  for (int64_t b = 0; b < d->n_bonds; b++) {
    t->bonds.push_back({(size_t)d->bonds[3 * b], (size_t)d->bonds[3 * b + 1]});
    t->bond_types.push_back(d->bonds[3 * b + 2]);
  }
  t->bond_k.assign(d->bond_k, d->bond_k + d->n_bond_types);
  t->bond_req.assign(d->bond_req, d->bond_req + d->n_bond_types);
  for (int64_t a = 0; a < d->n_angles; a++)
    t->angles.push_back({(size_t)d->angles[4 * a], (size_t)d->angles[4 * a + 1], (size_t)d->angles[4 * a + 2],
                         (size_t)d->angles[4 * a + 3]});
  t->angle_k.assign(d->angle_k, d->angle_k + d->n_angle_types);
  t->angle_teq.assign(d->angle_teq, d->angle_teq + d->n_angle_types);
  for (int64_t k = 0; k < d->n_dihedrals; k++) {
    const int64_t* q = d->dihedrals + 6 * k;
    t->dihedrals.push_back({(size_t)q[0], (size_t)q[1], (size_t)q[2], (size_t)q[3], (size_t)q[4], q[5] != 0});
  }
  t->dih_pk.assign(d->dih_pk, d->dih_pk + d->n_dihedral_types);
  t->dih_pn.assign(d->dih_pn, d->dih_pn + d->n_dihedral_types);
  t->dih_phase.assign(d->dih_phase, d->dih_phase + d->n_dihedral_types);
  for (int64_t i = 0; i < d->n_atoms; i++) t->num_excluded.push_back(d->num_excluded ? d->num_excluded[i] : 0);
  for (int64_t k = 0; k < d->n_excluded; k++)
    t->excluded_list.push_back(d->excluded_list[k] < 0 ? SIZE_MAX : (size_t)d->excluded_list[k]);
  t->scee = d->scee;
  t->scnb = d->scnb;
  t->lj_a.assign(d->lj_a, d->lj_a + d->n_lj);
  t->lj_b.assign(d->lj_b, d->lj_b + d->n_lj);
  t->nb_index.assign(d->nb_index, d->nb_index + d->n_types * d->n_types);
  return t;
}

void orc_topology_free(void* h) { delete T(h); }
int64_t orc_topology_n_atoms(void* h) { return (int64_t)T(h)->n_atoms; }
int64_t orc_topology_n_residues(void* h) { return (int64_t)T(h)->n_residues; }

void orc_topology_arrays(void* h, double* charges, double* charges_amber, double* radii, double* screen,
                         int64_t* type_idx, int64_t* res_ptr) {
  Topology* t = T(h);
  for (size_t i = 0; i < t->n_atoms; i++) {
    charges[i] = t->charges[i];
    charges_amber[i] = t->charges_amber[i];
    radii[i] = t->radii[i];
    screen[i] = t->screen[i];
    type_idx[i] = (int64_t)t->type_idx[i];
  }
  for (size_t r = 0; r < t->n_residues; r++) res_ptr[r] = (int64_t)t->residue_pointers[r];
}

void orc_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}
int orc_get_threads(void) { return omp_get_max_threads(); }

double orc_kappa(double salt, double eps, double temp) { return kappa(salt, eps, temp); }

double orc_gb_energy(void* h, const double* xyz_A, const orc_gb_params* p, int accurate, double* born_out) {
  Topology* t = T(h);
  auto x = coords(xyz_A, t->n_atoms);
  GbParams g = gbp(p);
  auto R = born_radii(*t, x, g, accurate != 0);
  if (born_out) memcpy(born_out, R.data(), sizeof(double) * R.size());
  return gb_energy_from_radii(*t, x, g, R, accurate != 0);
}

// compute_gb_energy_from_radii with given radii (gb_energy.rs:283-355), the
// energy compute_gb_energy_cached returns on a cache hit (gb_energy.rs:372-387).
double orc_gb_energy_from_radii(void* h, const double* xyz_A, const orc_gb_params* p, const double* radii) {
  Topology* t = T(h);
  auto x = coords(xyz_A, t->n_atoms);
  std::vector<double> r(radii, radii + t->n_atoms);
  return gb_energy_from_radii(*t, x, gbp(p), r, false);
}

void orc_mm_energy(void* h, const double* xyz_A, int accurate, double* out7) {
  Topology* t = T(h);
  MmEnergy e = mm_energy(*t, coords(xyz_A, t->n_atoms), accurate != 0);
  double v[7] = {e.bond, e.angle, e.dihedral, e.vdw, e.elec, e.vdw_14, e.elec_14};
  memcpy(out7, v, sizeof(v));
}

double orc_sa_energy(void* h, const double* xyz_A, const orc_sa_params* p, double* total_sasa, double* per_atom) {
  Topology* t = T(h);
  SaParams s = sap(p);
  auto v = sasa_per_atom(coords(xyz_A, t->n_atoms), t->radii, s.probe, s.n_points);
  double tot = 0.0;
  for (double a : v) tot += a;
  if (per_atom) memcpy(per_atom, v.data(), sizeof(double) * v.size());
  if (total_sasa) *total_sasa = tot;
  return s.surface_tension * tot + s.offset;
}

// Raw SASA on arrays (sasa.rs SASAEngine): per-atom areas.
void orc_sasa_raw(int64_t n, const double* xyz, const double* radii, double probe, int64_t n_points,
                  double* per_atom) {
  std::vector<double> r(radii, radii + n);
  auto v = sasa_per_atom(coords(xyz, n), r, probe, (size_t)n_points);
  memcpy(per_atom, v.data(), sizeof(double) * n);
}

void orc_fibonacci(int64_t n, double* out) {
  auto v = fibonacci_sphere((size_t)n);
  for (size_t i = 0; i < v.size(); i++) {
    out[3 * i] = v[i].x;
    out[3 * i + 1] = v[i].y;
    out[3 * i + 2] = v[i].z;
  }
}

double orc_pb_energy(void* h, const double* xyz_A, const orc_pb_params* p, int64_t* iters2, double* res2,
                     int32_t* conv2, int32_t* dims3) {
  Topology* t = T(h);
  PbDiag d;
  double e = pb_energy(coords(xyz_A, t->n_atoms), t->charges, t->radii, pbp(p), &d);
  if (iters2) {
    iters2[0] = d.iterations[0];
    iters2[1] = d.iterations[1];
  }
  if (res2) {
    res2[0] = d.residual[0];
    res2[1] = d.residual[1];
  }
  if (conv2) {
    conv2[0] = d.converged[0];
    conv2[1] = d.converged[1];
  }
  if (dims3)
    for (int k = 0; k < 3; k++) dims3[k] = d.dims[k];
  return e;
}

// PB on raw arrays (charges in e), used by the Born-ion known-answer test.
double orc_pb_energy_raw(int64_t n, const double* xyz, const double* q_e, const double* radii,
                         const orc_pb_params* p) {
  std::vector<double> q(q_e, q_e + n), r(radii, radii + n);
  return pb_energy(coords(xyz, n), q, r, pbp(p), nullptr);
}

// Grid set-up maps of one solve (for exact map comparisons): dims/origin out,
// arrays sized by a previous call with nulls (returns the point count).
int64_t orc_pb_maps(int64_t n, const double* xyz, const double* q_e, const double* radii, double h, double buffer,
                    double probe, double ion_radius, double eps_in, double eps_out, double kappa_bulk,
                    double eps_solvent, int use_ionic, int64_t* dims3, double* origin3, double* charge,
                    uint8_t* inside, double* ex, double* ey, double* ez, double* k2, double* boundary_phi) {
  std::vector<double> q(q_e, q_e + n), r(radii, radii + n);
  auto x = coords(xyz, n);
  Grid g = auto_grid(x, h, buffer);
  for (int k = 0; k < 3; k++) {
    dims3[k] = (int64_t)g.dims[k];
    origin3[k] = g.origin[k];
  }
  if (!charge) return (int64_t)g.len();
  auto c = map_charges(g, x, q);
  memcpy(charge, c.data(), sizeof(double) * c.size());
  if (inside) {
    auto in = inside_ses(g, x, r, probe);
    memcpy(inside, in.data(), in.size());
  }
  Diel D = assign_dielectrics(g, x, r, probe, eps_in, eps_out);
  memcpy(ex, D.ex.data(), sizeof(double) * D.ex.size());
  memcpy(ey, D.ey.data(), sizeof(double) * D.ey.size());
  memcpy(ez, D.ez.data(), sizeof(double) * D.ez.size());
  std::vector<double> K =
      use_ionic ? assign_kappa(g, x, r, ion_radius, kappa_bulk, eps_solvent) : std::vector<double>(g.len(), 0.0);
  memcpy(k2, K.data(), sizeof(double) * K.size());
  std::vector<double> phi(g.len(), 0.0);
  set_dh_boundary(phi, g, x, q, use_ionic ? kappa_bulk : 0.0, eps_out);
  memcpy(boundary_phi, phi.data(), sizeof(double) * phi.size());
  return (int64_t)g.len();
}

// Multigrid solve on given maps (DH boundary from atoms): potential out.
int64_t orc_pb_solve(int64_t n, const double* xyz, const double* q_e, const int64_t* dims3, const double* origin3,
                     double h, const double* charge, const double* ex, const double* ey, const double* ez,
                     const double* k2, double kappa_bc, double eps_bc, double tol, int64_t max_iter, double* phi_out,
                     double* residual, int32_t* converged, double* energy) {
  Grid g;
  for (int k = 0; k < 3; k++) {
    g.dims[k] = (size_t)dims3[k];
    g.origin[k] = origin3[k];
    g.h[k] = h;
  }
  size_t N = g.len();
  std::vector<double> q(q_e, q_e + n), rho(charge, charge + N), K(k2, k2 + N);
  Diel D;
  D.ex.assign(ex, ex + N);
  D.ey.assign(ey, ey + N);
  D.ez.assign(ez, ez + N);
  BC bc;
  bc.kind = 1;
  auto x = coords(xyz, n);
  SolveResult R = solve_multigrid(g, rho, D, K, bc, x, q, kappa_bc, eps_bc, tol, (size_t)max_iter);
  memcpy(phi_out, R.phi.data(), sizeof(double) * N);
  if (residual) *residual = R.residual;
  if (converged) *converged = R.converged;
  if (energy) *energy = elec_energy(g, R.phi, x, q);
  return (int64_t)R.iterations;
}

// restrict/prolong known-answer (pb_solver.rs:1260-1283): 9^3 constant 3.0.
void orc_restrict_prolong_constant(double value, double* coarse_out125, double* fine_out729) {
  size_t fd[3] = {9, 9, 9}, cd[3] = {5, 5, 5};
  std::vector<double> f(729, value), c(125, 0.0), fo(729, 0.0);
  restrict_into(f.data(), fd, c.data(), cd, 1.0);
  prolongate_add(c.data(), cd, fo.data(), fd);
  memcpy(coarse_out125, c.data(), sizeof(double) * 125);
  memcpy(fine_out729, fo.data(), sizeof(double) * 729);
}

// Total charge after spreading (pb_grid.rs:1013-1025 known-answer).
double orc_charge_total(int64_t n, const double* xyz, const double* q_e, double h, double buffer) {
  std::vector<double> q(q_e, q_e + n);
  auto x = coords(xyz, n);
  Grid g = auto_grid(x, h, buffer);
  auto c = map_charges(g, x, q);
  double s = 0.0;
  for (double v : c) s += v;
  return s * g.h[0] * g.h[1] * g.h[2];
}

static bool split_from(void* h, const int64_t* rr, int64_t nr, const int64_t* lr, int64_t nl, Split& s,
                       char* err, int errlen) {
  std::vector<size_t> R(rr, rr + nr), L(lr, lr + nl);
  std::string e;
  if (!make_split(*T(h), R, L, s, e)) {
    seterr(err, errlen, e);
    return false;
  }
  return true;
}

// One frame of the binding workflow (binding.rs:333-415, 749-786).
// out13 = c.mm c.polar c.sa r.mm r.polar r.sa l.mm l.polar l.sa d_mm d_polar d_sa d_total
int orc_binding_frame(void* h, const double* xyz_A, const int64_t* rr, int64_t nr, const int64_t* lr, int64_t nl,
                      int method, const orc_gb_params* gb, const orc_pb_params* pb, const orc_sa_params* sa,
                      int accurate, double* out13, char* err, int errlen) {
  Split s;
  if (!split_from(h, rr, nr, lr, nl, s, err, errlen)) return 1;
  std::vector<V3> x = coords(xyz_A, T(h)->n_atoms);
  if (!s.complex_atoms.empty()) x = gather(x, s.complex_atoms);
  Method m;
  m.kind = method;
  m.gb = gbp(gb);
  m.pb = pbp(pb);
  FrameEnergy f;
  frame_energy(s, x, m, sap(sa), accurate != 0, f);
  double v[13] = {f.c.mm, f.c.polar, f.c.sa, f.r.mm, f.r.polar, f.r.sa, f.l.mm,
                  f.l.polar, f.l.sa, f.d_mm, f.d_polar, f.d_sa, f.d_total};
  memcpy(out13, v, sizeof(v));
  return 0;
}

// Many frames (frames_A: F x n_atoms x 3 in the topology's atom order),
// parallel over frames as binding.rs:520-539 does when the batch has at least
// as many frames as threads; otherwise frames run in order with the inner
// loops parallel.
int orc_binding_frames(void* h, const double* frames_A, int64_t F, const int64_t* rr, int64_t nr,
                       const int64_t* lr, int64_t nl, int method, const orc_gb_params* gb, const orc_pb_params* pb,
                       const orc_sa_params* sa, int accurate, double* out13F, char* err, int errlen) {
  Split s;
  if (!split_from(h, rr, nr, lr, nl, s, err, errlen)) return 1;
  size_t n = T(h)->n_atoms;
  Method m;
  m.kind = method;
  m.gb = gbp(gb);
  m.pb = pbp(pb);
  SaParams sp = sap(sa);
  int nt = omp_get_max_threads();
  auto one = [&](int64_t f) {
    std::vector<V3> x = coords(frames_A + (size_t)f * n * 3, n);
    if (!s.complex_atoms.empty()) x = gather(x, s.complex_atoms);
    FrameEnergy e;
    frame_energy(s, x, m, sp, accurate != 0, e);
    double v[13] = {e.c.mm, e.c.polar, e.c.sa, e.r.mm, e.r.polar, e.r.sa, e.l.mm,
                    e.l.polar, e.l.sa, e.d_mm, e.d_polar, e.d_sa, e.d_total};
    memcpy(out13F + 13 * f, v, sizeof(v));
  };
  if (F >= nt) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t f = 0; f < F; f++) one(f);
  } else {
    for (int64_t f = 0; f < F; f++) one(f);
  }
  return 0;
}

// decomposition.rs:75-92; out arrays are n_res x 4 (vdw, elec, polar, sa).
int orc_decompose(void* h, const double* xyz_A, const int64_t* rr, int64_t nr, const int64_t* lr, int64_t nl,
                  const orc_gb_params* gb, const orc_sa_params* sa, int accurate, double* rec_out, double* lig_out,
                  char* err, int errlen) {
  Split s;
  if (!split_from(h, rr, nr, lr, nl, s, err, errlen)) return 1;
  std::vector<V3> x = coords(xyz_A, T(h)->n_atoms);
  if (!s.complex_atoms.empty()) x = gather(x, s.complex_atoms);
  std::vector<Residue> R, L;
  decompose(s, x, gbp(gb), sap(sa), accurate != 0, R, L);
  for (size_t k = 0; k < R.size(); k++) {
    rec_out[4 * k] = R[k].vdw;
    rec_out[4 * k + 1] = R[k].elec;
    rec_out[4 * k + 2] = R[k].polar;
    rec_out[4 * k + 3] = R[k].sa;
  }
  for (size_t k = 0; k < L.size(); k++) {
    lig_out[4 * k] = L[k].vdw;
    lig_out[4 * k + 1] = L[k].elec;
    lig_out[4 * k + 2] = L[k].polar;
    lig_out[4 * k + 3] = L[k].sa;
  }
  return 0;
}

// DCD reader (dcd.rs): returns frame count, fills nm coordinates if out given.
int64_t orc_read_dcd(const char* path, double* out_nm, int64_t max_values, int64_t* n_atoms, char* err, int errlen) {
  std::vector<std::vector<V3>> fr;
  std::string e;
  if (!read_dcd(path, fr, e)) {
    seterr(err, errlen, e);
    return -1;
  }
  *n_atoms = fr.empty() ? 0 : (int64_t)fr[0].size();
  if (out_nm) {
    int64_t k = 0;
    for (auto& f : fr)
      for (auto& v : f) {
        if (k + 3 > max_values) break;
        out_nm[k++] = v.x;
        out_nm[k++] = v.y;
        out_nm[k++] = v.z;
      }
  }
  return (int64_t)fr.size();
}

}  // extern "C"
