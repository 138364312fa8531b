// CPU restatement of the reference hot path: topology, trajectory, GB, MM, SA.
// TEST INFRASTRUCTURE ONLY (see oracle.hpp).  Each function cites the
// reference file:line it restates (paths relative to the reference project).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <map>
#include <sstream>
#include <unordered_map>

#include "oracle.hpp"

namespace orc {

static const double PI = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// prmtop parsing: core/src/amber/prmtop.rs:331-733
// ---------------------------------------------------------------------------
namespace {
struct Sections {
  std::map<std::string, std::vector<std::string>> data;
  const std::vector<std::string>* get(const std::string& k) const {
    auto it = data.find(k);
    return it == data.end() ? nullptr : &it->second;
  }
};

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) a++;
  while (b > a && isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

bool ints(const Sections& s, const std::string& flag, std::vector<int64_t>& out, std::string& err) {
  auto lines = s.get(flag);
  if (!lines) {
    err = "Missing section: " + flag;
    return false;
  }
  out.clear();
  for (auto& ln : *lines) {
    std::istringstream is(ln);
    std::string w;
    while (is >> w) {
      char* end = nullptr;
      long long v = strtoll(w.c_str(), &end, 10);
      if (*end != 0) {
        err = "Failed to parse integer in " + flag;
        return false;
      }
      out.push_back(v);
    }
  }
  return true;
}

bool floats(const Sections& s, const std::string& flag, std::vector<double>& out, std::string& err) {
  auto lines = s.get(flag);
  if (!lines) {
    err = "Missing section: " + flag;
    return false;
  }
  out.clear();
  for (auto& ln : *lines) {
    std::istringstream is(ln);
    std::string w;
    while (is >> w) {
      char* end = nullptr;
      double v = strtod(w.c_str(), &end);
      if (*end != 0) {
        err = "Failed to parse float in " + flag;
        return false;
      }
      out.push_back(v);
    }
  }
  return true;
}

bool strings(const Sections& s, const std::string& flag, size_t width, std::vector<std::string>& out,
             std::string& err) {
  auto lines = s.get(flag);
  if (!lines) {
    err = "Missing section: " + flag;
    return false;
  }
  out.clear();
  for (auto& ln : *lines) {
    size_t pos = 0;
    while (pos + width <= ln.size()) {
      out.push_back(trim(ln.substr(pos, width)));
      pos += width;
    }
    if (pos < ln.size()) {
      std::string r = trim(ln.substr(pos));
      if (!r.empty()) out.push_back(r);
    }
  }
  return true;
}
}  // namespace

std::vector<size_t> Topology::atom_residue_indices() const {
  // prmtop.rs:120-132
  std::vector<size_t> r(n_atoms, 0);
  for (size_t k = 0; k < n_residues; k++) {
    size_t a = residue_pointers[k];
    size_t b = (k + 1 < n_residues) ? residue_pointers[k + 1] : n_atoms;
    for (size_t i = a; i < b; i++) r[i] = k;
  }
  return r;
}

bool Topology::build_selection(const std::vector<size_t>& residues, std::vector<size_t>& atoms,
                               std::string& err) const {
  // prmtop.rs:165-204
  for (size_t r : residues) {
    if (r >= n_residues) {
      err = "Residue index " + std::to_string(r) + " out of range (0-" +
            std::to_string(n_residues - 1) + ")";
      return false;
    }
  }
  atoms.clear();
  for (size_t r : residues) {
    size_t a = residue_pointers[r];
    size_t b = (r + 1 < n_residues) ? residue_pointers[r + 1] : n_atoms;
    for (size_t i = a; i < b; i++) atoms.push_back(i);
  }
  return true;
}

bool parse_prmtop(const std::string& path, Topology& t, std::string& err) {
  std::ifstream f(path);
  if (!f) {
    err = "Failed to open prmtop file: " + path;
    return false;
  }
  Sections s;
  std::string line, flag;
  bool have = false;
  std::vector<std::string> cur;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.rfind("%FLAG", 0) == 0) {
      if (have) s.data[flag] = cur;
      cur.clear();
      flag = trim(line.substr(5));
      have = true;
    } else if (line.rfind("%FORMAT", 0) == 0 || line.rfind("%VERSION", 0) == 0 ||
               line.rfind("%COMMENT", 0) == 0) {
      continue;
    } else if (have) {
      cur.push_back(line);
    }
  }
  if (have) s.data[flag] = cur;

  std::vector<int64_t> ptr;
  if (!ints(s, "POINTERS", ptr, err)) return false;
  if (ptr.size() < 12) {
    err = "POINTERS section too short";
    return false;
  }
  if (ptr[0] < 0 || ptr[1] < 0 || ptr[11] < 0) {
    err = "POINTERS contains negative values";
    return false;
  }
  t.n_atoms = (size_t)ptr[0];
  t.n_types = (size_t)ptr[1];
  t.n_residues = (size_t)ptr[11];
  if (!strings(s, "ATOM_NAME", 4, t.atom_names, err)) return false;
  if (t.atom_names.size() < t.n_atoms) {
    err = "ATOM_NAME too short";
    return false;
  }
  t.atom_names.resize(t.n_atoms);
  std::vector<int64_t> ti;
  if (!ints(s, "ATOM_TYPE_INDEX", ti, err)) return false;
  t.type_idx.clear();
  for (size_t i = 0; i < ti.size() && i < t.n_atoms; i++) {
    if (ti[i] < 1) {
      err = "Invalid ATOM_TYPE_INDEX";
      return false;
    }
    t.type_idx.push_back((size_t)(ti[i] - 1));
  }
  std::vector<double> q;
  if (!floats(s, "CHARGE", q, err)) return false;
  t.charges.clear();
  t.charges_amber.clear();
  for (size_t i = 0; i < q.size() && i < t.n_atoms; i++) {
    t.charges.push_back(q[i] / 18.2223);
    t.charges_amber.push_back(q[i]);
  }
  if (!strings(s, "RESIDUE_LABEL", 4, t.residue_labels, err)) return false;
  if (t.residue_labels.size() > t.n_residues) t.residue_labels.resize(t.n_residues);
  std::vector<int64_t> rp;
  if (!ints(s, "RESIDUE_POINTER", rp, err)) return false;
  t.residue_pointers.clear();
  for (size_t i = 0; i < rp.size() && i < t.n_residues; i++) {
    if (rp[i] < 1) {
      err = "Invalid RESIDUE_POINTER";
      return false;
    }
    t.residue_pointers.push_back((size_t)(rp[i] - 1));
  }
  if (!floats(s, "LENNARD_JONES_ACOEF", t.lj_a, err)) return false;
  if (!floats(s, "LENNARD_JONES_BCOEF", t.lj_b, err)) return false;
  if (!ints(s, "NONBONDED_PARM_INDEX", t.nb_index, err)) return false;
  if (t.nb_index.size() < t.n_types * t.n_types && t.n_types > 0) {
    err = "NONBONDED_PARM_INDEX out of bounds";
    return false;
  }
  std::string e2;
  std::vector<int64_t> raw;
  t.bonds.clear();
  t.bond_types.clear();
  for (const char* sec : {"BONDS_INC_HYDROGEN", "BONDS_WITHOUT_HYDROGEN"}) {
    if (!ints(s, sec, raw, e2)) continue;
    for (size_t k = 0; k + 3 <= raw.size(); k += 3) {
      if (raw[k] < 0 || raw[k + 1] < 0 || raw[k + 2] < 1) continue;
      t.bonds.push_back({(size_t)(raw[k] / 3), (size_t)(raw[k + 1] / 3)});
      t.bond_types.push_back((size_t)(raw[k + 2] - 1));
    }
  }
  auto opt = [&](const char* sec, std::vector<double>& v, double dflt, size_t n) {
    if (!floats(s, sec, v, e2)) v.assign(n, dflt);
  };
  opt("MASS", t.masses, 0.0, t.n_atoms);
  opt("RADII", t.radii, 0.0, t.n_atoms);
  opt("SCREEN", t.screen, 0.0, t.n_atoms);
  opt("BOND_FORCE_CONSTANT", t.bond_k, 0.0, 0);
  opt("BOND_EQUIL_VALUE", t.bond_req, 0.0, 0);
  opt("ANGLE_FORCE_CONSTANT", t.angle_k, 0.0, 0);
  opt("ANGLE_EQUIL_VALUE", t.angle_teq, 0.0, 0);
  opt("DIHEDRAL_FORCE_CONSTANT", t.dih_pk, 0.0, 0);
  opt("DIHEDRAL_PERIODICITY", t.dih_pn, 0.0, 0);
  opt("DIHEDRAL_PHASE", t.dih_phase, 0.0, 0);
  t.angles.clear();
  for (const char* sec : {"ANGLES_INC_HYDROGEN", "ANGLES_WITHOUT_HYDROGEN"}) {
    if (!ints(s, sec, raw, e2)) continue;
    for (size_t k = 0; k + 4 <= raw.size(); k += 4) {
      if (raw[k] < 0 || raw[k + 1] < 0 || raw[k + 2] < 0 || raw[k + 3] < 1) continue;
      t.angles.push_back({(size_t)(raw[k] / 3), (size_t)(raw[k + 1] / 3), (size_t)(raw[k + 2] / 3),
                          (size_t)(raw[k + 3] - 1)});
    }
  }
  t.dihedrals.clear();
  for (const char* sec : {"DIHEDRALS_INC_HYDROGEN", "DIHEDRALS_WITHOUT_HYDROGEN"}) {
    if (!ints(s, sec, raw, e2)) continue;
    for (size_t k = 0; k + 5 <= raw.size(); k += 5) {
      if (raw[k + 4] < 1) continue;
      Topology::Dihedral d;
      d.i = (size_t)(std::llabs(raw[k]) / 3);
      d.j = (size_t)(std::llabs(raw[k + 1]) / 3);
      d.k = (size_t)(std::llabs(raw[k + 2]) / 3);
      d.l = (size_t)(std::llabs(raw[k + 3]) / 3);
      d.t = (size_t)(raw[k + 4] - 1);
      d.ignore_14 = raw[k + 2] < 0 || raw[k + 3] < 0;
      t.dihedrals.push_back(d);
    }
  }
  t.num_excluded.clear();
  if (ints(s, "NUMBER_EXCLUDED_ATOMS", raw, e2))
    for (auto v : raw) t.num_excluded.push_back((size_t)v);
  t.excluded_list.clear();
  if (ints(s, "EXCLUDED_ATOMS_LIST", raw, e2))
    for (auto v : raw) t.excluded_list.push_back(v > 0 ? (size_t)(v - 1) : SIZE_MAX);
  std::vector<double> sc;
  t.scee = (floats(s, "SCEE_SCALE_FACTOR", sc, e2) && !sc.empty()) ? sc[0] : 1.2;
  t.scnb = (floats(s, "SCNB_SCALE_FACTOR", sc, e2) && !sc.empty()) ? sc[0] : 2.0;
  return true;
}

// subsystem.rs:22-169
Topology extract_subtopology(const Topology& t, const std::vector<size_t>& atoms) {
  Topology s;
  std::unordered_map<size_t, size_t> o2n;
  for (size_t k = 0; k < atoms.size(); k++) o2n[atoms[k]] = k;
  s.n_atoms = atoms.size();
  s.n_types = t.n_types;
  for (size_t a : atoms) {
    s.atom_names.push_back(t.atom_names.size() > a ? t.atom_names[a] : "");
    s.type_idx.push_back(t.type_idx[a]);
    s.charges.push_back(t.charges[a]);
    s.charges_amber.push_back(t.charges_amber[a]);
    s.masses.push_back(t.masses.size() > a ? t.masses[a] : 0.0);
    s.radii.push_back(t.radii[a]);
    s.screen.push_back(t.screen[a]);
  }
  auto ar = t.atom_residue_indices();
  bool have_last = false;
  size_t last = 0;
  for (size_t k = 0; k < atoms.size(); k++) {
    size_t r = ar[atoms[k]];
    if (!have_last || last != r) {
      s.residue_labels.push_back(t.residue_labels.size() > r ? t.residue_labels[r] : "");
      s.residue_pointers.push_back(k);
      last = r;
      have_last = true;
    }
  }
  s.n_residues = s.residue_labels.size();
  for (size_t b = 0; b < t.bonds.size(); b++) {
    auto ia = o2n.find(t.bonds[b].first), ib = o2n.find(t.bonds[b].second);
    if (ia != o2n.end() && ib != o2n.end()) {
      s.bonds.push_back({ia->second, ib->second});
      s.bond_types.push_back(t.bond_types[b]);
    }
  }
  for (auto& a : t.angles) {
    auto i = o2n.find(a.i), j = o2n.find(a.j), k = o2n.find(a.k);
    if (i != o2n.end() && j != o2n.end() && k != o2n.end())
      s.angles.push_back({i->second, j->second, k->second, a.t});
  }
  for (auto& d : t.dihedrals) {
    auto i = o2n.find(d.i), j = o2n.find(d.j), k = o2n.find(d.k), l = o2n.find(d.l);
    if (i != o2n.end() && j != o2n.end() && k != o2n.end() && l != o2n.end())
      s.dihedrals.push_back({i->second, j->second, k->second, l->second, d.t, d.ignore_14});
  }
  s.num_excluded.assign(s.n_atoms, 0);
  size_t off = 0;
  for (size_t i = 0; i < t.n_atoms; i++) {
    size_t cnt = i < t.num_excluded.size() ? t.num_excluded[i] : 0;
    auto ni = o2n.find(i);
    if (ni != o2n.end()) {
      size_t c = 0;
      for (size_t k = 0; k < cnt; k++) {
        if (off + k < t.excluded_list.size()) {
          auto nj = o2n.find(t.excluded_list[off + k]);
          if (nj != o2n.end()) {
            s.excluded_list.push_back(nj->second);
            c++;
          }
        }
      }
      s.num_excluded[ni->second] = c;
    }
    off += cnt;
  }
  s.scee = t.scee;
  s.scnb = t.scnb;
  s.bond_k = t.bond_k;
  s.bond_req = t.bond_req;
  s.angle_k = t.angle_k;
  s.angle_teq = t.angle_teq;
  s.dih_pk = t.dih_pk;
  s.dih_pn = t.dih_pn;
  s.dih_phase = t.dih_phase;
  s.lj_a = t.lj_a;
  s.lj_b = t.lj_b;
  s.nb_index = t.nb_index;
  return s;
}

// ---------------------------------------------------------------------------
// DCD: core/src/trajectory/dcd.rs:217-444 (little/big endian, optional cell)
// ---------------------------------------------------------------------------
bool read_dcd(const std::string& path, std::vector<std::vector<V3>>& frames, std::string& err) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) {
    err = "Failed to open DCD file: " + path;
    return false;
  }
  std::vector<unsigned char> buf;
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  buf.resize(sz);
  if (sz > 0 && fread(buf.data(), 1, sz, f) != (size_t)sz) {
    fclose(f);
    err = "short read";
    return false;
  }
  fclose(f);
  size_t pos = 0;
  bool be = false;
  auto rd32 = [&](int32_t& v) {
    if (pos + 4 > buf.size()) return false;
    uint32_t u;
    memcpy(&u, &buf[pos], 4);
    if (be) u = __builtin_bswap32(u);
    memcpy(&v, &u, 4);
    pos += 4;
    return true;
  };
  auto rdf32 = [&](float& v) {  // coordinates are read little-endian (dcd.rs:152-159)
    if (pos + 4 > buf.size()) return false;
    memcpy(&v, &buf[pos], 4);
    pos += 4;
    return true;
  };
  if (buf.size() < 4) {
    err = "Failed to read block size";
    return false;
  }
  int32_t le;
  memcpy(&le, &buf[0], 4);
  if (le != 84) {
    be = true;
    int32_t t0;
    if (!rd32(t0) || t0 != 84) {
      err = "Invalid DCD header";
      return false;
    }
    pos = 0;
  }
  int32_t b1 = 0, nfr = 0, tmp = 0;
  if (!rd32(b1) || b1 != 84) {
    err = "Invalid DCD header size";
    return false;
  }
  if (pos + 4 > buf.size() || memcmp(&buf[pos], "CORD", 4) != 0) {
    err = "Invalid DCD magic";
    return false;
  }
  pos += 4;
  if (!rd32(nfr) || nfr < 0) {
    err = "Invalid number of frames";
    return false;
  }
  for (int k = 0; k < 8; k++) rd32(tmp);
  pos += 4;  // timestep f32
  int32_t cell = 0;
  rd32(cell);
  pos += 32;
  rd32(tmp);  // charmm version
  rd32(tmp);  // block end
  int32_t b2 = 0, nt = 0;
  rd32(b2);
  rd32(nt);
  if (b2 < 4 || nt < 0 || 4 + nt * 80 > b2) {
    err = "Invalid title block";
    return false;
  }
  pos += (size_t)b2 - 4;
  rd32(tmp);
  rd32(tmp);
  int32_t na = 0;
  if (!rd32(na) || na < 0) {
    err = "Invalid number of atoms";
    return false;
  }
  rd32(tmp);
  frames.clear();
  for (int fr = 0; fr < nfr; fr++) {
    if (cell) pos += 4 + 48 + 4;
    std::vector<float> xyz[3];
    for (int d = 0; d < 3; d++) {
      int32_t m;
      if (!rd32(m)) {
        err = "Failed to read i32";
        return false;
      }
      xyz[d].resize(na);
      for (int i = 0; i < na; i++)
        if (!rdf32(xyz[d][i])) {
          err = "Failed to read f32";
          return false;
        }
      rd32(m);
    }
    std::vector<V3> fr_nm(na);
    for (int i = 0; i < na; i++)
      fr_nm[i] = {(double)xyz[0][i] * 0.1, (double)xyz[1][i] * 0.1, (double)xyz[2][i] * 0.1};
    frames.push_back(std::move(fr_nm));
  }
  return true;
}

// ---------------------------------------------------------------------------
// GB: crates/mmpbsa/src/gb_energy.rs
// ---------------------------------------------------------------------------
double kappa(double salt, double eps, double temperature) {
  // gb_energy.rs:126-139 (identical copy at pb_energy.rs:78-86)
  if (salt <= 0.0) return 0.0;
  double kb = 0.00198688, na = 6.022e-4;
  double factor = 8.0 * PI * 332.0522 * na;
  return std::sqrt(factor * salt / (eps * kb * temperature));
}

// One ordered-pair HCT descreening term, gb_energy.rs:177-212.  Returns false
// when the pair is skipped.
static inline bool hct_term(double r2, double rho_i, double sj, double& out) {
  double r = std::sqrt(r2);
  if (r == 0.0) return false;
  if (rho_i >= r + sj) return false;
  double u = r + sj;
  double l = (rho_i > std::fabs(r - sj)) ? rho_i : std::fabs(r - sj);
  double l_inv = 1.0 / l, u_inv = 1.0 / u;
  double contrib = 0.5 * (l_inv - u_inv + 0.25 * (u_inv * u_inv - l_inv * l_inv) * (r - sj * sj / r) +
                          std::log(l / u) / (2.0 * r));
  if (rho_i < sj - r)
    out = contrib + 2.0 * (1.0 / rho_i - l_inv);
  else
    out = contrib;
  return true;
}

// gb_energy.rs:219-255, the HCT / OBC conversion of psi to a Born radius.
static inline double radius_from_psi(double psi, double rho_i, double radius_i, const GbParams& p) {
  double alpha = 1.0, beta = 0.0, gamma = 0.0;
  if (p.model == 1) {
    alpha = 0.8;
    beta = 0.0;
    gamma = 2.909125;
  } else if (p.model == 2) {
    alpha = 1.0;
    beta = 0.8;
    gamma = 4.85;
  }
  double R;
  if (p.model == 0) {
    double inv_r = 1.0 / rho_i - psi;
    R = inv_r > 0.0 ? 1.0 / inv_r : p.rgbmax;
  } else {
    double pr = psi * rho_i, p2 = pr * pr, p3 = p2 * pr;
    double tv = std::tanh(alpha * pr - beta * p2 + gamma * p3);
    double inv_r = 1.0 / rho_i - tv / radius_i;
    R = inv_r > 0.0 ? 1.0 / inv_r : p.rgbmax;
  }
  if (R > p.rgbmax) R = p.rgbmax;
  return R;
}

// gb_energy.rs:144-258
std::vector<double> born_radii(const Topology& t, const std::vector<V3>& x, const GbParams& p,
                               bool accurate) {
  size_t n = t.n_atoms;
  std::vector<double> rho(n), R(n);
  for (size_t i = 0; i < n; i++) rho[i] = t.radii[i] - p.offset;
  double cut2 = p.cutoff * p.cutoff;
#pragma omp parallel for schedule(dynamic, 16)
  for (long ii = 0; ii < (long)n; ii++) {
    size_t i = (size_t)ii;
    double psi = 0.0;
    long double psil = 0.0L;
    for (size_t j = 0; j < n; j++) {
      if (i == j) continue;
      double dx = x[i].x - x[j].x, dy = x[i].y - x[j].y, dz = x[i].z - x[j].z;
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > cut2) continue;
      double sj = t.screen[j] * rho[j];
      double term;
      if (!hct_term(r2, rho[i], sj, term)) continue;
      if (accurate)
        psil += term;
      else
        psi += term;
    }
    if (accurate) psi = (double)psil;
    R[i] = radius_from_psi(psi, rho[i], t.radii[i], p);
  }
  return R;
}

static inline double gb_pair(double qi, double qj, double r2, double Ri, double Rj, double kap,
                             double inv_ein, double inv_eout, bool no_salt, double diel_ns) {
  // gb_energy.rs:339-346
  const double KSCALE = 0.73;
  double rr = Ri * Rj;
  double f = std::sqrt(r2 + rr * std::exp(-r2 / (4.0 * rr)));
  if (no_salt) return diel_ns * qi * qj / f;
  return -0.5 * qi * qj * (inv_ein - std::exp(-KSCALE * kap * f) * inv_eout) / f;
}

static inline double gb_self(double qi, double Ri, double kap, double inv_ein, double inv_eout,
                             bool no_salt, double diel_ns) {
  // gb_energy.rs:310-318
  const double KSCALE = 0.73;
  if (no_salt) return diel_ns * qi * qi / Ri;
  return -0.5 * qi * qi * (inv_ein - std::exp(-KSCALE * kap * Ri) * inv_eout) / Ri;
}

// gb_energy.rs:283-355
double gb_energy_from_radii(const Topology& t, const std::vector<V3>& x, const GbParams& p,
                            const std::vector<double>& R, bool accurate) {
  size_t n = t.n_atoms;
  double kap = kappa(p.salt, p.solvent_dielectric, p.temperature);
  double cut2 = p.cutoff * p.cutoff;
  double inv_ein = 1.0 / p.solute_dielectric, inv_eout = 1.0 / p.solvent_dielectric;
  bool no_salt = kap <= 0.0;
  double diel_ns = -0.5 * (inv_ein - inv_eout);
  double energy = 0.0;
  long double el = 0.0L;
  for (size_t i = 0; i < n; i++) {
    double s = gb_self(t.charges_amber[i], R[i], kap, inv_ein, inv_eout, no_salt, diel_ns);
    energy += s;
    el += s;
  }
  std::vector<double> part(n, 0.0);
  std::vector<long double> partl(n, 0.0L);
#pragma omp parallel for schedule(dynamic, 16)
  for (long ii = 0; ii < (long)n; ii++) {
    size_t i = (size_t)ii;
    double qi = t.charges_amber[i], sum = 0.0;
    long double suml = 0.0L;
    for (size_t j = i + 1; j < n; j++) {
      double dx = x[i].x - x[j].x, dy = x[i].y - x[j].y, dz = x[i].z - x[j].z;
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > cut2) continue;
      double pe = gb_pair(qi, t.charges_amber[j], r2, R[i], R[j], kap, inv_ein, inv_eout, no_salt,
                          diel_ns);
      sum += 2.0 * pe;
      suml += 2.0L * (long double)pe;
    }
    part[i] = sum;
    partl[i] = suml;
  }
  if (accurate) {
    for (size_t i = 0; i < n; i++) el += partl[i];
    return (double)el;
  }
  double cross = 0.0;
  for (size_t i = 0; i < n; i++) cross += part[i];
  energy += cross;
  return energy;
}

// ---------------------------------------------------------------------------
// MM: crates/mmpbsa/src/mm_energy.rs
// ---------------------------------------------------------------------------
struct PairBitmap {  // mm_energy.rs:8-39
  std::vector<uint64_t> w;
  explicit PairBitmap(size_t n) { w.assign((n * (n - 1) / 2 + 63) / 64, 0); }
  void set(size_t i, size_t j) {
    size_t k = j * (j - 1) / 2 + i;
    w[k / 64] |= 1ull << (k % 64);
  }
  bool has(size_t i, size_t j) const {
    size_t k = j * (j - 1) / 2 + i;
    return (w[k / 64] >> (k % 64)) & 1;
  }
};

static PairBitmap exclusion_set(const Topology& t) {  // mm_energy.rs:61-83
  PairBitmap b(std::max<size_t>(t.n_atoms, 2));
  size_t off = 0;
  for (size_t i = 0; i < t.n_atoms; i++) {
    size_t cnt = i < t.num_excluded.size() ? t.num_excluded[i] : 0;
    for (size_t k = 0; k < cnt; k++) {
      if (off + k < t.excluded_list.size()) {
        size_t j = t.excluded_list[off + k];
        if (j < t.n_atoms) b.set(std::min(i, j), std::max(i, j));
      }
    }
    off += cnt;
  }
  return b;
}

static PairBitmap pairs_14(const Topology& t) {  // mm_energy.rs:86-95
  PairBitmap b(std::max<size_t>(t.n_atoms, 2));
  for (auto& d : t.dihedrals)
    if (!d.ignore_14) b.set(std::min(d.i, d.l), std::max(d.i, d.l));
  return b;
}

static inline void lj_ab(const Topology& t, size_t i, size_t j, double& a, double& b) {
  // mm_energy.rs:152-161
  int64_t idx = t.nb_index[t.n_types * t.type_idx[i] + t.type_idx[j]];
  if (idx < 1) {
    a = 0;
    b = 0;
    return;
  }
  a = t.lj_a[idx - 1];
  b = t.lj_b[idx - 1];
}

static inline double vdot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline void vcross(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// Bonded terms, mm_energy.rs:97-149,187-212.  Returns {bond, angle, dihedral}.
static void bonded(const Topology& t, const std::vector<V3>& x, double out[3]) {
  double eb = 0, ea = 0, ed = 0;
  for (size_t b = 0; b < t.bonds.size(); b++) {
    size_t ty = t.bond_types[b];
    double k = t.bond_k[ty], req = t.bond_req[ty];
    const V3 &A = x[t.bonds[b].first], &B = x[t.bonds[b].second];
    double dx = A.x - B.x, dy = A.y - B.y, dz = A.z - B.z;
    double r = std::sqrt(dx * dx + dy * dy + dz * dz);
    eb += k * (r - req) * (r - req);
  }
  for (auto& an : t.angles) {
    double ka = t.angle_k[an.t], teq = t.angle_teq[an.t];
    const V3 &A = x[an.i], &B = x[an.j], &C = x[an.k];
    double ba[3] = {A.x - B.x, A.y - B.y, A.z - B.z}, bc[3] = {C.x - B.x, C.y - B.y, C.z - B.z};
    double dot = vdot(ba, bc);
    double m1 = std::sqrt(vdot(ba, ba)), m2 = std::sqrt(vdot(bc, bc));
    double c = dot / (m1 * m2);
    c = std::min(1.0, std::max(-1.0, c));
    double th = std::acos(c);
    ea += ka * (th - teq) * (th - teq);
  }
  for (auto& d : t.dihedrals) {
    double pk = t.dih_pk[d.t], pn = t.dih_pn[d.t], ph = t.dih_phase[d.t];
    const V3 &A = x[d.i], &B = x[d.j], &C = x[d.k], &D = x[d.l];
    double b1[3] = {B.x - A.x, B.y - A.y, B.z - A.z}, b2[3] = {C.x - B.x, C.y - B.y, C.z - B.z},
           b3[3] = {D.x - C.x, D.y - C.y, D.z - C.z};
    double n1[3], n2[3], m1[3], b2n[3];
    vcross(b1, b2, n1);
    vcross(b2, b3, n2);
    double len = std::sqrt(b2[0] * b2[0] + b2[1] * b2[1] + b2[2] * b2[2]);
    if (len < 1e-20) {
      b2n[0] = b2n[1] = b2n[2] = 0;
    } else {
      b2n[0] = b2[0] / len;
      b2n[1] = b2[1] / len;
      b2n[2] = b2[2] / len;
    }
    vcross(n1, b2n, m1);
    double xx = vdot(n1, n2), yy = vdot(m1, n2);
    double phi = std::atan2(-yy, xx);
    ed += pk * (1.0 + std::cos(pn * phi - ph));
  }
  out[0] = eb;
  out[1] = ea;
  out[2] = ed;
}

// mm_energy.rs:179-267
MmEnergy mm_energy(const Topology& t, const std::vector<V3>& x, bool accurate) {
  MmEnergy e;
  double b[3];
  bonded(t, x, b);
  e.bond = b[0];
  e.angle = b[1];
  e.dihedral = b[2];
  PairBitmap ex = exclusion_set(t), p14 = pairs_14(t);
  size_t n = t.n_atoms;
  std::vector<double> pv(n), pe(n), pv14(n), pe14(n);
  std::vector<long double> lv(n), le(n), lv14(n), le14(n);
  double scee = t.scee, scnb = t.scnb;
#pragma omp parallel for schedule(dynamic, 16)
  for (long ii = 0; ii < (long)n; ii++) {
    size_t i = (size_t)ii;
    double vdw = 0, elec = 0, v14 = 0, e14 = 0;
    long double a_v = 0, a_e = 0, a_v14 = 0, a_e14 = 0;
    for (size_t j = i + 1; j < n; j++) {
      double dx = x[i].x - x[j].x, dy = x[i].y - x[j].y, dz = x[i].z - x[j].z;
      double r2 = dx * dx + dy * dy + dz * dz;
      if (p14.has(i, j)) {
        double r = std::sqrt(r2), r6 = r2 * r2 * r2, r12 = r6 * r6, A, B;
        lj_ab(t, i, j, A, B);
        double v = (A / r12 - B / r6) / scnb;
        double c = t.charges_amber[i] * t.charges_amber[j] / r / scee;
        v14 += v;
        e14 += c;
        a_v14 += v;
        a_e14 += c;
      } else if (!ex.has(i, j)) {
        double r = std::sqrt(r2), r6 = r2 * r2 * r2, r12 = r6 * r6, A, B;
        lj_ab(t, i, j, A, B);
        double v = A / r12 - B / r6;
        double c = t.charges_amber[i] * t.charges_amber[j] / r;
        vdw += v;
        elec += c;
        a_v += v;
        a_e += c;
      }
    }
    pv[i] = vdw;
    pe[i] = elec;
    pv14[i] = v14;
    pe14[i] = e14;
    lv[i] = a_v;
    le[i] = a_e;
    lv14[i] = a_v14;
    le14[i] = a_e14;
  }
  if (accurate) {
    long double s[4] = {0, 0, 0, 0};
    for (size_t i = 0; i < n; i++) {
      s[0] += lv[i];
      s[1] += le[i];
      s[2] += lv14[i];
      s[3] += le14[i];
    }
    e.vdw = (double)s[0];
    e.elec = (double)s[1];
    e.vdw_14 = (double)s[2];
    e.elec_14 = (double)s[3];
  } else {
    for (size_t i = 0; i < n; i++) {
      e.vdw += pv[i];
      e.elec += pe[i];
      e.vdw_14 += pv14[i];
      e.elec_14 += pe14[i];
    }
  }
  return e;
}

// ---------------------------------------------------------------------------
// SASA: core/src/sasa.rs:147-289, sa_energy.rs:51-75
// ---------------------------------------------------------------------------
std::vector<V3> fibonacci_sphere(size_t n) {  // sasa.rs:147-169
  std::vector<V3> pts;
  if (n == 0) return pts;
  if (n == 1) return {{0.0, 1.0, 0.0}};
  double phi = PI * (3.0 - std::sqrt(5.0));
  for (size_t i = 0; i < n; i++) {
    double y = 1.0 - ((double)i / (double)(n - 1)) * 2.0;
    double rad = std::sqrt(1.0 - y * y);
    double th = phi * (double)i;
    pts.push_back({std::cos(th) * rad, y, std::sin(th) * rad});
  }
  return pts;
}

std::vector<double> sasa_per_atom(const std::vector<V3>& x, const std::vector<double>& radii,
                                  double probe, size_t n_points) {
  size_t n = x.size();
  std::vector<V3> sp = fibonacci_sphere(n_points);
  double maxr = 0.0;
  for (double r : radii) maxr = std::max(maxr, r);
  double max_ext = maxr + probe;  // sasa.rs:213-214
  std::vector<double> out(n);
#pragma omp parallel for schedule(dynamic, 8)
  for (long ii = 0; ii < (long)n; ii++) {
    size_t i = (size_t)ii;
    double er = radii[i] + probe, er2 = er * er, search = er + max_ext, s2 = search * search;
    // The KD-tree radius query (sasa.rs:88-143) returns exactly the atoms with
    // distance_squared <= search^2; an exhaustive scan returns the same set.
    std::vector<size_t> nb;
    for (size_t j = 0; j < n; j++) {
      double dx = x[j].x - x[i].x, dy = x[j].y - x[i].y, dz = x[j].z - x[i].z;
      if (dx * dx + dy * dy + dz * dz <= s2) nb.push_back(j);
    }
    size_t acc = 0;
    for (const V3& p : sp) {  // sasa.rs:247-270
      double tx = x[i].x + p.x * er, ty = x[i].y + p.y * er, tz = x[i].z + p.z * er;
      bool ok = true;
      for (size_t j : nb) {
        if (j == i) continue;
        double oer = radii[j] + probe;
        double dx = tx - x[j].x, dy = ty - x[j].y, dz = tz - x[j].z;
        double d2 = dx * dx + dy * dy + dz * dz;
        if (!(d2 > oer * oer)) {
          ok = false;
          break;
        }
      }
      if (ok) acc++;
    }
    double frac = (double)acc / (double)n_points;
    double area = 4.0 * PI * er2;
    out[i] = frac * area;
  }
  return out;
}

}  // namespace orc
