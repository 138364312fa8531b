// Host-side topology: prmtop parsing (core/src/amber/prmtop.rs:331-733),
// sub-topology extraction (crates/mmpbsa/src/subsystem.rs:22-169),
// non-bonded pair classes (crates/mmpbsa/src/mm_energy.rs:61-95) and the
// receptor/ligand split (crates/mmpbsa/src/binding.rs:142-211).
#include <algorithm>
#include <cstring>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <unordered_map>

#include "internal.hpp"

namespace rstg {

namespace {
std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) a++;
  while (b > a && isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

struct Sections {
  std::map<std::string, std::vector<std::string>> m;
  bool has(const std::string& k) const { return m.count(k) > 0; }
  const std::vector<std::string>& at(const std::string& k) const {
    auto it = m.find(k);
    if (it == m.end()) throw Error(RSTG_ERR_IO, "Missing section: " + k);
    return it->second;
  }
  std::vector<int64_t> ints(const std::string& k) const {
    std::vector<int64_t> v;
    for (auto& ln : at(k)) {
      std::istringstream is(ln);
      std::string w;
      while (is >> w) {
        char* e = nullptr;
        long long x = strtoll(w.c_str(), &e, 10);
        if (*e) throw Error(RSTG_ERR_IO, "Failed to parse integer in " + k + ": " + w);
        v.push_back(x);
      }
    }
    return v;
  }
  std::vector<double> floats(const std::string& k) const {
    std::vector<double> v;
    for (auto& ln : at(k)) {
      std::istringstream is(ln);
      std::string w;
      while (is >> w) {
        char* e = nullptr;
        double x = strtod(w.c_str(), &e);
        if (*e) throw Error(RSTG_ERR_IO, "Failed to parse float in " + k + ": " + w);
        v.push_back(x);
      }
    }
    return v;
  }
  std::vector<std::string> strings(const std::string& k, size_t w) const {
    std::vector<std::string> v;
    for (auto& ln : at(k)) {
      size_t p = 0;
      for (; p + w <= ln.size(); p += w) v.push_back(trim(ln.substr(p, w)));
      if (p < ln.size()) {
        std::string r = trim(ln.substr(p));
        if (!r.empty()) v.push_back(r);
      }
    }
    return v;
  }
};
}  // namespace

std::vector<int64_t> Topology::atom_residue_indices() const {
  std::vector<int64_t> r(n_atoms, 0);
  for (int64_t k = 0; k < n_residues; k++) {
    int64_t a = residue_pointers[k], b = k + 1 < n_residues ? residue_pointers[k + 1] : n_atoms;
    for (int64_t i = a; i < b; i++) r[i] = k;
  }
  return r;
}

std::vector<int64_t> Topology::select(const std::vector<int64_t>& residues) const {
  for (int64_t r : residues)
    if (r < 0 || r >= n_residues)
      throw Error(RSTG_ERR_INVALID, "Residue index " + std::to_string(r) + " out of range (0-" +
                                        std::to_string(n_residues - 1) + ")");
  std::vector<int64_t> a;
  for (int64_t r : residues) {
    int64_t s = residue_pointers[r], e = r + 1 < n_residues ? residue_pointers[r + 1] : n_atoms;
    for (int64_t i = s; i < e; i++) a.push_back(i);
  }
  return a;
}

Topology parse_prmtop(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw Error(RSTG_ERR_IO, "Failed to open prmtop file: " + path);
  Sections S;
  std::string line, flag;
  bool have = false;
  std::vector<std::string> cur;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.rfind("%FLAG", 0) == 0) {
      if (have) S.m[flag] = std::move(cur);
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
  if (have) S.m[flag] = std::move(cur);

  Topology t;
  auto ptr = S.ints("POINTERS");
  if (ptr.size() < 12) throw Error(RSTG_ERR_IO, "POINTERS section too short");
  if (ptr[0] < 0 || ptr[1] < 0 || ptr[11] < 0) throw Error(RSTG_ERR_IO, "POINTERS contains negative values");
  t.n_atoms = ptr[0];
  t.n_types = ptr[1];
  t.n_residues = ptr[11];
  t.atom_names = S.strings("ATOM_NAME", 4);
  if ((int64_t)t.atom_names.size() < t.n_atoms) throw Error(RSTG_ERR_IO, "ATOM_NAME has too few entries");
  t.atom_names.resize(t.n_atoms);
  auto ti = S.ints("ATOM_TYPE_INDEX");
  if ((int64_t)ti.size() < t.n_atoms) throw Error(RSTG_ERR_IO, "ATOM_TYPE_INDEX has too few entries");
  for (int64_t i = 0; i < t.n_atoms; i++) {
    if (ti[i] < 1) throw Error(RSTG_ERR_IO, "Invalid ATOM_TYPE_INDEX at position " + std::to_string(i));
    if (ti[i] > t.n_types) throw Error(RSTG_ERR_IO, "ATOM_TYPE_INDEX exceeds the number of types");
    t.type_idx.push_back(ti[i] - 1);
  }
  auto q = S.floats("CHARGE");
  if ((int64_t)q.size() < t.n_atoms) throw Error(RSTG_ERR_IO, "CHARGE has too few entries");
  for (int64_t i = 0; i < t.n_atoms; i++) {
    t.charges.push_back(q[i] / 18.2223);
    t.charges_amber.push_back(q[i]);
  }
  t.residue_labels = S.strings("RESIDUE_LABEL", 4);
  if ((int64_t)t.residue_labels.size() > t.n_residues) t.residue_labels.resize(t.n_residues);
  while ((int64_t)t.residue_labels.size() < t.n_residues) t.residue_labels.push_back("");
  auto rp = S.ints("RESIDUE_POINTER");
  if ((int64_t)rp.size() < t.n_residues) throw Error(RSTG_ERR_IO, "RESIDUE_POINTER has too few entries");
  for (int64_t i = 0; i < t.n_residues; i++) {
    if (rp[i] < 1 || rp[i] > t.n_atoms)
      throw Error(RSTG_ERR_IO, "Invalid RESIDUE_POINTER at position " + std::to_string(i));
    t.residue_pointers.push_back(rp[i] - 1);
  }
  t.lj_a = S.floats("LENNARD_JONES_ACOEF");
  t.lj_b = S.floats("LENNARD_JONES_BCOEF");
  t.nb_index = S.ints("NONBONDED_PARM_INDEX");
  if ((int64_t)t.nb_index.size() < t.n_types * t.n_types)
    throw Error(RSTG_ERR_IO, "NONBONDED_PARM_INDEX out of bounds");
  for (int64_t k = 0; k < t.n_types * t.n_types; k++)
    if (t.nb_index[k] > (int64_t)std::min(t.lj_a.size(), t.lj_b.size()))
      throw Error(RSTG_ERR_IO, "NONBONDED_PARM_INDEX entry exceeds the LJ tables");
  auto opt_f = [&](const char* k, std::vector<double>& v, size_t n) {
    if (S.has(k))
      v = S.floats(k);
    else
      v.assign(n, 0.0);
  };
  opt_f("MASS", t.masses, t.n_atoms);
  opt_f("RADII", t.radii, t.n_atoms);
  opt_f("SCREEN", t.screen, t.n_atoms);
  if ((int64_t)t.radii.size() < t.n_atoms || (int64_t)t.screen.size() < t.n_atoms ||
      (int64_t)t.masses.size() < t.n_atoms)
    throw Error(RSTG_ERR_IO, "RADII/SCREEN/MASS have too few entries");
  opt_f("BOND_FORCE_CONSTANT", t.bond_k, 0);
  opt_f("BOND_EQUIL_VALUE", t.bond_req, 0);
  opt_f("ANGLE_FORCE_CONSTANT", t.angle_k, 0);
  opt_f("ANGLE_EQUIL_VALUE", t.angle_teq, 0);
  opt_f("DIHEDRAL_FORCE_CONSTANT", t.dih_pk, 0);
  opt_f("DIHEDRAL_PERIODICITY", t.dih_pn, 0);
  opt_f("DIHEDRAL_PHASE", t.dih_phase, 0);
  auto chk = [&](int64_t atom) {
    if (atom < 0 || atom >= t.n_atoms) throw Error(RSTG_ERR_IO, "bonded term references atom out of range");
  };
  for (const char* k : {"BONDS_INC_HYDROGEN", "BONDS_WITHOUT_HYDROGEN"}) {
    if (!S.has(k)) continue;
    auto v = S.ints(k);
    for (size_t c = 0; c + 3 <= v.size(); c += 3) {
      if (v[c] < 0 || v[c + 1] < 0 || v[c + 2] < 1) continue;
      chk(v[c] / 3);
      chk(v[c + 1] / 3);
      if (v[c + 2] > (int64_t)std::min(t.bond_k.size(), t.bond_req.size()))
        throw Error(RSTG_ERR_IO, "bond type out of range");
      t.bond_i.push_back(v[c] / 3);
      t.bond_j.push_back(v[c + 1] / 3);
      t.bond_t.push_back(v[c + 2] - 1);
    }
  }
  for (const char* k : {"ANGLES_INC_HYDROGEN", "ANGLES_WITHOUT_HYDROGEN"}) {
    if (!S.has(k)) continue;
    auto v = S.ints(k);
    for (size_t c = 0; c + 4 <= v.size(); c += 4) {
      if (v[c] < 0 || v[c + 1] < 0 || v[c + 2] < 0 || v[c + 3] < 1) continue;
      chk(v[c] / 3);
      chk(v[c + 1] / 3);
      chk(v[c + 2] / 3);
      if (v[c + 3] > (int64_t)std::min(t.angle_k.size(), t.angle_teq.size()))
        throw Error(RSTG_ERR_IO, "angle type out of range");
      t.ang_i.push_back(v[c] / 3);
      t.ang_j.push_back(v[c + 1] / 3);
      t.ang_k.push_back(v[c + 2] / 3);
      t.ang_t.push_back(v[c + 3] - 1);
    }
  }
  for (const char* k : {"DIHEDRALS_INC_HYDROGEN", "DIHEDRALS_WITHOUT_HYDROGEN"}) {
    if (!S.has(k)) continue;
    auto v = S.ints(k);
    for (size_t c = 0; c + 5 <= v.size(); c += 5) {
      if (v[c + 4] < 1) continue;
      int64_t a = std::llabs(v[c]) / 3, b = std::llabs(v[c + 1]) / 3, cc = std::llabs(v[c + 2]) / 3,
              d = std::llabs(v[c + 3]) / 3;
      chk(a);
      chk(b);
      chk(cc);
      chk(d);
      if (v[c + 4] > (int64_t)std::min({t.dih_pk.size(), t.dih_pn.size(), t.dih_phase.size()}))
        throw Error(RSTG_ERR_IO, "dihedral type out of range");
      t.dih_i.push_back(a);
      t.dih_j.push_back(b);
      t.dih_k.push_back(cc);
      t.dih_l.push_back(d);
      t.dih_t.push_back(v[c + 4] - 1);
      t.dih_ignore14.push_back(v[c + 2] < 0 || v[c + 3] < 0);
    }
  }
  if (S.has("NUMBER_EXCLUDED_ATOMS"))
    for (auto v : S.ints("NUMBER_EXCLUDED_ATOMS")) t.num_excluded.push_back(v < 0 ? 0 : v);
  if (S.has("EXCLUDED_ATOMS_LIST"))
    for (auto v : S.ints("EXCLUDED_ATOMS_LIST")) t.excluded_list.push_back(v > 0 ? v - 1 : -1);
  if (S.has("SCEE_SCALE_FACTOR")) {
    auto v = S.floats("SCEE_SCALE_FACTOR");
    if (!v.empty()) t.scee = v[0];
  }
  if (S.has("SCNB_SCALE_FACTOR")) {
    auto v = S.floats("SCNB_SCALE_FACTOR");
    if (!v.empty()) t.scnb = v[0];
  }
  return t;
}

Topology extract_subtopology(const Topology& t, const std::vector<int64_t>& atoms) {
  Topology s;
  std::unordered_map<int64_t, int64_t> o2n;
  o2n.reserve(atoms.size() * 2);
  for (size_t k = 0; k < atoms.size(); k++) {
    if (atoms[k] < 0 || atoms[k] >= t.n_atoms) throw Error(RSTG_ERR_INVALID, "atom index out of range");
    o2n[atoms[k]] = (int64_t)k;
  }
  s.n_atoms = atoms.size();
  s.n_types = t.n_types;
  for (int64_t a : atoms) {
    s.atom_names.push_back(a < (int64_t)t.atom_names.size() ? t.atom_names[a] : "");
    s.type_idx.push_back(t.type_idx[a]);
    s.charges.push_back(t.charges[a]);
    s.charges_amber.push_back(t.charges_amber[a]);
    s.masses.push_back(t.masses[a]);
    s.radii.push_back(t.radii[a]);
    s.screen.push_back(t.screen[a]);
  }
  auto ar = t.atom_residue_indices();
  int64_t last = -1;
  for (size_t k = 0; k < atoms.size(); k++) {
    int64_t r = ar[atoms[k]];
    if (r != last) {
      s.residue_labels.push_back(t.residue_labels[r]);
      s.residue_pointers.push_back((int64_t)k);
      last = r;
    }
  }
  s.n_residues = s.residue_pointers.size();
  auto get = [&](int64_t a, int64_t& o) {
    auto it = o2n.find(a);
    if (it == o2n.end()) return false;
    o = it->second;
    return true;
  };
  for (size_t b = 0; b < t.bond_i.size(); b++) {
    int64_t x, y;
    if (get(t.bond_i[b], x) && get(t.bond_j[b], y)) {
      s.bond_i.push_back(x);
      s.bond_j.push_back(y);
      s.bond_t.push_back(t.bond_t[b]);
    }
  }
  for (size_t a = 0; a < t.ang_i.size(); a++) {
    int64_t x, y, z;
    if (get(t.ang_i[a], x) && get(t.ang_j[a], y) && get(t.ang_k[a], z)) {
      s.ang_i.push_back(x);
      s.ang_j.push_back(y);
      s.ang_k.push_back(z);
      s.ang_t.push_back(t.ang_t[a]);
    }
  }
  for (size_t d = 0; d < t.dih_i.size(); d++) {
    int64_t w, x, y, z;
    if (get(t.dih_i[d], w) && get(t.dih_j[d], x) && get(t.dih_k[d], y) && get(t.dih_l[d], z)) {
      s.dih_i.push_back(w);
      s.dih_j.push_back(x);
      s.dih_k.push_back(y);
      s.dih_l.push_back(z);
      s.dih_t.push_back(t.dih_t[d]);
      s.dih_ignore14.push_back(t.dih_ignore14[d]);
    }
  }
  s.num_excluded.assign(s.n_atoms, 0);
  int64_t off = 0;
  for (int64_t i = 0; i < t.n_atoms; i++) {
    int64_t cnt = i < (int64_t)t.num_excluded.size() ? t.num_excluded[i] : 0;
    int64_t ni;
    if (get(i, ni)) {
      int64_t c = 0;
      for (int64_t k = 0; k < cnt; k++) {
        if (off + k >= (int64_t)t.excluded_list.size()) continue;
        int64_t nj;
        int64_t j = t.excluded_list[off + k];
        if (j >= 0 && get(j, nj)) {
          s.excluded_list.push_back(nj);
          c++;
        }
      }
      s.num_excluded[ni] = c;
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

static inline uint64_t key(int64_t i, int64_t j) {
  if (i > j) std::swap(i, j);
  return ((uint64_t)i << 32) | (uint64_t)j;
}

PairClasses PairClasses::build(const Topology& t) {
  PairClasses pc;
  int64_t n = std::max<int64_t>(t.n_atoms, 2);
  size_t words = (size_t)((n * (n - 1) / 2 + 63) / 64);
  pc.excl_bits.assign(words, 0);
  pc.p14_bits.assign(words, 0);
  auto setb = [&](std::vector<uint64_t>& b, int64_t i, int64_t j) {
    if (i > j) std::swap(i, j);
    uint64_t k = (uint64_t)j * (j - 1) / 2 + i;
    b[k / 64] |= 1ull << (k % 64);
  };
  int64_t off = 0;
  for (int64_t i = 0; i < t.n_atoms; i++) {
    int64_t cnt = i < (int64_t)t.num_excluded.size() ? t.num_excluded[i] : 0;
    for (int64_t k = 0; k < cnt; k++) {
      if (off + k >= (int64_t)t.excluded_list.size()) continue;
      int64_t j = t.excluded_list[off + k];
      if (j >= 0 && j < t.n_atoms && j != i) {
        setb(pc.excl_bits, i, j);
        pc.excl_keys.push_back(key(i, j));
      }
    }
    off += cnt;
  }
  for (size_t d = 0; d < t.dih_i.size(); d++) {
    if (t.dih_ignore14[d]) continue;
    if (t.dih_i[d] == t.dih_l[d]) continue;
    setb(pc.p14_bits, t.dih_i[d], t.dih_l[d]);
    pc.p14_keys.push_back(key(t.dih_i[d], t.dih_l[d]));
  }
  for (auto* v : {&pc.excl_keys, &pc.p14_keys}) {
    std::sort(v->begin(), v->end());
    v->erase(std::unique(v->begin(), v->end()), v->end());
  }
  return pc;
}

int PairClasses::cls(int64_t i, int64_t j) const {
  uint64_t k = key(i, j);
  if (std::binary_search(p14_keys.begin(), p14_keys.end(), k)) return 2;
  if (std::binary_search(excl_keys.begin(), excl_keys.end(), k)) return 0;
  return 1;
}

Split Split::make(const Topology& t, const std::vector<int64_t>& rres, const std::vector<int64_t>& lres) {
  Split s;
  std::set<int64_t> cs(rres.begin(), rres.end());
  cs.insert(lres.begin(), lres.end());
  std::vector<int64_t> cres(cs.begin(), cs.end());
  std::vector<int64_t> catoms = t.select(cres);
  if ((int64_t)catoms.size() == t.n_atoms) {
    s.complex = t;
    s.rec_res = rres;
    s.lig_res = lres;
  } else {
    s.complex = extract_subtopology(t, catoms);
    s.complex_atoms = catoms;
    std::unordered_map<int64_t, int64_t> m;
    for (size_t k = 0; k < cres.size(); k++) m[cres[k]] = (int64_t)k;
    for (int64_t r : rres) s.rec_res.push_back(m[r]);
    for (int64_t r : lres) s.lig_res.push_back(m[r]);
  }
  s.rec_atoms = s.complex.select(s.rec_res);
  s.lig_atoms = s.complex.select(s.lig_res);
  s.rec = extract_subtopology(s.complex, s.rec_atoms);
  s.lig = extract_subtopology(s.complex, s.lig_atoms);
  return s;
}

}  // namespace rstg
