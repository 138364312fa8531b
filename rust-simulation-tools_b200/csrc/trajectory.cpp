// Trajectory readers: DCD (core/src/trajectory/dcd.rs:217-444) and AMBER
// ASCII mdcrd (crates/mmpbsa/src/mdcrd.rs:26-108).
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "internal.hpp"
#include "trajectory.hpp"

namespace rstg {

DcdData read_dcd(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) throw Error(RSTG_ERR_IO, "Failed to open DCD file: " + path);
  std::vector<unsigned char> buf;
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  buf.resize(sz > 0 ? sz : 0);
  size_t got = sz > 0 ? fread(buf.data(), 1, sz, f) : 0;
  fclose(f);
  if ((long)got != sz) throw Error(RSTG_ERR_IO, "Failed to read DCD file: " + path);
  size_t pos = 0;
  bool be = false;
  auto need = [&](size_t k, const char* what) {
    if (pos + k > buf.size()) throw Error(RSTG_ERR_IO, std::string("Failed to read ") + what);
  };
  auto i32 = [&]() {
    need(4, "i32");
    uint32_t u;
    memcpy(&u, &buf[pos], 4);
    if (be) u = __builtin_bswap32(u);
    pos += 4;
    int32_t v;
    memcpy(&v, &u, 4);
    return v;
  };
  need(4, "block size");
  int32_t le;
  memcpy(&le, &buf[0], 4);
  uint32_t sw = __builtin_bswap32((uint32_t)le);
  if (le == 84)
    be = false;
  else if ((int32_t)sw == 84)
    be = true;
  else
    throw Error(RSTG_ERR_IO, "Invalid DCD header: first block size is not 84");
  if (i32() != 84) throw Error(RSTG_ERR_IO, "Invalid DCD header size");
  need(4, "magic");
  if (memcmp(&buf[pos], "CORD", 4) != 0) throw Error(RSTG_ERR_IO, "Invalid DCD magic");
  pos += 4;
  int32_t nfr = i32();
  if (nfr < 0) throw Error(RSTG_ERR_IO, "Invalid number of frames");
  for (int k = 0; k < 8; k++) i32();
  need(4, "timestep");
  pos += 4;
  bool cell = i32() != 0;
  need(32, "header");
  pos += 32;
  i32();  // CHARMM version
  i32();  // end of block 1
  int32_t b2 = i32();
  if (b2 < 4) throw Error(RSTG_ERR_IO, "Invalid title block size");
  int32_t nt = i32();
  if (nt < 0 || 4 + (int64_t)nt * 80 > b2) throw Error(RSTG_ERR_IO, "Title block size mismatch");
  need((size_t)b2 - 4, "titles");
  pos += (size_t)b2 - 4;
  i32();
  i32();
  int32_t na = i32();
  if (na < 0 || na > 100000000) throw Error(RSTG_ERR_IO, "Invalid number of atoms");
  i32();
  DcdData d;
  d.n_atoms = na;
  d.n_frames = nfr;
  d.has_cell = cell;
  d.xyz.resize((size_t)nfr * na * 3);
  std::vector<float> col(na);
  for (int32_t fr = 0; fr < nfr; fr++) {
    if (cell) {
      need(56, "unit cell");
      double c6[6];
      memcpy(c6, &buf[pos + 4], 48);
      pos += 56;
      // a, b, c (CHARMM order a, gamma, b, beta, alpha, c); the reference
      // stores them in nm (dcd.rs:383-400) and scales by 10 for reimaging
      // (binding.rs:635-642): the same roundings here
      d.boxes.push_back({(c6[0] * 0.1) * 10.0, (c6[2] * 0.1) * 10.0, (c6[5] * 0.1) * 10.0});
    }
    for (int dim = 0; dim < 3; dim++) {
      i32();
      need((size_t)na * 4, "f32");
      memcpy(col.data(), &buf[pos], (size_t)na * 4);  // coordinates are little-endian (dcd.rs:152-159)
      pos += (size_t)na * 4;
      i32();
      for (int32_t a = 0; a < na; a++) d.xyz[((size_t)fr * na + a) * 3 + dim] = col[a];
    }
  }
  return d;
}

std::vector<double> read_mdcrd(const std::string& path, int64_t n_atoms, bool has_box,
                               std::vector<std::array<double, 3>>* boxes) {
  std::ifstream f(path);
  if (!f) throw Error(RSTG_ERR_IO, "Failed to open mdcrd: " + path);
  std::string line;
  std::getline(f, line);  // title
  int64_t nv = n_atoms * 3 + (has_box ? 3 : 0);
  std::vector<double> out, vals;
  int64_t frame = 0;
  for (;;) {
    vals.clear();
    bool eof = false;
    while ((int64_t)vals.size() < nv) {
      if (!std::getline(f, line)) {
        eof = true;
        break;
      }
      while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
      for (size_t p = 0; p < line.size() && (int64_t)vals.size() < nv; p += 8) {
        std::string fld = line.substr(p, 8);
        size_t a = fld.find_first_not_of(" \t"), b = fld.find_last_not_of(" \t");
        std::string t = a == std::string::npos ? "" : fld.substr(a, b - a + 1);
        char* e = nullptr;
        double v = strtod(t.c_str(), &e);
        if (t.empty() || *e)
          throw Error(RSTG_ERR_INVALID,
                      "Failed to parse mdcrd value '" + t + "' at frame " + std::to_string(frame));
        vals.push_back(v);
      }
    }
    if (eof) {
      if (vals.empty()) break;
      throw Error(RSTG_ERR_INVALID, "Unexpected EOF at frame " + std::to_string(frame));
    }
    out.insert(out.end(), vals.begin(), vals.begin() + n_atoms * 3);
    if (has_box && boxes) boxes->push_back({vals[n_atoms * 3], vals[n_atoms * 3 + 1], vals[n_atoms * 3 + 2]});
    frame++;
  }
  return out;
}

}  // namespace rstg
