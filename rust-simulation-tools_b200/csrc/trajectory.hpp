#pragma once
#include <array>
#include <string>
#include <vector>

namespace rstg {

struct DcdData {
  int64_t n_frames = 0, n_atoms = 0;
  bool has_cell = false;
  std::vector<float> xyz;  // [frames][atoms][3] Angstrom as stored
  std::vector<std::array<double, 3>> boxes;  // Angstrom, when has_cell
};

DcdData read_dcd(const std::string& path);
// Angstrom [frames][atoms][3]
std::vector<double> read_mdcrd(const std::string& path, int64_t n_atoms, bool has_box,
                               std::vector<std::array<double, 3>>* boxes);

}  // namespace rstg
