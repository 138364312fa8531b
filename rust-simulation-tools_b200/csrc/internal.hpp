// Internal host-side structures of librstg.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "rstg.h"

namespace rstg {

// Error carrying an rstg_status; converted to the C status at the ABI edge.
struct Error : std::runtime_error {
  rstg_status code;
  Error(rstg_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& m);

#define RSTG_CUDA(expr)                                                                              \
  do {                                                                                               \
    cudaError_t e_ = (expr);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      throw ::rstg::Error(RSTG_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));      \
  } while (0)

// AmberTopology (core/src/amber/prmtop.rs:34-105), host copy.
struct Topology {
  int64_t n_atoms = 0, n_residues = 0, n_types = 0;
  std::vector<std::string> atom_names, residue_labels;
  std::vector<int64_t> type_idx, residue_pointers;
  std::vector<double> charges, charges_amber, masses, radii, screen;
  std::vector<int64_t> bond_i, bond_j, bond_t;
  std::vector<double> bond_k, bond_req, angle_k, angle_teq, dih_pk, dih_pn, dih_phase;
  std::vector<int64_t> ang_i, ang_j, ang_k, ang_t;
  std::vector<int64_t> dih_i, dih_j, dih_k, dih_l, dih_t;
  std::vector<uint8_t> dih_ignore14;
  std::vector<int64_t> num_excluded, excluded_list;  // -1 = placeholder
  double scee = 1.2, scnb = 2.0;
  std::vector<double> lj_a, lj_b;
  std::vector<int64_t> nb_index;

  std::vector<int64_t> atom_residue_indices() const;
  std::vector<int64_t> select(const std::vector<int64_t>& residues) const;  // throws on range
};

Topology parse_prmtop(const std::string& path);
Topology extract_subtopology(const Topology& t, const std::vector<int64_t>& atoms);

// Non-bonded pair classes of one topology: the reference checks 1-4 first
// (scaled), then exclusion (skipped), else full (mm_energy.rs:230-252).
// Stored as sorted (i < j) key lists for O(log) host lookups and as the
// triangular bitmaps the plain kernels read (mm_energy.rs:8-39).
struct PairClasses {
  std::vector<uint64_t> excl_bits, p14_bits;  // triangular j(j-1)/2 + i
  std::vector<uint64_t> excl_keys, p14_keys;  // (i << 32) | j, sorted, unique
  static PairClasses build(const Topology& t);
  int cls(int64_t i, int64_t j) const;  // 0 skip, 1 full, 2 scaled 1-4
};

// The receptor/ligand split of binding.rs:142-211 / decomposition.rs:125-208.
struct Split {
  Topology complex, rec, lig;
  std::vector<int64_t> complex_atoms;  // topology atom of each complex atom
  std::vector<int64_t> rec_atoms, lig_atoms;  // complex numbering
  std::vector<int64_t> rec_res, lig_res;  // complex residue numbering
  static Split make(const Topology& t, const std::vector<int64_t>& rres, const std::vector<int64_t>& lres);
};

// Stream-ordered device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t s = nullptr;
  DevBuf() = default;
  DevBuf(size_t n, cudaStream_t st);
  ~DevBuf();
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes), s(o.s) { o.p = nullptr; }
  DevBuf& operator=(DevBuf&& o) noexcept;
  template <class T>
  T* as() const {
    return (T*)p;
  }
};

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::recursive_mutex mu;
  std::atomic<int64_t> launches{0};
  cudaDeviceProp prop{};
  void bind() const { cudaSetDevice(device); }
};

// Records a kernel launch for the context's counter and checks the launch.
void launched(Ctx* c, int n = 1);

}  // namespace rstg

struct rstg_ctx : rstg::Ctx {};
struct rstg_topology : rstg::Topology {};
