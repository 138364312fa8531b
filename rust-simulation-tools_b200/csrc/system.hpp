// Device-resident batched binding engine (rstg_system).
#pragma once
#include <memory>

#include "frame_plain.hpp"
#include "internal.hpp"
#include "pb_batch.hpp"

namespace rstg {

constexpr int kTile = 128;  // rows per CTA and columns per shared-memory tile

struct FusedParams;  // system.cu

struct System {
  Ctx* ctx = nullptr;
  std::recursive_mutex mu;        // one run at a time per system
  cudaStream_t stream_ = nullptr;  // fused-mode stream (null: the context's)
  cudaStream_t stream() const { return stream_ ? stream_ : ctx->stream; }
  rstg_solvation solv{};
  rstg_sa_params sa{};
  rstg_system_opts opts{};
  Split split;
  int64_t n_top = 0;  // atoms per input frame (topology atoms)
  int64_t nC = 0, nR = 0, nL = 0, n_res_rec = 0, n_res_lig = 0;

  // plain mode (and PB): per-frame FP64 evaluation
  std::unique_ptr<PlainFrameEval> plain;

  // fused mode
  bool perm_ready = false;
  std::vector<int64_t> slot_atom;  // slot -> complex atom
  std::vector<int32_t> slot_src;   // slot -> topology atom (input frame index)
  std::unique_ptr<FusedParams> fp;
  int64_t batch = 0;  // frames per device batch
  int nbr_cap = 320;
  // launch shapes (picked by tune() on the first run when opts.autotune)
  int pairs_variant = 0;  // index into the k_pairs shape table (system.cu)
  int psi_variant = 0;    // index into the k_psi shape table
  int pairs_per_sm[8] = {};  // resident k_pairs blocks per SM of each shape (persistent grid), 0 until queried
  int sasa_warps = 2;     // warps (atoms) per k_sasa block
  bool tuned = false;
  int64_t tune_frames = 0;
  double tune_ms[12] = {};  // candidate times of the tuning run (k_pairs, k_sasa, k_psi shapes)
  void tuning(int32_t* shape12, double* ms12) const;

  // per-batch buffers (fused)
  DevBuf in_frames, xyz64, xyz32, R64, Rf, dRf, nbr, nbrcnt, sasa, k1part, k2part, rows, cols, bpart, res_buf, dec_buf,
      diag;
  int64_t buf_frames = 0;
  cudaGraphExec_t graph = nullptr;
  int64_t graph_frames = 0;
  int graph_input_f64 = -1;
  const void* graph_src = nullptr;
  void* graph_out = nullptr;
  void* graph_decomp = nullptr;
  int64_t last_stats[4] = {0, 0, 0, 0};

  // fused mode with PB solvation: polar terms from the batched PB engine
  std::unique_ptr<PbBatchEngine> pbe;
  int64_t pb_frames_per_batch = 0;  // 0: from the device memory budget
  bool pb_profile = false;          // time the level-0 PB kernels
  double pb_rel_tol = 0.0;          // > 0: PB grids solved to this relative residual (not the reference's rule)

  System(Ctx* c, const Topology& t, const std::vector<int64_t>& rres, const std::vector<int64_t>& lres,
         const rstg_solvation& s, const rstg_sa_params& sa, const rstg_system_opts& o);
  ~System();
  int64_t footprint(int64_t frames) const;
  void release_buffers();  // frees the per-batch device buffers
  // frames: [F][n_top][3]; f64 selects float64 Angstrom input (else float32
  // Angstrom through the DCD nm round trip).  host_* true: host pointers.
  void run(const void* frames, bool f64, bool host_in, int64_t F, rstg_frame_energy* out, bool host_out,
           rstg_residue_energy* decomp);

 private:
  void prepare_fused(const double* first_frame_complex);
  void ensure_buffers(int64_t frames);
  // prof (optional): events recorded before the first and after every kernel;
  // names/flops/bytes receive one entry per kernel.
  struct Prof {
    cudaEvent_t ev[9];
    const char* names[8];
    double flops[8], bytes[8];
    int n = 0;
  };
  void launch_batch(const void* d_frames, bool f64, int64_t F, rstg_frame_energy* d_out,
                    rstg_residue_energy* d_decomp, Prof* prof = nullptr);
  void launch_pairs(int variant, int64_t F);
  void launch_psi(int variant, int64_t F);
  void launch_sasa(int warps, int64_t F);
  void tune(const void* frames, bool f64, bool host_in, int64_t F);

 public:
  void profile(const float* d_frames, int64_t F, int32_t* n, char* names, double* ms, double* flops, double* bytes);

 private:
  void run_plain(const void* frames, bool f64, bool host_in, int64_t F, rstg_frame_energy* out, bool host_out,
                 rstg_residue_energy* decomp);
  // PB polar terms of F frames replace the placeholder polar terms in out.
  void run_pb(const void* frames, bool f64, bool host_in, int64_t F, rstg_frame_energy* out, bool host_out);
  int64_t pb_points_estimate() const;
  int graph_kernels() const;
};

}  // namespace rstg

struct rstg_system : rstg::System {
  using rstg::System::System;
};
