// Batched mixed-precision Poisson-Boltzmann engine (pb_batch.cu).
#pragma once
#include <memory>
#include <vector>

#include "pb.cuh"

namespace rstg {

// One grid solve of a batch.
struct PbJob {
  PbGeom g;
  const AtomsDev* atoms = nullptr;
  bool uniform = false;  // reference solve: dielectric ein everywhere, kbar^2 = 0
  bool ionic = false;    // kbar^2 map from the ion-accessible region
  double ein = 1.0, eout = 80.0, kap = 0.0;
  BcSpec bc;             // Debye-Hueckel, or interpolated from bc.cphi on *bc.cg
  double tol = 1e-6;
  int64_t maxit = 10000;
  double rtol = 0.0;     // > 0: consistent multigrid, stop on this relative FP64 residual (not the reference's rule)
  bool energy = true;    // 0.5 sum q phi(atom) wanted
  int rho_of = -1;       // index of an earlier job of the batch with the same grid and atoms: use its charge map
  // results
  PbSolveStats stats{};
  double e = 0.0;        // energy (kcal/mol) when requested
  double maxabs = 0.0;   // max |phi| over the grid
  bool fallback = false; // solved by the FP64 path (grid too small for multigrid, or divergence)
};

struct PbBatchStats {
  int64_t cycles = 0;      // lock-step cycles run
  int64_t fallbacks = 0;   // jobs solved by the FP64 path
  int64_t jobs = 0;
  double ms_setup = 0.0;   // maps and boundary values
  double ms_cycles = 0.0;  // lock-step multigrid cycles
  double ms_finish = 0.0;  // FP64 fallbacks, energies
};

// Per-kernel device time of the level-0 multigrid kernels (profile mode):
// 0 colour sweep, 1 FP32 residual, 2 FP64 residual, 3 update; bytes are the
// algorithmic (compulsory) DRAM bytes of the timed launches.
constexpr int kProfKernels = 4;
// Per kernel family and multigrid level: sweep, FP32 residual, restriction,
// prolongation, coarsest level, FP64 residual, update, norm, SOR fallback.
constexpr int kProfDetail = 9, kProfLevels = 16;
struct PbProfile {
  double ms[kProfKernels] = {}, bytes[kProfKernels] = {};
  int64_t launches[kProfKernels] = {};
  double detail_ms[kProfDetail][kProfLevels] = {};
  int64_t detail_n[kProfDetail][kProfLevels] = {};
};

class PbBatchEngine {
 public:
  PbBatchEngine(Ctx* c, cudaStream_t st) : c_(c), st_(st) {}
  ~PbBatchEngine();
  // Builds maps and boundary values of every job, solves them in lock step
  // and fills stats / e / maxabs.  keep_phi: copy each job's potential into
  // phi_out[j] (device arrays of g.n() doubles, may be null per job).
  void solve(std::vector<PbJob>& jobs, const rstg_pb_params& p, const std::vector<double*>* phi_out = nullptr);
  void set_stream(cudaStream_t s) { st_ = s; }
  // Frees the device pools (kept between solves otherwise); statistics stay.
  void release();
  PbBatchStats stats;
  PbProfile prof;
  bool profile = false;  // time the level-0 kernels with events (no graph capture)
  int chunk_cycles = 8;  // cycles per graph launch between status reads

 private:
  Ctx* c_;
  cudaStream_t st_;
  DevBuf pool64_, pool32_, pool8_, desc_, part_, small_, lists_;
  cudaGraphExec_t graph_ = nullptr;
  static constexpr int kSetupWorkers = 8;       // threads (and streams) of the per-grid set-up
  std::vector<cudaStream_t> setup_streams_;
  std::vector<cudaEvent_t> setup_events_;
  cudaEvent_t start_event_ = nullptr;
  std::vector<cudaEvent_t> prof_events_;
};

// Polar PB energies (E_solvated - E_reference, pb_energy.rs:332-438) of
// n_sets atom sets, batched.  xyz[i]: host Angstrom coordinates; q in e.
// out[i] receives the energy, diag[i] (optional) the solve statistics.
// rtol > 0 solves every grid (focusing coarse grids included) to that
// relative FP64 residual with the consistent multigrid instead of the
// reference's schedule.
void pb_polar_batch(Ctx* c, cudaStream_t st, PbBatchEngine& eng, const rstg_pb_params& p,
                    const std::vector<const std::vector<double>*>& xyz, const std::vector<const std::vector<double>*>& q,
                    const std::vector<const std::vector<double>*>& r, double* out, rstg_pb_diag* diag,
                    double rtol = 0.0);

}  // namespace rstg
