// Poisson-Boltzmann engine (pb_grid.rs, pb_solver.rs, pb_energy.rs).
#include "frame_plain.hpp"

namespace rstg {

double pb_energy_run(Ctx*, const std::vector<double>&, const std::vector<double>&, const std::vector<double>&,
                     const rstg_pb_params&, rstg_pb_diag*) {
  throw Error(RSTG_ERR_INVALID, "the PB engine is not part of this build yet");
}

}  // namespace rstg
