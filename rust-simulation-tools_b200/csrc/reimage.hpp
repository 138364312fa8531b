// Periodic reimaging of the complex (reimage_complex, binding.rs:234-308),
// host and device forms with the same arithmetic and order.
#pragma once
#include <array>
#include <cstdint>
#include <vector>

#include "internal.hpp"

namespace rstg {

// Host form, one frame: x holds the n complex atoms' coordinates (Angstrom,
// complex numbering), t the complex topology (its bonds).
void reimage_host(double* x, int64_t n, const Topology& t, const std::array<double, 3>& box);

// Device form: F frames in topology order ([F][n_top][3] Angstrom, device
// memory, reimaged in place), the complex of `sp`, per-frame box edges
// [F][3] (device memory).  Launches on `st`.
void reimage_device(Ctx* ctx, cudaStream_t st, const Split& sp, int64_t n_top, double* d_frames,
                    const double* d_boxes, int64_t F);

}  // namespace rstg
