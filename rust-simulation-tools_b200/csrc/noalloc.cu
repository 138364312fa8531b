// GB energy for callers that must not allocate device memory.
//
// Some callers cannot call cudaMalloc (or any allocating routine) at the point
// where they need an energy: code running under an allocator owned by a host
// framework that forbids side allocations, latency-critical loops that must
// not hit the driver's allocator, or code running where an allocation would
// synchronise the device.  This entry point takes device inputs and device
// outputs and keeps its scratch -- the Born radii when the caller does not
// want them, and one partial sum per warp -- in a file-scope device array.
//
// The array is kGbScratchDoubles doubles (1.5 MiB) and every GPU that loads
// this library holds it until the process exits.  Host code cannot use the
// array's name as a device address, so the first call on each device resolves
// the address with cudaGetSymbolAddress (with that device current) and caches
// it with the id of the device's context (a device reset gives a new context,
// and the address is then resolved again); that first call on a device, or
// after a reset, should therefore come before any stream capture.  All
// calls on a device share the array: calls whose kernels overlap on the GPU
// (for example on two streams) race and must be serialised by the caller.
// Every scratch element a call reads is written earlier in the same call, so
// nothing needs clearing between calls.
#include <mutex>

#include "plain.cuh"

namespace rstg {

constexpr int64_t kGbScratchDoubles = 3 * 65536;  // radii [n] + warp partials [(n + 1) / 2]
constexpr int64_t kGbNoAllocMaxAtoms = 131072;    // n + (n + 1) / 2 <= kGbScratchDoubles
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_gb_scratch[kGbScratchDoubles];

static std::mutex g_scratch_mu;
static double* g_scratch_addr[kMaxDevices] = {};
static unsigned long long g_scratch_ctx[kMaxDevices] = {};

// Process-unique id of the calling thread's current CUDA context (0 when it
// cannot be read).  After cudaDeviceReset the device gets a new primary
// context, the module is loaded again and the array may sit at a new
// address; the id tells the cached address apart from a stale one.  The
// driver functions come through the runtime's entry-point query, so the
// library needs no link against libcuda.
static unsigned long long current_ctx_id() {
  typedef int (*GetCurrent)(void**);
  typedef int (*GetId)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (GetCurrent)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (GetId)f;
    looked_up = true;
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&ctx) == 0 && ctx && get_id(ctx, &id) == 0) return id;
  return 0;
}

// Device address of g_gb_scratch on the current device.  Resolved once per
// device and context (the caller has made the device current), and again
// only when the device's context has changed.
static double* scratch_on(int device) {
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  unsigned long long id = current_ctx_id();
  if (!g_scratch_addr[device] || g_scratch_ctx[device] != id) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_gb_scratch);
    if (e != cudaSuccess || !p)
      throw Error(RSTG_ERR_CUDA, std::string("cudaGetSymbolAddress of the GB scratch array failed: ") +
                                     cudaGetErrorString(e));
    g_scratch_addr[device] = (double*)p;
    g_scratch_ctx[device] = id;
  }
  return g_scratch_addr[device];
}

}  // namespace rstg

using namespace rstg;

extern "C" rstg_status rstg_gb_energy_noalloc_async(const double* d_xyz, const double* d_charges_amber,
                                                    const double* d_radii, const double* d_screen, int64_t n_atoms,
                                                    const rstg_gb_params* params, double* d_total,
                                                    double* d_born_radii, void* stream) {
  try {
    if (!d_xyz || !d_charges_amber || !d_radii || !d_screen || !d_total)
      throw Error(RSTG_ERR_INVALID, "coordinate, charge, radius, screen and total pointers must not be NULL");
    if (n_atoms < 1 || n_atoms > kGbNoAllocMaxAtoms)
      throw Error(RSTG_ERR_INVALID, "rstg_gb_energy_noalloc_async supports 1 to " +
                                        std::to_string(kGbNoAllocMaxAtoms) + " atoms, got " +
                                        std::to_string(n_atoms));
    rstg_gb_params p;
    if (params)
      p = *params;
    else
      rstg_gb_params_default(&p);
    if (p.model < 0 || p.model > 2) throw Error(RSTG_ERR_INVALID, "unknown GB model");
    int dev = 0;
    RSTG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error(RSTG_ERR_INVALID, "device ordinal out of range");
    double* scratch = scratch_on(dev);
    cudaStream_t st = (cudaStream_t)stream;
    int n = (int)n_atoms;
    int64_t nw = (n_atoms + 1) / 2;
    double* R = d_born_radii ? d_born_radii : scratch;
    double* part = scratch + n_atoms;
    k_born_radii_plain<<<(unsigned)((n_atoms + 7) / 8), 256, 0, st>>>(n, d_xyz, d_radii, d_screen, p.offset,
                                                                       p.cutoff * p.cutoff, p.model, p.rgbmax, R);
    k_gb_plain<<<(unsigned)((nw + 7) / 8), 256, 0, st>>>(n, d_xyz, d_charges_amber, R, gb_const(p), part);
    k_sum_columns<<<1, 512, 0, st>>>(part, nw, 1, d_total);
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw Error(RSTG_ERR_CUDA, std::string("kernel launch failed: ") + cudaGetErrorString(e));
    }
    return RSTG_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  }
}
