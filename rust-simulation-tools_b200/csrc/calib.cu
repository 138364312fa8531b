// Peak rates of the non-tensor pipes this library's pair kernels use:
// FP32 FMA, FP64 FMA and the MUFU ex2 unit, measured with dependent-chain
// loops (8 independent chains per thread) over every SM.
#include "internal.hpp"

namespace rstg {

__global__ void k_fma32(float* out, int iters) {
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = (float)(threadIdx.x + k) * 1e-6f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = fmaf(a[k], 0.999999f, 1e-7f);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; k++) s += a[k];
  if (s == 123.456f) out[0] = s;  // keeps the chains live
}

__global__ void k_fma64(double* out, int iters) {
  double a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = (double)(threadIdx.x + k) * 1e-6;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = fma(a[k], 0.999999, 1e-7);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += a[k];
  if (s == 123.456) out[0] = s;
}

__global__ void k_ex2(float* out, int iters, long long* ticks) {
  long long t0 = clock64();
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = (float)(threadIdx.x + k) * -1e-6f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) {
      float r;
      asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a[k]));
      a[k] = r * -0.5f;
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; k++) s += a[k];
  if (s == 123.456f) out[0] = s;
  if (blockIdx.x == 0 && threadIdx.x == 0) *ticks = clock64() - t0;
}

}  // namespace rstg

using namespace rstg;

extern "C" rstg_status rstg_calibrate(int device, double* out4) {
  try {
    if (!out4) throw Error(RSTG_ERR_INVALID, "out must not be NULL");
    RSTG_CUDA(cudaSetDevice(device));
    cudaDeviceProp p;
    RSTG_CUDA(cudaGetDeviceProperties(&p, device));
    int blocks = p.multiProcessorCount * 8, threads = 256, iters = 4096;
    void* buf;
    long long* ticks;
    RSTG_CUDA(cudaMalloc(&buf, 64));
    ticks = (long long*)((char*)buf + 32);
    cudaEvent_t a, b;
    RSTG_CUDA(cudaEventCreate(&a));
    RSTG_CUDA(cudaEventCreate(&b));
    auto timed = [&](auto launch) {
      launch();  // warm-up
      RSTG_CUDA(cudaEventRecord(a));
      for (int r = 0; r < 5; r++) launch();
      RSTG_CUDA(cudaEventRecord(b));
      RSTG_CUDA(cudaEventSynchronize(b));
      float ms = 0.f;
      RSTG_CUDA(cudaEventElapsedTime(&ms, a, b));
      return ms / 5.0;
    };
    double n = (double)blocks * threads * iters * 8;
    double t32 = timed([&] { k_fma32<<<blocks, threads>>>((float*)buf, iters); });
    double t64 = timed([&] { k_fma64<<<blocks, threads>>>((double*)buf, iters / 4); });
    double tex = timed([&] { k_ex2<<<blocks, threads>>>((float*)buf, iters / 4, ticks); });
    long long tk = 0;
    RSTG_CUDA(cudaMemcpy(&tk, ticks, 8, cudaMemcpyDeviceToHost));
    RSTG_CUDA(cudaGetLastError());
    out4[0] = 2.0 * n / (t32 * 1e-3) / 1e12;
    out4[1] = 2.0 * (n / 4) / (t64 * 1e-3) / 1e12;
    out4[2] = (n / 4) / (tex * 1e-3) / 1e9;
    int khz = 0;
    RSTG_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, device));
    out4[3] = khz / 1000.0;  // nominal maximum SM clock
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(buf);
    return RSTG_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  }
}
