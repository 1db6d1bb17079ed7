// FP64 FMA throughput probe: the denominator of the FP64-pipe roofline of
// the pointwise thermochemistry kernel (the measured HBM and bf16 peaks of
// the device carry no FP64 figure). No counterpart in the reference.
#include <cuda_runtime.h>

#include "senga_gpu.h"
#include "senga_internal.h"

namespace senga {
namespace {

constexpr int kChains = 8;     // independent FMA chains per thread (hides the pipe latency)
constexpr int kIters = 4096;   // FMAs per chain
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_dfma(double a, double b, double* out) {
  double x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = (double)(threadIdx.x + c) * 1e-3;
#pragma unroll 4
  for (int i = 0; i < kIters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  if (s == 1234.5678) out[0] = s;  // keeps the chains live; never true for these inputs
}

}  // namespace
}  // namespace senga

extern "C" int senga_fp64_peak(int device, double* tflops) {
  using namespace senga;
  if (!tflops) return fail(SENGA_ERR_ARG, "senga_fp64_peak: null output");
  int sms = 0;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return fail(SENGA_ERR_CUDA, "senga_fp64_peak: no such device");
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return fail(SENGA_ERR_CUDA, "senga_fp64_peak: cudaMalloc");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int grid = sms * 8;
  senga::k_dfma<<<grid, kThreads>>>(0.999999, 1e-9, out);  // warm-up
  cudaEventRecord(e0);
  const int reps = 5;
  for (int r = 0; r < reps; ++r) senga::k_dfma<<<grid, kThreads>>>(0.999999, 1e-9, out);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess || ms <= 0.f) return fail(SENGA_ERR_CUDA, "senga_fp64_peak: launch failed");
  const double flops = 2.0 * kChains * (double)kIters * kThreads * grid * reps;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return SENGA_OK;
}
