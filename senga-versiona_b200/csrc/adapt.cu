// Device part of ADAPTT (src/adaptt.f:53-330): per conserved field the
// maximum over the box of |ERR| / (|RUN| + norm). The PID controller itself
// is a handful of scalar operations and runs on the host between steps
// (senga_capi.cu), in the reference's order of operations.
#include <cuda_runtime.h>

#include "senga_internal.h"

namespace senga {
namespace {

constexpr int kRedBlock = 256;

// Non-negative doubles order like their bit patterns read as unsigned
// integers, so a 64-bit atomicMax on the bits is a max on the values.
__global__ void __launch_bounds__(kRedBlock) k_errmax(int64_t n, const double* __restrict__ err,
                                                      const double* __restrict__ run, ErrNorms nrm,
                                                      unsigned long long* __restrict__ out) {
  const int fl = blockIdx.y;
  const double* e = err + (int64_t)fl * n;
  const double* r = run + (int64_t)fl * n;
  const double den0 = nrm.v[fl];
  double m = 0.0;
  for (int64_t q = (int64_t)blockIdx.x * kRedBlock + threadIdx.x; q < n; q += (int64_t)gridDim.x * kRedBlock) {
    const double v = fabs(e[q]) / (fabs(r[q]) + den0);
    m = v > m ? v : m;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_xor_sync(0xffffffffu, m, o);
    m = w > m ? w : m;
  }
  __shared__ double wm[kRedBlock / 32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = wm[0];
    for (int w = 1; w < kRedBlock / 32; ++w) b = wm[w] > b ? wm[w] : b;
    atomicMax(out + fl, (unsigned long long)__double_as_longlong(b));
  }
}

}  // namespace

void launch_errmax(int64_t n, int nc, const double* err, const double* run, const ErrNorms& nrm,
                   unsigned long long* out, int sms, cudaStream_t s) {
  cudaMemsetAsync(out, 0, nc * sizeof(unsigned long long), s);
  int64_t blocks = (n + kRedBlock - 1) / kRedBlock;
  const int64_t cap = (int64_t)sms * 4;
  if (blocks > cap) blocks = cap;
  k_errmax<<<dim3((unsigned)blocks, (unsigned)nc), kRedBlock, 0, s>>>(n, err, run, nrm, out);
}

}  // namespace senga
