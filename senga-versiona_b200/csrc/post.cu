// Post-processing output on the device download path: the record SENGA2
// writes every NTDUMP steps for post-processing (src/output.f:240-265):
//   DRUN, URUN/DRUN, VRUN/DRUN, WRUN/DRUN, ERUN/DRUN, TRUN, PRUN,
//   YRUN(:,:,:,k)/DRUN (NSPEC fields), RRTE (NSPCMX fields), ETIME
// TRUN and PRUN are those of the last TEMPER (the fifth substage), RRTE the
// CHRATE rates saved by RHSCAL (src/rhscal.f:828) in that substage. The
// primitive fields are formed here on the device, then copied to the host in
// one transfer; the file itself is written by senga_post_write.
#include <cuda_runtime.h>

#include "senga_gpu.h"
#include "senga_internal.h"

namespace senga {
namespace {

constexpr int kPostBlock = 256;

__global__ void __launch_bounds__(kPostBlock) k_post(int64_t n, int nspec, const double* __restrict__ run,
                                                      const double* __restrict__ t, const double* __restrict__ p,
                                                      double* __restrict__ out) {
  const int64_t q = (int64_t)blockIdx.x * kPostBlock + threadIdx.x;
  if (q >= n) return;
  const double d = run[q];
  out[q] = d;
  for (int fl = 1; fl < 5; ++fl) out[fl * n + q] = run[fl * n + q] / d;
  out[5 * n + q] = t[q];
  out[6 * n + q] = p[q];
  for (int k = 0; k < nspec; ++k) out[(7 + k) * n + q] = run[(5 + k) * n + q] / d;
}

}  // namespace

void launch_post(int64_t n, int nspec, const double* run, const double* t, const double* p, double* out,
                 cudaStream_t s) {
  k_post<<<(unsigned)((n + kPostBlock - 1) / kPostBlock), kPostBlock, 0, s>>>(n, nspec, run, t, p, out);
}

}  // namespace senga
