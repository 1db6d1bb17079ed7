// Start-up temperature and pressure, TEMPIN (src/tempin.f:58-524).
//
// One thread per interior point, reading the conserved state of the U
// register: the energy residual R(T) = sum_k rhoY_k e_k(T) + 1/2 rho|u|^2
// - rho E, each species' polynomial taken from the interval that holds T
// (:75-140), is bracketed from the guess TRIN by 50 K steps inside
// [200, 3000] K (:150-352) and then bisected until |R| < 1e-4 (:364-436);
// ITNDEX and p = T sum_k rhoY_k R_k follow at the root (:444-508). The sums
// and the Horner evaluation are rounded without contraction, so every branch
// decision and the returned T equal a host evaluation in IEEE double bit
// for bit. Where the source stops (no sign change inside the limits) the
// point keeps its last iterate and sets status bit 1; the source bisects
// without limit, here 200 halvings at most, after which status bit 2 is set.
#include "itndex.cuh"
#include "senga_internal.h"

namespace senga {
namespace {

constexpr double kTolTmp = 1.0e-4;  // TOLTMP
constexpr double kTinInc = 5.0e1;   // TININC
constexpr double kTLimLo = 2.0e2, kTLimHi = 3.0e3;
constexpr int kNctMax = 5;          // NCTMAX: degree of the energy polynomial
constexpr int kMaxSteps = 1 << 16;  // bracketing steps (the limits end them first for any finite guess)
constexpr int kBlock = 256;

__device__ __forceinline__ int interval_at(const senga_chem* __restrict__ C, int s, double T) {
  int it = 0;
  while (T > C->tinthi[s][it] && it + 1 < C->ntint[s]) ++it;
  return it;
}

__device__ double residual(const senga_chem* __restrict__ C, int nspec, const double* ry, double tuk2me, double T) {
  double tc[kNctMax + 1] = {tuk2me, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int s = 0; s < nspec; ++s) {
    const int it = interval_at(C, s, T);
    const double y = ry[s];
    const double* et = C->amasct[s][it];
    tc[0] = __dadd_rn(tc[0], __dmul_rn(y, C->amascp[s][it][C->ncenth[s][it] - 1]));
    tc[1] = __dadd_rn(tc[1], __dmul_rn(y, et[0]));
    const int np = C->ncpoly[s][it] < kNctMax ? C->ncpoly[s][it] : kNctMax;
    for (int icp = 2; icp <= np; ++icp) tc[icp] = __dadd_rn(tc[icp], __dmul_rn(y, et[icp - 1]));
  }
  double r = tc[kNctMax];
  for (int icp = kNctMax - 1; icp >= 1; --icp) r = __dadd_rn(tc[icp], __dmul_rn(r, T));
  return __dadd_rn(tc[0], __dmul_rn(r, T));
}

__global__ void __launch_bounds__(kBlock) k_tempin(int64_t n, int nspec, const double* __restrict__ U,
                                                   const senga_chem* __restrict__ C, double trin, int maxbis,
                                                   double* __restrict__ t, int32_t* __restrict__ itn,
                                                   double* __restrict__ p, unsigned int* status) {
  const int64_t q = (int64_t)blockIdx.x * kBlock + threadIdx.x;
  if (q >= n) return;
  const double rho = U[q], ru = U[n + q], rv = U[2 * n + q], rw = U[3 * n + q], re = U[4 * n + q];
  double ry[SENGA_NSPCMX];
  for (int s = 0; s < nspec; ++s) ry[s] = U[(5 + s) * n + q];
  const double ukuk = __dadd_rn(__dadd_rn(__dmul_rn(ru, ru), __dmul_rn(rv, rv)), __dmul_rn(rw, rw)) / rho;
  const double tuk2me = __dsub_rn(__dmul_rn(0.5, ukuk), re);

  double tlo = kTLimLo, thi = kTLimHi, T = trin;
  bool conv = false, lost = false;
  double r = residual(C, nspec, ry, tuk2me, T);
  if (fabs(r) < kTolTmp) {
    conv = true;
  } else if (r < 0.0) {  // guess too low: step up
    for (int k = 0;; ++k) {
      tlo = T;
      T = __dadd_rn(T, kTinInc);
      r = residual(C, nspec, ry, tuk2me, T);
      if (fabs(r) < kTolTmp) { conv = true; break; }
      if (r < 0.0) {
        if (T < kTLimHi && k < kMaxSteps) continue;
        lost = true;
        break;
      }
      if (r > 0.0) thi = T;
      break;
    }
  } else if (r > 0.0) {  // guess too high: step down
    for (int k = 0;; ++k) {
      thi = T;
      T = __dsub_rn(T, kTinInc);
      r = residual(C, nspec, ry, tuk2me, T);
      if (fabs(r) < kTolTmp) { conv = true; break; }
      if (r > 0.0) {
        if (T > kTLimLo && k < kMaxSteps) continue;
        lost = true;
        break;
      }
      if (r < 0.0) tlo = T;
      break;
    }
  }
  if (lost) {
    atomicOr(status, 2u);
  } else if (!conv) {
    int it = 0;
    for (; it < maxbis; ++it) {
      T = __dmul_rn(0.5, __dadd_rn(tlo, thi));
      r = residual(C, nspec, ry, tuk2me, T);
      if (fabs(r) < kTolTmp) break;
      if (r < 0.0) tlo = T;
      else if (r > 0.0) thi = T;
      else break;  // NaN: the source leaves the loop as well
    }
    if (it == maxbis) atomicOr(status, 4u);
  }
  uint64_t code = 0;
  double rmix = 0.0;
  for (int s = 0; s < nspec; ++s) {
    code += (uint64_t)interval_at(C, s, T) << (2 * s);
    rmix = __dadd_rn(rmix, __dmul_rn(ry[s], C->rgspec[s]));
  }
  t[q] = T;
  itn_store(itn, n, q, nspec, code);
  p[q] = __dmul_rn(T, rmix);
}

}  // namespace

void launch_tempin(int64_t n, int nspec, const double* U, const senga_chem* dchem, double trin, double* t,
                   int32_t* itn, double* p, unsigned int* status, cudaStream_t s) {
  const unsigned grid = (unsigned)((n + kBlock - 1) / kBlock);
  k_tempin<<<grid, kBlock, 0, s>>>(n, nspec, U, dchem, trin, 200, t, itn, p, status);
}

}  // namespace senga
