// Molar-mass, pressure, Soret and Dufour terms of mixture-averaged transport
// (the cont.dat transport switches NFMIXW, NFMIXP, NFMSOR, NFMDUF with the
// light-species molar-mass limit WMLTDR; flags from src/diffin.f:384-406).
//
// The reference evaluates them inside RHSCAL's species loop
// (src/rhscal.f:946-1003 derivatives of ln W_mix, ln p, ln(T/TDIFGB);
// :1352-1403 thermal diffusion ratio TDRMIX; :1552-1564 Dufour term in the
// species enthalpy; :1966-2357 molar-mass, :2361-2757 pressure and
// :2760-3765 Soret branches). Every one of them adds to the species source
// RATE, the correction-velocity sums UCOR/VCOR/WCOR and VTMP, or ERHS, so
// here they run as three extra passes between the species kernel and the
// species+RK kernel, which consume those sums:
//   k_mixt_pre      pointwise: W_mix, the three logarithms, TDRMIX per light
//                   species;
//   k_mixt_grad     first derivatives of each logarithm and the sum of its
//                   second derivatives (x part zeroed on diffusion-flux
//                   faces, as ZEROXL/XR do to WD2X/PD2X/TD2X);
//   k_mixt_species  per point, all species: the branch terms, and the
//                   Dufour part of the main heat-flux terms (the species
//                   kernel formed those with the plain enthalpy h_k; the
//                   reference uses h_k + R_k T TDRMIX_k, so the difference,
//                   linear in the enthalpy, is added here).
// Neighbour values come from global memory through the read-only cache:
// these passes are off by default and sit outside the headline step.
//
// Kept as coded: in the molar-mass and pressure branches the x component of
// the "species enthalpy gradient" is STORE4, which the code before them
// overwrote with DIFMIX (src/rhscal.f:1882-1891); the term is restated with
// that value.
#include <cuda_runtime.h>

#include "senga_gpu.h"
#include "senga_internal.h"
#include "stencil.cuh"

namespace senga {
namespace {

constexpr int kMixBlock = 128;

__global__ void __launch_bounds__(kMixBlock) k_mixt_pre(Geo g, Fields f, MixtParams m, const senga_chem* __restrict__ ch,
                                                        const senga_diff* __restrict__ df, int nspec) {
  const int64_t q = (int64_t)blockIdx.x * kMixBlock + threadIdx.x;
  if (q >= g.n) return;
  const int64_t n = g.n;
  // W_mix = rho / sum_k (rho Y_k / W_k)  (rhscal.f mixture-averaged conductivity block)
  double c3 = 0.0;
  for (int k = 0; k < nspec; ++k) c3 = c3 + f.uin[(5 + k) * n + q] * ch->ovwmol[k];
  c3 = 1.0 / c3;
  const double wmix = f.uin[q] * c3;
  m.wmix[q] = wmix;
  const double T = f.t[q];
  if (m.w) m.lng[0][q] = log(wmix);
  if (m.p) m.lng[1][q] = log(f.p[q]);
  if (m.t) m.lng[2][q] = log(T / df->tdifgb);
  if (!m.tdr) return;
  const double combo2 = T / df->tdifgb;
  const int nct = df->ncotdr;
  for (int k = 0; k < nspec; ++k) {
    if (!((m.tdr >> k) & 1u)) continue;
    double acc = 0.0;
    for (int j = 0; j < nspec; ++j) {
      if (!((m.tdr >> j) & 1u) || j == k) continue;
      double c = df->tdrcco[k][j][nct - 1];
      for (int icp = nct - 2; icp >= 0; --icp) c = c * combo2 + df->tdrcco[k][j][icp];
      const double fornow = f.y[j * n + q] * ch->ovwmol[j];
      acc = acc + fornow * wmix * c;
    }
    m.tdrmix[k * n + q] = acc * f.y[k * n + q] * wmix * ch->ovwmol[k];
  }
}

__global__ void __launch_bounds__(kMixBlock) k_mixt_grad(Geo g, MixtParams m) {
  const int64_t q = (int64_t)blockIdx.x * kMixBlock + threadIdx.x;
  if (q >= g.n) return;
  const int64_t n = g.n;
  const Pt pt = point_of(g, q);
  const bool dif = !g.per[0] && (face_bits(g, pt.i) & BF_DIF);
  const int on[3] = {m.w, m.p, m.t};
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    if (!on[b]) continue;
    const Ld F{m.lng[b]};
    m.g1[b][q] = D1<0>(g, pt, F);
    m.g1[b][n + q] = D1<1>(g, pt, F);
    m.g1[b][2 * n + q] = D1<2>(g, pt, F);
    const double d2x = dif ? 0.0 : D2<0>(g, pt, F);
    m.g2[b][q] = d2x + D2<1>(g, pt, F) + D2<2>(g, pt, F);
  }
}

// value of a pointwise function of the fields at a neighbour, for D1
template <class Fn>
struct At {
  Fn fn;
  __device__ __forceinline__ double operator()(int64_t q) const { return fn(q); }
};
template <class Fn>
__device__ __forceinline__ At<Fn> at(Fn fn) {
  return At<Fn>{fn};
}

template <class F>
__device__ __forceinline__ void grad(const Geo& g, const Pt& pt, const F& acc, bool zero_x, double d[3]) {
  d[0] = zero_x ? 0.0 : D1<0>(g, pt, acc);
  d[1] = D1<1>(g, pt, acc);
  d[2] = D1<2>(g, pt, acc);
}
__device__ __forceinline__ double dot(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

__global__ void __launch_bounds__(kMixBlock) k_mixt_species(Geo g, Fields f, MixtParams m, const senga_chem* __restrict__ ch,
                                                            int nspec) {
  const int64_t q = (int64_t)blockIdx.x * kMixBlock + threadIdx.x;
  if (q >= g.n) return;
  const int64_t n = g.n;
  const Pt pt = point_of(g, q);
  const bool dif = !g.per[0] && (face_bits(g, pt.i) & BF_DIF);
  const double* __restrict__ T = f.t;
  const double* __restrict__ wm = m.wmix;
  double gW[3] = {0, 0, 0}, gP[3] = {0, 0, 0}, gT[3] = {0, 0, 0};
  double lW = 0.0, lP = 0.0, lT = 0.0;
  for (int d = 0; d < 3; ++d) {
    if (m.w) gW[d] = m.g1[0][d * n + q];
    if (m.p) gP[d] = m.g1[1][d * n + q];
    if (m.t) gT[d] = m.g1[2][d * n + q];
  }
  if (m.w) lW = m.g2[0][q];
  if (m.p) lP = m.g2[1][q];
  if (m.t) lT = m.g2[2][q];
  double vc[3] = {0.0, 0.0, 0.0}, vt = 0.0, eacc = 0.0;
  for (int k = 0; k < nspec; ++k) {
    const double* __restrict__ rdk = f.rd + k * n;
    const double* __restrict__ yk = f.y + k * n;
    const double* __restrict__ hk = f.h + k * n;
    const double* __restrict__ tk = m.tdrmix ? m.tdrmix + k * n : nullptr;
    const bool duf = (m.duf >> k) & 1u, sor = (m.sor >> k) & 1u;
    const double rg = ch->rgspec[k], wk = ch->wmolar[k];
    const double rd = rdk[q], y = yk[q], h = hk[q];
    const double delta = duf ? rg * T[q] * tk[q] : 0.0;
    const double hp = duf ? h + delta : h;  // UTMP with the Dufour term
    double src = 0.0;                       // added to RATE
    double dY[3];
    if (duf) {
      // the Dufour part of the main heat-flux terms: (grad rhoD . grad Y) dh,
      // (grad dh . grad Y) rhoD, (rhoD lap Y) dh, dh = R_k T TDRMIX_k
      grad(g, pt, Ld{yk}, false, dY);
      double dRD[3], dDl[3];
      grad(g, pt, Ld{rdk}, dif, dRD);
      grad(g, pt, at([=](int64_t r) { return rg * T[r] * tk[r]; }), dif, dDl);
      const Ld Y{yk};
      const double lapY = (dif ? 0.0 : D2<0>(g, pt, Y)) + D2<1>(g, pt, Y) + D2<2>(g, pt, Y);
      eacc = eacc + dot(dRD, dY) * delta + dot(dDl, dY) * rd + lapY * rd * delta;
    }
    // molar-mass and pressure branches share the enthalpy gradient: x part
    // DIFMIX (see the file comment), y/z parts those of h_k + Dufour term
    double hy = 0.0, hz = 0.0;
    if (m.w || m.p) {
      if (duf) {
        const auto hpa = at([=](int64_t r) { return hk[r] + rg * T[r] * tk[r]; });
        hy = D1<1>(g, pt, hpa);
        hz = D1<2>(g, pt, hpa);
      } else {
        hy = D1<1>(g, pt, Ld{hk});
        hz = D1<2>(g, pt, Ld{hk});
      }
    }
    const double hx = dif ? 0.0 : rd;
    auto branch = [&](double s7, const double dS[3], const double gG[3], double lG) {
      for (int d = 0; d < 3; ++d) vc[d] = vc[d] + s7 * gG[d];
      const double f1 = dot(dS, gG);
      const double f2 = lG * s7;
      src = src + f1 + f2;
      vt = vt + f1 + f2;
      eacc = eacc + f1 * hp + (hx * gG[0] + hy * gG[1] + hz * gG[2]) * s7 + f2 * hp;
    };
    if (m.w) {
      double dS[3];
      grad(g, pt, LdMul{rdk, yk}, dif, dS);
      branch(rd * y, dS, gW, lW);
    }
    if (m.p) {
      double dS[3];
      grad(g, pt, at([=](int64_t r) { return rdk[r] * yk[r] * (1.0 - wk / wm[r]); }), dif, dS);
      branch(rd * y * (1.0 - wk / wm[q]), dS, gP, lP);
    }
    if (sor) {
      const double s7 = rd * y * tk[q];
      double dS[3], dU[3];
      grad(g, pt, at([=](int64_t r) { return rdk[r] * yk[r] * tk[r]; }), dif, dS);
      // UTMP with the Dufour term taken out again, and its gradient
      const double u = duf ? hp - delta : h;
      if (duf)
        grad(g, pt, at([=](int64_t r) {
               const double dl = rg * T[r] * tk[r];
               return (hk[r] + dl) - dl;
             }),
             dif, dU);
      else
        grad(g, pt, Ld{hk}, dif, dU);
      for (int d = 0; d < 3; ++d) vc[d] = vc[d] + s7 * gT[d];
      const double f1 = dot(dS, gT);
      const double f2 = lT * s7;
      src = src + f1 + f2;
      vt = vt + f1 + f2;
      eacc = eacc + f1 * u + dot(dU, gT) * s7 + f2 * u;
    }
    if (src != 0.0) f.wdot[k * n + q] += src;
  }
  f.vc[q] += vc[0];
  f.vc[n + q] += vc[1];
  f.vc[2 * n + q] += vc[2];
  f.vtmp[q] += vt;
  f.rhs[4 * n + q] += eacc;
}

inline unsigned grid_of(int64_t n) { return (unsigned)((n + kMixBlock - 1) / kMixBlock); }

}  // namespace

int launch_mixt(const Geo& g, const Fields& f, const MixtParams& m, const senga_chem* dchem, const senga_diff* ddiff,
                int nspec, cudaStream_t s) {
  const unsigned gr = grid_of(g.n);
  k_mixt_pre<<<gr, kMixBlock, 0, s>>>(g, f, m, dchem, ddiff, nspec);
  int nl = 1;
  if (m.w || m.p || m.t) {
    k_mixt_grad<<<gr, kMixBlock, 0, s>>>(g, m);
    ++nl;
  }
  k_mixt_species<<<gr, kMixBlock, 0, s>>>(g, f, m, dchem, nspec);
  return nl + 1;
}

}  // namespace senga
