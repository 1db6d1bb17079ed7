// Per-point thermochemistry of the substage, shared by the pointwise kernels
// (kernels.cu) and the persistent batch kernel (kernels_tiled.cu): CHRATE
// (src/chrate.f:146-741), the mechanism policies (table-driven MechTables and
// the generated straight-line policies of mech_gen.cuh) and thermo_point,
// which fuses TEMPER (src/temper.f:58-219), the primitive variables,
// transport properties, species enthalpies and CHRATE at one grid point.
// Everything here has internal linkage: each translation unit that includes
// it compiles its own copy.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "itndex.cuh"
#include "mech_gen.cuh"
#include "senga_internal.h"

namespace senga {
namespace {
constexpr double kPrantl = 7.0e-1;  // src/com_senga2.h:115
constexpr double kRlamda = 7.0e-1;  // :113
constexpr double kYsmall = 1.0e-30, kYdenom = 1.0e-15;  // src/chrate.f:40
constexpr double kDfctol = 1.0e-12;                     // src/com_senga2.h:187
constexpr int kBlock = 256;

// Interval of species s packed in ITNDEX (2 bits per species). NTINMX = 2,
// so only 0/1 are valid; the mask keeps a corrupt upload inside the tables.
__device__ __forceinline__ int tint_of(uint64_t itn, int s) { return (int)(itn >> (2 * s)) & 1; }

// Select-by-index update of a register array (keeps the array in registers
// when the index comes from a table).
template <int NSM>
__device__ __forceinline__ void add_at(double (&a)[NSM], int k, double v) {
#pragma unroll
  for (int s = 0; s < NSM; ++s)
    if (s == k) a[s] += v;
}
template <int NSM>
__device__ __forceinline__ double get_at(const double (&a)[NSM], int k) {
  double r = 0.0;
#pragma unroll
  for (int s = 0; s < NSM; ++s)
    if (s == k) r = a[s];
  return r;
}

// -------------------------------------------------------------------------
// CHRATE for one point. ry: rho*Y_k, T, itn (updated interval index).
// Gibbs functions and log T are hoisted out of the step loop: the reference
// evaluates the same expressions per step, so the values are identical.
template <int NSM>
__device__ void chrate_point(const senga_chem* __restrict__ C, int nspec, const double (&ry)[NSM], double T,
                             uint64_t itn, double (&rate)[NSM]) {
  const double lnT = log(T);
  const double ovT = 1.0 / T;
  double gib[NSM];
#pragma unroll
  for (int s = 0; s < NSM; ++s) {
    rate[s] = 0.0;
    gib[s] = 0.0;
    if (s < nspec && C->ngibb > 0) {
      const int it = tint_of(itn, s);
      const int np = C->ncpoly[s][it];
      const double* gb = C->amolgb[s][it];
      double g = gb[np - 1];
      for (int icp = np - 1; icp >= 1; --icp) g = gb[icp - 1] + g * T;
      gib[s] = gb[C->ncenth[s][it] - 1] / T - gb[C->ncenpy[s][it] - 1] * lnT - g;
    }
  }
  double s3 = 0.0;
  for (int st = 0; st < C->nstep; ++st) {
    bool flthrd = true;
    const int ib = C->mblist[st];
    if (ib != 0) {
      s3 = 0.0;
#pragma unroll
      for (int s = 0; s < NSM; ++s)
        if (s < nspec) s3 += ry[s] * (C->ovwmol[s] * C->effy3b[ib - 1][s]);
    }
    double s2 = C->rparam[st][0] + C->rparam[st][1] * lnT - C->rparam[st][2] * ovT;
    double s1 = exp(s2);
    if (C->mllist[st] != 0) {
      const double* rl = C->rclind[C->mllist[st] - 1];
      const double flcnst = (double)(float)rl[3];  // implicit REAL in the reference
      const double s4 = exp(rl[0] + rl[1] * lnT - rl[2] * ovT);
      const double pr = s3 * s4 / s1;
      s1 = s1 * (flcnst * pr / (1.0 + pr));
      s2 = log(s1);
      flthrd = false;
    }
    if (C->mtlist[st] != 0) {
      const double* rt = C->rctroe[C->mtlist[st] - 1];
      const double talpha = (double)(float)rt[3];
      const double cf1 = (double)(float)rt[7], cf2 = (double)(float)rt[8];
      const double en1 = (double)(float)rt[9], en2 = (double)(float)rt[10], dtc = (double)(float)rt[11];
      const double s4 = exp(rt[0] + rt[1] * lnT - rt[2] * ovT);
      const double pr = s3 * s4 / s1;
      double ftc = (1.0 - talpha) * exp(T * rt[6]) + talpha * exp(T * rt[4]) + exp(-rt[5] / T);
      ftc = log10(ftc);
      const double cfa = cf1 + cf2 * ftc, enf = en1 + en2 * ftc;
      double fn = log10(pr) + cfa;
      fn = fn / (enf - dtc * fn);
      fn = 1.0 + fn * fn;
      const double fbroad = exp((ftc / fn) * 2.302585092994046);
      s1 = s1 * (fbroad * pr / (1.0 + pr));
      s2 = log(s1);
      flthrd = false;
    }
    if (C->mslist[st] != 0) {
      const double* rs = C->rcsrif[C->mslist[st] - 1];
      const double s4 = exp(rs[0] + rs[1] * lnT - rs[2] * ovT);
      const double pr = s3 * s4 / s1;
      double fb = rs[3] * exp(rs[4] / T) + exp(T * rs[5]);
      const double fn = 1.0 / (1.0 + log10(log10(pr)));
      fb = rs[6] * exp(fn * log(fb));
      s1 = s1 * (fb * pr / (1.0 + pr));
      s2 = log(s1);
      flthrd = false;
    }
    for (int l = 0; l < C->nrslen[st]; ++l) {
      const int s = C->nrspec[st][l] - 1;
      s1 = s1 * fmax(get_at(ry, s) * C->ovwmol[s], 0.0);
    }
    for (int l = 0; l < C->nrclen[st]; ++l) {
      const int s = C->nrcpec[st][l] - 1;
      double fn = fmax(get_at(ry, s) * C->ovwmol[s], kYsmall);
      fn = exp(C->crspec[st][l] * log(fn));
      s1 = s1 * (fn / (1.0 + kYdenom * fn));
    }
    if (C->mglist[st] != 0) {
      for (int l = 0; l < C->nsslen[st]; ++l) s2 = s2 + C->diffmu[st][l] * get_at(gib, C->nsspec[st][l] - 1);
      s2 = exp(s2);
      for (int l = 0; l < C->npslen[st]; ++l) {
        const int s = C->npspec[st][l] - 1;
        s2 = s2 * fmax(get_at(ry, s) * C->ovwmol[s], 0.0);
      }
      for (int l = 0; l < C->npclen[st]; ++l) {
        const int s = C->npcpec[st][l] - 1;
        double fn = fmax(get_at(ry, s) * C->ovwmol[s], kYsmall);
        fn = exp(C->cpspec[st][l] * log(fn));
        s2 = s2 * (fn / (1.0 + kYdenom * fn));
      }
      s1 = s1 - s2;
    }
    if (ib != 0 && flthrd) s1 = s1 * s3;
    for (int l = 0; l < C->nsslen[st]; ++l) add_at(rate, C->nsspec[st][l] - 1, s1 * C->diffmw[st][l]);
  }
}

// -------------------------------------------------------------------------
// Mechanism policies. A policy supplies the per-point thermochemistry of one
// mechanism: TEMPER's e(T) polynomial (src/temper.f:84-122), interval
// location and mixture cp (:168-209), transport properties (src/rhscal.f:
// 515-571, 1292-1340, 3854-3885; src/rhsvel.f:933-952), species enthalpy
// (src/rhscal.f:1444-1466) and CHRATE. MechTables reads the tables of any
// chem.dat/diff.dat; generated policies (mech_gen.cuh) hard-code one
// mechanism and are selected only when the loaded tables match them exactly.
template <int NSM, bool MAVT_>
struct MechTables {
  static constexpr int NS = NSM;
  static constexpr bool MAVT = MAVT_;
  const senga_chem* __restrict__ C;
  const senga_diff* __restrict__ Dt;
  int nspec;

  __device__ __forceinline__ bool has(int s) const { return s < nspec; }
  __device__ __forceinline__ int count() const { return nspec; }

  __device__ __forceinline__ void temper_coeffs(const double (&ry)[NS], uint64_t itn0, double (&tc)[6], double (&td)[6],
                                                double& rmix) const {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      if (s >= nspec) continue;
      const int it = tint_of(itn0, s);
      const double y = ry[s];
      const int np = C->ncpoly[s][it];
      tc[0] = tc[0] + y * C->amascp[s][it][C->ncenth[s][it] - 1];
      tc[1] = tc[1] + y * C->amasct[s][it][0];
      td[1] = tc[1];
#pragma unroll
      for (int icp = 2; icp <= 5; ++icp)
        if (icp <= np) {
          tc[icp] = tc[icp] + y * C->amasct[s][it][icp - 1];
          td[icp] = td[icp] + y * C->amascp[s][it][icp - 1];
        }
      rmix = rmix + y * C->rgspec[s];
    }
  }
  // new interval index and sum_k rho Y_k cp_k (divided by rho by the caller)
  __device__ __forceinline__ void locate(double T, const double (&ry)[NS], uint64_t& itn, double& cpsum) const {
    itn = 0;
    cpsum = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      if (s >= nspec) continue;
      int it = 0;
      while (T > C->tinthi[s][it] && it + 1 < C->ntint[s]) ++it;
      itn += (uint64_t)it << (2 * s);
      const int np = C->ncpoly[s][it];
      const double* cp = C->amascp[s][it];
      double c = cp[np - 1];
      for (int icp = np - 1; icp >= 1; --icp) c = c * T + cp[icp - 1];
      cpsum = cpsum + ry[s] * c;
    }
  }
  __device__ __forceinline__ double alamda() const { return C->alamda; }
  __device__ __forceinline__ double olewis(int s) const { return C->olewis[s]; }
  // mixture-averaged transport: lambda, rho*D_k, mu
  __device__ __forceinline__ void mixture(double T, double p, double rho, const double (&ry)[NS], const double (&y)[NS],
                                          double& lam, double (&rd)[NS], double& mu) const {
    const double lt = log(T / Dt->tdifgb);
    double c1 = 0.0, c2 = 0.0, c3 = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      if (s >= nspec) continue;
      double fp = Dt->condco[s][Dt->ncocon - 1];
      for (int icp = Dt->ncocon - 1; icp >= 1; --icp) fp = fp * lt + Dt->condco[s][icp - 1];
      const double lk = exp(fp);
      const double fm = ry[s] * C->ovwmol[s];
      c1 = c1 + fm * lk;
      c2 = c2 + fm / lk;
      c3 = c3 + fm;
    }
    c3 = 1.0 / c3;
    c1 = c1 * c3;
    c2 = c2 * c3;
    lam = 0.5 * (c1 + 1.0 / c2);
    const double wmix = rho * c3;
    double sumy = 0.0;
    double den[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      den[s] = 0.0;
      if (s < nspec) sumy += y[s] + kDfctol;
    }
    const double povr = p / Dt->pdifgb;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
#pragma unroll
      for (int t = s + 1; t < NS; ++t) {
        if (t >= nspec) continue;
        const double* dc = Dt->diffco[s][t];
        double fp = dc[Dt->ncodif - 1];
        for (int icp = Dt->ncodif - 1; icp >= 1; --icp) fp = fp * lt + dc[icp - 1];
        const double inv = exp(-fp) * povr;  // 1/D_st (DIFFCO is symmetric: one exp per pair)
        den[s] += (y[t] + kDfctol) * C->ovwmol[t] * inv;
        den[t] += (y[s] + kDfctol) * C->ovwmol[s] * inv;
      }
    }
#pragma unroll
    for (int s = 0; s < NS; ++s)
      if (s < nspec) rd[s] = rho * (sumy - (y[s] + kDfctol)) / (den[s] * wmix);
    double mk[NS], sq[NS], rq[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      mk[s] = 1.0;
      if (s < nspec) {
        double fp = Dt->viscco[s][Dt->ncovis - 1];
        for (int icp = Dt->ncovis - 1; icp >= 1; --icp) fp = fp * lt + Dt->viscco[s][icp - 1];
        mk[s] = exp(fp);
      }
      sq[s] = sqrt(mk[s]);  // sqrt(mu_i/mu_j) evaluated as sqrt(mu_i)/sqrt(mu_j)
      rq[s] = 1.0 / sq[s];
    }
    mu = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      if (s >= nspec) continue;
      double cc = 0.0;
#pragma unroll
      for (int t = 0; t < NS; ++t) {
        if (t >= nspec) continue;
        double fw = 1.0 + sq[s] * rq[t] * Dt->wilko2[s][t];
        fw = Dt->wilko1[s][t] * fw * fw;
        cc = cc + y[t] * C->ovwmol[t] * fw;
      }
      mu = mu + y[s] * C->ovwmol[s] * (mk[s] / cc);
    }
  }
  __device__ __forceinline__ void enthalpy(double T, uint64_t itn, double (&h)[NS]) const {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      h[s] = 0.0;
      if (s >= nspec) continue;
      const int it = tint_of(itn, s);
      const int np = C->ncpoly[s][it];
      const double* ch = C->amasch[s][it];
      double v = ch[np - 1];
      for (int icp = np - 1; icp >= 1; --icp) v = v * T + ch[icp - 1];
      h[s] = ch[C->ncenth[s][it] - 1] + v * T;
    }
  }
  __device__ __forceinline__ void chrate(double T, uint64_t itn, const double (&ry)[NS], double (&rate)[NS]) const {
    chrate_point<NS>(C, nspec, ry, T, itn, rate);
  }
};

// -------------------------------------------------------------------------
// PART 0: everything; PART 1: all but CHRATE; PART 2: CHRATE only, from the
// T and interval index that PART 1 stored. The long mechanisms run as the
// two smaller kernels: fewer registers and a smaller instruction footprint
// each, so more warps hide the FP64 latency (1.27x on the H2 mechanism).
template <class M, int PART = 0>
__device__ __forceinline__ void thermo_point(const Geo& g, const Fields& f, const M& m, const int64_t q) {
  constexpr int NS = M::NS;
  const int64_t n = g.n;
  const double* U = f.uin;
  double ry[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) ry[s] = m.has(s) ? U[(5 + s) * n + q] : 0.0;
  if (PART == 2) {
    double rate[NS];
    m.chrate(f.t[q], itn_load(f, n, q, m.count()), ry, rate);
#pragma unroll
    for (int s = 0; s < NS; ++s)
      if (m.has(s)) f.wdot[s * n + q] = rate[s];
    return;
  }
  const double rho = U[q], ru = U[n + q], rv = U[2 * n + q], rw = U[3 * n + q], re = U[4 * n + q];

  // ---- TEMPER: Newton inversion of e(T) from the previous T ----
  const double ukuk = (ru * ru + rv * rv + rw * rw) / rho;
  double tc[6], td[6];
  tc[0] = 0.5 * ukuk - re;
#pragma unroll
  for (int i = 1; i < 6; ++i) tc[i] = td[i] = 0.0;
  double rmix = 0.0;
  m.temper_coeffs(ry, itn_load(f, n, q, m.count()), tc, td, rmix);
  const double toltmp = (double)1.0e-10f;  // TOLTMP is a single-precision literal
  double T = f.t[q];
  int iters = 1;
  for (;;) {
    double tf = tc[5], tdp = td[5];
#pragma unroll
    for (int icp = 4; icp >= 1; --icp) {
      tf = tc[icp] + tf * T;
      tdp = td[icp] + tdp * T;
    }
    tf = tc[0] + tf * T;
    const double del = -tf / tdp;
    if (fabs(del) > toltmp) {
      if (iters < 100) {
        T = T + del;
        ++iters;
        continue;
      }
      atomicOr(f.status, 1u);  // reported through senga_get_status
    }
    break;
  }
  uint64_t itn;
  double cpm;
  m.locate(T, ry, itn, cpm);
  cpm = cpm / rho;
  const double p = T * rmix;
  f.t[q] = T;
  itn_store(f.itn, n, q, m.count(), itn);
  f.p[q] = p;
  if (f.cp) {  // NSCBC face data (cp_mix, rho R_mix of TEMPER)
    f.cp[q] = cpm;
    f.rmix[q] = rmix;
  }

  // ---- primitive variables ----
  double y[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    y[s] = ry[s] / rho;
    if (m.has(s)) f.y[s * n + q] = y[s];
  }
  f.vel[q] = ru / rho;
  f.vel[n + q] = rv / rho;
  f.vel[2 * n + q] = rw / rho;
  if (f.mom) {
    f.mom[q] = ru;
    f.mom[n + q] = rv;
    f.mom[2 * n + q] = rw;
  }
  f.e[q] = re / rho;

  // ---- transport properties ----
  if (!M::MAVT) {
    const double lcp = m.alamda() * exp(kRlamda * log(T));
    f.lam[q] = lcp * cpm;
    f.lcp[q] = lcp;
    f.mu[q] = lcp * kPrantl;
#pragma unroll
    for (int s = 0; s < NS; ++s)
      if (m.has(s)) f.rd[s * n + q] = lcp * m.olewis(s);
  } else {
    double lam, mu, rd[NS];
    m.mixture(T, p, rho, ry, y, lam, rd, mu);
    f.lam[q] = lam;
    f.mu[q] = mu;
#pragma unroll
    for (int s = 0; s < NS; ++s)
      if (m.has(s)) f.rd[s * n + q] = rd[s];
  }

  // ---- species enthalpy and mixture enthalpy (new interval index) ----
  {
    double h[NS];
    m.enthalpy(T, itn, h);
    double hm = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      if (!m.has(s)) continue;
      f.h[s * n + q] = h[s];
      hm = hm + h[s] * y[s];
    }
    f.hmix[q] = hm;
  }

  // ---- CHRATE ----
  if (PART == 0) {
    double rate[NS];
    m.chrate(T, itn, ry, rate);
#pragma unroll
    for (int s = 0; s < NS; ++s)
      if (m.has(s)) f.wdot[s * n + q] = rate[s];
  }
}

}  // namespace
}  // namespace senga
