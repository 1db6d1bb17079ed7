// Initial flame, FLAMIN (src/flamin.f:44-322), and the conversion of the
// primitive start-up fields to the conserved state that INDATA performs after
// it (src/indata.f:1233-1394), one thread per interior point.
//
// FLAMIN: progress c = (1 + erf((x - 5 mm)/0.5 mm))/2 along the global x
// coordinate x = (i-1) L/(N-1) (:220-232; erf by ERFUNC, src/erfunc.f, the
// Abramowitz-Stegun 7.1.26 rational approximation); Y_k and T blended between
// the reactant (Y_1 = 0.011606960, Y_2 = 0.230295282, T = TRIN) and product
// (Y_2 = 0.139255233, Y_3 = 0.102581446, T = 1417.2 K written as a default
// REAL constant) states, the last species the remainder (:89-135, :240-276);
// u = DRIN URIN / rho (:300-318). INDATA then: rho = PRIN / (T sum_k R_k Y_k),
// ITNDEX from T, E = sum_k Y_k h_k(T) - T sum_k R_k Y_k + |u|^2/2 and the
// conserved products rho (1, u, v, w, E, Y_k) (:1233-1394).
#include "itndex.cuh"
#include "senga_internal.h"

namespace senga {
namespace {

constexpr int kBlock = 256;

// ERFUNC (src/erfunc.f:40-79): Abramowitz and Stegun 7.1.26
__device__ __forceinline__ double erfunc(double a) {
  const double pc = 0.3275911;
  const double ec[5] = {0.254829592, -0.284496736, 1.421413741, -1.453152027, 1.061405429};
  const double z = fabs(a);
  const double t = 1.0 / (1.0 + pc * z);
  double e = ec[4];
  for (int i = 3; i >= 0; --i) e = ec[i] + e * t;
  e = e * t;
  const double r = 1.0 - e * exp(-z * z);
  return a < 0.0 ? -r : r;
}

struct FlaminArgs {
  int64_t n;
  int nx, ny, nspec;
  double deltag, trin, prin, flxmas;
  double yr[SENGA_NSPCMX], yp[SENGA_NSPCMX];
};

__global__ void __launch_bounds__(kBlock) k_flamin(FlaminArgs a, const senga_chem* __restrict__ C,
                                                   const double* __restrict__ vin, const double* __restrict__ win,
                                                   double* __restrict__ run, double* __restrict__ uin,
                                                   double* __restrict__ t, int32_t* __restrict__ itn) {
  const int64_t q = (int64_t)blockIdx.x * kBlock + threadIdx.x;
  if (q >= a.n) return;
  const int64_t n = a.n;
  const int ic = (int)(q % a.nx);
  const double trinp = (double)1417.2f;  // TRINP = 1417.2, a default (single precision) REAL constant
  const double x = (double)(float)ic * a.deltag;
  const double crin = 0.5 * (1.0 + erfunc((x - 5.0e-3) / 5.0e-4));
  double y[SENGA_NSPCMX];
  const int last = a.nspec - 1;
  double ysum = 0.0;
  for (int s = 0; s < last; ++s) {
    y[s] = a.yr[s] + crin * (a.yp[s] - a.yr[s]);
    ysum = ysum + y[s];
  }
  y[last] = 1.0 - ysum;
  const double T = a.trin + crin * (trinp - a.trin);
  double st1 = 0.0;
  for (int s = 0; s < a.nspec; ++s) st1 = st1 + C->rgspec[s] * y[s];
  const double u = a.flxmas / (a.prin / (st1 * T));  // FLAMIN's own density
  const double rt = st1 * T;
  const double rho = a.prin / rt;
  uint64_t code = 0;
  double e = 0.0;
  for (int s = 0; s < a.nspec; ++s) {
    int it = 0;
    while (T > C->tinthi[s][it] && it + 1 < C->ntint[s]) ++it;
    code += (uint64_t)it << (2 * s);
    const double* ch = C->amasch[s][it];
    double h = ch[C->ncpoly[s][it] - 1];
    for (int icp = C->ncpom1[s][it]; icp >= 1; --icp) h = h * T + ch[icp - 1];
    h = ch[C->ncenth[s][it] - 1] + h * T;
    e = e + h * y[s];
  }
  const double v = vin ? vin[q] : 0.0, w = win ? win[q] : 0.0;
  e = e - rt + 0.5 * (u * u + v * v + w * w);
  double c[5 + SENGA_NSPCMX];
  c[0] = rho;
  c[1] = rho * u;
  c[2] = rho * v;
  c[3] = rho * w;
  c[4] = rho * e;
  for (int s = 0; s < a.nspec; ++s) c[5 + s] = rho * y[s];
  for (int f = 0; f < 5 + a.nspec; ++f) {
    run[f * n + q] = c[f];
    uin[f * n + q] = c[f];
  }
  t[q] = T;
  itn_store(itn, n, q, a.nspec, code);
}

}  // namespace

void launch_flamin(const Geo& g, int nspec, double xgdlen, double trin, double prin, double drin, double urin,
                   const senga_chem* dchem, const double* v, const double* w, double* run, double* uin, double* t,
                   int32_t* itn, cudaStream_t s) {
  FlaminArgs a{};
  a.n = g.n;
  a.nx = g.nx;
  a.ny = g.ny;
  a.nspec = nspec;
  a.deltag = xgdlen / (double)(float)(g.nx - 1);  // XGDLEN/REAL(NXGLBL-1)
  a.trin = trin;
  a.prin = prin;
  a.flxmas = drin * urin;
  a.yr[0] = 1.1606960e-2;
  a.yr[1] = 2.30295282e-1;
  a.yp[0] = 0.0;
  a.yp[1] = 1.39255233e-1;
  if (nspec > 2) a.yp[2] = 1.02581446e-1;
  const unsigned grid = (unsigned)((g.n + kBlock - 1) / kBlock);
  k_flamin<<<grid, kBlock, 0, s>>>(a, dchem, v, w, run, uin, t, itn);
}

}  // namespace senga
