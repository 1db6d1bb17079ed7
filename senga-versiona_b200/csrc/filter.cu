// Explicit 12th-order filter (FLTREM: src/fltrem.f:43-90; FILTRX/Y/Z:
// src/filtrx.f:56-295; coefficients src/flinit.f:42-…).
//
// F_i = c0 f_i + sum_{m=1..6} c_m (f_{i+m} + f_{i-m}) in the interior; the
// first/last six points of a bounded direction use the one-sided rows of
// FLINIT (6th..11th order). Three directional passes x -> y -> z, each over
// the output of the previous one; periodic neighbours at +-6 are reached by
// index wrap. The coefficient table is built on the host (filter_coef) with
// the same TWFACT = -EXP(-12 LOG 2) expression as FLINIT, sign-flipped on
// request (the coded sign amplifies the grid-scale mode: transfer 1 +
// sin^12(theta/2)).
//
// The filter is an O(N) pass run every few steps, not per substage: one thread
// per point, neighbours from global memory (L1/L2 serve the reuse).
#include <cuda_runtime.h>

#include <cmath>

#include "senga_internal.h"

namespace senga {

FilterCoef filter_coef(bool flip) {
  FilterCoef c{};
  const double tw0 = -std::exp(-1.2e1 * std::log(2.0));
  const double tw = flip ? -tw0 : tw0;
  const double ints[6] = {7.92e2, -4.95e2, 2.20e2, -6.60e1, 1.20e1, -1.00};
  for (int m = 0; m < 6; ++m) c.in[m] = ints[m] * tw;
  c.in[6] = 1.0 + (-9.24e2 * tw);
  // one-sided rows 1..6 (row r has r+6 entries; the diagonal one carries the
  // unit term), src/flinit.f FACF1X..FLCF6X
  const double rows[6][12] = {{-1, 6, -15, 20, -15, 6, -1},
                              {6, -37, 96, -135, 110, -51, 12, -1},
                              {-15, 96, -262, 396, -360, 200, -66, 12, -1},
                              {20, -135, 396, -662, 696, -480, 220, -66, 12, -1},
                              {-15, 110, -360, 696, -887, 786, -495, 220, -66, 12, -1},
                              {6, -51, 200, -480, 786, -923, 792, -495, 220, -66, 12, -1}};
  for (int r = 0; r < 6; ++r) {
    for (int e = 0; e < r + 7; ++e) c.bnd[r][e] = rows[r][e] * tw;
    c.bnd[r][r] = 1.0 + c.bnd[r][r];
  }
  return c;
}

namespace {

constexpr int kFiltBlock = 256;

template <int DIR>
__global__ void __launch_bounds__(kFiltBlock) k_filter(Geo g, const double* __restrict__ in,
                                                       double* __restrict__ out, FilterCoef c) {
  const int64_t q = (int64_t)blockIdx.x * kFiltBlock + threadIdx.x;
  if (q >= g.n) return;
  const int i = (int)(q % g.nx);
  const int j = (int)((q / g.nx) % g.ny);
  const int k = (int)(q / ((int64_t)g.nx * g.ny));
  const int n = DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
  const int cc = DIR == 0 ? i : DIR == 1 ? j : k;
  const int64_t st = DIR == 0 ? 1 : DIR == 1 ? (int64_t)g.nx : (int64_t)g.nx * g.ny;
  const double* base = in + (q - (int64_t)cc * st);  // the line through q
  auto f = [&](int a) {  // a = 0-based coordinate along DIR
    if (g.per[DIR]) {  // any extent, one-point directions included
      a %= n;
      if (a < 0) a += n;
    }
    return base[(int64_t)a * st];
  };
  double v;
  if (g.per[DIR] || (cc >= 6 && cc <= n - 7)) {
    v = c.in[0] * (f(cc + 1) + f(cc - 1)) + c.in[1] * (f(cc + 2) + f(cc - 2)) + c.in[2] * (f(cc + 3) + f(cc - 3)) +
        c.in[3] * (f(cc + 4) + f(cc - 4)) + c.in[4] * (f(cc + 5) + f(cc - 5)) + c.in[5] * (f(cc + 6) + f(cc - 6)) +
        c.in[6] * f(cc);
  } else if (cc < 6) {
    const int r = cc;
    v = c.bnd[r][0] * f(0);
    for (int e = 1; e < r + 7; ++e) v = v + c.bnd[r][e] * f(e);
  } else {
    const int r = n - 1 - cc;
    v = c.bnd[r][0] * f(n - 1);
    for (int e = 1; e < r + 7; ++e) v = v + c.bnd[r][e] * f(n - 1 - e);
  }
  out[q] = v;
}

}  // namespace

void launch_filter_field(const Geo& g, const double* in, double* out, double* t1, double* t2, const FilterCoef& c,
                         cudaStream_t s) {
  const unsigned grid = (unsigned)((g.n + kFiltBlock - 1) / kFiltBlock);
  k_filter<0><<<grid, kFiltBlock, 0, s>>>(g, in, t1, c);
  k_filter<1><<<grid, kFiltBlock, 0, s>>>(g, t1, t2, c);
  k_filter<2><<<grid, kFiltBlock, 0, s>>>(g, t2, out, c);
}

}  // namespace senga
