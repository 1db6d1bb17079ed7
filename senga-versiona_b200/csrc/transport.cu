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
//   k_mixt_species  one launch per kind of term (molar mass, pressure,
//                   Soret, and the Dufour part of the main heat-flux terms:
//                   the species kernel formed those with the plain enthalpy
//                   h_k; the reference uses h_k + R_k T TDRMIX_k, so the
//                   difference, linear in the enthalpy, is added here), each
//                   looping over the species of the point.
// The per-species terms use the tile machinery of the species kernels
// (shared-memory slabs for x/y, register columns for z).
//
// Kept as coded: in the molar-mass and pressure branches the x component of
// the "species enthalpy gradient" is STORE4, which the code before them
// overwrote with DIFMIX (src/rhscal.f:1882-1891); the term is restated with
// that value.
#include <cuda_runtime.h>

#include "senga_gpu.h"
#include "senga_internal.h"
#include "stencil.cuh"
#include "tiles.cuh"

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

// ---- per-species terms: one tile kernel per kind of term ----------------
// Tiles of 32 x 8 x 2 points as in the species kernels (tiles.cuh): each
// field a term differentiates is staged once per tile and species into a
// shared-memory slab (x, y halos) plus a register column per thread (z
// halo), the driving diffusivities as products formed while staging.
constexpr int MX = 32, MY = 8, MZ = 2, MNW = MX * MY / 32;
using MSlab = tile::Slab<MX, MY, MZ>;
using MCol = tile::Column<MZ>;
constexpr int kMixSmem = 3 * MSlab::SIZE;

enum { kBrW = 0, kBrP = 1, kBrT = 2, kBrDufour = 3 };

// DIFMIX * Y_k times a branch factor: 1 (molar mass), 1 - W_k/W_mix
// (pressure), TDRMIX_k (Soret)
template <int BR>
struct DrivingF {
  const double* __restrict__ rd;
  const double* __restrict__ y;
  const double* __restrict__ x;  // W_mix or TDRMIX_k
  double wk;
  __device__ __forceinline__ double operator()(int64_t q) const {
    if (BR == kBrW) return rd[q] * y[q];
    if (BR == kBrP) return rd[q] * y[q] * (1.0 - wk / x[q]);
    return rd[q] * y[q] * x[q];
  }
};
// UTMP as the reference holds it: h_k, + R_k T TDRMIX_k with Dufour
// (mode 1), and that with the Dufour term taken out again (mode 2)
struct EnthF {
  const double* __restrict__ h;
  const double* __restrict__ t;
  const double* __restrict__ tk;
  double rg;
  int mode;
  __device__ __forceinline__ double operator()(int64_t q) const {
    if (mode == 0) return h[q];
    const double dl = rg * t[q] * tk[q];
    return mode == 1 ? h[q] + dl : (h[q] + dl) - dl;
  }
};
// the Dufour enthalpy increment R_k T TDRMIX_k
struct DufF {
  const double* __restrict__ t;
  const double* __restrict__ tk;
  double rg;
  __device__ __forceinline__ double operator()(int64_t q) const { return rg * t[q] * tk[q]; }
};

template <int BR, bool P>
__global__ void __launch_bounds__(MX* MY, 2) k_mixt_species(Geo g, Fields f, MixtParams m,
                                                            const senga_chem* __restrict__ ch, int nspec) {
  using namespace tile;
  extern __shared__ double sm[];
  __shared__ Folds<MX, MY, MZ> fo;
  const Origin o{(int)blockIdx.x * MX, (int)blockIdx.y * MY, (int)blockIdx.z * MZ};
  const int tx = threadIdx.x % MX, ty = threadIdx.x / MX;
  fo.init(g, o);
  tile_sync();
  TP tp[MZ];
#pragma unroll
  for (int z = 0; z < MZ; ++z) tp[z] = make_tp(g, o, tx, ty, z);
  const int64_t n = g.n;
  const MSlab bA{sm}, bB{sm + MSlab::SIZE}, bC{sm + 2 * MSlab::SIZE};
  const int b = BR == kBrW ? 0 : BR == kBrP ? 1 : 2;
  double gG[MZ][3], lG[MZ], vc[MZ][3], vt[MZ], ea[MZ];
#pragma unroll
  for (int z = 0; z < MZ; ++z) {
    const int64_t q = tp[z].q;
    for (int d = 0; d < 3; ++d) {
      gG[z][d] = BR == kBrDufour ? 0.0 : m.g1[b][d * n + q];
      vc[z][d] = 0.0;
    }
    lG[z] = BR == kBrDufour ? 0.0 : m.g2[b][q];
    vt[z] = 0.0;
    ea[z] = 0.0;
  }
#pragma unroll 1
  for (int k = 0; k < nspec; ++k) {
    const bool duf = (m.duf >> k) & 1u, sor = (m.sor >> k) & 1u;
    if (BR == kBrDufour && !duf) continue;
    if (BR == kBrT && !sor) continue;
    const double* __restrict__ rdk = f.rd + k * n;
    const double* __restrict__ yk = f.y + k * n;
    const double* __restrict__ hk = f.h + k * n;
    const double* __restrict__ tk = m.tdrmix ? m.tdrmix + k * n : nullptr;
    const double rg = ch->rgspec[k];
    tile_sync();
    if (BR == kBrDufour) {
      // the Dufour part of the main heat-flux terms: (grad rhoD . grad Y) dh,
      // (grad dh . grad Y) rhoD, (rhoD lap Y) dh, dh = R_k T TDRMIX_k
      const DufF dl{f.t, tk, rg};
      MCol cY, cR, cD;
      cY.load(fo, tx, ty, Ld{yk});
      cR.load(fo, tx, ty, Ld{rdk});
      cD.load(fo, tx, ty, dl);
      bA.stage<MNW>(fo, Ld{yk});
      bB.stage<MNW>(fo, Ld{rdk});
      bC.stage<MNW>(fo, dl);
      tile_sync();
#pragma unroll
      for (int z = 0; z < MZ; ++z) {
        const TP& t = tp[z];
        const bool dif = !P && (face_bits(g, t.gx) & BF_DIF);
        const double dY[3] = {d1<0, P>(g, t, bA), d1<1, P>(g, t, bA), d1z<P>(g, t, cY)};
        const double dRD[3] = {dif ? 0.0 : d1<0, P>(g, t, bB), d1<1, P>(g, t, bB), d1z<P>(g, t, cR)};
        const double dDl[3] = {dif ? 0.0 : d1<0, P>(g, t, bC), d1<1, P>(g, t, bC), d1z<P>(g, t, cD)};
        const double lapY = (dif ? 0.0 : d2<0, P>(g, t, bA)) + d2<1, P>(g, t, bA) + d2z<P>(g, t, cY);
        const double rd = cR.c[z + H], delta = cD.c[z + H];
        ea[z] = ea[z] + (dRD[0] * dY[0] + dRD[1] * dY[1] + dRD[2] * dY[2]) * delta +
                (dDl[0] * dY[0] + dDl[1] * dY[1] + dDl[2] * dY[2]) * rd + lapY * rd * delta;
      }
      continue;
    }
    const DrivingF<BR> drv{rdk, yk, BR == kBrP ? m.wmix : tk, ch->wmolar[k]};
    // W, P: UTMP with the Dufour term; Soret: with it taken out again
    const EnthF en{hk, f.t, tk, rg, duf ? (BR == kBrT ? 2 : 1) : 0};
    MCol cA, cB;
    cA.load(fo, tx, ty, drv);
    cB.load(fo, tx, ty, en);
    bA.stage<MNW>(fo, drv);
    bB.stage<MNW>(fo, en);
    tile_sync();
#pragma unroll
    for (int z = 0; z < MZ; ++z) {
      const TP& t = tp[z];
      const bool dif = !P && (face_bits(g, t.gx) & BF_DIF);
      const double s7 = cA.c[z + H], u = cB.c[z + H];
      const double dS[3] = {dif ? 0.0 : d1<0, P>(g, t, bA), d1<1, P>(g, t, bA), d1z<P>(g, t, cA)};
      // molar-mass and pressure branches: the x part of the "enthalpy
      // gradient" is DIFMIX (see the file comment)
      double dHx;
      if (BR == kBrT) dHx = dif ? 0.0 : d1<0, P>(g, t, bB);
      else dHx = dif ? 0.0 : rdk[t.q];
      const double dH[3] = {dHx, d1<1, P>(g, t, bB), d1z<P>(g, t, cB)};
      for (int d = 0; d < 3; ++d) vc[z][d] = vc[z][d] + s7 * gG[z][d];
      const double f1 = dS[0] * gG[z][0] + dS[1] * gG[z][1] + dS[2] * gG[z][2];
      const double f2 = lG[z] * s7;
      vt[z] = vt[z] + f1 + f2;
      ea[z] = ea[z] + f1 * u + (dH[0] * gG[z][0] + dH[1] * gG[z][1] + dH[2] * gG[z][2]) * s7 + f2 * u;
      if (t.valid) f.wdot[k * n + t.q] += f1 + f2;
    }
  }
#pragma unroll
  for (int z = 0; z < MZ; ++z) {
    const TP& t = tp[z];
    if (!t.valid) continue;
    if (BR != kBrDufour) {
      f.vc[t.q] += vc[z][0];
      f.vc[n + t.q] += vc[z][1];
      f.vc[2 * n + t.q] += vc[z][2];
      f.vtmp[t.q] += vt[z];
    }
    f.rhs[4 * n + t.q] += ea[z];
  }
}

// Wall terms of the molar-mass, pressure and Soret branches at a W1/W2 wall
// (FxxDFW: src/rhscal.f:2116-2175, 2512-2571, 2925-2984): the one-sided
// fourth-order x derivative at the wall of the branch's driving diffusivity
// times its x gradient (ln W_mix, ln p or ln(T/TDIFGB), first derivatives
// with the bounded closures), over the wall and the four planes inward,
// added to the species rate and to VTMP of the wall point. Their energy
// parts, and the Dufour branch's wall terms (rhscal.f:3106-3160,
// 3402-3500), reach only the wall's energy RHS, which BOUNDS sets to zero
// at either wall kind, and are left out. One thread per wall point;
// blockIdx.y = side.
template <int BR>
__global__ void __launch_bounds__(kMixBlock) k_mixt_wall(Geo g, Fields f, MixtParams m,
                                                         const senga_chem* __restrict__ ch, int nspec) {
  const int jk = blockIdx.x * kMixBlock + threadIdx.x;
  const int side = blockIdx.y;
  if (jk >= g.ny * g.nz || !((side == 0 ? g.bxl : g.bxr) & BF_WALL)) return;
  const int i = side == 0 ? 0 : g.nx - 1, st = side == 0 ? 1 : -1;
  const int64_t n = g.n, q = (int64_t)i + (int64_t)g.nx * jk;
  const double* __restrict__ gx = m.g1[BR == kBrW ? 0 : BR == kBrP ? 1 : 2];  // x components
  const double c0 = (double)(25.0f / 12.0f), c3 = (double)(4.0f / 3.0f);  // single-precision literals as coded
  double vt = f.vtmp[q];
  for (int k = 0; k < nspec; ++k) {
    if (BR == kBrT && !((m.sor >> k) & 1u)) continue;
    const DrivingF<BR> drv{f.rd + k * n, f.y + k * n, BR == kBrP ? m.wmix : (BR == kBrT ? m.tdrmix + k * n : nullptr),
                           ch->wmolar[k]};
    double fv[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) fv[c] = drv(q + c * st) * gx[q + c * st];
    const double w = side == 0 ? ((-c0) * fv[0] + 4.0 * fv[1] - 3.0 * fv[2] + c3 * fv[3] - 0.25 * fv[4]) * g.ovd[0]
                               : (c0 * fv[0] - 4.0 * fv[1] + 3.0 * fv[2] - c3 * fv[3] + 0.25 * fv[4]) * g.ovd[0];
    f.wdot[k * n + q] = f.wdot[k * n + q] + w;
    vt = vt + w;
  }
  f.vtmp[q] = vt;
}

// launches the branch's tile kernel and, with a wall, its wall terms;
// returns the number of launches
template <int BR>
int launch_branch(const Geo& g, const Fields& f, const MixtParams& m, const senga_chem* dchem, int nspec,
                  cudaStream_t s) {
  const dim3 grid((unsigned)((g.nx + MX - 1) / MX), (unsigned)((g.ny + MY - 1) / MY), (unsigned)((g.nz + MZ - 1) / MZ));
  const bool per = g.per[0] && g.per[1] && g.per[2];
  if (per) k_mixt_species<BR, true><<<grid, MX * MY, kMixSmem * 8, s>>>(g, f, m, dchem, nspec);
  else k_mixt_species<BR, false><<<grid, MX * MY, kMixSmem * 8, s>>>(g, f, m, dchem, nspec);
  if (BR == kBrDufour || !((g.bxl | g.bxr) & BF_WALL)) return 1;
  k_mixt_wall<BR == kBrDufour ? kBrW : BR>
      <<<dim3((unsigned)((g.ny * g.nz + kMixBlock - 1) / kMixBlock), 2), kMixBlock, 0, s>>>(g, f, m, dchem, nspec);
  return 2;
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
  if (m.duf) nl += launch_branch<kBrDufour>(g, f, m, dchem, nspec, s);
  if (m.w) nl += launch_branch<kBrW>(g, f, m, dchem, nspec, s);
  if (m.p) nl += launch_branch<kBrP>(g, f, m, dchem, nspec, s);
  if (m.sor) nl += launch_branch<kBrT>(g, f, m, dchem, nspec, s);
  return nl;
}

}  // namespace senga
