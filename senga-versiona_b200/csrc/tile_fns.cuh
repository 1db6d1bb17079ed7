// Tile functions of the stencil kernels of the substage (see tiles.cuh),
// shared by the one-CTA-per-tile kernels (kernels_tiled.cu) and the
// persistent batch kernel (persist.cu):
//
//   flow_tile      continuity, momentum, energy convection, heat conduction,
//                  pressure and viscous terms (src/rhscal.f:141-793,
//                  src/rhsvel.f:48-2318) for a 32x8x2 tile; 7 staging phases.
//   species_tile   species convection/diffusion, correction velocity and the
//                  species enthalpy fluxes of the energy equation
//                  (src/rhscal.f:1030-1955) for a 32x8x2 tile, all species.
//   species_rk_tile diffusion-correction terms (src/rhscal.f:3782-3938) fused
//                  with the 2N-storage RK update (src/lincom.f:53-169,
//                  src/fincom.f:54-168).
// The physics and the association of every product follow the reference
// line by line within a term; terms are accumulated per grid point in a
// different order (FP64 rounding differences only). Template parameter NC
// selects the field loads: the read-only data path (kernels in which no
// CTA writes the fields they read) or coherent loads (persist.cu).
// Everything here has internal linkage.
#pragma once
#include <cuda_runtime.h>

#include "senga_internal.h"
#include "tiles.cuh"

namespace senga {
namespace {

using namespace tile;

// Tile shapes (x fastest; every library file is compiled with the same
// shapes, the launchers and work lists take them from here)
#ifndef SENGA_TILE_X
#define SENGA_TILE_X 32
#endif
#ifndef SENGA_TILE_Y
#define SENGA_TILE_Y 8
#endif
// flow tile
constexpr int FX = SENGA_TILE_X, FY = SENGA_TILE_Y, FZ = 2;
constexpr int FNW = FX * FY / 32;
// species tiles
constexpr int SX_ = SENGA_TILE_X, SY_ = SENGA_TILE_Y, SZ_ = 2;
constexpr int SNW = SX_ * SY_ / 32;
static_assert(FX * FY == 256 && SX_ * SY_ == 256, "the stencil kernels run 256 threads per tile");

using FStar = Star<FX, FY, FZ>;
using FBox = Box<FX, FY, FZ>;
using FXRow = XRow<FX, FY, FZ>;
using FYRow = YRow<FX, FY, FZ>;
using FZCol = ZCol<FX, FY, FZ>;

constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int kFlowSmem = cmax(cmax(FXRow::SIZE + FYRow::SIZE + FZCol::SIZE + FStar::SIZE, 2 * FStar::SIZE),
                                cmax(3 * FXRow::SIZE + 3 * FYRow::SIZE, FStar::SIZE + FBox::SIZE));

using SSlab = Slab<SX_, SY_, SZ_>;
using SXRow = XRow<SX_, SY_, SZ_>;
using SYRow = YRow<SX_, SY_, SZ_>;
using SCol = Column<SZ_>;
// the species kernel's rho w z-columns: one per thread, [k][thread]
constexpr int kSpecColW = (SZ_ + 2 * H) * SX_ * SY_;
constexpr int kSpecSmem = SXRow::SIZE + SYRow::SIZE + 3 * SSlab::SIZE + kSpecColW;
// species+RK: two slabs, then the prefetched S register and rate of the next
// species' own points, double-buffered: [buffer][run | rate][z][thread]
constexpr int kRkPre = 2 * SZ_ * SX_ * SY_;
constexpr int kSpecRkSmem = 2 * SSlab::SIZE + 2 * kRkPre;

// Staging of a plain field: bulk copies on the TMA engine (B) or per-element
// cp.async; and the wait for the group staged last (B: one mbarrier phase of
// `bytes`, a CTA-uniform barrier; returns true when the CTA must give up).
template <bool B, int NW, bool NC = true, class Buf, class FO>
__device__ __forceinline__ void stage_plain(const Buf& b, const FO& fo, const Geo& g, const Origin& o,
                                            const double* src, uint64_t* bar) {
  if constexpr (B) b.stage_bulk(fo, o.x0, g.nx, src, bar);
  else b.template stage<NW>(fo, LdT<NC>{src});
}
// Tensor maps of the species kernels (tensor-copy mode): the Y, rho D and h
// families as 4-D tensors [species][z][y][x] with boxes of one slab
// (SX x (TY+2H) x TZ), and the U register [field][z][y][x] with the x-row and
// y-row boxes of rho u and rho v; hmix as a one-field 4-D tensor.
struct SpecMaps {
  CUtensorMap y, rd, h, ux, vy;
};
struct RkMaps {
  CUtensorMap y, hm;
};
// a tile whose halo-extended x and y ranges lie inside the box takes one
// tensor copy per buffer; tiles at the periodic wrap copy rows
// (tensor copies land on 128-byte aligned buffers: the dynamic shared
// memory base is checked, the buffer offsets are multiples of 128 bytes)
template <int TX, int TY, int TZ>
__device__ __forceinline__ bool tensor_tile(const Geo& g, const Origin& o, const double* sm) {
  return (smem_u32(sm) & 127u) == 0 && o.x0 >= XH && o.x0 + TX + XH <= g.nx && o.y0 >= H &&
         o.y0 + TY + H <= g.ny && o.z0 + TZ <= g.nz;
}
static_assert((8 * SXRow::SIZE) % 128 == 0 && (8 * SYRow::SIZE) % 128 == 0 && (8 * SSlab::SIZE) % 128 == 0,
              "tensor-copy buffers start on 128-byte boundaries");

template <bool B>
__device__ __forceinline__ bool sync_staged(BulkBar& bb, unsigned bytes, unsigned int* status) {
  if constexpr (B) return bb.wait(bytes, status);
  tile_sync();
  return false;
}

template <bool P, bool B = false, bool NC = true>
__device__ __forceinline__ void flow_tile(const Geo& g, const Fields& f, const Origin o, double* sm,
                                          Folds<FX, FY, FZ>& fo, const ZDec& zd, uint64_t* bar = nullptr) {
  const int tx = threadIdx.x % FX, ty = threadIdx.x / FX;
  fo.init(g, o, zd);
  BulkBar bb{bar, 0u};
  if (B && threadIdx.x == 0) mbar_init(bar, 1);
  tile_sync();
  TP tp[FZ];
#pragma unroll
  for (int z = 0; z < FZ; ++z) tp[z] = make_tp(g, o, tx, ty, z);
  const int64_t n = g.n;
  const double* U = f.uin;
  double divm[FZ], rU[FZ], rV[FZ], rW[FZ], rE[FZ];

  // ---- phase 1: mass-flux divergence, energy convection ----
  {
    const FXRow bru{sm};
    const FYRow brv{sm + FXRow::SIZE};
    const FZCol brw{sm + FXRow::SIZE + FYRow::SIZE};
    const FStar bE{sm + FXRow::SIZE + FYRow::SIZE + FZCol::SIZE};
    stage_plain<B, FNW, NC>(bru, fo, g, o, U + n, bar);
    stage_plain<B, FNW, NC>(brv, fo, g, o, U + 2 * n, bar);
    stage_plain<B, FNW, NC>(brw, fo, g, o, U + 3 * n, bar);
    stage_plain<B, FNW, NC>(bE, fo, g, o, f.e, bar);
    if (sync_staged<B>(bb, FXRow::kBulkBytes + FYRow::kBulkBytes + FZCol::kBulkBytes + FStar::kBulkBytes, f.status))
      return;
#pragma unroll
    for (int z = 0; z < FZ; ++z) {
      const TP& t = tp[z];
      const double dv = d1<0, P>(g, t, bru) + d1<1, P>(g, t, brv) + d1<2, P>(g, t, brw);
      divm[z] = dv;
      const double s4 = bE.v(t.x, t.y, t.z) * dv + d1p<0, P>(g, t, bE, bru) + d1p<1, P>(g, t, bE, brv) +
                        d1p<2, P>(g, t, bE, brw);
      rE[z] = -0.5 * (s4 + d1<0, P>(g, t, bE) * bru.v(t.x, t.y, t.z) + d1<1, P>(g, t, bE) * brv.v(t.x, t.y, t.z) +
                      d1<2, P>(g, t, bE) * brw.v(t.x, t.y, t.z));
    }
    tile_sync();
  }
  // ---- phase 2: heat conduction ----
  {
    const FStar bT{sm}, bL{sm + FStar::SIZE};
    stage_plain<B, FNW, NC>(bT, fo, g, o, f.t, bar);
    stage_plain<B, FNW, NC>(bL, fo, g, o, f.lam, bar);
    if (sync_staged<B>(bb, 2 * FStar::kBulkBytes, f.status)) return;
#pragma unroll
    for (int z = 0; z < FZ; ++z) {
      const TP& t = tp[z];
      // FxxCON: the x conduction terms vanish on the face plane (rhscal.f:582,774)
      const bool con = !P && (face_bits(g, t.gx) & BF_CON);
      rE[z] = rE[z] + ((con ? 0.0 : d1<0, P>(g, t, bL) * d1<0, P>(g, t, bT)) + d1<1, P>(g, t, bL) * d1<1, P>(g, t, bT) +
                       d1<2, P>(g, t, bL) * d1<2, P>(g, t, bT));
      rE[z] = rE[z] + ((con ? 0.0 : d2<0, P>(g, t, bT)) + d2<1, P>(g, t, bT) + d2<2, P>(g, t, bT)) * bL.v(t.x, t.y, t.z);
    }
    tile_sync();
  }
  // ---- phase 3: pressure gradient (of p - p(1,1,1)) and pressure work ----
  {
    const FStar bPr{sm};
    const double p111 = ldf<NC>(f.p + zd.base[0]);  // p(1,1,1) lives in slab 0
    // the point's velocity, loaded before the staging wait so that its
    // latency overlaps the copies
    double pu[FZ], pv[FZ], pw[FZ];
    auto point_vel = [&] {
#pragma unroll
      for (int z = 0; z < FZ; ++z) {
        pu[z] = ldf<NC>(f.vel + tp[z].q);
        pv[z] = ldf<NC>(f.vel + n + tp[z].q);
        pw[z] = ldf<NC>(f.vel + 2 * n + tp[z].q);
      }
    };
    auto phase3 = [&](const auto& bP) {
#pragma unroll
      for (int z = 0; z < FZ; ++z) {
        const TP& t = tp[z];
        const double px = d1<0, P>(g, t, bP), py = d1<1, P>(g, t, bP), pz = d1<2, P>(g, t, bP);
        rU[z] = -px;
        rV[z] = -py;
        rW[z] = -pz;
        rE[z] = rE[z] - pu[z] * px - pv[z] * py - pw[z] * pz;
      }
    };
    if constexpr (B) {
      // raw p by bulk copies, p(1,1,1) subtracted where read: the same
      // subtraction as staging p - p(1,1,1), so the same values
      bPr.stage_bulk(fo, o.x0, g.nx, f.p, bar);
      point_vel();
      if (bb.wait(FStar::kBulkBytes, f.status)) return;
      phase3(Shifted<FStar>{bPr, p111});
    } else {
      bPr.stage<FNW>(fo, LdSubT<NC>{f.p, p111});
      point_vel();
      tile_sync();
      phase3(bPr);
    }
    tile_sync();
  }
  // ---- phase 4: momentum fluxes d/dx_j (rho u_i u_j) ----
  // x and y derivatives from products staged in x rows and y rows, z
  // derivatives from products of register z-columns; each flux summed x, y,
  // z in that order
  double S4[FZ], S5[FZ], S6[FZ];
  {
    const FXRow xA{sm}, xB{sm + FXRow::SIZE}, xC{sm + 2 * FXRow::SIZE};
    double* const sy = sm + 3 * FXRow::SIZE;
    const FYRow yA{sy}, yB{sy + FYRow::SIZE}, yC{sy + 2 * FYRow::SIZE};
    // the three x-row products share rho u, the three y-row ones v or rho v:
    // one pass of loads fills each group of three buffers
    const double* const pru = U + n;
    const double* const prv = U + 2 * n;
    const double* const pu = f.vel;
    const double* const pv = f.vel + n;
    const double* const pw = f.vel + 2 * n;
    xA.stage3<FNW, 2>(xB, xC, fo, [=](int64_t q, double& a, double& b, double& c) {
      const double m = ldf<NC>(pru + q);
      a = m * ldf<NC>(pu + q);  // rho u u
      b = m * ldf<NC>(pv + q);  // rho u v
      c = m * ldf<NC>(pw + q);  // rho u w
    });
    yA.stage3<FNW, 3>(yB, yC, fo, [=](int64_t q, double& a, double& b, double& c) {
      const double v = ldf<NC>(pv + q), m = ldf<NC>(prv + q);
      a = ldf<NC>(pru + q) * v;  // rho u v
      b = m * v;                 // rho v v
      c = m * ldf<NC>(pw + q);   // rho v w
    });
    Column<FZ> cw, cm;
    cw.load(fo, tx, ty, LdT<NC>{f.vel + 2 * n});
    cm.load(fo, tx, ty, LdT<NC>{U + n});
    tile_sync();
#pragma unroll
    for (int z = 0; z < FZ; ++z) {
      const TP& t = tp[z];
      S4[z] = d1<0, P>(g, t, xA);
      S5[z] = d1<0, P>(g, t, xB);
      S6[z] = d1<0, P>(g, t, xC);
      S4[z] = S4[z] + d1<1, P>(g, t, yA);
      S5[z] = S5[z] + d1<1, P>(g, t, yB);
      S6[z] = S6[z] + d1<1, P>(g, t, yC);
      S4[z] = S4[z] + d1zp<P>(g, t, cm, cw);  // rho u w
    }
    cm.load(fo, tx, ty, LdT<NC>{U + 2 * n});
#pragma unroll
    for (int z = 0; z < FZ; ++z) S5[z] = S5[z] + d1zp<P>(g, tp[z], cm, cw);  // rho v w
    cm.load(fo, tx, ty, LdT<NC>{U + 3 * n});
#pragma unroll
    for (int z = 0; z < FZ; ++z) S6[z] = S6[z] + d1zp<P>(g, tp[z], cm, cw);  // rho w w
    tile_sync_async();
  }
  // ---- phase 5: velocity derivatives, viscous stresses and work ----
  const FStar bM{sm};
  const FBox bX{sm + FStar::SIZE};
  stage_plain<B, FNW, NC>(bM, fo, g, o, f.mu, bar);
  double mux[FZ], muy[FZ], muz[FZ], ux[FZ], uy[FZ], uz[FZ], vx[FZ], vy[FZ], vz[FZ];
  // 5a: u
  stage_plain<B, FNW, NC>(bX, fo, g, o, f.vel, bar);
  // point values of 5a, loaded before the staging wait
  double qa[FZ], qb[FZ], qc[FZ];
#pragma unroll
  for (int z = 0; z < FZ; ++z) {
    qa[z] = ldf<NC>(f.vel + n + tp[z].q);
    qb[z] = ldf<NC>(f.vel + 2 * n + tp[z].q);
    qc[z] = ldf<NC>(U + n + tp[z].q);
  }
  if (sync_staged<B>(bb, FStar::kBulkBytes + FBox::kBulkBytes, f.status)) return;
#pragma unroll
  for (int z = 0; z < FZ; ++z) {
    const TP& t = tp[z];
    const double mu = bM.v(t.x, t.y, t.z);
    mux[z] = d1<0, P>(g, t, bM);
    muy[z] = d1<1, P>(g, t, bM);
    muz[z] = d1<2, P>(g, t, bM);
    ux[z] = d1<0, P>(g, t, bX);
    uy[z] = d1<1, P>(g, t, bX);
    uz[z] = d1<2, P>(g, t, bX);
    const double uq = bX.v(t.x, t.y, t.z);
    const double vq = qa[z], wq = qb[z];
    // x-face viscous flags (rhsvel.f: FxxVSN normal, FxxVST shear terms zeroed on the plane)
    const int bf = P ? 0 : face_bits(g, t.gx);
    const double vsn = (bf & BF_VSN) ? 0.0 : 1.0, vst = (bf & BF_VST) ? 0.0 : 1.0;
    rU[z] = rU[z] + -0.5 * (qc[z] * ux[z] + (S4[z] + uq * divm[z]));
    double fn = vsn * (mu * kFthd * d2<0, P>(g, t, bX));
    rU[z] += fn;
    rE[z] = rE[z] + fn * uq;
    fn = mu * d2<1, P>(g, t, bX);
    rU[z] += fn;
    rE[z] = rE[z] + uq * fn;
    fn = mu * d2<2, P>(g, t, bX);
    rU[z] += fn;
    rE[z] = rE[z] + uq * fn;
    const double uxy = dm<0, 1, P>(g, t, bX), uxz = dm<0, 2, P>(g, t, bX);
    fn = kTthd * mu * uxy;
    rV[z] -= fn;
    rE[z] = rE[z] - vq * fn;
    fn = vst * (mu * uxy);
    rV[z] += fn;
    rE[z] = rE[z] + vq * fn;
    fn = kTthd * mu * uxz;
    rW[z] -= fn;
    rE[z] = rE[z] - wq * fn;
    fn = vst * (mu * uxz);
    rW[z] += fn;
    rE[z] = rE[z] + wq * fn;
  }
  tile_sync();
  // 5b: v
  stage_plain<B, FNW, NC>(bX, fo, g, o, f.vel + n, bar);
#pragma unroll
  for (int z = 0; z < FZ; ++z) {
    qa[z] = ldf<NC>(f.vel + tp[z].q);
    qb[z] = ldf<NC>(f.vel + 2 * n + tp[z].q);
    qc[z] = ldf<NC>(U + 2 * n + tp[z].q);
  }
  if (sync_staged<B>(bb, FBox::kBulkBytes, f.status)) return;
#pragma unroll
  for (int z = 0; z < FZ; ++z) {
    const TP& t = tp[z];
    const double mu = bM.v(t.x, t.y, t.z);
    vx[z] = d1<0, P>(g, t, bX);
    vy[z] = d1<1, P>(g, t, bX);
    vz[z] = d1<2, P>(g, t, bX);
    const double vq = bX.v(t.x, t.y, t.z);
    const double uq = qa[z], wq = qb[z];
    const int bf = P ? 0 : face_bits(g, t.gx);
    const double vsn = (bf & BF_VSN) ? 0.0 : 1.0, vst = (bf & BF_VST) ? 0.0 : 1.0;
    rV[z] = rV[z] + -0.5 * (qc[z] * vy[z] + (S5[z] + vq * divm[z]));
    double fn = mu * kFthd * d2<1, P>(g, t, bX);
    rV[z] += fn;
    rE[z] = rE[z] + fn * vq;
    fn = vst * (mu * d2<0, P>(g, t, bX));
    rV[z] += fn;
    rE[z] = rE[z] + vq * fn;
    fn = mu * d2<2, P>(g, t, bX);
    rV[z] += fn;
    rE[z] = rE[z] + vq * fn;
    const double vxy = dm<0, 1, P>(g, t, bX), vyz = dm<1, 2, P>(g, t, bX);
    fn = vsn * (kTthd * mu * vxy);
    rU[z] -= fn;
    rE[z] = rE[z] - uq * fn;
    fn = mu * vxy;
    rU[z] += fn;
    rE[z] = rE[z] + uq * fn;
    fn = kTthd * mu * vyz;
    rW[z] -= fn;
    rE[z] = rE[z] - wq * fn;
    fn = mu * vyz;
    rW[z] += fn;
    rE[z] = rE[z] + wq * fn;
  }
  tile_sync();
  // 5c: w, then the first-derivative products
  stage_plain<B, FNW, NC>(bX, fo, g, o, f.vel + 2 * n, bar);
  double qd[FZ];
#pragma unroll
  for (int z = 0; z < FZ; ++z) {  // (an invalid point has q = 0: in bounds, unused)
    qa[z] = ldf<NC>(f.vel + tp[z].q);
    qb[z] = ldf<NC>(f.vel + n + tp[z].q);
    qc[z] = ldf<NC>(U + tp[z].q);
    qd[z] = ldf<NC>(U + 3 * n + tp[z].q);
  }
  if (sync_staged<B>(bb, FBox::kBulkBytes, f.status)) return;
#pragma unroll
  for (int z = 0; z < FZ; ++z) {
    const TP& t = tp[z];
    if (!t.valid) continue;
    const double mu = bM.v(t.x, t.y, t.z);
    const double wx = d1<0, P>(g, t, bX), wy = d1<1, P>(g, t, bX), wz = d1<2, P>(g, t, bX);
    const double wq = bX.v(t.x, t.y, t.z);
    const double uq = qa[z], vq = qb[z];
    const double rho = qc[z];
    const int bf = P ? 0 : face_bits(g, t.gx);
    const double vsn = (bf & BF_VSN) ? 0.0 : 1.0, vst = (bf & BF_VST) ? 0.0 : 1.0;
    rW[z] = rW[z] + -0.5 * (qd[z] * wz + (S6[z] + wq * divm[z]));
    double fn = mu * kFthd * d2<2, P>(g, t, bX);
    rW[z] += fn;
    rE[z] = rE[z] + fn * wq;
    fn = vst * (mu * d2<0, P>(g, t, bX));
    rW[z] += fn;
    rE[z] = rE[z] + wq * fn;
    fn = mu * d2<1, P>(g, t, bX);
    rW[z] += fn;
    rE[z] = rE[z] + wq * fn;
    const double wxz = dm<0, 2, P>(g, t, bX), wyz = dm<1, 2, P>(g, t, bX);
    fn = vsn * (kTthd * mu * wxz);
    rU[z] -= fn;
    rE[z] = rE[z] - uq * fn;
    fn = mu * wxz;
    rU[z] += fn;
    rE[z] = rE[z] + uq * fn;
    fn = kTthd * mu * wyz;
    rV[z] -= fn;
    rE[z] = rE[z] - vq * fn;
    fn = mu * wyz;
    rV[z] += fn;
    rE[z] = rE[z] + vq * fn;
    // pressure work p div u
    rE[z] = rE[z] - ldf<NC>(f.p + t.q) * (ux[z] + vy[z] + wz);
    // normal stresses with viscosity gradients (TAUxx b,e,f)
    double t6 = kFthd * ux[z] - kTthd * (vy[z] + wz);
    rE[z] = rE[z] + mu * t6 * ux[z];
    t6 = vsn * (t6 * mux[z]);
    rU[z] += t6;
    rE[z] = rE[z] + uq * t6;
    t6 = kFthd * vy[z] - kTthd * (ux[z] + wz);
    rE[z] = rE[z] + mu * t6 * vy[z];
    t6 = t6 * muy[z];
    rV[z] += t6;
    rE[z] = rE[z] + vq * t6;
    t6 = kFthd * wz - kTthd * (ux[z] + vy[z]);
    rE[z] = rE[z] + mu * t6 * wz;
    t6 = t6 * muz[z];
    rW[z] += t6;
    rE[z] = rE[z] + wq * t6;
    // xy
    rU[z] = rU[z] - 0.5 * rho * vq * uy[z];
    rV[z] = rV[z] - 0.5 * rho * uq * vx[z];
    double s7 = uy[z] + vx[z];
    fn = s7 * muy[z];
    rU[z] += fn;
    rE[z] = rE[z] + uq * fn;
    fn = vst * (s7 * mux[z]);
    rV[z] += fn;
    rE[z] = rE[z] + vq * fn;
    rE[z] = rE[z] + mu * s7 * s7;
    // xz
    rU[z] = rU[z] - 0.5 * rho * wq * uz[z];
    rW[z] = rW[z] - 0.5 * rho * uq * wx;
    s7 = uz[z] + wx;
    fn = s7 * muz[z];
    rU[z] += fn;
    rE[z] = rE[z] + uq * fn;
    fn = vst * (s7 * mux[z]);
    rW[z] += fn;
    rE[z] = rE[z] + wq * fn;
    rE[z] = rE[z] + mu * s7 * s7;
    // yz
    rV[z] = rV[z] - 0.5 * rho * wq * vz[z];
    rW[z] = rW[z] - 0.5 * rho * vq * wy;
    s7 = vz[z] + wy;
    fn = s7 * muz[z];
    rV[z] += fn;
    rE[z] = rE[z] + vq * fn;
    fn = s7 * muy[z];
    rW[z] += fn;
    rE[z] = rE[z] + wq * fn;
    rE[z] = rE[z] + mu * s7 * s7;

    f.rhs[t.q] = -divm[z];
    f.rhs[n + t.q] = rU[z];
    f.rhs[2 * n + t.q] = rV[z];
    f.rhs[3 * n + t.q] = rW[z];
    f.rhs[4 * n + t.q] = rE[z];
    f.divm[t.q] = divm[z];
  }
}

// -------------------------------------------------------------------------
// What the species pass hands to the species+RK pass when both run in one
// CTA (KEEP): each thread's correction velocity, VTMP and energy RHS in
// registers, the species rates in this CTA's shared memory (rate[(s * SZ_ +
// z) * 256 + thread]); without KEEP they go through the global scratch
// fields VC, VTMP, RHS(E) and WDOT.
struct SpecCarry {
  double vcx[SZ_], vcy[SZ_], vcz[SZ_], vt[SZ_], rE[SZ_];
  double* rate;
};
constexpr int kFuseMaxSpec = 9;  // species the fused kernel carries on chip
constexpr int kCarryRate = kFuseMaxSpec * SZ_ * SX_ * SY_;  // doubles of shared memory

// M: 0 per-element cp.async, 1 bulk row copies, 2 one tensor copy per buffer
// for tiles away from the wrap (bulk rows for the others)
template <bool P, int M = 0, bool NC = true, bool KEEP = false>
__device__ __forceinline__ void species_tile(const Geo& g, const Fields& f, int nspec, const Origin o, double* sm,
                                             Folds<SX_, SY_, SZ_>& fo, const ZDec& zd, uint64_t* bar = nullptr,
                                             const SpecMaps* tm = nullptr, SpecCarry* carry = nullptr) {
  constexpr bool B = M > 0;
  const bool tens = M == 2 && tensor_tile<SX_, SY_, SZ_>(g, o, sm);
  constexpr unsigned kSlabT = 8u * SSlab::SIZE;  // a tensor copy fills the whole slab
  const unsigned slab_bytes = tens ? kSlabT : SSlab::kBulkBytes;
  auto stage_f = [&](const SSlab& b, const CUtensorMap* m, int s, const double* src) {
    if (tens) {
      if (threadIdx.x == 0) tma_load_4d(b.p, m, o.x0 - XH, o.y0 - H, o.z0, s, bar);
    } else {
      stage_plain<B, SNW, NC>(b, fo, g, o, src, bar);
    }
  };
  const int tx = threadIdx.x % SX_, ty = threadIdx.x / SX_;
  fo.init(g, o, zd);
  BulkBar bb{bar, 0u};
  if (B && threadIdx.x == 0) mbar_init(bar, 1);
  tile_sync();
  TP tp[SZ_];
#pragma unroll
  for (int z = 0; z < SZ_; ++z) tp[z] = make_tp(g, o, tx, ty, z);
  const int64_t n = g.n;
  // rho u, rho v, rho w: fields 1..3 of U, or (KEEP) their copy, since this
  // CTA's RK pass and those of its neighbours rewrite U while tiles still read it
  const double* const ru = KEEP ? f.mom : f.uin + n;
  const double* const rv = KEEP ? f.mom + n : f.uin + 2 * n;
  const double* const rw = KEEP ? f.mom + 2 * n : f.uin + 3 * n;
  const SXRow bru{sm};
  const SYRow brv{sm + SXRow::SIZE};
  const SSlab bS{sm + SXRow::SIZE + SYRow::SIZE};
  const SSlab bH{sm + SXRow::SIZE + SYRow::SIZE + SSlab::SIZE};
  const SSlab bR{sm + SXRow::SIZE + SYRow::SIZE + 2 * SSlab::SIZE};
  if (tens) {
    if (threadIdx.x == 0) {
      tma_load_4d(bru.p, &tm->ux, o.x0 - XH, o.y0, o.z0, 1, bar);
      tma_load_4d(brv.p, &tm->vy, o.x0, o.y0 - H, o.z0, 2, bar);
    }
  } else {
    stage_plain<B, SNW, NC>(bru, fo, g, o, ru, bar);
    stage_plain<B, SNW, NC>(brv, fo, g, o, rv, bar);
  }
  // copies run one stage ahead: Y_s while the previous species' rho D and
  // h are used, rho D and h of species s while Y_s is used
  if (nspec > 0) stage_f(bS, tm ? &tm->y : nullptr, 0, f.y);
  // bytes of the group in flight (bulk paths): rho u, rho v and Y_0 first
  unsigned inflight = SXRow::kBulkBytes + SYRow::kBulkBytes + slab_bytes;
  // this thread's rho w z-column, kept in shared memory across the species
  // loop (in registers it would take 24 of them for the whole loop); the
  // fused kernel (KEEP), whose shared memory holds the species rates past
  // the slabs, keeps it in registers
  double* const colw = sm + SXRow::SIZE + SYRow::SIZE + 3 * SSlab::SIZE;
  SCol rwc;
  rwc.load(fo, tx, ty, LdT<NC>{rw});
  if constexpr (!KEEP) {
#pragma unroll
    for (int k = 0; k < SZ_ + 2 * H; ++k) colw[k * (SX_ * SY_) + threadIdx.x] = rwc.c[k];
  }
  auto wcol = [&](int k) {
    if constexpr (KEEP) return rwc.c[k];
    else return colw[k * (SX_ * SY_) + threadIdx.x];
  };
  double vcx[SZ_], vcy[SZ_], vcz[SZ_], vt[SZ_], rE[SZ_], dvm[SZ_];
#pragma unroll
  for (int z = 0; z < SZ_; ++z) {
    vcx[z] = vcy[z] = vcz[z] = vt[z] = 0.0;
    rE[z] = tp[z].valid ? f.rhs[4 * n + tp[z].q] : 0.0;
    dvm[z] = tp[z].valid ? f.divm[tp[z].q] : 0.0;
  }
  for (int s = 0; s < nspec; ++s) {
    double rate[SZ_], yx[SZ_], yy[SZ_], yz[SZ_], fn1[SZ_], fn3[SZ_], rd[SZ_];
    // Y_k: convection, gradient, Laplacian
    {
      SCol cy;
      cy.load(fo, tx, ty, LdT<NC>{f.y + s * n});
      // the chemistry rate of the thread's points, loaded before the wait
      // (an invalid point has q = 0: in bounds, unused)
      double w0[SZ_];
#pragma unroll
      for (int z = 0; z < SZ_; ++z) w0[z] = f.wdot[s * n + tp[z].q];
      // Y_s has landed in bS; the rho D and h slabs are free
      if (sync_staged<B>(bb, inflight, f.status)) return;
      stage_f(bR, tm ? &tm->rd : nullptr, s, f.rd + s * n);
      stage_f(bH, tm ? &tm->h : nullptr, s, f.h + s * n);
      inflight = 2 * slab_bytes;
#pragma unroll
      for (int z = 0; z < SZ_; ++z) {
        const TP& t = tp[z];
        const double yq = cy.c[z + H];
        double r = w0[z];
        r = r - 0.5 * yq * dvm[z];
        if constexpr (P) {
          // all periodic: each staged neighbour of Y, rho u, rho v read once
          // into registers and shared by the flux, first and second
          // derivatives (same arithmetic as the generic path)
          double d1px, d1py, d2x, d2y, uc, vc;
          {
            double yv[2 * H + 1], fv[2 * H + 1];
#pragma unroll
            for (int m = 0; m <= 2 * H; ++m) {
              yv[m] = bS.v(t.x + m - H, t.y, t.z);
              fv[m] = bru.v(t.x + m - H, t.y, t.z);
            }
            d1px = d1core([&](int m) { return yv[m + H] * fv[m + H]; }, t.gx, g.nx, 1) * g.ovd[0];
            yx[z] = d1core([&](int m) { return yv[m + H]; }, t.gx, g.nx, 1) * g.ovd[0];
            d2x = d2core([&](int m) { return yv[m + H]; }, t.gx, g.nx, 1) * g.ovd2[0];
            uc = fv[H];
          }
          {
            double yv[2 * H + 1], fv[2 * H + 1];
#pragma unroll
            for (int m = 0; m <= 2 * H; ++m) {
              yv[m] = bS.v(t.x, t.y + m - H, t.z);
              fv[m] = brv.v(t.x, t.y + m - H, t.z);
            }
            d1py = d1core([&](int m) { return yv[m + H] * fv[m + H]; }, t.gy, g.ny, 1) * g.ovd[1];
            yy[z] = d1core([&](int m) { return yv[m + H]; }, t.gy, g.ny, 1) * g.ovd[1];
            d2y = d2core([&](int m) { return yv[m + H]; }, t.gy, g.ny, 1) * g.ovd2[1];
            vc = fv[H];
          }
          r = r - 0.5 * (d1px + d1py + d1core([&](int m) { return cy.c[t.z + H + m] * wcol(t.z + H + m); }, t.gz, g.nz, 1) * g.ovd[2]);
          yz[z] = d1z<P>(g, t, cy);
          r = r - 0.5 * (yx[z] * uc + yy[z] * vc + yz[z] * wcol(z + H));
          rate[z] = r;
          fn3[z] = d2x + d2y + d2z<P>(g, t, cy);  // Laplacian for now
        } else {
          r = r - 0.5 * (d1p<0, P>(g, t, bS, bru) + d1p<1, P>(g, t, bS, brv) + d1core([&](int m) { return cy.c[t.z + H + m] * wcol(t.z + H + m); }, t.gz, g.nz, 1) * g.ovd[2]);
          yx[z] = d1<0, P>(g, t, bS);
          yy[z] = d1<1, P>(g, t, bS);
          yz[z] = d1z<P>(g, t, cy);
          r = r - 0.5 * (yx[z] * bru.v(t.x, t.y, t.z) + yy[z] * brv.v(t.x, t.y, t.z) + yz[z] * wcol(z + H));
          rate[z] = r;
          // FxxDIF/FxxADB zero the x diffusive terms on the face plane (rhscal.f:1581-1955)
          const bool dif = !P && (face_bits(g, t.gx) & BF_DIF);
          fn3[z] = (dif ? 0.0 : d2<0, P>(g, t, bS)) + d2<1, P>(g, t, bS) + d2z<P>(g, t, cy);  // Laplacian for now
        }
      }
    }
    // rho D_k and h_k staged together (one barrier pair): correction
    // velocity, diffusive flux divergence, enthalpy fluxes of the energy
    // equation
    {
      SCol cd, ch;
      cd.load(fo, tx, ty, LdT<NC>{f.rd + s * n});
      ch.load(fo, tx, ty, LdT<NC>{f.h + s * n});
      // rho D_s, h_s have landed; every thread is done with Y_s
      if (sync_staged<B>(bb, inflight, f.status)) return;
      if (s + 1 < nspec) stage_f(bS, tm ? &tm->y : nullptr, s + 1, f.y + (s + 1) * n);
      inflight = slab_bytes;
#pragma unroll
      for (int z = 0; z < SZ_; ++z) {
        const TP& t = tp[z];
        rd[z] = cd.c[z + H];
        vcx[z] = vcx[z] + rd[z] * yx[z];
        vcy[z] = vcy[z] + rd[z] * yy[z];
        vcz[z] = vcz[z] + rd[z] * yz[z];
        const bool dif = !P && (face_bits(g, t.gx) & BF_DIF);
        const double fn = (dif ? 0.0 : d1<0, P>(g, t, bR) * yx[z]) + d1<1, P>(g, t, bR) * yy[z] +
                          d1z<P>(g, t, cd) * yz[z];
        rate[z] = rate[z] + fn;
        vt[z] = vt[z] + fn;
        fn1[z] = fn;
        const double f3 = fn3[z] * rd[z];
        rate[z] = rate[z] + f3;
        vt[z] = vt[z] + f3;
        fn3[z] = f3;
        const double hk = ch.c[z + H];
        rE[z] = rE[z] + fn1[z] * hk;
        const double fn2 = (dif ? 0.0 : d1<0, P>(g, t, bH) * yx[z]) + d1<1, P>(g, t, bH) * yy[z] +
                           d1z<P>(g, t, ch) * yz[z];
        rE[z] = rE[z] + fn2 * rd[z];
        rE[z] = rE[z] + fn3[z] * hk;
        if constexpr (KEEP) carry->rate[(s * SZ_ + z) * (SX_ * SY_) + threadIdx.x] = rate[z];
        else if (t.valid) f.wdot[s * n + t.q] = rate[z];
      }
    }
  }
#pragma unroll
  for (int z = 0; z < SZ_; ++z) {
    if constexpr (KEEP) {
      carry->vcx[z] = vcx[z];
      carry->vcy[z] = vcy[z];
      carry->vcz[z] = vcz[z];
      carry->vt[z] = vt[z];
      carry->rE[z] = rE[z];
      continue;
    }
    const TP& t = tp[z];
    if (!t.valid) continue;
    f.vc[t.q] = vcx[z];
    f.vc[n + t.q] = vcy[z];
    f.vc[2 * n + t.q] = vcz[z];
    f.vtmp[t.q] = vt[z];
    f.rhs[4 * n + t.q] = rE[z];
  }
}

// -------------------------------------------------------------------------
template <bool P, int M = 0, bool NC = true, bool KEEP = false>
__device__ __forceinline__ void species_rk_tile(const Geo& g, const Fields& f, int nspec, const RK& rk,
                                                const Origin o, double* sm, Folds<SX_, SY_, SZ_>& fo,
                                                const ZDec& zd, uint64_t* bar = nullptr, const RkMaps* tm = nullptr,
                                                const SpecCarry* carry = nullptr) {
  constexpr bool B = M > 0;
  const bool tens = M == 2 && tensor_tile<SX_, SY_, SZ_>(g, o, sm);
  const unsigned slab_bytes = tens ? 8u * SSlab::SIZE : SSlab::kBulkBytes;
  auto stage_f = [&](const SSlab& b, const CUtensorMap* m, int s, const double* src) {
    if (tens) {
      if (threadIdx.x == 0) tma_load_4d(b.p, m, o.x0 - XH, o.y0 - H, o.z0, s, bar);
    } else {
      stage_plain<B, SNW, NC>(b, fo, g, o, src, bar);
    }
  };
  const int tx = threadIdx.x % SX_, ty = threadIdx.x / SX_;
  // KEEP: the species pass of this CTA built the same tables; the barrier
  // below also ends its reads of the buffers this pass fills
  if constexpr (!KEEP) fo.init(g, o, zd);
  BulkBar bb{bar, 0u};
  if (B && threadIdx.x == 0) mbar_init(bar, 1);
  tile_sync();
  TP tp[SZ_];
#pragma unroll
  for (int z = 0; z < SZ_; ++z) tp[z] = make_tp(g, o, tx, ty, z);
  const int64_t n = g.n;
  const SSlab bS{sm};
  const int nc = 5 + nspec;
  // bf: x-face bits of the point; NSCBC planes add the BOUNDS correction
  // (precomputed per face point), an I3 inflow plane integrates only E, an
  // I2 plane only D, a wall has zero momentum and energy RHS and integrates
  // no momentum (src/bcinit.f ranges ISTALD..ISTALY; a W2 wall's energy,
  // left out of the range too, is advanced by a zero RHS, which leaves both
  // registers where BOUNDT put them)
  auto advance = [&](int fld, const TP& t, int bf, double R, const double* srun = nullptr) {
    const int64_t q = t.q;
    const int64_t idx = (int64_t)fld * n + q;
    if (!P && (bf & BF_NSCBC)) {
      const int side = t.gx == 0 ? 0 : 1;
      R = R + f.face[((int64_t)side * nc + fld) * ((int64_t)g.ny * g.nz) + t.gy + (int64_t)g.ny * t.gz];
    }
    if (!P && (bf & BF_WALL) && fld >= 1 && fld <= 4) R = 0.0;
    if (rk.last < 0) {  // right-hand side only
      f.rhs[idx] = R;
      return;
    }
    if (!P && (bf & BF_IMPOSED) && fld != 4) return;
    if (!P && (bf & BF_IMPOSED_D) && fld != 0) return;
    if (!P && (bf & BF_WALL) && fld >= 1 && fld <= 3) return;
    if (f.err) f.err[idx] = f.err[idx] + rk.err * R;
    const double s0 = srun ? *srun : f.run[idx];
    if (!rk.last) {
      f.run[idx] = s0 + rk.lhs * R;
      f.uout[idx] = s0 + rk.rhs * R;
    } else {
      const double s = s0 + rk.lhs * R;
      f.run[idx] = s;
      f.uout[idx] = s;
    }
  };
  // per-element staging (cp.async), not fused: the rate of each species'
  // own points, and in the RK form their S register, are copied into shared
  // memory together with its slab, one species ahead, so their latency
  // overlaps the previous species' work; a thread reads back only the slots
  // it copied. The RHS-only form has no S register (its pointer may be null)
  // and copies only the rate.
  constexpr bool PRE = M == 0 && !KEEP;
  const bool pre_run = PRE && rk.last >= 0 && f.run != nullptr;
  double* const pre = sm + 2 * SSlab::SIZE;
  auto prefetch = [&](int s) {
    if constexpr (PRE) {
      double* b = pre + (s & 1) * kRkPre;
#pragma unroll
      for (int z = 0; z < SZ_; ++z) {
        if (!tp[z].valid) continue;
        if (pre_run) cp_async8(b + z * (SX_ * SY_) + threadIdx.x, f.run + (int64_t)(5 + s) * n + tp[z].q);
        cp_async8(b + (SZ_ + z) * (SX_ * SY_) + threadIdx.x, f.wdot + (int64_t)s * n + tp[z].q);
      }
    }
  };
  double vcx[SZ_], vcy[SZ_], vcz[SZ_], vt[SZ_];
#pragma unroll
  for (int z = 0; z < SZ_; ++z) {
    if constexpr (KEEP) {
      vcx[z] = carry->vcx[z];
      vcy[z] = carry->vcy[z];
      vcz[z] = carry->vcz[z];
      vt[z] = carry->vt[z];
      continue;
    }
    const int64_t q = tp[z].q;
    vcx[z] = f.vc[q];
    vcy[z] = f.vc[n + q];
    vcz[z] = f.vc[2 * n + q];
    vt[z] = f.vtmp[q];
  }
  // two slabs in turn: while one species' Y is differentiated, the next
  // one's copy (cp.async) is in flight into the other
  auto slab = [&](int i) { return SSlab{(i & 1) ? sm : sm + SSlab::SIZE}; };
  {
    SCol cm;
    cm.load(fo, tx, ty, LdT<NC>{f.hmix});
    stage_f(bS, tm ? &tm->hm : nullptr, 0, f.hmix);
    if (sync_staged<B>(bb, slab_bytes, f.status)) return;
    if (nspec > 0) {
      stage_f(slab(0), tm ? &tm->y : nullptr, 0, f.y);
      prefetch(0);
    }
#pragma unroll
    for (int z = 0; z < SZ_; ++z) {
      const TP& t = tp[z];
      if (!t.valid) continue;
      const int bf = P ? 0 : face_bits(g, t.gx);
      // FxxDIF/FxxADB: x gradient term and VTMP vanish on the face (rhscal.f:3782-3839)
      const bool dif = bf & BF_DIF;
      const double rE = (KEEP ? carry->rE[z] : f.rhs[4 * n + t.q]) - cm.c[z + H] * (dif ? 0.0 : vt[z]) -
                        (dif ? 0.0 : d1<0, P>(g, t, bS) * vcx[z]) - d1<1, P>(g, t, bS) * vcy[z] -
                        d1z<P>(g, t, cm) * vcz[z];
#pragma unroll
      for (int fl = 0; fl < 4; ++fl) advance(fl, t, bf, f.rhs[fl * n + t.q]);
      advance(4, t, bf, rE);
    }
  }
  for (int s = 0; s < nspec; ++s) {
    SCol cy;
    cy.load(fo, tx, ty, LdT<NC>{f.y + s * n});
    // Y_s has landed in slab(s); every thread is done with the other slab
    if (sync_staged<B>(bb, slab_bytes, f.status)) return;
    if (s + 1 < nspec) {
      stage_f(slab(s + 1), tm ? &tm->y : nullptr, s + 1, f.y + (s + 1) * n);
      prefetch(s + 1);
    }
    const SSlab bY = slab(s);
    const double* const pb = pre + (s & 1) * kRkPre;
#pragma unroll
    for (int z = 0; z < SZ_; ++z) {
      const TP& t = tp[z];
      if (!t.valid) continue;
      const int bf = P ? 0 : face_bits(g, t.gx);
      const bool dif = bf & BF_DIF;  // rhscal.f:3919: x gradient of Y zeroed on the face
      const double rate = KEEP  ? carry->rate[(s * SZ_ + z) * (SX_ * SY_) + threadIdx.x]
                          : PRE ? pb[(SZ_ + z) * (SX_ * SY_) + threadIdx.x]
                                : f.wdot[s * n + t.q];
      const double R = rate - cy.c[z + H] * vt[z] - (dif ? 0.0 : d1<0, P>(g, t, bY) * vcx[z]) -
                       d1<1, P>(g, t, bY) * vcy[z] - d1z<P>(g, t, cy) * vcz[z];
      advance(5 + s, t, bf, R, pre_run ? pb + z * (SX_ * SY_) + threadIdx.x : nullptr);
    }
  }
}

}  // namespace
}  // namespace senga
