// Navier-Stokes characteristic boundary conditions on the x faces.
//
// Restated from the reference (I1 subsonic non-reflecting laminar inflow,
// I4 Lodato-type inflow relaxed towards targets (x-left, as coded),
// I3 subsonic inflow with constant velocity,
// NXxPRM(1)=1, I2 subsonic reflecting inflow with specified temperature,
// O1 partially non-reflecting outflow, W1 adiabatic and W2 isothermal
// no-slip walls, on either x face; inflow on one face at most; both O1 faces
// take the same parameters):
//   BOUNDT  src/boundt.f:177-200 (x-left), 591- (x-right)   impose the
//           inflow state on the U register
//   face data gathered inside RHSCAL/RHSVEL (src/rhscal.f:70-90,159-180,
//           257-275,438-456,841-862,1140-1180,1483-1500,3966-3990;
//           src/rhsvel.f:62-200,558-570,764-800,1310-1325,1630-1650)
//   BOUNDS  src/bounds.f:115-157 (x-left preliminaries), 213-372 (O1 left),
//           610-675 (I3 left), 1198-1240 (x-right preliminaries), 1296-1450
//           (O1 right), 1688- (I3 right)
//   BOUNTT  src/bountt.f:203-252 (x-left), 709- (x-right)   both registers
//           of the inflow plane reset
//   W1      boundt.f:243-356, 657-768 and bountt.f:290-428, 767- (wall
//           temperature extrapolated, zero momentum, internal energy);
//           bounds.f:917-1056, 1833-1974 (reflected wave); rhscal.f:1698-1760
//           (wall diffusion flux); lincom.f/fincom.f:171-210 (zero-gradient
//           mass fractions)
//   W2      the same with the wall temperature imposed (boundt.f:358-470,
//           bountt.f:429-560 and their x-right blocks; bounds.f:1058-1190,
//           1975-), energy not integrated on the wall
// Every face quantity is a pointwise value or a derivative at the face plane,
// so one thread per face point computes them from the thermochemistry
// kernel's outputs and the U register right after that kernel (before the
// species kernel overwrites the chemistry rate), folds BOUNDS into one
// additive correction per conserved field, and the fused RK epilogue adds it
// on the face planes (face_bits BF_NSCBC). This is O(ny*nz) work.
#include <cuda_runtime.h>

#include "senga_internal.h"
#include "itndex.cuh"
#include "stencil.cuh"

namespace senga {
namespace {

constexpr int kFaceBlock = 128;

// value m points along DIR from (i, j, k); y and z periodic, x bounded (the
// closures read only inward points). A box split along z (zd.nr > 1) reads
// the z neighbours from the slab that owns their plane.
template <int DIR>
__device__ __forceinline__ double at(const Geo& g, const ZDec& zd, const double* a, int i, int j, int k, int m) {
  if (DIR == 0) i += m;
  if (DIR == 1) j = ((j + m) % g.ny + g.ny) % g.ny;
  int64_t base = 0;
  if (DIR == 2) {
    if (zd.nr > 1) {
      const int zg = ((zd.rank * g.nz + k + m) % zd.nzg + zd.nzg) % zd.nzg;
      const int r = zg / g.nz;
      base = zd.base[r];
      k = zg - r * g.nz;
    } else {
      k = ((k + m) % g.nz + g.nz) % g.nz;
    }
  }
  return a[base + (int64_t)i + (int64_t)g.nx * (j + (int64_t)g.ny * k)];
}
template <int DIR>
__device__ __forceinline__ double dd(const Geo& g, const ZDec& zd, const double* a, int i, int j, int k) {
  const int c = DIR == 0 ? i : DIR == 1 ? j : k;
  const int n = DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
  return d1core([&](int m) { return at<DIR>(g, zd, a, i, j, k, m); }, c, n, g.per[DIR]) * g.ovd[DIR];
}
// derivative of (a - c) along DIR: the pressure gradient of RHSVEL is taken of
// p - p(1,1,1) (src/rhsvel.f:730-752)
template <int DIR>
__device__ __forceinline__ double dd_sub(const Geo& g, const ZDec& zd, const double* a, double c0, int i, int j,
                                         int k) {
  const int c = DIR == 0 ? i : DIR == 1 ? j : k;
  const int n = DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
  return d1core([&](int m) { return at<DIR>(g, zd, a, i, j, k, m) - c0; }, c, n, g.per[DIR]) * g.ovd[DIR];
}

// h_k(T) per unit mass of interval `it` (AMASCH polynomial, boundt.f:316-324)
__device__ __forceinline__ double enthalpy(const senga_chem* chem, int s, int it, double t) {
  const double* c = chem->amasch[s][it];
  double h = c[chem->ncpoly[s][it] - 1];
  for (int icp = chem->ncpom1[s][it]; icp >= 1; --icp) h = h * t + c[icp - 1];
  return c[chem->ncenth[s][it] - 1] + h * t;
}
__device__ __forceinline__ uint64_t interval_index(const senga_chem* chem, int nspec, double t) {
  uint64_t itn = 0;
  for (int s = 0; s < nspec; ++s) {
    int it = 0;
    while (t > chem->tinthi[s][it] && it + 1 < chem->ntint[s]) ++it;
    itn += (uint64_t)it << (2 * s);
  }
  return itn;
}
// W1 wall temperature (boundt.f:252-260): T_w = (48 T_1 - 36 T_2 + 16 T_3 -
// 3 T_4)/25 over the four planes inward, st = +1 (x-left) or -1 (x-right)
__device__ __forceinline__ double wall_t(const double* t, int64_t q, int st) {
  return (48.0 * t[q + st] - 36.0 * t[q + 2 * st] + 16.0 * t[q + 3 * st] - 3.0 * t[q + 4 * st]) / 25.0;
}

// one thread per face point; blockIdx.y = side (0: x-left, 1: x-right)
__global__ void __launch_bounds__(kFaceBlock)
    k_boundt(Geo g, Fields f, NscbcParams bc, int nspec, int both, const senga_chem* chem) {
  const int jk = blockIdx.x * kFaceBlock + threadIdx.x;
  if (jk >= g.ny * g.nz) return;
  const int64_t n = g.n;
  const int side = blockIdx.y;
  const int kind = side == 0 ? bc.xl : bc.xr;
  if (kind != 12 && kind != 13 && kind != 31 && kind != 32) return;
  const int i = side == 0 ? 0 : g.nx - 1;  // the face plane
  const int64_t q = (int64_t)i + (int64_t)g.nx * jk;
  double* regs[2] = {f.uin, f.run};
  if (kind == 31 || kind == 32) {
    // W1 (boundt.f:243-356 / 657-768; bountt.f:290-428 / 767-): wall
    // temperature from the last TEMPER's planes inward, its ITNDEX, zero
    // momentum, rho E = sum_k (h_k(T) - R_k T) rho Y_k. W2 (boundt.f:
    // 358-470, bountt.f:429-560): the imposed temperature, TRUN untouched.
    double t;
    if (kind == 31) {
      t = wall_t(f.t, q, side == 0 ? 1 : -1);
      f.t[q] = t;
    } else {
      t = bc.t_wall[side];
    }
    const uint64_t itn = interval_index(chem, nspec, t);
    itn_store(f.itn, n, q, nspec, itn);
    double e = 0.0;
    e = f.uin[q] * e;
    for (int s = 0; s < nspec; ++s)
      e = e + (enthalpy(chem, s, (int)(itn >> (2 * s)) & 3, t) - chem->rgspec[s] * t) * f.uin[(5 + s) * n + q];
    for (int r = 0; r < (both ? 2 : 1); ++r) {
      double* U = regs[r];
      U[n + q] = 0.0;
      U[2 * n + q] = 0.0;
      U[3 * n + q] = 0.0;
      U[4 * n + q] = e;
    }
    if (both && f.err)  // BOUNTT: momentum and energy errors zeroed
      for (int fl = 1; fl < 5; ++fl) f.err[fl * n + q] = 0.0;
    return;
  }
  if (kind == 12) {
    // I2 (boundt.f:81-176, bountt.f:84-200): ITNDEX of TRIN, then velocity,
    // energy and species from the face density of the U register
    const double t = bc.t_in, u = bc.u_in, v = 0.0, w = 0.0;
    const uint64_t itn = interval_index(chem, nspec, t);
    itn_store(f.itn, n, q, nspec, itn);
    const double d = f.uin[q];
    double e = 0.5 * (u * u + v * v + w * w);
    e = d * e;
    double ys[SENGA_NSPCMX];
    for (int s = 0; s < nspec; ++s) {
      const double h = enthalpy(chem, s, (int)(itn >> (2 * s)) & 3, t);
      ys[s] = d * bc.y_in[s];
      e = e + (h - chem->rgspec[s] * t) * ys[s];
    }
    for (int r = 0; r < (both ? 2 : 1); ++r) {
      double* U = regs[r];
      U[n + q] = d * u;
      U[2 * n + q] = d * v;
      U[3 * n + q] = d * w;
      U[4 * n + q] = e;
      for (int s = 0; s < nspec; ++s) U[(5 + s) * n + q] = ys[s];
    }
    if (both && f.err) {  // BOUNTT: error of the imposed fields zeroed (not the density's)
      for (int fl = 1; fl < 5; ++fl) f.err[fl * n + q] = 0.0;
      for (int s = 0; s < nspec; ++s) f.err[(5 + s) * n + q] = 0.0;
    }
    return;
  }
  const double r = bc.rho_in;
  // BCUTXL: constant U_in, or the synthetic inflow (bcutxl.f:492-498, VFAC = 1)
  const bool syn = bc.uinf2 != nullptr;
  const double su = syn ? (bc.u_in * 1.0 + bc.uinf2[jk]) * 1.0 + bc.coflow : bc.u_in;
  const double sv = syn ? bc.vinf2[jk] * 1.0 : 0.0, sw = syn ? bc.winf2[jk] * 1.0 : 0.0;
  for (int w = 0; w < (both ? 2 : 1); ++w) {
    double* U = regs[w];
    U[q] = r;
    U[n + q] = r * su;
    U[2 * n + q] = r * sv;
    U[3 * n + q] = r * sw;
    for (int s = 0; s < nspec; ++s) U[(5 + s) * n + q] = r * bc.y_in[s];
  }
  if (both && f.err) {  // BOUNTT: error of the imposed fields zeroed
    for (int fl = 0; fl < 4; ++fl) f.err[fl * n + q] = 0.0;
    for (int s = 0; s < nspec; ++s) f.err[(5 + s) * n + q] = 0.0;
  }
}

__global__ void __launch_bounds__(kFaceBlock) k_face(Geo g, Fields f, NscbcParams bc, int nspec, const senga_chem* chem,
                                                   ZDec zd) {
  const int nyz = g.ny * g.nz;
  const int jk = blockIdx.x * kFaceBlock + threadIdx.x;
  const int side = blockIdx.y;  // 0: x-left, 1: x-right
  const int kind = side == 0 ? bc.xl : bc.xr;
  if (jk >= nyz || kind == 0) return;
  const int j = jk % g.ny, k = jk / g.ny;
  const int i = side == 0 ? 0 : g.nx - 1;
  const int64_t n = g.n;
  const int64_t q = (int64_t)i + (int64_t)g.nx * jk;
  const int nc = 5 + nspec;
  const double* U = f.uin;
  const double* vel = f.vel;
  const double pref = __ldg(f.p + zd.base[0]);  // p(1,1,1) lives in slab 0
  // ---- face data ----
  const double d = U[q], u = vel[q], v = vel[n + q], w = vel[2 * n + q];
  const double p = f.p[q], t = f.t[q], rr = f.rmix[q] / d, cp = f.cp[q];
  double e = f.e[q];
  const double bcl1 = dd<0>(g, zd, vel, i, j, k), bcl2 = dd<0>(g, zd, U, i, j, k);
  const double bcl3 = dd<0>(g, zd, vel + n, i, j, k), bcl4 = dd<0>(g, zd, vel + 2 * n, i, j, k);
  const double bcl5 = dd_sub<0>(g, zd, f.p, pref, i, j, k);
  const double t2b = -v * dd<1>(g, zd, vel, i, j, k) - w * dd<2>(g, zd, vel, i, j, k);
  const double py = dd_sub<1>(g, zd, f.p, pref, i, j, k), pz = dd_sub<2>(g, zd, f.p, pref, i, j, k);
  const double t51b = -v * py - w * pz;
  const double t52b = -p * (dd<1>(g, zd, vel + n, i, j, k) + dd<2>(g, zd, vel + 2 * n, i, j, k));
  // ---- BOUNDS preliminaries (bounds.f:115-157 / 1198-1240) ----
  double gam1 = cp - rr;
  e = e - gam1 * t;
  gam1 = rr / gam1;
  const double ovgm = 1.0 / gam1;
  const double fornow0 = cp * gam1 * t;
  const double acou = sqrt(fornow0);
  const double ova2 = 1.0 / fornow0;
  double* corr = f.face + (int64_t)side * nc * nyz + jk;
  for (int fl = 0; fl < nc; ++fl) corr[(int64_t)fl * nyz] = 0.0;
  auto hprime = [&](int s) { return f.h[s * n + q] - cp * t * chem->rgspec[s] / rr; };
  if (kind == 12) {  // I2 inflow (bounds.f:522-608 left, 1600-1684 right): u, T, Y imposed, DRHS corrected
    double sydt = 0.0, sorp = 0.0;
    for (int s = 0; s < nspec; ++s) {
      sydt = sydt + 0.0 * chem->rgspec[s];
      sorp = sorp + hprime(s) * f.wdot[s * n + q];
    }
    sydt = sydt / rr;
    sorp = -sorp * gam1;
    const double fornow = d * acou * bcl1;
    double b1 = 0.5 * (u - acou) * (bcl5 - fornow);
    double b2 = u * (bcl2 - bcl5 * ova2);
    double b5 = 0.5 * (u + acou) * (bcl5 + fornow);
    if (side == 0) b5 = b1 - d * acou * 0.0 - b5;  // L1 unchanged
    else b1 = b5 + d * acou * 0.0 - b1;            // L5 unchanged
    b2 = gam1 * ova2 * (b1 + b5) + d * (0.0 / t - sorp / p + sydt) - b2;
    corr[0] = -b2 - (side == 0 ? b5 : b1) * ova2;
  } else if (kind == 14) {  // I4 inflow at x-left (bounds.f:686-845): waves relaxed towards the targets
    const double m2max = 0.001;  // bounds.f:101
    const double xl = bc.xlen, c = acou;
    const double n2 = bc.nrieta[1], n3 = bc.nrieta[2], n4 = bc.nrieta[3], n5 = bc.nrieta[4], n6 = bc.nrieta[5];
    // transverse terms (bounds.f:185-204 from rhscal.f:159-180, rhsvel.f:62-200, 764-800)
    const double t1b = -(dd<1>(g, zd, U + 2 * n, i, j, k) + dd<2>(g, zd, U + 3 * n, i, j, k));
    const double rho_inv = 1.0 / d;
    const double t3b = -v * dd<1>(g, zd, vel + n, i, j, k) - w * dd<2>(g, zd, vel + n, i, j, k) - py * rho_inv;
    const double t4b = -v * dd<1>(g, zd, vel + 2 * n, i, j, k) - w * dd<2>(g, zd, vel + 2 * n, i, j, k) - pz * rho_inv;
    const double tt2 = c * c * t1b - t51b - (gam1 + 1.0) * t52b;
    const double tt5 = t51b + t52b * (gam1 + 1.0) + d * c * t2b;
    const double fornow = d * c * bcl1;
    double b2 = u * (bcl2 - bcl5 * ova2);
    double b3 = u * bcl3;
    double b4 = u * bcl4;
    double b5 = 0.5 * (u + c) * (bcl5 + fornow);
    b2 = n2 * d * rr / (xl * c) * (t - bc.t_in) + tt2 * ova2 - b2;
    b3 = n3 * c / xl * (v - 0.0) + t3b - b3;
    b4 = n4 * c / xl * (w - 0.0) + t4b - b4;
    b5 = n5 * d * c * c * (1.0 - m2max) / (2.0 * xl) * (u - bc.u_in) + 0.5 * tt5 - b5;
    corr[0] = -b2 - b5 * ova2;
    corr[(int64_t)nyz] = -b2 * u - b5 * ova2 * (u + c);
    corr[2 * (int64_t)nyz] = -b2 * v - b3 * d - b5 * ova2 * v;
    corr[3 * (int64_t)nyz] = -b2 * w - b4 * d - b5 * ova2 * w;
    double ce = -b2 * e - b3 * d * v - b4 * d * w - b5 * (ova2 * e + u / c + ovgm);
    for (int s = 0; s < nspec; ++s) {
      const double* ys = f.y + s * n;
      const double t6b = -dd<1>(g, zd, ys, i, j, k) * v - dd<2>(g, zd, ys, i, j, k) * w;
      double bcly = u * dd<0>(g, zd, ys, i, j, k);
      bcly = n6 * c / xl * (ys[q] - bc.y_in[s]) + t6b - bcly;
      const double fn = bcly * d;
      ce = ce - fn * hprime(s);
      corr[(int64_t)(5 + s) * nyz] = -(b2 + b5 * ova2) * ys[q] - fn;
    }
    corr[4 * (int64_t)nyz] = ce;
  } else if (kind == 11) {  // I1 inflow (bounds.f:387-520 left, 1465-1598 right): nothing imposed
    double sorp = 0.0;
    for (int s = 0; s < nspec; ++s) sorp = sorp + hprime(s) * f.wdot[s * n + q];
    sorp = -sorp * gam1;
    const double cobc = 0.0, pinf = 0.0;  // COBCxx, PINFxx: set by BCINIT only for an O1 face
    const double fornow = d * acou * bcl1;
    double b1 = 0.5 * (u - acou) * (bcl5 - fornow);
    double b2 = u * (bcl2 - bcl5 * ova2);
    double b3 = u * bcl3;
    double b4 = u * bcl4;
    double b5 = 0.5 * (u + acou) * (bcl5 + fornow);
    b2 = -b2;
    b3 = -b3;
    b4 = -b4;
    double ce;
    if (side == 0) {  // L5 enters
      b5 = 0.5 * sorp + cobc * acou * (p - pinf) - b5;
      corr[0] = -b2 - b5 * ova2;
      corr[(int64_t)nyz] = -b2 * u - b5 * ova2 * (u + acou);
      corr[2 * (int64_t)nyz] = -b2 * v - b3 * d - b5 * ova2 * v;
      corr[3 * (int64_t)nyz] = -b2 * w - b4 * d - b5 * ova2 * w;
      ce = -b2 * e - b3 * d * v - b4 * d * w - b5 * (ova2 * e + u / acou + ovgm);
    } else {  // L1 enters
      b1 = 0.5 * sorp + cobc * acou * (p - pinf) - b1;
      corr[0] = -b1 * ova2 - b2;
      corr[(int64_t)nyz] = -b1 * ova2 * (u - acou) - b2 * u;
      corr[2 * (int64_t)nyz] = -b1 * ova2 * v - b2 * v - b3 * d;
      corr[3 * (int64_t)nyz] = -b1 * ova2 * w - b2 * w - b4 * d;
      ce = -b1 * (ova2 * e - u / acou + ovgm) - b2 * e - b3 * d * v - b4 * d * w;
    }
    const double lw = side == 0 ? b5 : b1;
    for (int s = 0; s < nspec; ++s) {
      double bcly = u * dd<0>(g, zd, f.y + s * n, i, j, k);
      bcly = f.wdot[s * n + q] / d - bcly;
      const double fn = bcly * d;
      ce = ce - fn * hprime(s);
      corr[(int64_t)(5 + s) * nyz] = -(b2 + lw * ova2) * f.y[s * n + q] - fn;
    }
    corr[4 * (int64_t)nyz] = ce;
  } else if (kind == 31 || kind == 32) {  // W1/W2 wall (bounds.f:917-1056, 1058-1190 left; 1833-1974, 1975- right)
    // the outgoing wave reflected (L5 = L1 - L5 on the left, L1 = L5 - L1 on
    // the right), L2 = L3 = L4 = LY = 0; U, V, W, E RHS zeroed in the RK
    // epilogue (BF_WALL)
    const double fornow = d * acou * bcl1;
    const double b1 = 0.5 * (u - acou) * (bcl5 - fornow);
    const double b5 = 0.5 * (u + acou) * (bcl5 + fornow);
    const double lw = side == 0 ? b1 - b5 : b5 - b1;
    const double b2 = 0.0;
    corr[0] = side == 0 ? -b2 - lw * ova2 : -lw * ova2 - b2;
    for (int s = 0; s < nspec; ++s) corr[(int64_t)(5 + s) * nyz] = -(b2 + lw * ova2) * f.y[s * n + q];
  } else if (kind == 13 && side == 1) {  // I3 inflow at x-right (bounds.f:1688-): L1 enters
    double fornow = d * acou * bcl1;
    double b1 = 0.5 * (u - acou) * (bcl5 - fornow);
    double b2 = u * (bcl2 - bcl5 * ova2);
    double b3 = u * bcl3;
    double b4 = u * bcl4;
    const double b5 = 0.5 * (u + acou) * (bcl5 + fornow);
    fornow = b5 + d * acou * 0.0;
    b1 = fornow - b1;
    b2 = -0.0 - ova2 * (b5 + fornow) - b2;
    b3 = -0.0 - b3;
    b4 = -0.0 - b4;
    double ce = -b1 * (ova2 * e - u / acou + ovgm) - b2 * e - b3 * d * v - b4 * d * w;
    for (int s = 0; s < nspec; ++s) {
      const double bcly = f.wdot[s * n + q] / d - 0.0 - u * dd<0>(g, zd, f.y + s * n, i, j, k);
      ce = ce - bcly * d * hprime(s);
    }
    corr[4 * (int64_t)nyz] = ce;
  } else if (kind == 21 && side == 0) {  // O1 outflow at x-left (bounds.f:213-372): L5 relaxed
    double sorp = 0.0;
    for (int s = 0; s < nspec; ++s) sorp = sorp + hprime(s) * f.wdot[s * n + q];
    sorp = -sorp * gam1;
    const double tt5 = t51b + t52b * (gam1 + 1.0) + d * acou * t2b;
    double b2 = u * (bcl2 - bcl5 * ova2);
    double b3 = u * bcl3;
    double b4 = u * bcl4;
    double b5 = 0.5 * (u + acou) * (bcl5 + d * acou * bcl1);
    double bet = bc.bet;
    if (bc.betloc == 1) bet = sqrt(u * u + v * v + w * w) / acou;
    const bool pio = u > 0.0 && bc.pio == 1;
    if (pio) {
      b2 = -b2 - ova2 * sorp;
      b3 = (double)0.1f * (v - 0.0) - b3;
      b4 = (double)0.1f * (w - 0.0) - b4;
      b5 = 0.5 * sorp + bc.cobc * acou * (p - bc.p_inf) + 0.5 * (1.0 - bet) * tt5 - b5 +
           100.0 * d * (1.0 / bc.xlen) * (pow(acou, 2.0) - pow(u, 2.0)) * (u - 0.0);
      corr[0] = -b2 - b5 * ova2;
      corr[(int64_t)nyz] = -b2 * u - b5 * ova2 * (u + acou);
      corr[2 * (int64_t)nyz] = -b2 * v - b3 * d - b5 * ova2 * v;
      corr[3 * (int64_t)nyz] = -b2 * w - b4 * d - b5 * ova2 * w;
      double ce = -b2 * e - b3 * d * v - b4 * d * w - b5 * (ova2 * e + u / acou + ovgm);
      for (int s = 0; s < nspec; ++s) {
        const double fn = dd<0>(g, zd, f.y + s * n, i, j, k) * d;
        ce = ce - fn * hprime(s);
        corr[(int64_t)(5 + s) * nyz] = -(b2 + b5 * ova2) * f.y[s * n + q] - fn;
      }
      corr[4 * (int64_t)nyz] = ce;
    } else {
      b5 = 0.5 * sorp + bc.cobc * acou * (p - bc.p_inf) + 0.5 * (1.0 - bet) * tt5 - b5;
      corr[0] = -b5 * ova2;
      corr[(int64_t)nyz] = -b5 * ova2 * (u + acou);
      corr[2 * (int64_t)nyz] = -b5 * ova2 * v;
      corr[3 * (int64_t)nyz] = -b5 * ova2 * w;
      corr[4 * (int64_t)nyz] = -b5 * (ova2 * e + u / acou + ovgm);
      for (int s = 0; s < nspec; ++s) corr[(int64_t)(5 + s) * nyz] = -b5 * ova2 * f.y[s * n + q];
    }
  } else if (kind == 13) {  // I3 inflow at x-left: rho and Y constant (DDDT = DYDT = 0)
    // DUDT, DVDT, DWDT: zero for a constant u_in; the synthetic inflow's
    // (bcutxl.f:501-506, VFAC = 1, DVFDT = 0)
    const bool syn = bc.uinf2 != nullptr;
    const double dudt = syn ? (bc.uinf2[jk] - bc.uinf1[jk]) / bc.tstep * 1.0 + (bc.u_in * 1.0 + bc.uinf2[jk]) * 0.0 : 0.0;
    const double dvdt = syn ? (bc.vinf2[jk] - bc.vinf1[jk]) / bc.tstep * 1.0 + bc.vinf2[jk] * 0.0 : 0.0;
    const double dwdt = syn ? (bc.winf2[jk] - bc.winf1[jk]) / bc.tstep * 1.0 + bc.winf2[jk] * 0.0 : 0.0;
    double fornow = d * acou * bcl1;
    const double b1 = 0.5 * (u - acou) * (bcl5 - fornow);
    double b2 = u * (bcl2 - bcl5 * ova2);
    double b3 = u * bcl3;
    double b4 = u * bcl4;
    double b5 = 0.5 * (u + acou) * (bcl5 + fornow);
    fornow = b1 - d * acou * dudt;
    b2 = -0.0 - ova2 * (b1 + fornow) - b2;
    b3 = -dvdt - b3;
    b4 = -dwdt - b4;
    b5 = fornow - b5;
    double ce = -b2 * e - b3 * d * v - b4 * d * w - b5 * (ova2 * e + u / acou + ovgm);
    for (int s = 0; s < nspec; ++s) {
      const double bcly = f.wdot[s * n + q] / d - 0.0 - u * dd<0>(g, zd, f.y + s * n, i, j, k);
      ce = ce - bcly * d * hprime(s);
    }
    corr[4 * (int64_t)nyz] = ce;
  } else {  // O1 outflow at x-right
    double sorp = 0.0;
    for (int s = 0; s < nspec; ++s) sorp = sorp + hprime(s) * f.wdot[s * n + q];
    sorp = -sorp * gam1;
    const double tt1 = t51b + t52b * (gam1 + 1.0) - d * acou * t2b;
    double b2 = u * (bcl2 - ova2 * bcl5);
    double b3 = u * bcl3;
    double b4 = u * bcl4;
    double b1 = 0.5 * (u - acou) * (bcl5 - d * acou * bcl1);
    double bet = bc.bet;
    if (bc.betloc == 1) bet = sqrt(u * u + v * v + w * w) / acou;
    const bool pio = u < 0.0 && bc.pio == 1;
    if (pio) {
      b2 = -ova2 * sorp - b2;
      b3 = (double)0.1f * (v - 0.0) - b3;
      b4 = (double)0.1f * (w - 0.0) - b4;
      b1 = 0.5 * sorp + bc.cobc * acou * (p - bc.p_inf) + 0.5 * (1.0 - bet) * tt1 - b1 -
           100.0 * d * (1.0 / bc.xlen) * (pow(acou, 2.0) - pow(u, 2.0)) * (u - 0.0);
      corr[0] = -b1 * ova2 - b2;
      corr[(int64_t)nyz] = -b1 * ova2 * (u - acou) - b2 * u;
      corr[2 * (int64_t)nyz] = -b1 * ova2 * v - b2 * v - b3 * d;
      corr[3 * (int64_t)nyz] = -b1 * ova2 * w - b2 * w - b4 * d;
      double ce = -b1 * (ova2 * e - u / acou + ovgm) - b2 * e - b3 * d * v - b4 * d * w;
      for (int s = 0; s < nspec; ++s) {
        const double fn = dd<0>(g, zd, f.y + s * n, i, j, k) * d;
        ce = ce - fn * hprime(s);
        corr[(int64_t)(5 + s) * nyz] = -(b2 + b1 * ova2) * f.y[s * n + q] - fn;
      }
      corr[4 * (int64_t)nyz] = ce;
    } else {
      b1 = 0.5 * sorp + bc.cobc * acou * (p - bc.p_inf) + 0.5 * (1.0 - bet) * tt1 - b1;
      corr[0] = -b1 * ova2;
      corr[(int64_t)nyz] = -b1 * ova2 * (u - acou);
      corr[2 * (int64_t)nyz] = -b1 * ova2 * v;
      corr[3 * (int64_t)nyz] = -b1 * ova2 * w;
      corr[4 * (int64_t)nyz] = -b1 * (ova2 * e - u / acou + ovgm);
      for (int s = 0; s < nspec; ++s) corr[(int64_t)(5 + s) * nyz] = -b1 * ova2 * f.y[s * n + q];
    }
  }
}

// W1 wall diffusion flux (rhscal.f:1698-1760, base transport): the one-sided
// fourth-order x derivative at the wall of rho D_k dY_k/dx over the wall and
// the four planes inward, added to species k's rate and to VTMP (its energy
// part is dropped: BOUNDS zeroes the wall's energy RHS).
__global__ void __launch_bounds__(kFaceBlock) k_wall_flux(Geo g, Fields f, NscbcParams bc, int nspec) {
  const int jk = blockIdx.x * kFaceBlock + threadIdx.x;
  const int side = blockIdx.y;
  const int kind = side == 0 ? bc.xl : bc.xr;
  if (jk >= g.ny * g.nz || (kind != 31 && kind != 32)) return;
  const int j = jk % g.ny, k = jk / g.ny;
  const int i = side == 0 ? 0 : g.nx - 1, st = side == 0 ? 1 : -1;
  const int64_t n = g.n, q = (int64_t)i + (int64_t)g.nx * jk;
  const double c0 = (double)(25.0f / 12.0f), c3 = (double)(4.0f / 3.0f);  // single-precision literals as coded
  double vt = f.vtmp[q];
  for (int s = 0; s < nspec; ++s) {
    double fv[5];
#pragma unroll
    for (int m = 0; m < 5; ++m)
      fv[m] = f.rd[s * n + q + m * st] * dd<0>(g, ZDec{}, f.y + s * n, i + m * st, j, k);  // x only: own slab
    const double w = side == 0 ? ((-c0) * fv[0] + 4.0 * fv[1] - 3.0 * fv[2] + c3 * fv[3] - 0.25 * fv[4]) * g.ovd[0]
                               : (c0 * fv[0] - 4.0 * fv[1] + 3.0 * fv[2] - c3 * fv[3] + 0.25 * fv[4]) * g.ovd[0];
    f.wdot[s * n + q] = f.wdot[s * n + q] + w;
    vt = vt + w;
  }
  f.vtmp[q] = vt;
}

// After the RK update at a W1 wall: the wall temperature re-extrapolated
// from this substage's TEMPER (bounds.f:925-933; not at a W2 wall) and, at
// either wall when rk, every mass
// fraction of the updated U register extrapolated with zero normal gradient,
// Y_w = (12/25)(4 Y_1 - 3 Y_2 + (4/3) Y_3 - Y_4/4), clipped to [0, 1], times
// the wall density, into both registers (lincom.f:171-210, fincom.f:171-210).
__global__ void __launch_bounds__(kFaceBlock) k_wall_fix(Geo g, Fields f, NscbcParams bc, int nspec, int rk) {
  const int jk = blockIdx.x * kFaceBlock + threadIdx.x;
  const int side = blockIdx.y;
  const int kind = side == 0 ? bc.xl : bc.xr;
  if (jk >= g.ny * g.nz || (kind != 31 && kind != 32)) return;
  const int st = side == 0 ? 1 : -1;
  const int64_t n = g.n, q = (side == 0 ? 0 : g.nx - 1) + (int64_t)g.nx * jk;
  if (kind == 31) f.t[q] = wall_t(f.t, q, st);
  if (!rk) return;
  const double* U = f.uout;
  const double c1 = (double)(12.0f / 25.0f), c3 = (double)(4.0f / 3.0f);
  for (int s = 0; s < nspec; ++s) {
    const double* y = U + (5 + s) * n;
    const double t1 = y[q + st] / U[q + st], t2 = y[q + 2 * st] / U[q + 2 * st];
    const double t3 = y[q + 3 * st] / U[q + 3 * st], t4 = y[q + 4 * st] / U[q + 4 * st];
    double yw = c1 * (4.0 * t1 - 3.0 * t2 + c3 * t3 - (0.25 * t4));
    yw = fmin(1.0, yw);
    yw = fmax(0.0, yw);
    yw = U[q] * yw;
    f.run[(5 + s) * n + q] = yw;
    f.uout[(5 + s) * n + q] = yw;
  }
}

}  // namespace

bool has_wall(const NscbcParams& bc) { return bc.xl == 31 || bc.xr == 31 || bc.xl == 32 || bc.xr == 32; }

void launch_boundt(const Geo& g, const Fields& f, const NscbcParams& bc, int nspec, bool both,
                   const senga_chem* dchem, cudaStream_t s) {
  auto imposed = [](int k) { return k == 12 || k == 13 || k == 31 || k == 32; };
  if (!imposed(bc.xl) && !imposed(bc.xr)) return;
  const int nyz = g.ny * g.nz;
  k_boundt<<<dim3((nyz + kFaceBlock - 1) / kFaceBlock, 2), kFaceBlock, 0, s>>>(g, f, bc, nspec, both ? 1 : 0, dchem);
}

void launch_wall_flux(const Geo& g, const Fields& f, const NscbcParams& bc, int nspec, cudaStream_t s) {
  if (!has_wall(bc)) return;
  const int nyz = g.ny * g.nz;
  k_wall_flux<<<dim3((nyz + kFaceBlock - 1) / kFaceBlock, 2), kFaceBlock, 0, s>>>(g, f, bc, nspec);
}

void launch_wall_fix(const Geo& g, const Fields& f, const NscbcParams& bc, int nspec, bool rk, cudaStream_t s) {
  if (!has_wall(bc)) return;
  const int nyz = g.ny * g.nz;
  k_wall_fix<<<dim3((nyz + kFaceBlock - 1) / kFaceBlock, 2), kFaceBlock, 0, s>>>(g, f, bc, nspec, rk ? 1 : 0);
}

void launch_face(const Geo& g, const Fields& f, const NscbcParams& bc, int nspec, const senga_chem* dchem,
                 cudaStream_t s, const ZDec& zd) {
  const int nyz = g.ny * g.nz;
  k_face<<<dim3((nyz + kFaceBlock - 1) / kFaceBlock, 2), kFaceBlock, 0, s>>>(g, f, bc, nspec, dchem, zd);
}

}  // namespace senga
