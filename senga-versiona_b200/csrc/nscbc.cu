// Navier-Stokes characteristic boundary conditions on the x faces.
//
// Restated from the reference (I3 subsonic inflow with constant velocity,
// NXxPRM(1)=1, I2 subsonic reflecting inflow with specified temperature,
// and O1 partially non-reflecting outflow, on either x face; inflow on one
// face at most; both O1 faces take the same parameters):
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
// Every face quantity is a pointwise value or a derivative at the face plane,
// so one thread per face point computes them from the thermochemistry
// kernel's outputs and the U register right after that kernel (before the
// species kernel overwrites the chemistry rate), folds BOUNDS into one
// additive correction per conserved field, and the fused RK epilogue adds it
// on the face planes (face_bits BF_NSCBC). This is O(ny*nz) work.
#include <cuda_runtime.h>

#include "senga_internal.h"
#include "stencil.cuh"

namespace senga {
namespace {

constexpr int kFaceBlock = 128;

// value m points along DIR from (i, j, k); y and z periodic, x bounded (the
// closures read only inward points)
template <int DIR>
__device__ __forceinline__ double at(const Geo& g, const double* a, int i, int j, int k, int m) {
  if (DIR == 0) i += m;
  if (DIR == 1) j = ((j + m) % g.ny + g.ny) % g.ny;
  if (DIR == 2) k = ((k + m) % g.nz + g.nz) % g.nz;
  return a[(int64_t)i + (int64_t)g.nx * (j + (int64_t)g.ny * k)];
}
template <int DIR>
__device__ __forceinline__ double dd(const Geo& g, const double* a, int i, int j, int k) {
  const int c = DIR == 0 ? i : DIR == 1 ? j : k;
  const int n = DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
  return d1core([&](int m) { return at<DIR>(g, a, i, j, k, m); }, c, n, g.per[DIR]) * g.ovd[DIR];
}
// derivative of (a - c) along DIR: the pressure gradient of RHSVEL is taken of
// p - p(1,1,1) (src/rhsvel.f:730-752)
template <int DIR>
__device__ __forceinline__ double dd_sub(const Geo& g, const double* a, double c0, int i, int j, int k) {
  const int c = DIR == 0 ? i : DIR == 1 ? j : k;
  const int n = DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
  return d1core([&](int m) { return at<DIR>(g, a, i, j, k, m) - c0; }, c, n, g.per[DIR]) * g.ovd[DIR];
}

__global__ void __launch_bounds__(kFaceBlock)
    k_boundt(Geo g, Fields f, NscbcParams bc, int nspec, int both, const senga_chem* chem) {
  const int jk = blockIdx.x * kFaceBlock + threadIdx.x;
  if (jk >= g.ny * g.nz) return;
  const int64_t n = g.n;
  const bool left = bc.xl == 13 || bc.xl == 12;
  const int kind = left ? bc.xl : bc.xr;
  const int i = left ? 0 : g.nx - 1;  // the inflow plane
  const int64_t q = (int64_t)i + (int64_t)g.nx * jk;
  double* regs[2] = {f.uin, f.run};
  if (kind == 12) {
    // I2 (boundt.f:81-176, bountt.f:84-200): ITNDEX of TRIN, then velocity,
    // energy and species from the face density of the U register
    const double t = bc.t_in, u = bc.u_in, v = 0.0, w = 0.0;
    int32_t itn = 0;
    for (int s = 0; s < nspec; ++s) {
      int it = 0;
      while (t > chem->tinthi[s][it] && it + 1 < chem->ntint[s]) ++it;
      itn += it << (2 * s);
    }
    f.itn[q] = itn;
    const double d = f.uin[q];
    double e = 0.5 * (u * u + v * v + w * w);
    e = d * e;
    double ys[SENGA_NSPCMX];
    for (int s = 0; s < nspec; ++s) {
      const int it = (itn >> (2 * s)) & 3;
      const double* c = chem->amasch[s][it];
      double h = c[chem->ncpoly[s][it] - 1];
      for (int icp = chem->ncpom1[s][it]; icp >= 1; --icp) h = h * t + c[icp - 1];
      h = c[chem->ncenth[s][it] - 1] + h * t;
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
  for (int w = 0; w < (both ? 2 : 1); ++w) {
    double* U = regs[w];
    U[q] = r;
    U[n + q] = r * bc.u_in;
    U[2 * n + q] = r * 0.0;
    U[3 * n + q] = r * 0.0;
    for (int s = 0; s < nspec; ++s) U[(5 + s) * n + q] = r * bc.y_in[s];
  }
  if (both && f.err) {  // BOUNTT: error of the imposed fields zeroed
    for (int fl = 0; fl < 4; ++fl) f.err[fl * n + q] = 0.0;
    for (int s = 0; s < nspec; ++s) f.err[(5 + s) * n + q] = 0.0;
  }
}

__global__ void __launch_bounds__(kFaceBlock) k_face(Geo g, Fields f, NscbcParams bc, int nspec, const senga_chem* chem) {
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
  const double pref = __ldg(f.p);
  // ---- face data ----
  const double d = U[q], u = vel[q], v = vel[n + q], w = vel[2 * n + q];
  const double p = f.p[q], t = f.t[q], rr = f.rmix[q] / d, cp = f.cp[q];
  double e = f.e[q];
  const double bcl1 = dd<0>(g, vel, i, j, k), bcl2 = dd<0>(g, U, i, j, k);
  const double bcl3 = dd<0>(g, vel + n, i, j, k), bcl4 = dd<0>(g, vel + 2 * n, i, j, k);
  const double bcl5 = dd_sub<0>(g, f.p, pref, i, j, k);
  const double t2b = -v * dd<1>(g, vel, i, j, k) - w * dd<2>(g, vel, i, j, k);
  const double py = dd_sub<1>(g, f.p, pref, i, j, k), pz = dd_sub<2>(g, f.p, pref, i, j, k);
  const double t51b = -v * py - w * pz;
  const double t52b = -p * (dd<1>(g, vel + n, i, j, k) + dd<2>(g, vel + 2 * n, i, j, k));
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
      const double bcly = f.wdot[s * n + q] / d - 0.0 - u * dd<0>(g, f.y + s * n, i, j, k);
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
        const double fn = dd<0>(g, f.y + s * n, i, j, k) * d;
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
  } else if (kind == 13) {  // I3 inflow at x-left, constant u, rho and Y (DUDT = DDDT = DYDT = 0)
    double fornow = d * acou * bcl1;
    const double b1 = 0.5 * (u - acou) * (bcl5 - fornow);
    double b2 = u * (bcl2 - bcl5 * ova2);
    double b3 = u * bcl3;
    double b4 = u * bcl4;
    double b5 = 0.5 * (u + acou) * (bcl5 + fornow);
    fornow = b1 - d * acou * 0.0;
    b2 = -0.0 - ova2 * (b1 + fornow) - b2;
    b3 = -0.0 - b3;
    b4 = -0.0 - b4;
    b5 = fornow - b5;
    double ce = -b2 * e - b3 * d * v - b4 * d * w - b5 * (ova2 * e + u / acou + ovgm);
    for (int s = 0; s < nspec; ++s) {
      const double bcly = f.wdot[s * n + q] / d - 0.0 - u * dd<0>(g, f.y + s * n, i, j, k);
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
        const double fn = dd<0>(g, f.y + s * n, i, j, k) * d;
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

}  // namespace

void launch_boundt(const Geo& g, const Fields& f, const NscbcParams& bc, int nspec, bool both,
                   const senga_chem* dchem, cudaStream_t s) {
  if (bc.xl != 13 && bc.xr != 13 && bc.xl != 12 && bc.xr != 12) return;
  const int nyz = g.ny * g.nz;
  k_boundt<<<(nyz + kFaceBlock - 1) / kFaceBlock, kFaceBlock, 0, s>>>(g, f, bc, nspec, both ? 1 : 0, dchem);
}

void launch_face(const Geo& g, const Fields& f, const NscbcParams& bc, int nspec, const senga_chem* dchem,
                 cudaStream_t s) {
  const int nyz = g.ny * g.nz;
  k_face<<<dim3((nyz + kFaceBlock - 1) / kFaceBlock, 2), kFaceBlock, 0, s>>>(g, f, bc, nspec, dchem);
}

}  // namespace senga
