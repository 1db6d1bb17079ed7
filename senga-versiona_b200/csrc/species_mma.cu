// Species pass of the substage (the terms of species_tile: species
// convection, diffusion, correction velocity and the species enthalpy fluxes
// of the energy equation, src/rhscal.f:1030-1955) for all-periodic boxes, with
// the x derivatives on the FP64 tensor cores.
//
// A CTA covers an 8x8x8 tile. Warp w is the tile's y row w; lane l holds the
// two grid points (x = l/4, y = w, z = 2(l%4) + b), b = 0, 1, which are the row
// and the two columns of its accumulator fragment in an m8n8k4 FP64 mma
// (rows x, columns z).
//
// x derivatives: the interior first and second derivative operators along x
// (src/dfbydx.f:67-105, src/d2fdx2.f:96-111) are band matrices of 8 outputs by
// 20 staged inputs (x0-6 .. x0+13). D F for a staged field F is five mma
// k-steps, A = the band (per lane, from a small shared table) and B = F's
// values (4 x by 8 z). Every column of B is shifted by its value at x0+4
// first: the band's rows sum to zero, so the shift leaves D F unchanged and
// keeps the products of the sum small (the reference forms differences first).
// y and z derivatives are the stencils evaluated per point from shared memory
// in the reference's association; a lane's two points are z neighbours and
// share one 12-plane z window. Within a term the x, y and z parts are summed
// in the reference's order; the convective and Laplacian sums add their x and
// z parts before the y part (FP64 rounding differences only).
//
// Staging (cp.async, 16 bytes): per field, one buffer of 18 planes z0-5 ..
// z0+12 (stride 164 doubles, rows of 20 doubles: the in-tile planes with
// their x halos, the z-halo planes at in-tile x only) followed by the y-halo
// rows [8 z][10][8] (plane stride 164 as well). Fields go through three such
// buffers in turn (Y_k, rho D_k, h_k, Y_k+1, ...): the next two fields are
// copied while this one is used, one barrier per field, one CTA per SM (252
// registers a thread, no spills). rho v ([8 z][18 y][8], plane
// 148), rho w ([18 z][8 y][8], plane 68) and rho u (the in-tile planes of a
// field buffer) are staged once per tile. The plane strides put the 32 doubles
// of every warp-wide read below on distinct bank pairs (two wavefronts).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <string>

#include "senga_internal.h"
#include "stencil.cuh"
#include "tiles.cuh"

namespace senga {
namespace {

constexpr int MX = 8, MY = 8, MZ = 8;
constexpr int MH = 5;                        // stencil half width
constexpr int RW = MX + 12;                  // staged x row: x0-6 .. x0+13
constexpr int PS = MY * RW + 4;              // plane stride of a field buffer
constexpr int NPL = MZ + 2 * MH;             // planes z0-5 .. z0+12
constexpr int YHOFF = NPL * PS;              // y-halo rows [z][10][MX] after the planes
constexpr int FBUF = YHOFF + MZ * PS;        // one field buffer
constexpr int VPS = (MY + 2 * MH) * MX + 4;  // rho v: [z][y0-5 .. y0+12][x]
constexpr int VBUF = MZ * VPS;
constexpr int WPS = MY * MX + 4;             // rho w: [z0-5 .. z0+12][y][x]
constexpr int WBUF = NPL * WPS;
constexpr int UBUF = MZ * PS;                // rho u: the in-tile planes of a field buffer
constexpr int BTAB = 5 * 32;                 // one band's A operands: [k-step][lane]
constexpr int NB = 3;                        // field buffers: two fields in flight
constexpr int kMmaSmem = NB * FBUF + VBUF + WBUF + UBUF + 2 * BTAB;  // doubles
static_assert(MH == tile::H, "one stencil half width");
static_assert(MY == MZ, "y and z halos share one row mapping");
static_assert(PS % 16 == 4, "B operands: 8 planes x 4 doubles on distinct banks");
static_assert((2 * PS) % 16 == 8 && (2 * VPS) % 16 == 8 && (2 * WPS) % 16 == 8,
              "windows: 4 planes two apart x 8 doubles on distinct banks");
static_assert(PS % 2 == 0 && RW % 2 == 0 && FBUF % 2 == 0 && VPS % 2 == 0 && WPS % 2 == 0 && VBUF % 2 == 0 &&
                  WBUF % 2 == 0 && UBUF % 2 == 0,
              "16-byte copies need even offsets");
static_assert(8 * kMmaSmem <= 227 * 1024, "one CTA per SM");

__device__ __forceinline__ void cp16(double* dst, const double* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(tile::smem_u32(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ int wrap(int c, int n) { return c < 0 ? c + n : (c >= n ? c - n : c); }

// d += A B for one m8n8k4 FP64 fragment (A: row l/4, column l%4; B: row l%4,
// column l/4; d: row l/4, columns 2(l%4), 2(l%4)+1)
__device__ __forceinline__ void mma8(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

// band coefficients at offset j (input minus output), unscaled
__device__ __forceinline__ double band1(int j) {
  using namespace fdc;
  const int a = j < 0 ? -j : j;
  const double c = a == 1 ? a1 : a == 2 ? b1 : a == 3 ? c1 : a == 4 ? d1 : a == 5 ? e1 : 0.0;
  return j < 0 ? -c : c;
}
__device__ __forceinline__ double band2(int j) {
  using namespace fdc;
  const int a = j < 0 ? -j : j;
  return a == 0 ? -2.0 * (a2 + b2 + c2 + d2 + e2)
                : a == 1 ? a2 : a == 2 ? b2 : a == 3 ? c2 : a == 4 ? d2 : a == 5 ? e2 : 0.0;
}

__global__ void __launch_bounds__(256, 1) k_species_mma(Geo g, Fields f, int nspec) {
  extern __shared__ __align__(128) double sm[];
  double* const sv = sm + NB * FBUF;
  double* const sw = sv + VBUF;
  double* const su = sw + WBUF;
  double* const a1t = su + UBUF;
  double* const a2t = a1t + BTAB;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, gx = lane >> 2, qz = lane & 3;
  const int x0 = blockIdx.x * MX, y0 = blockIdx.y * MY, z0 = blockIdx.z * MZ;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int64_t nxy = (int64_t)nx * ny, n = g.n;

  // one field (a species slice) into a buffer: warp w copies the in-tile
  // rows of y row w, the z-halo rows of y row w and the y-halo rows of plane w
  auto stage = [&](double* dst, const double* src) {
    {
      const int r = lane / 10, c = lane - 10 * r;
      const double* s = src + wrap(x0 - 6 + 2 * c, nx) + (int64_t)(y0 + w) * nx + (int64_t)z0 * nxy;
      double* d = dst + MH * PS + w * RW + 2 * c;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const int z = 3 * j + r;
        if (r < 3 && z < MZ) cp16(d + z * PS, s + (int64_t)z * nxy);
      }
    }
    const int rr = lane >> 2, c = lane & 3;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int hr = 8 * j + rr;
      if (hr < 2 * MH) {
        const int dh = hr < MH ? hr - MH : hr + MZ - MH;  // -5..-1, 8..12
        cp16(dst + (dh + MH) * PS + w * RW + 6 + 2 * c,
             src + x0 + 2 * c + (int64_t)(y0 + w) * nx + (int64_t)wrap(z0 + dh, nz) * nxy);
        cp16(dst + YHOFF + w * PS + hr * MX + 2 * c,
             src + x0 + 2 * c + (int64_t)wrap(y0 + dh, ny) * nx + (int64_t)(z0 + w) * nxy);
      }
    }
  };
  // rho u (in-tile rows of y row w), rho v (y rows of plane w) and rho w (z
  // rows of y row w), once per tile
  {
    const int r = lane / 10, c = lane - 10 * r;
    const double* s = f.uin + n + wrap(x0 - 6 + 2 * c, nx) + (int64_t)(y0 + w) * nx + (int64_t)z0 * nxy;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int z = 3 * j + r;
      if (r < 3 && z < MZ) cp16(su + z * PS + w * RW + 2 * c, s + (int64_t)z * nxy);
    }
  }
  {
    const int rr = lane >> 2, c = lane & 3;
    const double* rv = f.uin + 2 * n;
    const double* rw = f.uin + 3 * n;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const int k = 8 * j + rr;
      if (k < MY + 2 * MH) {
        cp16(sv + w * VPS + k * MX + 2 * c,
             rv + x0 + 2 * c + (int64_t)wrap(y0 + k - MH, ny) * nx + (int64_t)(z0 + w) * nxy);
        cp16(sw + k * WPS + w * MX + 2 * c,
             rw + x0 + 2 * c + (int64_t)(y0 + w) * nx + (int64_t)wrap(z0 + k - MH, nz) * nxy);
      }
    }
  }
  // groups: G0 = rho u, v, w and Y_0; G1 = rho D_0; then one per field
  auto field_src = [&](int k) -> const double* {
    const int s3 = k / 3, r3 = k - 3 * s3;
    const double* base = r3 == 0 ? f.y : r3 == 1 ? f.rd : f.h;
    return base + (int64_t)s3 * n;
  };
  const int nfield = 3 * nspec;
  if (nfield > 0) stage(sm, f.y);
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  if (nfield > 1) stage(sm + FBUF, f.rd);
  asm volatile("cp.async.commit_group;\n" ::: "memory");

  // A operands: the bands' rows x = gx, columns 4kk + qz of the staged row
  if (threadIdx.x < BTAB) {
    const int kk = threadIdx.x >> 5;
    a1t[threadIdx.x] = band1(4 * kk + qz - gx - 6);
    a2t[threadIdx.x] = band2(4 * kk + qz - gx - 6);
  }
  int64_t qp[2];
  double vcx[2], vcy[2], vcz[2], vt[2], rE[2];
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    qp[b] = (int64_t)(x0 + gx) + (int64_t)(y0 + w) * nx + (int64_t)(z0 + 2 * qz + b) * nxy;
    rE[b] = f.rhs[4 * n + qp[b]];
    vcx[b] = vcy[b] = vcz[b] = vt[b] = 0.0;
  }
  const double ox = g.ovd[0], oy = g.ovd[1], oz = g.ovd[2];
  const double ox2 = g.ovd2[0], oy2 = g.ovd2[1], oz2 = g.ovd2[2];
  const int src_lane = (gx << 2) | 2;  // holds the B column's value at staged x 10

  // B operands of a buffer's field: rows 4kk + qz of plane gx, y row w
  auto bops = [&](const double* buf, double (&bv)[5]) {
#pragma unroll
    for (int kk = 0; kk < 5; ++kk) bv[kk] = buf[(gx + MH) * PS + w * RW + 4 * kk + qz];
  };
  // y window of point b at offset m: in-tile rows from the planes, halo rows
  // from the y-halo block (w + m is warp-uniform)
  auto yidx = [&](int b, int m) {
    const int yy = w + m;
    const int lanepart = (2 * qz + b) * PS + gx;
    if (yy >= 0 && yy < MY) return lanepart + MH * PS + yy * RW + 6;
    return lanepart + YHOFF + (yy < 0 ? yy + MH : yy - MY + MH) * MX;
  };
  auto zidx = [&](int mm) { return (2 * qz + mm) * PS + w * RW + gx + 6; };
  // scaled first z derivatives and the values of a buffer's field at the
  // lane's two points
  auto zpass = [&](const double* buf, double (&d)[2], double (&c)[2]) {
    double zv[12];
#pragma unroll
    for (int mm = 0; mm < 12; ++mm) zv[mm] = buf[zidx(mm)];
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      d[b] = d1core([&](int m) { return zv[b + MH + m]; }, 0, 1, 1) * oz;
      c[b] = zv[b + MH];
    }
  };
  // scaled first y derivative at point b
  auto ypass = [&](const double* buf, int b) {
    double yv[11];
#pragma unroll
    for (int m = -MH; m <= MH; ++m) yv[m + MH] = m == 0 ? 0.0 : buf[yidx(b, m)];
    return d1core([&](int m) { return yv[m + MH]; }, 0, 1, 1) * oy;
  };
  // first x derivative (scaled) of a buffer's field at the lane's two points
  auto xpass = [&](const double* buf, double (&e)[2]) {
    double bv[5];
    bops(buf, bv);
    const double r0 = __shfl_sync(0xffffffffu, bv[2], src_lane);
    e[0] = e[1] = 0.0;
#pragma unroll
    for (int kk = 0; kk < 5; ++kk) mma8(e, a1t[kk * 32 + lane], bv[kk] - r0);
    e[0] *= ox;
    e[1] *= ox;
  };

  // field fi has landed (its group and all earlier ones complete; the group
  // of fi+1 may still be in flight) and every thread is done with field
  // fi-1, whose buffer then takes field fi+2
  auto next_field = [&](int k) {
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    __syncthreads();
    if (k + 2 < nfield) stage(sm + ((k + 2) % NB) * FBUF, field_src(k + 2));
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  int fi = 0;  // fields consumed so far: buffer fi & 1 holds the current one
  for (int s = 0; s < nspec; ++s) {
    double yx[2], yy[2], yz[2], lap[2], rate[2], rdc[2], fn1[2];
    // ---- Y_s: convection, gradient, Laplacian ----
    {
      const double* cur = sm + (fi % NB) * FBUF;
      next_field(fi);
      double by[5], bf[5];
      bops(cur, by);
#pragma unroll
      for (int kk = 0; kk < 5; ++kk) bf[kk] = by[kk] * su[gx * PS + w * RW + 4 * kk + qz];
      const double ry = __shfl_sync(0xffffffffu, by[2], src_lane);
      const double rf = __shfl_sync(0xffffffffu, bf[2], src_lane);
      double e1[2] = {0.0, 0.0}, e2[2] = {0.0, 0.0}, ef[2] = {0.0, 0.0};
#pragma unroll
      for (int kk = 0; kk < 5; ++kk) {
        const double v = by[kk] - ry;
        mma8(e1, a1t[kk * 32 + lane], v);
        mma8(e2, a2t[kk * 32 + lane], v);
        mma8(ef, a1t[kk * 32 + lane], bf[kk] - rf);
      }
      // x and z parts of every term first (the lane's two points share one z
      // window), then each point's y window
      double fxz[2], cxz[2];
      {
        double zv[12], wv[12];
#pragma unroll
        for (int mm = 0; mm < 12; ++mm) {
          zv[mm] = cur[zidx(mm)];
          wv[mm] = sw[(2 * qz + mm) * WPS + w * MX + gx];
        }
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          yx[b] = e1[b] * ox;
          yz[b] = d1core([&](int m) { return zv[b + MH + m]; }, 0, 1, 1) * oz;
          const double r = f.wdot[(int64_t)s * n + qp[b]];
          rate[b] = r - 0.5 * zv[b + MH] * __ldg(f.divm + qp[b]);
          fxz[b] = ef[b] * ox + d1core([&](int m) { return zv[b + MH + m] * wv[b + MH + m]; }, 0, 1, 1) * oz;
          cxz[b] = yx[b] * su[(2 * qz + b) * PS + w * RW + gx + 6] + yz[b] * wv[b + MH];
          lap[b] = e2[b] * ox2 + d2core([&](int m) { return zv[b + MH + m]; }, 0, 1, 1) * oz2;
        }
      }
#pragma unroll
      for (int b = 0; b < 2; ++b) {

        double yv[11], vv[11];
#pragma unroll
        for (int m = -MH; m <= MH; ++m) {
          yv[m + MH] = cur[yidx(b, m)];
          vv[m + MH] = sv[(2 * qz + b) * VPS + (w + m + MH) * MX + gx];
        }
        auto yvf = [&](int m) { return yv[m + MH]; };
        const double d1py = d1core([&](int m) { return yv[m + MH] * vv[m + MH]; }, 0, 1, 1) * oy;
        yy[b] = d1core(yvf, 0, 1, 1) * oy;
        rate[b] = rate[b] - 0.5 * (fxz[b] + d1py);
        rate[b] = rate[b] - 0.5 * (cxz[b] + yy[b] * vv[MH]);
        lap[b] = lap[b] + d2core(yvf, 0, 1, 1) * oy2;
      }
      ++fi;
    }
    // ---- rho D_s: correction velocity, diffusive flux divergence ----
    {
      const double* cur = sm + (fi % NB) * FBUF;
      next_field(fi);
      double ex[2], dz[2], cz[2];
      xpass(cur, ex);
      zpass(cur, dz, cz);
#pragma unroll
      for (int b = 0; b < 2; ++b) {

        const double dy = ypass(cur, b);
        const double rd = cz[b];
        rdc[b] = rd;
        vcx[b] = vcx[b] + rd * yx[b];
        vcy[b] = vcy[b] + rd * yy[b];
        vcz[b] = vcz[b] + rd * yz[b];
        const double fn = ex[b] * yx[b] + dy * yy[b] + dz[b] * yz[b];
        rate[b] = rate[b] + fn;
        vt[b] = vt[b] + fn;
        fn1[b] = fn;
        const double f3 = lap[b] * rd;
        rate[b] = rate[b] + f3;
        vt[b] = vt[b] + f3;
        lap[b] = f3;  // fn3 from here on
      }
      ++fi;
    }
    // ---- h_s: enthalpy fluxes of the energy equation ----
    {
      const double* cur = sm + (fi % NB) * FBUF;
      next_field(fi);
      double ex[2], dz[2], cz[2];
      xpass(cur, ex);
      zpass(cur, dz, cz);
#pragma unroll
      for (int b = 0; b < 2; ++b) {

        const double dy = ypass(cur, b);
        const double hk = cz[b];
        rE[b] = rE[b] + fn1[b] * hk;
        const double fn2 = ex[b] * yx[b] + dy * yy[b] + dz[b] * yz[b];
        rE[b] = rE[b] + fn2 * rdc[b];
        rE[b] = rE[b] + lap[b] * hk;
        f.wdot[(int64_t)s * n + qp[b]] = rate[b];
      }
      ++fi;
    }
  }
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    f.vc[qp[b]] = vcx[b];
    f.vc[n + qp[b]] = vcy[b];
    f.vc[2 * n + qp[b]] = vcz[b];
    f.vtmp[qp[b]] = vt[b];
    f.rhs[4 * n + qp[b]] = rE[b];
  }
}

bool al16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace

// The tensor-core species kernel serves all-periodic single-context boxes
// whose extents are multiples of 8 (every halo then wraps at most once) with
// 16-byte aligned fields, when SENGA_SPECIES_MMA=1 is set. It is opt-in: on
// the 256^3 H2 box it takes 8.35 ms per launch against 6.47 ms for the
// stencil form. Its shared-memory reads per point are fewer, but the 8^3
// tile stages 5.2 values per point per field (halos) and runs one CTA of
// 8 warps per SM, and the kernel is latency-bound there.
bool species_mma_ok(const Geo& g, const Fields& f, const ZDec& zd) {
  const char* e = getenv("SENGA_SPECIES_MMA");
  if (!e || std::string(e) != "1") return false;
  return g.per[0] && g.per[1] && g.per[2] && zd.nr == 1 && g.nx % MX == 0 && g.ny % MY == 0 &&
         g.nz % MZ == 0 && g.nx >= MX && g.ny >= MY && g.nz >= MZ && al16(f.y) && al16(f.rd) && al16(f.h) &&
         al16(f.uin);
}

void launch_species_mma(const Geo& g, const Fields& f, int nspec, cudaStream_t s) {
  static bool attr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  if (!attr[dev]) {
    cudaFuncSetAttribute(k_species_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, kMmaSmem * 8);
    attr[dev] = true;
  }
  const dim3 grid((unsigned)(g.nx / MX), (unsigned)(g.ny / MY), (unsigned)(g.nz / MZ));
  k_species_mma<<<grid, 256, kMmaSmem * 8, s>>>(g, f, nspec);
}

}  // namespace senga
