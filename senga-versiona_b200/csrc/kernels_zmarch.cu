// Species + RK update marching along z (the last kernel of a substage).
//
// Same arithmetic as k_species_rk_t (kernels_tiled.cu): the diffusion
// correction terms of the energy and species equations (src/rhscal.f:
// 3782-3938, ERHS -= h_mix div V_c + grad h_mix . V_c, YRHS = RATE -
// Y div V_c - grad Y . V_c) fused with the 2N-storage RK update of all Nc
// fields (src/lincom.f:53-169, src/fincom.f:54-168). Every field's update is
// independent of the others, so instead of holding all species of a small
// 3-D tile, a CTA owns a 32 x 8 column of the box and marches a chunk of z
// planes one field after the other (h_mix, then Y_1 .. Y_S):
//   * each plane of a field, with its x and y halos (44 x 18 points), is
//     copied into a ring of 8 shared-memory slots by the TMA engine: one
//     tensor copy (cp.async.bulk.tensor) for columns away from the periodic
//     wrap in x and y, one bulk copy per row (cut at the wrap) for the
//     others; the copy of plane t+3 is in flight while plane t is used;
//   * every thread keeps the 11 values of its own z-column in registers
//     (pushed from the ring as each plane lands), so the z derivative costs
//     no further memory access;
//   * the x and y derivatives at output plane z are read from the ring slot
//     of plane z, which is still resident when plane z+5 lands.
// A plane is read once per chunk plus a 5-plane halo on either side.
// All-periodic boxes of one context with even nx (16-byte aligned rows).
#include <cuda_runtime.h>

#include "senga_internal.h"
#include "tiles.cuh"

namespace senga {
namespace {

using namespace tile;

constexpr int ZX = 32, ZY = 8;           // CTA column (one thread per (x, y))
constexpr int ZC = 32;                   // planes per chunk
constexpr int RING = 8;                  // ring slots (6 in use, 2 in flight)
constexpr int PX = ZX + 2 * XH, PY = ZY + 2 * H, PLANE = PX * PY;
constexpr unsigned kPlaneBytes = 8u * PLANE;     // bytes one plane copy delivers
constexpr int SLOT = (PLANE + 15) / 16 * 16;     // slot stride (doubles): 128-byte aligned slots
static_assert((8 * SLOT) % 128 == 0, "ring slots start on 128-byte boundaries");

struct ZMaps {
  CUtensorMap y, hm;  // [field][z][y][x] families, box 44 x 18 x 1 x 1
};

__device__ __forceinline__ double pv(const double* pl, int x, int y) { return pl[(y + H) * PX + (x + XH)]; }

__global__ void __launch_bounds__(ZX* ZY, 3)
    k_species_rk_z(Geo g, Fields f, int nspec, RK rk, const __grid_constant__ ZMaps tm) {
  extern __shared__ __align__(128) double ring[];
  __shared__ uint64_t bars[RING];
  __shared__ int64_t oy[PY];
  const int tx = threadIdx.x % ZX, ty = threadIdx.x / ZX;
  const int x0 = blockIdx.x * ZX, y0 = blockIdx.y * ZY, z0 = blockIdx.z * ZC;
  const int zc = min(ZC, g.nz - z0);
  const int64_t n = g.n, plane = (int64_t)g.nx * g.ny;
  if (threadIdx.x < RING) mbar_init(&bars[threadIdx.x], 1);
  if (threadIdx.x < PY) oy[threadIdx.x] = (int64_t)fold(y0 + (int)threadIdx.x - H, g.ny, 1) * g.nx;
  __syncthreads();
  const bool tensor = (smem_u32(ring) & 127u) == 0 && x0 >= XH && x0 + ZX + XH <= g.nx && y0 >= H &&
                      y0 + ZY + H <= g.ny;
  const int spf = zc + 2 * H;        // planes per field
  const int total = (nspec + 1) * spf;  // h_mix, then the species

  // copy plane t of the stream (field t / spf, z = z0 - H + t % spf) into
  // ring slot t % RING
  auto issue = [&](int t) {
    const int fld = t / spf;
    const int z = fold(z0 - H + t % spf, g.nz, 1);
    double* dst = ring + (t % RING) * SLOT;
    uint64_t* bar = &bars[t % RING];
    if (tensor) {
      if (threadIdx.x == 0) {
        mbar_expect_tx(bar, kPlaneBytes);
        tma_load_4d(dst, fld == 0 ? &tm.hm : &tm.y, x0 - XH, y0 - H, z, fld == 0 ? 0 : fld - 1, bar);
      }
    } else {
      if (threadIdx.x == 0) mbar_expect_tx(bar, kPlaneBytes);
      if (threadIdx.x < PY) {
        const double* src = (fld == 0 ? f.hmix : f.y + (int64_t)(fld - 1) * n) + oy[threadIdx.x] + (int64_t)z * plane;
        double* drow = dst + threadIdx.x * PX;
        int c = x0 - XH;
        const int e = c + PX;
        int xs = c % g.nx;
        if (xs < 0) xs += g.nx;
        int off = 0;
        while (c < e) {
          const int len = min(e - c, g.nx - xs);
          bulk_g2s(drow + off, src + xs, (unsigned)len * 8u, bar);
          off += len;
          c += len;
          xs = 0;
        }
      }
    }
  };

  const int gx = x0 + tx, gy = y0 + ty;
  const bool valid = gx < g.nx && gy < g.ny;
  const int64_t qxy = (int64_t)gx + (int64_t)g.nx * gy;
  auto advance = [&](int fld, int64_t q, double R) {
    const int64_t idx = (int64_t)fld * n + q;
    if (rk.last < 0) {  // right-hand side only
      f.rhs[idx] = R;
      return;
    }
    if (f.err) f.err[idx] = f.err[idx] + rk.err * R;
    if (!rk.last) {
      const double s = f.run[idx];
      f.run[idx] = s + rk.lhs * R;
      f.uout[idx] = s + rk.rhs * R;
    } else {
      const double s = f.run[idx] + rk.lhs * R;
      f.run[idx] = s;
      f.uout[idx] = s;
    }
  };

  for (int t = 0; t < 3 && t < total; ++t) issue(t);
  double q[2 * H + 1];
#pragma unroll
  for (int k = 0; k <= 2 * H; ++k) q[k] = 0.0;
  for (int t = 0; t < total; ++t) {
    const int fld = t / spf, j = t % spf;
    const bool ok = mbar_wait(&bars[t % RING], (unsigned)(t / RING) & 1u);
#pragma unroll
    for (int k = 0; k < 2 * H; ++k) q[k] = q[k + 1];
    q[2 * H] = ok ? pv(ring + (t % RING) * SLOT, tx, ty) : 0.0;
    if (ok && j >= 2 * H && valid) {
      const int gz = z0 + j - 2 * H;  // output plane: centre of the queue
      const double* pl = ring + ((t - H) % RING) * SLOT;
      const int64_t qq = qxy + (int64_t)gz * plane;
      const double vcx = f.vc[qq], vcy = f.vc[n + qq], vcz = f.vc[2 * n + qq], vt = f.vtmp[qq];
      const double dx = d1core([&](int m) { return pv(pl, tx + m, ty); }, gx, g.nx, 1) * g.ovd[0];
      const double dy = d1core([&](int m) { return pv(pl, tx, ty + m); }, gy, g.ny, 1) * g.ovd[1];
      const double dz = d1core([&](int m) { return q[H + m]; }, gz, g.nz, 1) * g.ovd[2];
      if (fld == 0) {
        const double rE = f.rhs[4 * n + qq] - q[H] * vt - dx * vcx - dy * vcy - dz * vcz;
#pragma unroll
        for (int fl = 0; fl < 4; ++fl) advance(fl, qq, f.rhs[fl * n + qq]);
        advance(4, qq, rE);
      } else {
        const int s = fld - 1;
        const double R = f.wdot[s * n + qq] - q[H] * vt - dx * vcx - dy * vcy - dz * vcz;
        advance(5 + s, qq, R);
      }
    }
    // every thread is done with the slot of plane t - H: refill it with
    // plane t + 3 (a CTA-uniform decision on a copy that did not land)
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0 && f.status) atomicOr(f.status, kStatusStageTimeout);
      // let the copies in flight (planes t .. t+2) land before leaving
      for (int u = t; u < t + 3 && u < total; ++u) mbar_wait(&bars[u % RING], (unsigned)(u / RING) & 1u);
      return;
    }
    if (t + 3 < total) issue(t + 3);
  }
}

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encoder() {
  static EncodeTiled fn = [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &qr) != cudaSuccess ||
        qr != cudaDriverEntryPointSuccess)
      return (EncodeTiled) nullptr;
    return (EncodeTiled)ptr;
  }();
  return fn;
}
bool plane_map(CUtensorMap* m, const double* base, const Geo& g, int nk) {
  EncodeTiled enc = encoder();
  if (!enc || !base) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz, (cuuint64_t)nk};
  const cuuint64_t strides[3] = {(cuuint64_t)g.nx * 8, (cuuint64_t)g.nx * g.ny * 8, (cuuint64_t)g.n * 8};
  const cuuint32_t box[4] = {PX, PY, 1, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

// Launches the z-marching form when the box qualifies (all periodic, one
// context, even nx, 16-byte aligned fields, the encoder available); returns
// false otherwise so the caller launches the tiled form.
bool launch_species_b_rk_z(const Geo& g, const Fields& f, int nspec, const RK& rk, cudaStream_t s,
                           const ZDec& zd) {
  if (!(g.per[0] && g.per[1] && g.per[2]) || zd.nr > 1 || (g.nx & 1)) return false;
  const void* ptrs[] = {f.y, f.hmix, f.run, f.uout, f.rhs, f.wdot, f.vc, f.vtmp};
  for (const void* p : ptrs)
    if (p && ((uintptr_t)p & 15u)) return false;
  ZMaps tm{};
  if (!plane_map(&tm.y, f.y, g, nspec) || !plane_map(&tm.hm, f.hmix, g, 1)) return false;
  static bool attr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  if (!attr[dev]) {
    cudaFuncSetAttribute(k_species_rk_z, cudaFuncAttributeMaxDynamicSharedMemorySize, RING * SLOT * 8);
    attr[dev] = true;
  }
  const dim3 grid((unsigned)((g.nx + ZX - 1) / ZX), (unsigned)((g.ny + ZY - 1) / ZY), (unsigned)((g.nz + ZC - 1) / ZC));
  k_species_rk_z<<<grid, ZX * ZY, RING * SLOT * 8, s>>>(g, f, nspec, rk, tm);
  return true;
}

}  // namespace senga
