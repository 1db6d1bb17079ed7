// Shared-memory tiles for the fused stencil kernels.
//
// A CTA owns a TX x TY x TZ block of grid points; thread (tx, ty) owns the TZ
// points of one z-column. Every field a kernel differentiates is staged once
// per tile into shared memory with exactly the halo its derivatives need (5
// points, the half-width of the 11-point stencils), then all derivatives of
// that field at the tile's points are read from shared memory. Halo points of
// periodic directions are wrapped into the domain (the single-rank halo copy
// of src/parfer.f:840-873); in a bounded direction they are clamped and never
// read, because the one-sided closures only look inward.
//
// Buffer layouts (doubles; SX = TX + 2*XH, one column more than the 5-point
// halo on each side so that every row starts on a 16-byte boundary):
//   Star : slab[TZ][TY+2H][SX] + zhalo[2H][TY][TX]   first/second derivatives
//          in x, y, z (+ xy corners for the xy mixed derivative when loaded)
//   Box  : [TZ+2H][TY+2H][SX]                         all mixed derivatives
//   XRow : [TZ][TY][SX]    YRow : [TZ][TY+2H][TX]    ZCol : [TZ+2H][TY][TX]
//
// Two ways of filling them. stage(): per-element cp.async by every thread
// (any box; the default). stage_bulk(): each row is one bulk copy on the TMA
// engine (cp.async.bulk, completion counted on an mbarrier), split in two
// where a periodic x direction wraps; no LSU instruction per element. The
// bulk path needs an all-periodic box of even nx, 16-byte aligned fields and
// one context (the launcher checks), because each copy must start on a
// 16-byte boundary and be a multiple of 16 bytes long.
#pragma once
#include <cuda.h>  // CUtensorMap (the descriptor type only)

#include <cstdint>

#include "stencil.cuh"

namespace senga {
namespace tile {

constexpr int H = 5;
constexpr int XH = 6;  // x halo allocated in shared memory (5 read + 1 for alignment)

struct Origin {
  int x0, y0, z0;
};

// Fold a coordinate into the domain: periodic wrap, or clamp (bounded
// directions: the clamped halo values are never read by the closures).
__device__ __forceinline__ int fold(int c, int n, int per) {
  if (per) {
    while (c < 0) c += n;
    while (c >= n) c -= n;
    return c;
  }
  return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

// Element offsets of the tile's (halo-extended) x, y and z coordinates,
// folded into the domain once per CTA: ox[x+H], oy[y+H]*nx, oz[z+H]*nx*ny.
template <int TX, int TY, int TZ>
struct Folds {
  static constexpr int NX = TX + 2 * H, NY = TY + 2 * H, NZ = TZ + 2 * H;
  int64_t ox[NX], oy[NY], oz[NZ];
  __device__ void init(const Geo& g, const Origin& o, const ZDec& zd = ZDec{}) {
    for (int e = threadIdx.x; e < NX + NY + NZ; e += blockDim.x) {
      if (e < NX) ox[e] = fold(o.x0 + e - H, g.nx, g.per[0]);
      else if (e < NX + NY) oy[e - NX] = (int64_t)fold(o.y0 + (e - NX) - H, g.ny, g.per[1]) * g.nx;
      else oz[e - NX - NY] = zplane(g, zd, o.z0 + (e - NX - NY) - H);
    }
  }
  // element offset of local plane z: folded in this box, or for a z-split
  // box the plane of the owning slab (the whole box is periodic in z)
  __device__ static int64_t zplane(const Geo& g, const ZDec& zd, int z) {
    const int64_t plane = (int64_t)g.nx * g.ny;
    if (zd.nr <= 1) return (int64_t)fold(z, g.nz, g.per[2]) * plane;
    int zg = (zd.rank * g.nz + z) % zd.nzg;
    if (zg < 0) zg += zd.nzg;
    const int r = zg / g.nz;
    return zd.base[r] + (int64_t)(zg - r * g.nz) * plane;
  }
};

// Stage NR rows of a region (NW warps per CTA). Row r covers tile-local x in
// [XLO, XLO+XL) at tile-local (y, z) and lands at dst[d*DS + (x - XLO)], where
// rowyz(r, y, z, d) gives y, z and the destination row d. Warps take rows,
// lanes take x; rows are processed four at a time so that every thread keeps
// several global loads in flight before it writes shared memory.
// Asynchronous global -> shared copies (cp.async, 8 bytes each): a plain
// field (Ld) is staged without passing through registers, every row of a
// buffer in flight at once; tile_sync() waits for the copies of this thread
// and then for the block.
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void tile_sync() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
}
// tile_sync before bulk copies overwrite buffers that threads wrote with
// ordinary stores: every thread orders its writes before the async proxy
// (after reads alone the barrier suffices)
__device__ __forceinline__ void tile_sync_async() {
  asm volatile("cp.async.wait_all;\n fence.proxy.async.shared::cta;\n" ::: "memory");
  __syncthreads();
}
// ---- bulk copies on the TMA engine, completion on an mbarrier ----
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
// initialise, and make the initialised barrier visible to the async proxy
// (the TMA engine) before any copy can signal it
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n fence.mbarrier_init.release.cluster;\n" ::"r"(
                   smem_u32(bar)),
               "r"(count)
               : "memory");
}
// the single arrival of a phase, announcing the bytes its copies will deliver
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// prior generic-proxy accesses of shared memory by this thread are ordered
// before its later bulk copies (which write through the async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_g2s(double* dst, const double* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// One tiled tensor copy (TMA) of a 4-D box starting at coordinates
// {c0 (x, innermost), c1, c2, c3} of the tensor `map` describes, into dst
// (128-byte aligned), completion counted on bar. The map lives in the
// kernel's parameter space (a __grid_constant__ argument).
__device__ __forceinline__ void tma_load_4d(double* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
// Waits for phase `parity` of bar to complete, for at most about one second
// of SM clock; returns false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  const long long t0 = clock64();
  for (;;) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > (1ll << 31)) return false;
  }
}

// Status bit set when a stencil kernel's bulk copies did not complete in
// time (the tile's results are then not written).
constexpr unsigned kStatusStageTimeout = 8u;

// One mbarrier driving the bulk fills of a tile, phase by phase.
struct BulkBar {
  uint64_t* bar;
  unsigned parity;
  // thread 0 announces the bytes of this phase's copies (issued by any
  // threads, before or after); everyone then waits. Returns true when the
  // CTA must give up (a time-out anywhere in the CTA), uniformly.
  __device__ __forceinline__ bool wait(unsigned bytes, unsigned int* status) {
    if (threadIdx.x == 0) mbar_expect_tx(bar, bytes);
    bool ok = mbar_wait(bar, parity);
    parity ^= 1u;
    if (!ok) {
      // give the copies in flight a second bound to land before leaving
      mbar_wait(bar, parity ^ 1u);
      if (status) atomicOr(status, kStatusStageTimeout);
    }
    return __syncthreads_or(!ok) != 0;
  }
};

// Bulk copies of NR rows: row r covers global x in [x0 + XLO, x0 + XLO + XL)
// at the folded (y, z) that rowyz(r) gives and lands at dst[d*DS + (x - XLO)].
// The periodic x range is cut at every wrap; with nx, x0 + XLO and XL even
// every piece starts on an even x and has an even length, i.e. 16-byte
// aligned and a multiple of 16 bytes. Rows are spread over the CTA's threads.
template <int XL, int XLO, int NR, class FO, class RowYZ>
__device__ __forceinline__ void stage_bulk(double* dst, int DS, const FO& fo, int x0, int nx, const RowYZ& rowyz,
                                           const double* src, uint64_t* bar) {
  static_assert(XL % 2 == 0 && XLO % 2 == 0, "bulk rows must be 16-byte aligned");
  for (int r = threadIdx.x; r < NR; r += blockDim.x) {
    int y, z, d;
    rowyz(r, y, z, d);
    const double* row = src + fo.oy[y + H] + fo.oz[z + H];
    double* drow = dst + d * DS;
    int c = x0 + XLO;
    const int e = c + XL;
    int xs = c % nx;
    if (xs < 0) xs += nx;
    int off = 0;
    while (c < e) {
      const int len = min(e - c, nx - xs);
      bulk_g2s(drow + off, row + xs, (unsigned)len * 8u, bar);
      off += len;
      c += len;
      xs = 0;
    }
  }
}

template <class F>
struct PlainLoad {
  static constexpr bool value = false;
};
template <bool NC>
struct PlainLoad<LdT<NC>> {
  static constexpr bool value = true;
};

template <int XL, int XLO, int NR, int NW, class FO, class RowYZ, class F>
__device__ __forceinline__ void stage_rows(double* dst, int DS, const FO& fo, const RowYZ& rowyz, const F& f) {
  constexpr int NK = (XL + 31) / 32;
  constexpr int ITER = (NR + NW - 1) / NW;
  constexpr int UB = 4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t gx[NK];
#pragma unroll
  for (int k = 0; k < NK; ++k) gx[k] = (lane + 32 * k < XL) ? fo.ox[XLO + H + lane + 32 * k] : 0;
  if constexpr (PlainLoad<F>::value) {
#pragma unroll 2
    for (int i = 0; i < ITER; ++i) {
      const int r = warp + i * NW;
      if (r < NR) {
        int y, z, d;
        rowyz(r, y, z, d);
        const int64_t base = fo.oy[y + H] + fo.oz[z + H];
#pragma unroll
        for (int k = 0; k < NK; ++k)
          if (lane + 32 * k < XL) cp_async8(dst + d * DS + lane + 32 * k, f.a + base + gx[k]);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    return;
  }
#pragma unroll 1
  for (int i0 = 0; i0 < ITER; i0 += UB) {
    double val[UB][NK];
    int drow[UB];
#pragma unroll
    for (int u = 0; u < UB; ++u) {
      const int r = warp + (i0 + u) * NW;
      drow[u] = -1;
      if (i0 + u < ITER && r < NR) {
        int y, z;
        rowyz(r, y, z, drow[u]);
        const int64_t base = fo.oy[y + H] + fo.oz[z + H];
#pragma unroll
        for (int k = 0; k < NK; ++k)
          if (lane + 32 * k < XL) val[u][k] = f(base + gx[k]);
      }
    }
#pragma unroll
    for (int u = 0; u < UB; ++u)
      if (drow[u] >= 0) {
#pragma unroll
        for (int k = 0; k < NK; ++k)
          if (lane + 32 * k < XL) dst[drow[u] * DS + lane + 32 * k] = val[u][k];
      }
  }
}

// As stage_rows (register path), for three buffers of the same layout filled
// from one pass: f(q, v0, v1, v2) forms the three values of point q, so
// products that share a factor load it once and every round of loads fills
// three buffers.
template <int XL, int XLO, int NR, int NW, int UB, class FO, class RowYZ, class F>
__device__ __forceinline__ void stage_rows3(double* d0, double* d1, double* d2, int DS, const FO& fo,
                                            const RowYZ& rowyz, const F& f) {
  constexpr int NK = (XL + 31) / 32;
  constexpr int ITER = (NR + NW - 1) / NW;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t gx[NK];
#pragma unroll
  for (int k = 0; k < NK; ++k) gx[k] = (lane + 32 * k < XL) ? fo.ox[XLO + H + lane + 32 * k] : 0;
#pragma unroll 1
  for (int i0 = 0; i0 < ITER; i0 += UB) {
    double v[UB][NK][3];
    int drow[UB];
#pragma unroll
    for (int u = 0; u < UB; ++u) {
      const int r = warp + (i0 + u) * NW;
      drow[u] = -1;
      if (i0 + u < ITER && r < NR) {
        int y, z;
        rowyz(r, y, z, drow[u]);
        const int64_t base = fo.oy[y + H] + fo.oz[z + H];
#pragma unroll
        for (int k = 0; k < NK; ++k)
          if (lane + 32 * k < XL) f(base + gx[k], v[u][k][0], v[u][k][1], v[u][k][2]);
      }
    }
#pragma unroll
    for (int u = 0; u < UB; ++u)
      if (drow[u] >= 0) {
#pragma unroll
        for (int k = 0; k < NK; ++k)
          if (lane + 32 * k < XL) {
            const int e = drow[u] * DS + lane + 32 * k;
            d0[e] = v[u][k][0];
            d1[e] = v[u][k][1];
            d2[e] = v[u][k][2];
          }
      }
  }
}

template <int TX, int TY, int TZ>
struct Star {
  static constexpr int SX = TX + 2 * XH, SY = TY + 2 * H;
  static constexpr int SLAB = TZ * SY * SX;
  static constexpr int SIZE = SLAB + 2 * H * TY * TX;
  double* p;
  __device__ __forceinline__ double v(int x, int y, int z) const {
    if (z >= 0 && z < TZ) return p[(z * SY + (y + H)) * SX + (x + XH)];
    const int zz = z < 0 ? z + H : z - TZ + H;
    return p[SLAB + (zz * TY + y) * TX + x];
  }
  // XYC: also load the xy corners (only the xy mixed derivative reads them)
  template <int NW, bool XYC = false, class F>
  __device__ void stage(const Folds<TX, TY, TZ>& fo, const F& f) const {
    // in-tile rows of every in-tile plane, with the x halos
    stage_rows<TX + 2 * H, -H, TY * TZ, NW>(p + (XH - H), SX, fo,
                                            [](int r, int& y, int& z, int& d) {
                                              y = r % TY;
                                              z = r / TY;
                                              d = z * SY + y + H;
                                            },
                                            f);
    // the y-halo rows of every in-tile plane (with or without the corners)
    auto yh = [](int r, int& y, int& z, int& d) {
      const int k = r % (2 * H);
      y = k < H ? k - H : TY + k - H;
      z = r / (2 * H);
      d = z * SY + y + H;
    };
    if (XYC) stage_rows<TX + 2 * H, -H, 2 * H * TZ, NW>(p + (XH - H), SX, fo, yh, f);
    else stage_rows<TX, 0, 2 * H * TZ, NW>(p + XH, SX, fo, yh, f);
    // z halos: in-tile rows of the 2H planes below and above the tile
    stage_rows<TX, 0, 2 * H * TY, NW>(p + SLAB, TX, fo,
                                      [](int r, int& y, int& z, int& d) {
                                        y = r % TY;
                                        const int zz = r / TY;
                                        z = zz < H ? zz - H : TZ + zz - H;
                                        d = r;
                                      },
                                      f);
  }
  // bulk form: every row one copy; the y-halo rows without the corners
  // (the bulk-staged Stars feed first and second derivatives only)
  static constexpr unsigned kBulkBytes = 8u * (unsigned)(SX * TY * TZ + TX * 2 * H * TZ + TX * 2 * H * TY);
  __device__ void stage_bulk(const Folds<TX, TY, TZ>& fo, int x0, int nx, const double* src, uint64_t* bar) const {
    tile::stage_bulk<SX, -XH, TY * TZ>(p, SX, fo, x0, nx,
                                      [](int r, int& y, int& z, int& d) {
                                        y = r % TY;
                                        z = r / TY;
                                        d = z * SY + y + H;
                                      },
                                      src, bar);
    tile::stage_bulk<TX, 0, 2 * H * TZ>(p + XH, SX, fo, x0, nx,
                                        [](int r, int& y, int& z, int& d) {
                                          const int k = r % (2 * H);
                                          y = k < H ? k - H : TY + k - H;
                                          z = r / (2 * H);
                                          d = z * SY + y + H;
                                        },
                                        src, bar);
    tile::stage_bulk<TX, 0, 2 * H * TY>(p + SLAB, TX, fo, x0, nx,
                                        [](int r, int& y, int& z, int& d) {
                                          y = r % TY;
                                          const int zz = r / TY;
                                          z = zz < H ? zz - H : TZ + zz - H;
                                          d = r;
                                        },
                                        src, bar);
  }
};

template <int TX, int TY, int TZ>
struct Box {
  static constexpr int SX = TX + 2 * XH, SY = TY + 2 * H, SZ = TZ + 2 * H;
  static constexpr int SIZE = SX * SY * SZ;
  double* p;
  __device__ __forceinline__ double v(int x, int y, int z) const { return p[((z + H) * SY + (y + H)) * SX + (x + XH)]; }
  template <int NW, class F>
  __device__ void stage(const Folds<TX, TY, TZ>& fo, const F& f) const {
    stage_rows<TX + 2 * H, -H, SY * SZ, NW>(p + (XH - H), SX, fo,
                                            [](int r, int& y, int& z, int& d) {
                                              y = r % SY - H;
                                              z = r / SY - H;
                                              d = r;
                                            },
                                            f);
  }
  static constexpr unsigned kBulkBytes = 8u * (unsigned)(SX * SY * SZ);
  __device__ void stage_bulk(const Folds<TX, TY, TZ>& fo, int x0, int nx, const double* src, uint64_t* bar) const {
    tile::stage_bulk<SX, -XH, SY * SZ>(p, SX, fo, x0, nx,
                                      [](int r, int& y, int& z, int& d) {
                                        y = r % SY - H;
                                        z = r / SY - H;
                                        d = r;
                                      },
                                      src, bar);
  }
};

// One-direction halo buffers (for fluxes differentiated along one axis only)
template <int TX, int TY, int TZ>
struct XRow {
  static constexpr int SX = TX + 2 * XH, SIZE = TZ * TY * SX;
  double* p;
  __device__ __forceinline__ double v(int x, int y, int z) const { return p[(z * TY + y) * SX + (x + XH)]; }
  template <int NW, class F>
  __device__ void stage(const Folds<TX, TY, TZ>& fo, const F& f) const {
    stage_rows<TX + 2 * H, -H, TY * TZ, NW>(p + (XH - H), SX, fo,
                                            [](int r, int& y, int& z, int& d) {
                                              y = r % TY;
                                              z = r / TY;
                                              d = r;
                                            },
                                            f);
  }
  // this buffer and b, c (same shape) from one pass of f (stage_rows3)
  template <int NW, int UB, class F>
  __device__ void stage3(const XRow& b, const XRow& c, const Folds<TX, TY, TZ>& fo, const F& f) const {
    stage_rows3<TX + 2 * H, -H, TY * TZ, NW, UB>(p + (XH - H), b.p + (XH - H), c.p + (XH - H), SX, fo,
                                                 [](int r, int& y, int& z, int& d) {
                                                   y = r % TY;
                                                   z = r / TY;
                                                   d = r;
                                                 },
                                                 f);
  }
  static constexpr unsigned kBulkBytes = 8u * (unsigned)SIZE;
  __device__ void stage_bulk(const Folds<TX, TY, TZ>& fo, int x0, int nx, const double* src, uint64_t* bar) const {
    tile::stage_bulk<SX, -XH, TY * TZ>(p, SX, fo, x0, nx,
                                      [](int r, int& y, int& z, int& d) {
                                        y = r % TY;
                                        z = r / TY;
                                        d = r;
                                      },
                                      src, bar);
  }
};
template <int TX, int TY, int TZ>
struct YRow {
  static constexpr int SY = TY + 2 * H, SIZE = TZ * SY * TX;
  double* p;
  __device__ __forceinline__ double v(int x, int y, int z) const { return p[(z * SY + (y + H)) * TX + x]; }
  template <int NW, class F>
  __device__ void stage(const Folds<TX, TY, TZ>& fo, const F& f) const {
    stage_rows<TX, 0, SY * TZ, NW>(p, TX, fo,
                                   [](int r, int& y, int& z, int& d) {
                                     y = r % SY - H;
                                     z = r / SY;
                                     d = r;
                                   },
                                   f);
  }
  // this buffer and b, c (same shape) from one pass of f (stage_rows3)
  template <int NW, int UB, class F>
  __device__ void stage3(const YRow& b, const YRow& c, const Folds<TX, TY, TZ>& fo, const F& f) const {
    stage_rows3<TX, 0, SY * TZ, NW, UB>(p, b.p, c.p, TX, fo,
                                        [](int r, int& y, int& z, int& d) {
                                          y = r % SY - H;
                                          z = r / SY;
                                          d = r;
                                        },
                                        f);
  }
  static constexpr unsigned kBulkBytes = 8u * (unsigned)SIZE;
  __device__ void stage_bulk(const Folds<TX, TY, TZ>& fo, int x0, int nx, const double* src, uint64_t* bar) const {
    tile::stage_bulk<TX, 0, SY * TZ>(p, TX, fo, x0, nx,
                                     [](int r, int& y, int& z, int& d) {
                                       y = r % SY - H;
                                       z = r / SY;
                                       d = r;
                                     },
                                     src, bar);
  }
};
template <int TX, int TY, int TZ>
struct ZCol {
  static constexpr int SZ = TZ + 2 * H, SIZE = SZ * TY * TX;
  double* p;
  __device__ __forceinline__ double v(int x, int y, int z) const { return p[((z + H) * TY + y) * TX + x]; }
  template <int NW, class F>
  __device__ void stage(const Folds<TX, TY, TZ>& fo, const F& f) const {
    stage_rows<TX, 0, TY * SZ, NW>(p, TX, fo,
                                   [](int r, int& y, int& z, int& d) {
                                     y = r % TY;
                                     z = r / TY - H;
                                     d = r;
                                   },
                                   f);
  }
  static constexpr unsigned kBulkBytes = 8u * (unsigned)SIZE;
  __device__ void stage_bulk(const Folds<TX, TY, TZ>& fo, int x0, int nx, const double* src, uint64_t* bar) const {
    tile::stage_bulk<TX, 0, TY * SZ>(p, TX, fo, x0, nx,
                                     [](int r, int& y, int& z, int& d) {
                                       y = r % TY;
                                       z = r / TY - H;
                                       d = r;
                                     },
                                     src, bar);
  }
};

// Slab: the in-tile planes with x and y halos only, [TZ][TY+2H][TX+2H]. Used
// with a per-thread register column for the z direction (Column below): the
// z-halo values of a column are only read by the thread that owns it.
template <int TX, int TY, int TZ>
struct Slab {
  static constexpr int SX = TX + 2 * XH, SY = TY + 2 * H;
  static constexpr int SIZE = TZ * SY * SX;
  double* p;
  __device__ __forceinline__ double v(int x, int y, int z) const { return p[(z * SY + (y + H)) * SX + (x + XH)]; }
  template <int NW, bool XYC = false, class F>
  __device__ void stage(const Folds<TX, TY, TZ>& fo, const F& f) const {
    stage_rows<TX + 2 * H, -H, TY * TZ, NW>(p + (XH - H), SX, fo,
                                            [](int r, int& y, int& z, int& d) {
                                              y = r % TY;
                                              z = r / TY;
                                              d = z * SY + y + H;
                                            },
                                            f);
    auto yh = [](int r, int& y, int& z, int& d) {
      const int k = r % (2 * H);
      y = k < H ? k - H : TY + k - H;
      z = r / (2 * H);
      d = z * SY + y + H;
    };
    if (XYC) stage_rows<TX + 2 * H, -H, 2 * H * TZ, NW>(p + (XH - H), SX, fo, yh, f);
    else stage_rows<TX, 0, 2 * H * TZ, NW>(p + XH, SX, fo, yh, f);
  }
  // bulk form: the in-tile rows with their x halos, the y-halo rows without
  // the corners (the same footprint as the per-element form)
  static constexpr unsigned kBulkBytes = 8u * (unsigned)(SX * TY * TZ + TX * 2 * H * TZ);
  __device__ void stage_bulk(const Folds<TX, TY, TZ>& fo, int x0, int nx, const double* src, uint64_t* bar) const {
    tile::stage_bulk<SX, -XH, TY * TZ>(p, SX, fo, x0, nx,
                                      [](int r, int& y, int& z, int& d) {
                                        y = r % TY;
                                        z = r / TY;
                                        d = z * SY + y + H;
                                      },
                                      src, bar);
    tile::stage_bulk<TX, 0, 2 * H * TZ>(p + XH, SX, fo, x0, nx,
                                        [](int r, int& y, int& z, int& d) {
                                          const int k = r % (2 * H);
                                          y = k < H ? k - H : TY + k - H;
                                          z = r / (2 * H);
                                          d = z * SY + y + H;
                                        },
                                        src, bar);
  }
};

// The thread's own z-column of a field, tile-local z in [-H, TZ+H), held in
// registers: c[z + H]. load() reads it straight from global memory (a warp
// reads 32 consecutive x per row: coalesced).
template <int TZ>
struct Column {
  double c[TZ + 2 * H];
  template <int TX, int TY, class F>
  __device__ __forceinline__ void load(const Folds<TX, TY, TZ>& fo, int tx, int ty, const F& f) {
    const int64_t b = fo.ox[tx + H] + fo.oy[ty + H];
#pragma unroll
    for (int k = 0; k < TZ + 2 * H; ++k) c[k] = f(b + fo.oz[k]);
  }
};

// A staged buffer read with a constant subtracted from every value (the
// pressure gradient of p - p(1,1,1), src/rhsvel.f:741-746).
template <class Buf>
struct Shifted {
  Buf b;
  double c;
  __device__ __forceinline__ double v(int x, int y, int z) const { return b.v(x, y, z) - c; }
};

// A grid point of the tile as seen by one thread.
struct TP {
  int x, y, z;      // tile-local
  int gx, gy, gz;   // global
  int64_t q;        // global linear index
  bool valid;       // inside the domain (partial edge tiles)
};

__device__ __forceinline__ TP make_tp(const Geo& g, const Origin& o, int x, int y, int z) {
  TP t;
  t.x = x;
  t.y = y;
  t.z = z;
  t.gx = o.x0 + x;
  t.gy = o.y0 + y;
  t.gz = o.z0 + z;
  t.valid = t.gx < g.nx && t.gy < g.ny && t.gz < g.nz;
  t.q = t.valid ? (int64_t)t.gx + (int64_t)g.nx * ((int64_t)t.gy + (int64_t)g.ny * t.gz) : 0;
  return t;
}

// ---- derivatives of staged fields (scaled) ----
// P = true: every direction is periodic (known at compile time, no closure
// branch); P = false: the box's per-direction flags select the closures.
template <int DIR, bool P, class B>
__device__ __forceinline__ double d1(const Geo& g, const TP& t, const B& b) {
  if (DIR == 0) return d1core([&](int m) { return b.v(t.x + m, t.y, t.z); }, t.gx, g.nx, P ? 1 : g.per[0]) * g.ovd[0];
  if (DIR == 1) return d1core([&](int m) { return b.v(t.x, t.y + m, t.z); }, t.gy, g.ny, P ? 1 : g.per[1]) * g.ovd[1];
  return d1core([&](int m) { return b.v(t.x, t.y, t.z + m); }, t.gz, g.nz, P ? 1 : g.per[2]) * g.ovd[2];
}
// derivative of the pointwise product of two staged fields
template <int DIR, bool P, class A, class B>
__device__ __forceinline__ double d1p(const Geo& g, const TP& t, const A& a, const B& b) {
  if (DIR == 0)
    return d1core([&](int m) { return a.v(t.x + m, t.y, t.z) * b.v(t.x + m, t.y, t.z); }, t.gx, g.nx, P ? 1 : g.per[0]) * g.ovd[0];
  if (DIR == 1)
    return d1core([&](int m) { return a.v(t.x, t.y + m, t.z) * b.v(t.x, t.y + m, t.z); }, t.gy, g.ny, P ? 1 : g.per[1]) * g.ovd[1];
  return d1core([&](int m) { return a.v(t.x, t.y, t.z + m) * b.v(t.x, t.y, t.z + m); }, t.gz, g.nz, P ? 1 : g.per[2]) * g.ovd[2];
}
template <int DIR, bool P, class B>
__device__ __forceinline__ double d2(const Geo& g, const TP& t, const B& b) {
  if (DIR == 0) return d2core([&](int m) { return b.v(t.x + m, t.y, t.z); }, t.gx, g.nx, P ? 1 : g.per[0]) * g.ovd2[0];
  if (DIR == 1) return d2core([&](int m) { return b.v(t.x, t.y + m, t.z); }, t.gy, g.ny, P ? 1 : g.per[1]) * g.ovd2[1];
  return d2core([&](int m) { return b.v(t.x, t.y, t.z + m); }, t.gz, g.nz, P ? 1 : g.per[2]) * g.ovd2[2];
}
template <int DA, int DB, bool P, class B>
__device__ __forceinline__ double dm(const Geo& g, const TP& t, const B& b) {
  auto v = [&](int ma, int mb) {
    const int dx = (DA == 0 ? ma : 0) + (DB == 0 ? mb : 0);
    const int dy = (DA == 1 ? ma : 0) + (DB == 1 ? mb : 0);
    const int dz = (DA == 2 ? ma : 0) + (DB == 2 ? mb : 0);
    return b.v(t.x + dx, t.y + dy, t.z + dz);
  };
  if (!P && !g.per[DA]) {
    const int c = DA == 0 ? t.gx : DA == 1 ? t.gy : t.gz;
    const int n = DA == 0 ? g.nx : DA == 1 ? g.ny : g.nz;
    return dmcore_b(v, c, n) * g.ovd[DA] * g.ovd[DB];
  }
  return dmcore(v) * g.ovd[DA] * g.ovd[DB];
}

// z derivatives from a register column (z in-tile, compile-time after
// unrolling). z is periodic on every box these tile kernels run on (boxes
// bounded in y or z are refused before any right-hand-side launch), so the
// interior scheme is compiled in and the column stays in registers.
template <bool P, int TZ>
__device__ __forceinline__ double d1z(const Geo& g, const TP& t, const Column<TZ>& col) {
  return d1core([&](int m) { return col.c[t.z + H + m]; }, t.gz, g.nz, 1) * g.ovd[2];
}
template <bool P, int TZ>
__device__ __forceinline__ double d2z(const Geo& g, const TP& t, const Column<TZ>& col) {
  return d2core([&](int m) { return col.c[t.z + H + m]; }, t.gz, g.nz, 1) * g.ovd2[2];
}
template <bool P, int TZ>
__device__ __forceinline__ double d1zp(const Geo& g, const TP& t, const Column<TZ>& a, const Column<TZ>& b) {
  return d1core([&](int m) { return a.c[t.z + H + m] * b.c[t.z + H + m]; }, t.gz, g.nz, 1) * g.ovd[2];
}

}  // namespace tile
}  // namespace senga
