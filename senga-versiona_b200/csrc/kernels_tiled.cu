// Shared-memory-tiled stencil kernels of the substage: one CTA per tile
// (k_flow_t, k_species_t, k_species_rk_t over one box; k_flow_b, k_species_b,
// k_species_rk_b over the (box, tile) items of a batch), running the tile
// functions of tile_fns.cuh, and their launchers.
#include <cuda_runtime.h>

#include <cstdlib>
#include <string>

#include "senga_internal.h"
#include "tile_fns.cuh"
#include "tiles.cuh"

namespace senga {

namespace {

using namespace tile;

// Resident CTAs per SM asked of the compiler (register cap 65536/(256*n)).
#ifndef SENGA_FLOW_MINB
#define SENGA_FLOW_MINB 2
#endif
#ifndef SENGA_SPEC_MINB
#define SENGA_SPEC_MINB 2
#endif
#ifndef SENGA_SPECRK_MINB
#define SENGA_SPECRK_MINB 4
#endif

// ---- single-box launches: one CTA per tile ----
// B: plain fields staged by bulk copies on the TMA engine (all-periodic
// boxes of even nx, one context, 16-byte aligned fields; the launcher checks)
template <bool P, bool B>
__global__ void __launch_bounds__(FX* FY, SENGA_FLOW_MINB) k_flow_t(Geo g, Fields f, ZDec zd) {
  extern __shared__ __align__(16) double sm[];
  __shared__ Folds<FX, FY, FZ> fo;
  __shared__ uint64_t bar;
  flow_tile<P, B>(g, f, Origin{(int)blockIdx.x * FX, (int)blockIdx.y * FY, (int)blockIdx.z * FZ}, sm, fo, zd, &bar);
}
template <bool P, int M>
__global__ void __launch_bounds__(SX_* SY_, SENGA_SPEC_MINB)
    k_species_t(Geo g, Fields f, int nspec, ZDec zd, const __grid_constant__ SpecMaps tm) {
  extern __shared__ __align__(128) double sm[];
  __shared__ Folds<SX_, SY_, SZ_> fo;
  __shared__ uint64_t bar;
  species_tile<P, M>(g, f, nspec, Origin{(int)blockIdx.x * SX_, (int)blockIdx.y * SY_, (int)blockIdx.z * SZ_}, sm,
                     fo, zd, &bar, &tm);
}
template <bool P, int M>
__global__ void __launch_bounds__(SX_* SY_, SENGA_SPECRK_MINB)
    k_species_rk_t(Geo g, Fields f, int nspec, RK rk, ZDec zd, const __grid_constant__ RkMaps tm) {
  extern __shared__ __align__(128) double sm[];
  __shared__ Folds<SX_, SY_, SZ_> fo;
  __shared__ uint64_t bar;
  species_rk_tile<P, M>(g, f, nspec, rk,
                        Origin{(int)blockIdx.x * SX_, (int)blockIdx.y * SY_, (int)blockIdx.z * SZ_}, sm, fo, zd,
                        &bar, &tm);
}

// Species pass and species+RK pass of one tile in one CTA, for all-periodic
// boxes of one context without the transport switches: the species rates
// stay in this CTA's shared memory and V_c, VTMP and the energy RHS in
// registers between the passes, instead of going through HBM (WDOT, VC,
// VTMP, RHS(E): 28 doubles written and read back per point).
constexpr int kSpecFusedSmem = kSpecSmem - kSpecColW + kCarryRate;  // rates in place of the rho w slots
__global__ void __launch_bounds__(SX_* SY_, SENGA_SPEC_MINB) k_species_fused_t(Geo g, Fields f, int nspec, RK rk) {
  extern __shared__ __align__(128) double sm[];
  __shared__ Folds<SX_, SY_, SZ_> fo;
  SpecCarry c;
  c.rate = sm + (kSpecSmem - kSpecColW);
  const Origin o{(int)blockIdx.x * SX_, (int)blockIdx.y * SY_, (int)blockIdx.z * SZ_};
  species_tile<true, 0, true, true>(g, f, nspec, o, sm, fo, ZDec{}, nullptr, nullptr, &c);
  species_rk_tile<true, 0, true, true>(g, f, nspec, rk, o, sm, fo, ZDec{}, nullptr, nullptr, &c);
}

// ---- batched launches: one CTA per (box, tile) work item; box descriptors
// come from the launch's parameter table (persist.cu runs the same tile
// functions as one persistent launch per substage) ----
template <bool P>
__global__ void __launch_bounds__(FX* FY, 2) k_flow_b(const __grid_constant__ BoxTable t,
                                                      const WorkItem* __restrict__ items) {
  extern __shared__ double sm[];
  __shared__ Folds<FX, FY, FZ> fo;
  const WorkItem w = items[blockIdx.x];
  const BoxDesc& sd = t.d[w.box];
  flow_tile<P>(sd.g, sd.f, Origin{w.x0, w.y0, w.z0}, sm, fo, ZDec{});
}
template <bool P>
__global__ void __launch_bounds__(SX_* SY_, 2) k_species_b(const __grid_constant__ BoxTable t,
                                                           const WorkItem* __restrict__ items) {
  extern __shared__ double sm[];
  __shared__ Folds<SX_, SY_, SZ_> fo;
  const WorkItem w = items[blockIdx.x];
  const BoxDesc& sd = t.d[w.box];
  species_tile<P>(sd.g, sd.f, sd.nspec, Origin{w.x0, w.y0, w.z0}, sm, fo, ZDec{});
}
template <bool P>
__global__ void __launch_bounds__(SX_* SY_, 2) k_species_rk_b(const __grid_constant__ BoxTable t,
                                                              const WorkItem* __restrict__ items, int irk) {
  extern __shared__ double sm[];
  __shared__ Folds<SX_, SY_, SZ_> fo;
  const WorkItem w = items[blockIdx.x];
  const BoxDesc& sd = t.d[w.box];
  species_rk_tile<P>(sd.g, sd.f, sd.nspec, sd.rk[irk], Origin{w.x0, w.y0, w.z0}, sm, fo, ZDec{});
}

dim3 tiles(const Geo& g, int tx, int ty, int tz) {
  return dim3((unsigned)((g.nx + tx - 1) / tx), (unsigned)((g.ny + ty - 1) / ty), (unsigned)((g.nz + tz - 1) / tz));
}

// Shared-memory opt-in per kernel, once per device (the attribute belongs
// to the current device's context).
template <bool P>
void set_attrs() {
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  if (done[dev]) return;
  cudaFuncSetAttribute(k_flow_t<P, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFlowSmem * 8);
  cudaFuncSetAttribute(k_species_t<P, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSpecSmem * 8);
  cudaFuncSetAttribute(k_species_rk_t<P, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSpecRkSmem * 8);
  if (P) {
    cudaFuncSetAttribute(k_flow_t<P, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFlowSmem * 8);
    cudaFuncSetAttribute(k_species_t<P, P ? 1 : 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSpecSmem * 8);
    cudaFuncSetAttribute(k_species_rk_t<P, P ? 1 : 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kSpecRkSmem * 8);
    cudaFuncSetAttribute(k_species_t<P, P ? 2 : 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSpecSmem * 8);
    cudaFuncSetAttribute(k_species_rk_t<P, P ? 2 : 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kSpecRkSmem * 8);
  }
  cudaFuncSetAttribute(k_flow_b<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFlowSmem * 8);
  cudaFuncSetAttribute(k_species_b<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSpecSmem * 8);
  cudaFuncSetAttribute(k_species_rk_b<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSpecRkSmem * 8);
  done[dev] = true;
}

bool all_periodic(const Geo& g) { return g.per[0] && g.per[1] && g.per[2]; }

bool al16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// Staging mode of the stencil tiles, from SENGA_STAGE (read at every launch
// or graph capture): 0 per-element cp.async, 1 rows copied by the TMA engine,
// 2 one tensor copy per buffer for tiles away from the periodic wrap (rows
// for the others; species kernels). Unset: rows for flow, cp.async for the
// species kernels; "cpasync", "bulk", "tma" force one mode ("tma" leaves flow
// on rows). Bulk and tensor modes apply to all-periodic boxes of one context
// with even nx whose staged fields start on 16-byte boundaries; other boxes
// use cp.async. Measured per launch on the 256^3 H2 box (cp.async / rows /
// tensor): flow 5.13 / 4.92 / -, species 6.47 / 8.18 / 8.28, species+RK
// 2.95 / 3.21 / 3.44 ms. The species kernels read their z neighbours from
// register columns loaded through L1, which the cp.async.ca fills of the
// same tile warm; copies on the TMA engine bypass L1, so those loads go to
// L2 (long-scoreboard stalls 7.9 against 1.4 per issue). Flow's buffers hold
// their z halos in shared memory and gain from the rows.
enum Kern { KFlow, KSpecies };
int stage_mode(const Geo& g, const Fields& f, const ZDec& zd, Kern k) {
  const char* e = getenv("SENGA_STAGE");
  const std::string v = e ? e : "";
  int m = k == KFlow ? 1 : 0;
  if (v == "cpasync") m = 0;
  else if (v == "bulk") m = 1;
  else if (v == "tma") m = k == KFlow ? 1 : 2;
  if (!m || !all_periodic(g) || zd.nr > 1 || (g.nx & 1)) return 0;
  const void* ptrs[] = {f.uin, f.e, f.t, f.lam, f.mu, f.vel, f.y, f.rd, f.h, f.hmix, f.p};
  for (const void* p : ptrs)
    if (p && !al16(p)) return 0;
  return m;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library)
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encoder() {
  static EncodeTiled fn = [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiled) nullptr;
    return (EncodeTiled)ptr;
  }();
  return fn;
}
// [k][z][y][x] FP64 tensor of nk fields of the box, x fastest, box
// bx x by x bz x 1; returns false when the encoder refuses it
bool make_map(CUtensorMap* m, const double* base, const Geo& g, int nk, unsigned bx, unsigned by, unsigned bz) {
  EncodeTiled enc = encoder();
  if (!enc || !base) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)g.nx, (cuuint64_t)g.ny, (cuuint64_t)g.nz, (cuuint64_t)nk};
  const cuuint64_t strides[3] = {(cuuint64_t)g.nx * 8, (cuuint64_t)g.nx * g.ny * 8, (cuuint64_t)g.n * 8};
  const cuuint32_t box[4] = {bx, by, bz, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(base), dims, strides, box, es,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

void launch_flow(const Geo& g, const Fields& f, int, cudaStream_t s, const ZDec& zd) {
  if (all_periodic(g)) {
    set_attrs<true>();
    if (stage_mode(g, f, zd, KFlow) == 1)
      k_flow_t<true, true><<<tiles(g, FX, FY, FZ), FX * FY, kFlowSmem * 8, s>>>(g, f, zd);
    else
      k_flow_t<true, false><<<tiles(g, FX, FY, FZ), FX * FY, kFlowSmem * 8, s>>>(g, f, zd);
  } else {
    set_attrs<false>();
    k_flow_t<false, false><<<tiles(g, FX, FY, FZ), FX * FY, kFlowSmem * 8, s>>>(g, f, zd);
  }
}

void launch_species_a(const Geo& g, const Fields& f, int nspec, cudaStream_t s, const ZDec& zd) {
  if (species_mma_ok(g, f, zd)) {
    launch_species_mma(g, f, nspec, s);
    return;
  }
  const dim3 grid = tiles(g, SX_, SY_, SZ_);
  SpecMaps tm{};
  if (all_periodic(g)) {
    set_attrs<true>();
    int m = stage_mode(g, f, zd, KSpecies);
    if (m == 2 && !(make_map(&tm.y, f.y, g, nspec, SSlab::SX, SSlab::SY, SZ_) &&
                    make_map(&tm.rd, f.rd, g, nspec, SSlab::SX, SSlab::SY, SZ_) &&
                    make_map(&tm.h, f.h, g, nspec, SSlab::SX, SSlab::SY, SZ_) &&
                    make_map(&tm.ux, f.uin, g, 5 + nspec, SXRow::SX, SY_, SZ_) &&
                    make_map(&tm.vy, f.uin, g, 5 + nspec, SX_, SYRow::SY, SZ_)))
      m = 1;
    if (m == 2) k_species_t<true, 2><<<grid, SX_ * SY_, kSpecSmem * 8, s>>>(g, f, nspec, zd, tm);
    else if (m == 1) k_species_t<true, 1><<<grid, SX_ * SY_, kSpecSmem * 8, s>>>(g, f, nspec, zd, tm);
    else k_species_t<true, 0><<<grid, SX_ * SY_, kSpecSmem * 8, s>>>(g, f, nspec, zd, tm);
  } else {
    set_attrs<false>();
    k_species_t<false, 0><<<grid, SX_ * SY_, kSpecSmem * 8, s>>>(g, f, nspec, zd, tm);
  }
}

// Opt-in (SENGA_FUSE=1, read at every launch or graph capture): measured on
// the 256^3 H2 box, the fused kernel takes 9.53 ms per substage against
// 6.48 + 2.93 ms for the two kernels. It saves 224 B per point of HBM
// traffic, but its RK pass runs at the species pass's two CTAs per SM
// (128 registers) instead of four, and is latency-bound there.
bool species_fusable(const Geo& g, const ZDec& zd) {
  const char* e = getenv("SENGA_FUSE");
  return all_periodic(g) && zd.nr == 1 && e && std::string(e) == "1";
}

void launch_species_fused(const Geo& g, const Fields& f, int nspec, const RK& rk, cudaStream_t s) {
  static bool attr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  if (!attr[dev]) {
    cudaFuncSetAttribute(k_species_fused_t, cudaFuncAttributeMaxDynamicSharedMemorySize, kSpecFusedSmem * 8);
    attr[dev] = true;
  }
  k_species_fused_t<<<tiles(g, SX_, SY_, SZ_), SX_ * SY_, kSpecFusedSmem * 8, s>>>(g, f, nspec, rk);
}

void launch_species_b_rk(const Geo& g, const Fields& f, int nspec, const RK& rk, cudaStream_t s, const ZDec& zd) {
  {
    const char* e = getenv("SENGA_SPECRK");
    if (e && std::string(e) == "z" && launch_species_b_rk_z(g, f, nspec, rk, s, zd)) return;
  }
  const dim3 grid = tiles(g, SX_, SY_, SZ_);
  RkMaps tm{};
  if (all_periodic(g)) {
    set_attrs<true>();
    int m = stage_mode(g, f, zd, KSpecies);
    if (m == 2 && !(make_map(&tm.y, f.y, g, nspec, SSlab::SX, SSlab::SY, SZ_) &&
                    make_map(&tm.hm, f.hmix, g, 1, SSlab::SX, SSlab::SY, SZ_)))
      m = 1;
    if (m == 2) k_species_rk_t<true, 2><<<grid, SX_ * SY_, kSpecRkSmem * 8, s>>>(g, f, nspec, rk, zd, tm);
    else if (m == 1) k_species_rk_t<true, 1><<<grid, SX_ * SY_, kSpecRkSmem * 8, s>>>(g, f, nspec, rk, zd, tm);
    else k_species_rk_t<true, 0><<<grid, SX_ * SY_, kSpecRkSmem * 8, s>>>(g, f, nspec, rk, zd, tm);
  } else {
    set_attrs<false>();
    k_species_rk_t<false, 0><<<grid, SX_ * SY_, kSpecRkSmem * 8, s>>>(g, f, nspec, rk, zd, tm);
  }
}

void tile_shape(int* tx, int* ty, int* tz) {
  static_assert(FX == SX_ && FY == SY_ && FZ == SZ_, "batched work lists assume one tile shape");
  *tx = FX;
  *ty = FY;
  *tz = FZ;
}

void launch_batch_stencil(const BoxTable& boxes, const WorkItem* items, int nitems, int irk, int phase,
                          cudaStream_t s) {
  set_attrs<true>();
  if (nitems <= 0) return;
  if (phase < 0 || phase == 0) k_flow_b<true><<<nitems, FX * FY, kFlowSmem * 8, s>>>(boxes, items);
  if (phase < 0 || phase == 1) k_species_b<true><<<nitems, SX_ * SY_, kSpecSmem * 8, s>>>(boxes, items);
  if (phase < 0 || phase == 2) k_species_rk_b<true><<<nitems, SX_ * SY_, kSpecRkSmem * 8, s>>>(boxes, items, irk);
}

}  // namespace senga
