// One persistent launch per RK substage for a batched ensemble.
//
// A grid of resident CTAs takes work items from a device-wide dispenser in
// phase-major order: the thermochemistry chunks of every box (256 points,
// thermo_point: TEMPER, primitives, transport, h_k, CHRATE), then every
// box's flow tiles, species tiles and species+RK tiles (the tile functions
// of tile_fns.cuh). An item of phase p of box b starts once all of b's
// phase p-1 items have completed: each finishing CTA releases its writes
// and counts the item on a per-(box, phase) counter, and the next phase's
// CTA acquires that counter before it reads. So the four phases of a
// substage overlap across boxes instead of draining between four kernels,
// and the fields are read with coherent loads (NC = false), never through
// the read-only path, since other CTAs of the same launch wrote them.
//
// Items are handed out in list order and a CTA waits only for items handed
// out before its own, which running CTAs hold; the earliest unfinished item
// never waits, so every wait ends. Each wait is still bounded (about one
// second of SM clock): on time-out the CTA sets kStatusPersistTimeout in the
// box's status word, raises the launch's abort flag and leaves; every other
// CTA leaves at its next item or wait. No part of this is in the reference,
// whose substage runs the boxes one at a time.
#include <cuda_runtime.h>

#include "senga_internal.h"
#include "stencil.cuh"
#include "thermo.cuh"
#include "tile_fns.cuh"
#include "tiles.cuh"

namespace senga {
namespace {

using namespace tile;

static_assert(FX == SX_ && FY == SY_ && FZ == SZ_, "one tile shape for every stencil phase");
static_assert(FX * FY == kBlock, "a thermochemistry chunk is one point per thread");

constexpr int kPersistSmem = cmax(kFlowSmem, cmax(kSpecSmem, kSpecRkSmem));

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// thread 0 of a CTA: true once *c reaches target; false when the launch is
// aborted or the wait runs out (which aborts the launch)
__device__ bool await_count(const int* c, int target, int* abort_flag, unsigned int* status) {
  const long long t0 = clock64();
  for (;;) {
    if (ld_acquire(c) >= target) return true;
    if (ld_acquire(abort_flag)) return false;
    if (clock64() - t0 > (1ll << 31)) {
      if (status) atomicOr(status, kStatusPersistTimeout);
      atomicExch(abort_flag, 1);
      return false;
    }
    __nanosleep(100);
  }
}

#ifndef SENGA_PERSIST_MINB
#define SENGA_PERSIST_MINB 2
#endif

// The four phases of an item.
template <class M>
__device__ __forceinline__ void phase_thermo(const BoxDesc& sd, const M& m, int chunk) {
  const int64_t q = (int64_t)chunk * kBlock + threadIdx.x;
  if (q < sd.g.n) thermo_point(sd.g, sd.f, m, q);
}
__device__ __forceinline__ void phase_flow(const BoxDesc& sd, Origin o, double* sm, Folds<FX, FY, FZ>& fo) {
  flow_tile<true, false, false>(sd.g, sd.f, o, sm, fo, ZDec{});
}
__device__ __forceinline__ void phase_species(const BoxDesc& sd, Origin o, double* sm, Folds<FX, FY, FZ>& fo) {
  species_tile<true, 0, false>(sd.g, sd.f, sd.nspec, o, sm, fo, ZDec{});
}
__device__ __forceinline__ void phase_species_rk(const BoxDesc& sd, int irk, Origin o, double* sm,
                                              Folds<FX, FY, FZ>& fo) {
  species_rk_tile<true, 0, false>(sd.g, sd.f, sd.nspec, sd.rk[irk], o, sm, fo, ZDec{});
}

template <class M>
__global__ void __launch_bounds__(FX* FY, SENGA_PERSIST_MINB)
    k_substage_persist(const __grid_constant__ BoxTable t, const PersistArgs a, const M m) {
  extern __shared__ __align__(16) double sm[];
  __shared__ Folds<FX, FY, FZ> fo;
  __shared__ int s_item, s_go;
  const int total = a.off[4];
  for (;;) {
    if (threadIdx.x == 0) s_item = ld_acquire(&a.ctr[1]) ? total : atomicAdd(&a.ctr[0], 1);
    __syncthreads();
    const int it = s_item;
    if (it >= total) return;
    const int phase = (it >= a.off[1]) + (it >= a.off[2]) + (it >= a.off[3]);
    const WorkItem w = a.items[it];
    const BoxDesc& sd = t.d[w.box];
    if (phase > 0) {
      if (threadIdx.x == 0)
        s_go = await_count(&a.ctr[2 + 4 * w.box + phase - 1], a.need[4 * w.box + phase - 1], &a.ctr[1],
                           sd.f.status);
      __syncthreads();
      if (!s_go) return;
    }
    const Origin o{w.x0, w.y0, w.z0};
    if (phase == 0) phase_thermo(sd, m, w.x0);
    else if (phase == 1) phase_flow(sd, o, sm, fo);
    else if (phase == 2) phase_species(sd, o, sm, fo);
    else phase_species_rk(sd, a.irk, o, sm, fo);
    // every thread's writes of the item, then one release per item
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(&a.ctr[2 + 4 * w.box + phase], 1);
    }
  }
}

template <class M>
void launch_one(const BoxTable& boxes, const PersistArgs& a, const M& m, int grid, cudaStream_t s) {
  static bool attr[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  if (!attr[dev]) {
    cudaFuncSetAttribute(k_substage_persist<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPersistSmem * 8);
    attr[dev] = true;
  }
  k_substage_persist<M><<<grid, FX * FY, kPersistSmem * 8, s>>>(boxes, a, m);
}

}  // namespace

int persist_ctas_per_sm(int mech, int nspec, int flmavt) {
  int n = 0;
  auto occ = [&](auto kern) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kPersistSmem * 8);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, FX * FY, kPersistSmem * 8);
  };
  if (mech == 1) occ(k_substage_persist<gen::Mech_onestep>);
  else if (mech == 2) occ(k_substage_persist<gen::Mech_h2>);
  else if (nspec <= 2) flmavt ? occ(k_substage_persist<MechTables<2, true>>) : occ(k_substage_persist<MechTables<2, false>>);
  else flmavt ? occ(k_substage_persist<MechTables<9, true>>) : occ(k_substage_persist<MechTables<9, false>>);
  return n;
}

void launch_batch_persist(const BoxTable& boxes, const PersistArgs& a, int grid, int mech, const senga_chem* dchem,
                          const senga_diff* ddiff, int nspec, int flmavt, cudaStream_t s) {
  if (a.off[4] <= 0) return;
  cudaMemsetAsync(a.ctr, 0, (size_t)kPersistCounters * sizeof(int), s);
  if (mech == 1) launch_one(boxes, a, gen::Mech_onestep{}, grid, s);
  else if (mech == 2) launch_one(boxes, a, gen::Mech_h2{}, grid, s);
  else if (nspec <= 2) {
    if (flmavt) launch_one(boxes, a, MechTables<2, true>{dchem, ddiff, nspec}, grid, s);
    else launch_one(boxes, a, MechTables<2, false>{dchem, ddiff, nspec}, grid, s);
  } else {
    if (flmavt) launch_one(boxes, a, MechTables<9, true>{dchem, ddiff, nspec}, grid, s);
    else launch_one(boxes, a, MechTables<9, false>{dchem, ddiff, nspec}, grid, s);
  }
}

}  // namespace senga
