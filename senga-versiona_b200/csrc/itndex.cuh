// ITNDEX, the per-point index of each species' thermodynamic temperature
// interval: base-4 digits (NTBASE = 4), NSPIMX = 15 species per 32-bit word,
// (nspec + 14) / 15 words per point stored words slowest ([word][n])
// (src/com_senga2.h:93-98, src/temper.f:196-205). In registers it is one
// packed value: word 1 lands 30 bits up, so species s is always at bits 2s,
// 2s+1.
#pragma once
#include <cstdint>

#include "senga_internal.h"

namespace senga {
namespace {

__device__ __forceinline__ uint64_t itn_load(const Fields& f, int64_t n, int64_t q, int nspec) {
  uint64_t v = (uint32_t)f.itn[q];
  if (nspec > SENGA_NSPIMX) v |= (uint64_t)(uint32_t)f.itn[n + q] << (2 * SENGA_NSPIMX);
  return v;
}
__device__ __forceinline__ void itn_store(int32_t* itn, int64_t n, int64_t q, int nspec, uint64_t v) {
  itn[q] = (int32_t)(v & ((1ull << (2 * SENGA_NSPIMX)) - 1));
  if (nspec > SENGA_NSPIMX) itn[n + q] = (int32_t)(v >> (2 * SENGA_NSPIMX));
}

}  // namespace
}  // namespace senga
