// Pointwise kernel of the B200 RHS + RK path and the operator-level stencils.
//
//   k_thermo      pointwise: TEMPER (src/temper.f:58-219), transport
//                 properties (src/rhscal.f:515-571, 1292-1340, 3854-3885;
//                 src/rhsvel.f:933-952), species enthalpy (rhscal.f:1444-1466)
//                 and CHRATE (src/chrate.f:146-741), fused per grid point.
//   k_deriv       operator-level derivative family (DFBYDX..D2FDYZ) reading
//                 global memory, for the unit entry points.
// The stencil kernels of the substage are in kernels_tiled.cu.
#include <cuda_runtime.h>

#include <cstdint>

#include <cstdlib>
#include <cstring>

#include "mech_gen.cuh"
#include "senga_internal.h"
#include "stencil.cuh"
#include "thermo.cuh"

namespace senga {

namespace {

// Resident blocks per SM asked of the compiler for a policy (register cap
// 65536 / (256 * blocks)): more warps hide the FP64 dependency chains of the
// long straight-line mechanisms.
template <class M>
struct ThermoOcc {
  static constexpr int blocks = 1;
};
#ifndef SENGA_THERMO_H2_MINB
#define SENGA_THERMO_H2_MINB 2
#endif
template <>
struct ThermoOcc<gen::Mech_h2> {
  static constexpr int blocks = SENGA_THERMO_H2_MINB;
};

template <class M>
__global__ void __launch_bounds__(kBlock, ThermoOcc<M>::blocks) k_thermo(Geo g, Fields f, M m) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= g.n) return;
  thermo_point(g, f, m, q);
}
// The two halves of the thermochemistry: PART 1 at three blocks per SM (the
// mixture-averaged transport wants ~128 registers; at 80 it spills some, and
// the extra warps still win: 5.17 against 5.35 ms per substage on the 256^3
// H2 box), PART 2 (CHRATE) at three.
#ifndef SENGA_THERMO_P1_MINB
#define SENGA_THERMO_P1_MINB 3
#endif
#ifndef SENGA_THERMO_P2_MINB
#define SENGA_THERMO_P2_MINB 3
#endif
#ifndef SENGA_THERMO_P1_BLOCK
#define SENGA_THERMO_P1_BLOCK kBlock
#endif
#ifndef SENGA_THERMO_P2_BLOCK
#define SENGA_THERMO_P2_BLOCK kBlock
#endif
template <int PART>
constexpr int kPartBlock = PART == 1 ? SENGA_THERMO_P1_BLOCK : SENGA_THERMO_P2_BLOCK;
template <class M, int PART>
__global__ void __launch_bounds__(kPartBlock<PART>, PART == 1 ? SENGA_THERMO_P1_MINB : SENGA_THERMO_P2_MINB)
    k_thermo_part(Geo g, Fields f, M m) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= g.n) return;
  thermo_point<M, PART>(g, f, m, q);
}

// Batched: CTAs stride over (box, 256-point chunk) items.
template <class M>
__global__ void __launch_bounds__(kBlock) k_thermo_b(const __grid_constant__ BoxTable t,
                                                     const WorkItem* __restrict__ chunks, int nchunks, M m) {
  for (int it = blockIdx.x; it < nchunks; it += gridDim.x) {
    const WorkItem w = chunks[it];
    const BoxDesc& sd = t.d[w.box];
    const int64_t q = (int64_t)w.x0 * kBlock + threadIdx.x;
    if (q < sd.g.n) thermo_point(sd.g, sd.f, m, q);
  }
}

// -------------------------------------------------------------------------
__global__ void k_deriv(Geo g, int kind, const double* __restrict__ in, double* __restrict__ out) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= g.n) return;
  const Pt pt = point_of(g, q);
  const Ld F{in};
  double r = 0.0;
  switch (kind) {
    case 0: r = D1<0>(g, pt, F); break;
    case 1: r = D1<1>(g, pt, F); break;
    case 2: r = D1<2>(g, pt, F); break;
    case 3: r = D2<0>(g, pt, F); break;
    case 4: r = D2<1>(g, pt, F); break;
    case 5: r = D2<2>(g, pt, F); break;
    case 6: r = DM<0, 1>(g, pt, F); break;
    case 7: r = DM<0, 2>(g, pt, F); break;
    default: r = DM<1, 2>(g, pt, F); break;
  }
  out[q] = r;
}

// The same operators on the reference's own array shape: `in` is the
// halo-extended FUNCTN(1-5:nx+5, 1-5:ny+5, 1-5:nz+5) (x fastest) and the
// result the interior FDERIV(nx, ny, nz) (src/dfbydx.f:36-37). Neighbours are
// read from the halo as given (PARFER's copies in a periodic direction, or a
// neighbour rank's planes), never folded; a bounded direction uses the
// one-sided closures, which read interior points only.
__global__ void k_deriv_big(Geo g, int kind, const double* __restrict__ in, double* __restrict__ out) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= g.n) return;
  const Pt pt = point_of(g, q);
  constexpr int H = 5;
  const int64_t bx = g.nx + 2 * H, bxy = bx * (g.ny + 2 * H);
  const int64_t qb = (pt.i + H) + bx * (pt.j + H) + bxy * (pt.k + H);
  const int64_t st[3] = {1, bx, bxy};
  const int c3[3] = {pt.i, pt.j, pt.k};
  const int n3[3] = {g.nx, g.ny, g.nz};
  auto f = [&](int64_t o) { return __ldg(in + qb + o); };
  double r = 0.0;
  if (kind < 6) {
    const int d = kind % 3;
    auto v = [&](int m) { return f(m * st[d]); };
    r = kind < 3 ? d1core(v, c3[d], n3[d], g.per[d]) * g.ovd[d] : d2core(v, c3[d], n3[d], g.per[d]) * g.ovd2[d];
  } else {
    const int da = kind == 8 ? 1 : 0, db = kind == 6 ? 1 : 2;
    auto v = [&](int ma, int mb) { return f(ma * st[da] + mb * st[db]); };
    if (!g.per[db]) {
      constexpr int kFar = 1 << 20;
      const int ca = c3[da], cb = c3[db];
      const int la = g.per[da] ? kFar : ca, ra = g.per[da] ? kFar : n3[da] - 1 - ca;
      const int lb = cb, rb = n3[db] - 1 - cb;
      r = dmcore_ends(v, la < ra ? la : ra, ra < la, lb < rb ? lb : rb, rb < lb);
    } else if (!g.per[da]) {
      r = dmcore_b(v, c3[da], n3[da]);
    } else {
      r = dmcore(v);
    }
    r = r * g.ovd[da] * g.ovd[db];
  }
  out[q] = r;
}

inline unsigned grid_of(int64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

}  // namespace

int select_mech(const senga_chem& chem, const senga_diff& diff) {
  const char* env = std::getenv("SENGA_MECH");
  if (env && std::strcmp(env, "generic") == 0) return 0;
  if (gen::Mech_onestep::matches(chem, diff)) return 1;
  if (gen::Mech_h2::matches(chem, diff)) return 2;
  return 0;
}

int launch_thermo(const Geo& g, const Fields& f, const senga_chem* dchem, const senga_diff* ddiff, int nspec,
                  int flmavt, int mech, cudaStream_t s) {
  const unsigned gr = grid_of(g.n);
  if (mech == 1) {
    k_thermo<<<gr, kBlock, 0, s>>>(g, f, gen::Mech_onestep{});
  } else if (mech == 2) {
    k_thermo_part<gen::Mech_h2, 1>
        <<<(unsigned)((g.n + kPartBlock<1> - 1) / kPartBlock<1>), kPartBlock<1>, 0, s>>>(g, f, gen::Mech_h2{});
    k_thermo_part<gen::Mech_h2, 2>
        <<<(unsigned)((g.n + kPartBlock<2> - 1) / kPartBlock<2>), kPartBlock<2>, 0, s>>>(g, f, gen::Mech_h2{});
    return 2;
  } else if (nspec <= 2) {
    if (flmavt) k_thermo<<<gr, kBlock, 0, s>>>(g, f, MechTables<2, true>{dchem, ddiff, nspec});
    else k_thermo<<<gr, kBlock, 0, s>>>(g, f, MechTables<2, false>{dchem, ddiff, nspec});
  } else if (nspec <= 9) {
    if (flmavt) k_thermo<<<gr, kBlock, 0, s>>>(g, f, MechTables<9, true>{dchem, ddiff, nspec});
    else k_thermo<<<gr, kBlock, 0, s>>>(g, f, MechTables<9, false>{dchem, ddiff, nspec});
  } else {  // the reference's larger casefile mechanisms (16 and 18 species)
    if (flmavt) k_thermo<<<gr, kBlock, 0, s>>>(g, f, MechTables<SENGA_NSPCMX, true>{dchem, ddiff, nspec});
    else k_thermo<<<gr, kBlock, 0, s>>>(g, f, MechTables<SENGA_NSPCMX, false>{dchem, ddiff, nspec});
  }
  return 1;
}

void launch_batch_thermo(const BoxTable& boxes, const WorkItem* chunks, int nchunks, int grid, int mech,
                         const senga_chem* dchem, const senga_diff* ddiff, int nspec, int flmavt, cudaStream_t s) {
  if (mech == 1) {
    k_thermo_b<<<grid, kBlock, 0, s>>>(boxes, chunks, nchunks, gen::Mech_onestep{});
  } else if (mech == 2) {
    k_thermo_b<<<grid, kBlock, 0, s>>>(boxes, chunks, nchunks, gen::Mech_h2{});
  } else if (nspec <= 2) {
    if (flmavt) k_thermo_b<<<grid, kBlock, 0, s>>>(boxes, chunks, nchunks, MechTables<2, true>{dchem, ddiff, nspec});
    else k_thermo_b<<<grid, kBlock, 0, s>>>(boxes, chunks, nchunks, MechTables<2, false>{dchem, ddiff, nspec});
  } else {
    if (flmavt) k_thermo_b<<<grid, kBlock, 0, s>>>(boxes, chunks, nchunks, MechTables<9, true>{dchem, ddiff, nspec});
    else k_thermo_b<<<grid, kBlock, 0, s>>>(boxes, chunks, nchunks, MechTables<9, false>{dchem, ddiff, nspec});
  }
}

int thermo_block() { return kBlock; }

void launch_deriv(const Geo& g, int kind, const double* in, double* out, cudaStream_t s) {
  k_deriv<<<grid_of(g.n), kBlock, 0, s>>>(g, kind, in, out);
}

void launch_deriv_big(const Geo& g, int kind, const double* in, double* out, cudaStream_t s) {
  k_deriv_big<<<grid_of(g.n), kBlock, 0, s>>>(g, kind, in, out);
}

}  // namespace senga
