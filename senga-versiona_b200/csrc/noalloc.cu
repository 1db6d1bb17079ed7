// Allocation-free right-hand side: senga_rhs_noalloc.
//
// Some callers of this library cannot allocate device memory when they call
// it: a Fortran driver that reserves all device memory once at start-up and
// forbids allocation afterwards, or a host that embeds this library inside
// another framework's memory pool. For them this entry point evaluates
// RHSCAL + RHSVEL of one box from caller-owned device buffers and keeps every
// intermediate field in a fixed, file-scope device array instead of a
// context-owned pool. It calls no cudaMalloc, cudaFree or allocating library
// routine.
//
// Limits and sharing:
//   * the scratch array holds SENGA_NOALLOC_SCRATCH_BYTES (16 MiB) on every
//     GPU that loads the library, until the process exits; a box needs
//     (14 + 4*nspec) doubles of scratch per grid point, so e.g. 41,943 points
//     for the 9-species mechanism and 95,325 for the 2-species one; larger
//     boxes are rejected with SENGA_ERR_ARG;
//   * every call shares the array and leaves its contents behind; the status
//     word is cleared at the start of each call and all other scratch fields
//     are written before they are read; calls whose work overlaps on the GPU
//     (different streams, or different host threads) race on the array;
//   * the first call on a device, with that device current, looks up the
//     device addresses of the file-scope arrays (cudaGetSymbolAddress); make
//     that first call before any stream capture. Under CUDA's lazy module
//     loading (the default of recent CUDA releases) that first call is also
//     when the array and the kernels' code are loaded onto the device, so a
//     host that reserves all free device memory at start-up makes one call
//     per device before it does (or runs with CUDA_MODULE_LOADING=EAGER);
//   * the status word is required: it is the only place a TEMPER
//     non-convergence is reported.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "senga_gpu.h"
#include "senga_internal.h"

namespace {

constexpr size_t kScratchBytes = SENGA_NOALLOC_SCRATCH_BYTES;
constexpr size_t kScratchDoubles = kScratchBytes / sizeof(double);
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];
static __device__ __align__(256) senga_chem g_noalloc_chem;
static __device__ __align__(256) senga_diff g_noalloc_diff;

// Transport tables of constant-Lewis runs (diff == NULL): a zeroed table at a
// fixed host address, the source of the table copy below.
const senga_diff kNoDiff = {};

struct DevicePtrs {
  bool ready = false;
  double* scratch = nullptr;
  senga_chem* chem = nullptr;
  senga_diff* diff = nullptr;
};
DevicePtrs g_ptrs[kMaxDevices];
std::mutex g_mutex;

// RK4(3)5[2R+]C coefficients are not needed: the RK epilogue runs in
// "right-hand side only" mode (RK::last = -1).

int setup(int dev, DevicePtrs& out) {
  std::lock_guard<std::mutex> lock(g_mutex);
  DevicePtrs& p = g_ptrs[dev];
  if (!p.ready) {
    cudaError_t e = cudaGetSymbolAddress((void**)&p.scratch, g_noalloc_scratch);
    if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&p.chem, g_noalloc_chem);
    if (e == cudaSuccess) e = cudaGetSymbolAddress((void**)&p.diff, g_noalloc_diff);
    if (e != cudaSuccess)
      return senga::fail(SENGA_ERR_CUDA, std::string("senga_rhs_noalloc: cudaGetSymbolAddress: ") +
                                             cudaGetErrorString(e));
    p.ready = true;
  }
  out = p;
  return SENGA_OK;
}

}  // namespace

extern "C" int senga_rhs_noalloc(const senga_config* cfg, const senga_chem* chem, const senga_diff* diff,
                                 const double* state, double* trun, int32_t* itndex, double* rhs,
                                 unsigned int* status, void* stream) {
  if (!cfg || !chem || !state || !trun || !itndex || !rhs || !status)
    return senga::fail(SENGA_ERR_ARG, "senga_rhs_noalloc: null argument");
  const int nspec = chem->nspec;
  if (nspec < 1 || nspec > SENGA_NSPCMX) return senga::fail(SENGA_ERR_ARG, "senga_rhs_noalloc: nspec out of range");
  const int n3[3] = {cfg->nx, cfg->ny, cfg->nz};
  const double len[3] = {cfg->xgdlen, cfg->ygdlen, cfg->zgdlen};
  senga::Geo g{};
  for (int d = 0; d < 3; ++d) {
    // any periodic extent, as for a context (one point in the unused
    // directions of 1D and 2D runs)
    if (n3[d] < 1) return senga::fail(SENGA_ERR_ARG, "senga_rhs_noalloc: grid extent must be at least 1 point");
    if (cfg->nend[2 * d] != SENGA_NPERI || cfg->nend[2 * d + 1] != SENGA_NPERI)
      return senga::fail(SENGA_ERR_UNSUPPORTED, "senga_rhs_noalloc: periodic boxes only");
    g.per[d] = 1;
    const double delta = len[d] / (double)(float)(n3[d] - 1);
    g.ovd[d] = 1.0 / delta;
    g.ovd2[d] = g.ovd[d] * g.ovd[d];
  }
  g.nx = cfg->nx;
  g.ny = cfg->ny;
  g.nz = cfg->nz;
  g.n = (int64_t)cfg->nx * cfg->ny * cfg->nz;
  const int64_t per_point = 14 + 4 * (int64_t)nspec;
  if (g.n * per_point > (int64_t)kScratchDoubles)
    return senga::fail(SENGA_ERR_ARG, "senga_rhs_noalloc: box of " + std::to_string(g.n) + " points needs " +
                                          std::to_string(g.n * per_point * 8) + " bytes of scratch, limit " +
                                          std::to_string(kScratchBytes));
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return senga::fail(SENGA_ERR_CUDA, std::string("senga_rhs_noalloc: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return senga::fail(SENGA_ERR_ARG, "senga_rhs_noalloc: device ordinal too large");
  cudaStream_t s = (cudaStream_t)stream;
  // the tables go up from pageable host memory on every call: a captured
  // copy node would read the caller's host structs again at each replay,
  // so the call refuses to be captured (checked before the first call's
  // symbol lookup, which a capture would not allow either)
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess) return senga::fail(SENGA_ERR_CUDA, std::string("senga_rhs_noalloc: ") + cudaGetErrorString(e));
  if (cap != cudaStreamCaptureStatusNone)
    return senga::fail(SENGA_ERR_UNSUPPORTED, "senga_rhs_noalloc: the call cannot be captured into a CUDA graph");
  DevicePtrs ptr;
  int rc = setup(dev, ptr);
  if (rc != SENGA_OK) return rc;

  const senga_diff& dz = diff ? *diff : kNoDiff;
  e = cudaMemcpyAsync(ptr.chem, chem, sizeof(senga_chem), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ptr.diff, &dz, sizeof(senga_diff), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return senga::fail(SENGA_ERR_CUDA, std::string("senga_rhs_noalloc: ") + cudaGetErrorString(e));

  // carve the scratch fields; the caller's rhs buffer is the accumulator
  const int64_t n = g.n;
  double* q = ptr.scratch;
  auto take = [&](int64_t k) {
    double* r = q;
    q += k * n;
    return r;
  };
  senga::Fields f{};
  f.uin = const_cast<double*>(state);
  f.uout = nullptr;
  f.run = nullptr;
  f.err = nullptr;
  f.t = trun;
  f.itn = itndex;
  f.p = take(1);
  f.lam = take(1);
  f.lcp = take(1);
  f.mu = take(1);
  f.rd = take(nspec);
  f.h = take(nspec);
  f.hmix = take(1);
  f.wdot = take(nspec);
  f.vel = take(3);
  f.e = take(1);
  f.y = take(nspec);
  f.divm = take(1);
  f.vc = take(3);
  f.vtmp = take(1);
  f.rhs = rhs;
  f.status = status;

  const int flmavt = diff ? diff->flmavt : 0;
  senga::launch_thermo(g, f, ptr.chem, ptr.diff, nspec, flmavt, senga::select_mech(*chem, dz), s);
  senga::launch_flow(g, f, nspec, s);
  senga::launch_species_a(g, f, nspec, s);
  senga::RK rk{0.0, 0.0, 0.0, -1};
  senga::launch_species_b_rk(g, f, nspec, rk, s);
  e = cudaGetLastError();
  if (e != cudaSuccess) return senga::fail(SENGA_ERR_CUDA, std::string("senga_rhs_noalloc: ") + cudaGetErrorString(e));
  return SENGA_OK;
}
