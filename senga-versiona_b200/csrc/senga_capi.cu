// C ABI: device-resident context, state transfer, substage driver.
//
// The reference keeps every field in COMMON and calls, per substage,
// BOUNDT, PARFER, RHSCAL, RHSVEL, BOUNDS, LINCOM/FINCOM (src/senga2.f:113-159).
// Here one context owns the HBM-resident registers and scratch of one box and
// a substage is four kernels on the context's stream:
//   thermo (TEMPER + transport + enthalpy + CHRATE, pointwise)
//   flow   (continuity, momentum, energy convection/conduction/work)
//   species_a, species_b+RK (species equations, correction velocity, LINCOM).
// PARFER's single-rank periodic copy is replaced by index wrapping inside the
// stencils, so no halo exchange runs.
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "senga_gpu.h"
#include "senga_internal.h"

namespace senga {

static thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      throw Error(e_ == cudaErrorMemoryAllocation ? SENGA_ERR_NOMEM : SENGA_ERR_CUDA,         \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                        \
  } while (0)

// RK4(3)5[2R+]C of Kennedy, Carpenter & Lewis: src/dtinit.f:76-94.
static const double kAcof[5] = {970286171893.0 / 4311952581923.0, 6584761158862.0 / 12103376702013.0,
                                2251764453980.0 / 15575788980749.0, 26877169314380.0 / 34165994151039.0, 0.0};
static const double kBcof[5] = {1153189308089.0 / 22510343858157.0, 1772645290293.0 / 4653164025191.0,
                                -1672844663538.0 / 4480602732383.0, 2114624349019.0 / 3568978502595.0,
                                5198255086312.0 / 14908931495163.0};
static const double kBhat[5] = {1016888040809.0 / 7410784769900.0, 11231460423587.0 / 58533540763752.0,
                                -1563879915014.0 / 6823010717585.0, 606302364029.0 / 971179775848.0,
                                1097981568119.0 / 3980877426909.0};

}  // namespace senga

using namespace senga;

struct senga_ctx {
  senga_config cfg{};
  senga_chem chem{};
  senga_diff diff{};
  Geo geo{};
  int nspec = 0, nc = 0;
  cudaStream_t stream = nullptr;
  senga_chem* d_chem = nullptr;
  senga_diff* d_diff = nullptr;
  double* pool = nullptr;
  unsigned int* d_status = nullptr;
  Fields f{};
  double rklhs[5], rkrhs[5], rkerr[5];
  cudaGraphExec_t graph = nullptr;
  int mech = 0;  // thermochemistry policy (select_mech)
  // ADAPTT state (cfg.adaptive): current TSTEP, ERROLD/ERRLDR, last ERRMAX
  double tstep = 0.0, errold = 1.0e-4, errldr = 1.0e-4, errmax = 0.0;
  int inderr = 0, sms = 148;
  unsigned long long* d_errmax = nullptr;
  // molar-mass / pressure / Soret / Dufour transport terms (senga_set_transport)
  bool mixt = false;
  MixtParams mx{};
  double* mixt_pool = nullptr;
  // CHRATE rates of the last RHS evaluation (RRTE), kept on request
  double* rrte = nullptr;
  // radiation heat loss (senga_set_radiation)
  bool rad = false;
  RadParams rp{};
  // NSCBC x faces (senga_set_nscbc)
  bool nscbc = false;
  NscbcParams bc{};
  double* nscbc_pool = nullptr;
  SynthInflow* synth = nullptr;  // synthetic inflow velocity (senga_set_synthetic_inflow)
};

namespace {

void build_geo(const senga_config& c, Geo& g) {
  g.nx = c.nx;
  g.ny = c.ny;
  g.nz = c.nz;
  g.n = (int64_t)c.nx * c.ny * c.nz;
  const int n3[3] = {c.nx, c.ny, c.nz};
  const double len[3] = {c.xgdlen, c.ygdlen, c.zgdlen};
  for (int d = 0; d < 3; ++d) {
    g.per[d] = c.nend[2 * d] == SENGA_NPERI ? 1 : 0;
    // DELTAX = XGDLEN/REAL(NXGLBL-1): spacing L/(N-1) also for periodic boxes
    const double delta = len[d] / (double)(float)(n3[d] - 1);
    g.ovd[d] = 1.0 / delta;
    g.ovd2[d] = g.ovd[d] * g.ovd[d];
  }
}

void check_config(const senga_config& c, int nspec) {
  const int n3[3] = {c.nx, c.ny, c.nz};
  for (int d = 0; d < 3; ++d) {
    const int l = c.nend[2 * d], r = c.nend[2 * d + 1];
    // periodic: any extent (one point for the unused directions of 1D and
    // 2D runs: every derivative there is zero, the filter the identity);
    // bounded: the filter's one-sided rows read 12 points, the closures 11
    if (n3[d] < (l == SENGA_NPERI ? 1 : 12))
      throw Error(SENGA_ERR_ARG, "grid extent must be at least 12 points per bounded direction");
    if ((l == SENGA_NPERI) != (r == SENGA_NPERI))
      throw Error(SENGA_ERR_ARG, "periodic end conditions must be set on both faces of a direction");
    if (l != SENGA_NPERI && (l != SENGA_NBOUND || r != SENGA_NBOUND))
      throw Error(SENGA_ERR_UNSUPPORTED, "a bounded direction takes NBOUND on both of its faces");
  }
  if (c.tstep <= 0.0) throw Error(SENGA_ERR_ARG, "tstep must be positive");
  if (nspec < 1 || nspec > SENGA_NSPCMX) throw Error(SENGA_ERR_ARG, "nspec out of range");
}

void set_rk(senga_ctx* c, double tstep) {
  for (int i = 0; i < 5; ++i) {
    c->rklhs[i] = kBcof[i] * tstep;
    c->rkrhs[i] = kAcof[i] * tstep;
    c->rkerr[i] = (kBcof[i] - kBhat[i]) * tstep;
  }
}

// The right-hand side needs conditions on every bounded face: the x faces
// take NSCBC (senga_set_nscbc); no y or z face conditions are built, so a box
// bounded in y or z serves the operator-level derivatives and the filter only.
void require_rhs(const senga_ctx* c) {
  if (!c->geo.per[1] || !c->geo.per[2])
    throw Error(SENGA_ERR_UNSUPPORTED,
                "bounded y or z direction: only senga_deriv and the filter run on this box (no y/z face conditions)");
  if (!c->geo.per[0] && !c->nscbc)
    throw Error(SENGA_ERR_UNSUPPORTED, "a bounded x direction needs its face conditions (senga_set_nscbc)");
}

// species kernel and species+RK kernel as one launch (launch_species_fused)
bool fused(const senga_ctx* c) {
  return !c->mixt && !c->nscbc && c->nspec <= 9 && species_fusable(c->geo);  // the rates of 9 species fit on chip
}

// the fields the thermochemistry kernel writes: the momentum copy only for
// the fused species kernel
Fields thermo_fields(const senga_ctx* c) {
  Fields f = c->f;
  if (!fused(c)) f.mom = nullptr;
  return f;
}

// Everything of a substage up to the species kernel; with fused species
// kernels that kernel is left to the caller's species+RK launch.
void run_rhs(senga_ctx* c) {
  require_rhs(c);
  if (c->nscbc) launch_boundt(c->geo, c->f, c->bc, c->nspec, false, c->d_chem, c->stream);  // BOUNDT
  launch_thermo(c->geo, thermo_fields(c), c->d_chem, c->d_diff, c->nspec, c->diff.flmavt, c->mech, c->stream);
  if (c->rrte)  // RRTE = RATE (src/rhscal.f:828)
    CK(cudaMemcpyAsync(c->rrte, c->f.wdot, (size_t)c->nspec * c->geo.n * sizeof(double), cudaMemcpyDeviceToDevice,
                       c->stream));
  if (c->nscbc) launch_face(c->geo, c->f, c->bc, c->nspec, c->d_chem, c->stream);  // face data + BOUNDS
  launch_flow(c->geo, c->f, c->nspec, c->stream);
  if (c->rad) launch_radcal(c->geo, c->f, c->rp, c->stream);  // RADCAL
  if (fused(c)) return;
  launch_species_a(c->geo, c->f, c->nspec, c->stream);
  if (c->mixt) launch_mixt(c->geo, c->f, c->mx, c->d_chem, c->d_diff, c->nspec, c->stream);
  if (c->nscbc) launch_wall_flux(c->geo, c->f, c->bc, c->nspec, c->stream);  // W1 wall diffusion flux
}

// the species+RK work after run_rhs (rk.last = -1: the RHS only)
void run_species_rk(senga_ctx* c, const RK& rk) {
  if (fused(c)) launch_species_fused(c->geo, c->f, c->nspec, rk, c->stream);
  else launch_species_b_rk(c->geo, c->f, c->nspec, rk, c->stream);
}

void run_substage(senga_ctx* c, int irk) {
  run_rhs(c);
  RK rk{c->rklhs[irk - 1], c->rkrhs[irk - 1], c->rkerr[irk - 1], irk == 5 ? 1 : 0};
  run_species_rk(c, rk);
  if (c->nscbc) launch_wall_fix(c->geo, c->f, c->bc, c->nspec, true, c->stream);  // W1: LINCOM/FINCOM wall Y
}

// ADAPTT (src/adaptt.f:53-330) after a step: error maxima on the device, the
// PID controller on the host with the constants DTINIT leaves in force
// (src/dtinit.f:99-175), RK coefficients rescaled by TRATIO as the reference
// does (cumulatively), error register zeroed.
void adaptt(senga_ctx* c) {
  const int nc = c->nc;
  ErrNorms nrm{};
  const double base[5] = {0.0, 1.0e-6, 1.0e-6, 1.0e-6, 1.0e-2};
  for (int fl = 0; fl < nc; ++fl) nrm.v[fl] = fl < 5 ? base[fl] : 1.0e-10;
  launch_errmax(c->geo.n, nc, c->f.err, c->f.run, nrm, c->d_errmax, c->sms, c->stream);
  unsigned long long bits[5 + SENGA_NSPCMX];
  CK(cudaMemcpyAsync(bits, c->d_errmax, nc * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemsetAsync(c->f.err, 0, (size_t)nc * c->geo.n * sizeof(double), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  double tot[5 + SENGA_NSPCMX];
  std::memcpy(tot, bits, nc * sizeof(double));
  const double errtol = 1.0e-4, errlow = 1.0e-30, trmax = 1.01, trmin = 1.0e-2, tsmax = 1.0, tsmin = 1.0e-15;
  const double ctmult = 9.0e-1, ctalph = 4.9e-1 / 3.0, ctbeta = 3.4e-1 / 3.0, ctgama = 1.0e-1 / 3.0;
  // field order and strict comparisons of adaptt.f: D(-4), U(-1), V(-2), W(-3), E(0), Y_k(k)
  const int code[5] = {-4, -1, -2, -3, 0};
  double errmax = 0.0;
  for (int fl = 0; fl < nc; ++fl)
    if (tot[fl] > errmax) {
      errmax = tot[fl];
      c->inderr = fl < 5 ? code[fl] : fl - 4;
    }
  if (errmax < errlow) errmax = errlow;
  c->errmax = errmax;
  double tratio = ctmult * std::exp(ctalph * std::log(errtol / errmax) + ctbeta * std::log(c->errold / errtol) +
                                    ctgama * std::log(errtol / c->errldr));
  c->errldr = c->errold;
  c->errold = errmax;
  if (tratio > trmax) tratio = trmax;
  if (tratio < trmin) tratio = trmin;
  const double tstold = c->tstep;
  c->tstep = c->tstep * tratio;
  if (c->tstep > tsmax) c->tstep = tsmax;
  if (c->tstep < tsmin) c->tstep = tsmin;
  tratio = c->tstep / tstold;
  for (int i = 0; i < 5; ++i) {
    c->rklhs[i] = c->rklhs[i] * tratio;
    c->rkrhs[i] = c->rkrhs[i] * tratio;
    c->rkerr[i] = c->rkerr[i] * tratio;
  }
}

template <class Fn>
int guard(Fn&& fn) {
  try {
    fn();
    return SENGA_OK;
  } catch (const Error& e) {
    return fail(e.code, e.what());
  } catch (const std::exception& e) {
    return fail(SENGA_ERR_CUDA, e.what());
  }
}

}  // namespace

extern "C" {

const char* senga_last_error(void) { return g_last_error.c_str(); }

int senga_ctx_create(const senga_config* cfg, const senga_chem* chem, const senga_diff* diff, senga_ctx** out) {
  if (!cfg || !chem || !out) return fail(SENGA_ERR_ARG, "senga_ctx_create: null argument");
  *out = nullptr;
  senga_ctx* c = new senga_ctx();
  int rc = guard([&] {
    c->cfg = *cfg;
    c->chem = *chem;
    if (diff) c->diff = *diff;
    else std::memset(&c->diff, 0, sizeof(c->diff));
    c->nspec = chem->nspec;
    c->nc = 5 + c->nspec;
    check_config(*cfg, c->nspec);
    build_geo(*cfg, c->geo);
    set_rk(c, cfg->tstep);
    c->mech = select_mech(c->chem, c->diff);
    CK(cudaSetDevice(cfg->device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaMalloc(&c->d_chem, sizeof(senga_chem)));
    CK(cudaMalloc(&c->d_diff, sizeof(senga_diff)));
    CK(cudaMemcpy(c->d_chem, &c->chem, sizeof(senga_chem), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_diff, &c->diff, sizeof(senga_diff), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->d_status, sizeof(unsigned int)));
    CK(cudaMalloc(&c->d_errmax, (5 + SENGA_NSPCMX) * sizeof(unsigned long long)));
    CK(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, cfg->device));
    c->tstep = cfg->tstep;
    CK(cudaMemset(c->d_status, 0, sizeof(unsigned int)));
    const int64_t n = c->geo.n;
    const int S = c->nspec, nc = c->nc;
    // pool layout (doubles): run nc | u nc | err nc? | t | p lam lcp mu | rd S | h S |
    // hmix | wdot S | vel 3 | e | y S | rhs nc | divm | vc 3 | vtmp | mom 3 | itn (int32 words)
    const int64_t per_point = (int64_t)nc * 2 + (cfg->adaptive ? nc : 0) + 1 + 4 + 3 * S + 1 + 3 + 1 + S + nc + 1 + 3 + 1 + 3;
    const int64_t total = per_point * n + (itn_words(S) * n + 1) / 2 + 64;
    CK(cudaMalloc(&c->pool, (size_t)total * sizeof(double)));
    CK(cudaMemsetAsync(c->pool, 0, (size_t)total * sizeof(double), c->stream));
    double* p = c->pool;
    auto take = [&](int64_t k) {
      double* r = p;
      p += k * n;
      return r;
    };
    Fields& f = c->f;
    f.run = take(nc);
    f.uin = take(nc);
    f.uout = f.uin;  // the RK epilogue reads no neighbour of the U register
    f.err = cfg->adaptive ? take(nc) : nullptr;
    f.t = take(1);
    f.p = take(1);
    f.lam = take(1);
    f.lcp = take(1);
    f.mu = take(1);
    f.rd = take(S);
    f.h = take(S);
    f.hmix = take(1);
    f.wdot = take(S);
    f.vel = take(3);
    f.e = take(1);
    f.y = take(S);
    f.rhs = take(nc);
    f.divm = take(1);
    f.vc = take(3);
    f.vtmp = take(1);
    f.mom = take(3);
    f.itn = reinterpret_cast<int32_t*>(p);
    f.status = c->d_status;
    CK(cudaStreamSynchronize(c->stream));
  });
  if (rc != SENGA_OK) {
    senga_ctx_destroy(c);
    return rc;
  }
  *out = c;
  return SENGA_OK;
}

int senga_ctx_destroy(senga_ctx* c) {
  if (!c) return SENGA_OK;
  if (c->graph) cudaGraphExecDestroy(c->graph);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->pool);
  cudaFree(c->d_chem);
  cudaFree(c->d_diff);
  cudaFree(c->d_status);
  cudaFree(c->d_errmax);
  cudaFree(c->nscbc_pool);
  synth_destroy(c->synth);
  cudaFree(c->mixt_pool);
  cudaFree(c->rrte);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return SENGA_OK;
}

int senga_sync(senga_ctx* c) {
  if (!c) return fail(SENGA_ERR_ARG, "null context");
  return guard([&] { CK(cudaStreamSynchronize(c->stream)); });
}

void* senga_stream(senga_ctx* c) { return c ? (void*)c->stream : nullptr; }

int senga_upload_state_host(senga_ctx* c, const double* fields, const double* trun, const int32_t* itn) {
  if (!c || !fields || !trun || !itn) return fail(SENGA_ERR_ARG, "senga_upload_state_host: null argument");
  return guard([&] {
    const size_t bytes = (size_t)c->nc * c->geo.n * sizeof(double);
    CK(cudaMemcpyAsync(c->f.run, fields, bytes, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->f.uin, c->f.run, bytes, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->f.t, trun, c->geo.n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->f.itn, itn, itn_words(c->nspec) * c->geo.n * sizeof(int32_t), cudaMemcpyHostToDevice,
                       c->stream));
    if (c->f.err) CK(cudaMemsetAsync(c->f.err, 0, bytes, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int senga_upload_state_async(senga_ctx* c, const double* fields, const double* trun, const int32_t* itn) {
  if (!c || !fields || !trun || !itn) return fail(SENGA_ERR_ARG, "senga_upload_state_async: null argument");
  return guard([&] {
    const size_t bytes = (size_t)c->nc * c->geo.n * sizeof(double);
    CK(cudaMemcpyAsync(c->f.run, fields, bytes, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->f.uin, c->f.run, bytes, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->f.t, trun, c->geo.n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->f.itn, itn, itn_words(c->nspec) * c->geo.n * sizeof(int32_t), cudaMemcpyHostToDevice,
                       c->stream));
    if (c->f.err) CK(cudaMemsetAsync(c->f.err, 0, bytes, c->stream));
  });
}

int senga_download_state_async(senga_ctx* c, double* fields, double* trun, int32_t* itn) {
  if (!c || !fields) return fail(SENGA_ERR_ARG, "senga_download_state_async: null argument");
  return guard([&] {
    const size_t bytes = (size_t)c->nc * c->geo.n * sizeof(double);
    CK(cudaMemcpyAsync(fields, c->f.run, bytes, cudaMemcpyDeviceToHost, c->stream));
    if (trun) CK(cudaMemcpyAsync(trun, c->f.t, c->geo.n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (itn)
      CK(cudaMemcpyAsync(itn, c->f.itn, itn_words(c->nspec) * c->geo.n * sizeof(int32_t), cudaMemcpyDeviceToHost,
                         c->stream));
  });
}

int senga_download_state_host(senga_ctx* c, double* fields, double* trun, int32_t* itn) {
  if (!c || !fields) return fail(SENGA_ERR_ARG, "senga_download_state_host: null argument");
  return guard([&] {
    const size_t bytes = (size_t)c->nc * c->geo.n * sizeof(double);
    CK(cudaMemcpyAsync(fields, c->f.run, bytes, cudaMemcpyDeviceToHost, c->stream));
    if (trun) CK(cudaMemcpyAsync(trun, c->f.t, c->geo.n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (itn)
      CK(cudaMemcpyAsync(itn, c->f.itn, itn_words(c->nspec) * c->geo.n * sizeof(int32_t), cudaMemcpyDeviceToHost,
                         c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int senga_substage(senga_ctx* c, int irkstp) {
  if (!c || irkstp < 1 || irkstp > 5) return fail(SENGA_ERR_ARG, "senga_substage: bad argument");
  return guard([&] {
    if (irkstp == 1 && c->synth) synth_step(c->synth, c->cfg.xgdlen, c->geo.nx, c->tstep, c->bc, c->stream);
    run_substage(c, irkstp);
    CK(cudaGetLastError());
  });
}

int senga_step(senga_ctx* c, int nsteps) {
  if (!c || nsteps < 0) return fail(SENGA_ERR_ARG, "senga_step: bad argument");
  return guard([&] {
    for (int s = 0; s < nsteps; ++s) {
      // INFLOW ahead of the substages (src/senga2.f:100-103)
      if (c->synth) synth_step(c->synth, c->cfg.xgdlen, c->geo.nx, c->tstep, c->bc, c->stream);
      for (int irk = 1; irk <= 5; ++irk) run_substage(c, irk);
      if (c->nscbc) launch_boundt(c->geo, c->f, c->bc, c->nspec, true, c->d_chem, c->stream);  // BOUNTT
      if (c->cfg.adaptive) adaptt(c);
    }
    CK(cudaGetLastError());
  });
}

int senga_step_graph(senga_ctx* c, int nsteps) {
  if (!c || nsteps < 0) return fail(SENGA_ERR_ARG, "senga_step_graph: bad argument");
  // dt changes every step, or the synthetic inflow draws its planes on the
  // host every step: no fixed graph
  if (c->cfg.adaptive || c->synth) return senga_step(c, nsteps);
  return guard([&] {
    if (!c->graph) {
      require_rhs(c);  // before the capture, so a refusal leaves the stream uncaptured
      cudaGraph_t gr;
      CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      for (int irk = 1; irk <= 5; ++irk) run_substage(c, irk);
      if (c->nscbc) launch_boundt(c->geo, c->f, c->bc, c->nspec, true, c->d_chem, c->stream);  // BOUNTT
      CK(cudaStreamEndCapture(c->stream, &gr));
      CK(cudaGraphInstantiate(&c->graph, gr, 0));
      CK(cudaGraphDestroy(gr));
    }
    for (int s = 0; s < nsteps; ++s) CK(cudaGraphLaunch(c->graph, c->stream));
    CK(cudaGetLastError());
  });
}

int senga_rhs_host(senga_ctx* c, double* rhs, double* trun, double* prun) {
  if (!c || !rhs) return fail(SENGA_ERR_ARG, "senga_rhs_host: null argument");
  return guard([&] {
    run_rhs(c);
    RK rk{0.0, 0.0, 0.0, -1};  // last = -1: write R(U) into the rhs fields only
    run_species_rk(c, rk);
    if (c->nscbc) launch_wall_fix(c->geo, c->f, c->bc, c->nspec, false, c->stream);  // BOUNDS: wall T
    CK(cudaGetLastError());
    const int64_t n = c->geo.n;
    CK(cudaMemcpyAsync(rhs, c->f.rhs, (size_t)c->nc * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (trun) CK(cudaMemcpyAsync(trun, c->f.t, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (prun) CK(cudaMemcpyAsync(prun, c->f.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int senga_profile_step(senga_ctx* c, double* ms, int* launches) {
  if (!c || !ms) return fail(SENGA_ERR_ARG, "senga_profile_step: null argument");
  return guard([&] {
    require_rhs(c);
    cudaEvent_t ev[21];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    for (int k = 0; k < 4; ++k) ms[k] = 0.0;
    int nl = 0;
    // the face kernels of an NSCBC box are timed with the kernel they follow
    const bool imposed = c->nscbc && (c->bc.xl == 12 || c->bc.xl == 13 || c->bc.xr == 12 || c->bc.xr == 13 ||
                                      has_wall(c->bc));
    const bool wall = c->nscbc && has_wall(c->bc);
    const int nface = c->nscbc ? 1 + (imposed ? 1 : 0) + (wall ? 2 : 0) : 0;
    for (int irk = 1; irk <= 5; ++irk) {
      const int b = (irk - 1) * 4;
      CK(cudaEventRecord(ev[b], c->stream));
      if (c->nscbc) launch_boundt(c->geo, c->f, c->bc, c->nspec, false, c->d_chem, c->stream);
      const int nth =
          launch_thermo(c->geo, thermo_fields(c), c->d_chem, c->d_diff, c->nspec, c->diff.flmavt, c->mech, c->stream);
      CK(cudaEventRecord(ev[b + 1], c->stream));
      if (c->nscbc) launch_face(c->geo, c->f, c->bc, c->nspec, c->d_chem, c->stream);
      launch_flow(c->geo, c->f, c->nspec, c->stream);
      if (c->rad) launch_radcal(c->geo, c->f, c->rp, c->stream);
      CK(cudaEventRecord(ev[b + 2], c->stream));
      RK rk{c->rklhs[irk - 1], c->rkrhs[irk - 1], c->rkerr[irk - 1], irk == 5 ? 1 : 0};
      // fused species kernels: the one launch is timed as the species
      // kernel, the species+RK interval is then empty
      if (fused(c)) launch_species_fused(c->geo, c->f, c->nspec, rk, c->stream);
      else launch_species_a(c->geo, c->f, c->nspec, c->stream);
      const int nmx = c->mixt ? launch_mixt(c->geo, c->f, c->mx, c->d_chem, c->d_diff, c->nspec, c->stream) : 0;
      if (c->nscbc) launch_wall_flux(c->geo, c->f, c->bc, c->nspec, c->stream);
      CK(cudaEventRecord(ev[b + 3], c->stream));
      if (!fused(c)) launch_species_b_rk(c->geo, c->f, c->nspec, rk, c->stream);
      if (c->nscbc) launch_wall_fix(c->geo, c->f, c->bc, c->nspec, true, c->stream);
      if (irk == 5 && imposed) launch_boundt(c->geo, c->f, c->bc, c->nspec, true, c->d_chem, c->stream);  // BOUNTT
      CK(cudaEventRecord(irk < 5 ? ev[b + 4] : ev[20], c->stream));
      nl += (fused(c) ? 2 : 3) + nth + (c->rad ? 1 : 0) + nmx + nface + (irk == 5 && imposed ? 1 : 0);
    }
    CK(cudaStreamSynchronize(c->stream));
    for (int irk = 1; irk <= 5; ++irk) {
      const int b = (irk - 1) * 4;
      for (int k = 0; k < 4; ++k) {
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, ev[b + k], (b + k + 1 < 20) ? ev[b + k + 1] : ev[20]));
        ms[k] += t;
      }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (launches) *launches = nl;
  });
}

int senga_ctx_species_fused(senga_ctx* c, int* fused_kernels) {
  if (!c || !fused_kernels) return fail(SENGA_ERR_ARG, "senga_ctx_species_fused: null argument");
  *fused_kernels = fused(c) ? 1 : 0;
  return SENGA_OK;
}

int senga_ctx_species_mma(senga_ctx* c, int* mma) {
  if (!c || !mma) return fail(SENGA_ERR_ARG, "senga_ctx_species_mma: null argument");
  *mma = !fused(c) && species_mma_ok(c->geo, c->f, ZDec{}) ? 1 : 0;
  return SENGA_OK;
}

int senga_ctx_info(senga_ctx* c, int* mech, int64_t* device_bytes) {
  if (!c) return fail(SENGA_ERR_ARG, "senga_ctx_info: null context");
  if (mech) *mech = c->mech;
  if (device_bytes) {
    size_t bytes = 0;
    cudaPointerAttributes a;
    (void)a;
    const int64_t n = c->geo.n;
    const int S = c->nspec, nc = c->nc;
    bytes = (size_t)((int64_t)(3 * nc + 4 * S + 18 + (c->cfg.adaptive ? nc : 0)) * n + (n + 1) / 2 + 64) * sizeof(double);
    *device_bytes = (int64_t)bytes;
  }
  return SENGA_OK;
}

int senga_get_status(senga_ctx* c, int* status) {
  if (!c || !status) return fail(SENGA_ERR_ARG, "senga_get_status: null argument");
  return guard([&] {
    unsigned int s = 0;
    CK(cudaMemcpyAsync(&s, c->d_status, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *status = (int)s;
  });
}

int senga_flamin(senga_ctx* c, double trin, double prin, double drin, double urin, const double* v,
                 const double* w) {
  if (!c) return fail(SENGA_ERR_ARG, "senga_flamin: null context");
  if (c->nspec < 2) return fail(SENGA_ERR_ARG, "senga_flamin: needs at least two species");
  if (!(trin > 0.0) || !(prin > 0.0)) return fail(SENGA_ERR_ARG, "senga_flamin: trin and prin must be positive");
  return guard([&] {
    const int64_t n = c->geo.n;
    struct Staged {  // v and w on the device for the one launch, freed on every path
      double* p = nullptr;
      ~Staged() { if (p) cudaFree(p); }
    } dv, dw;
    if (v) CK(cudaMalloc(&dv.p, n * sizeof(double)));
    if (w) CK(cudaMalloc(&dw.p, n * sizeof(double)));
    if (v) CK(cudaMemcpyAsync(dv.p, v, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (w) CK(cudaMemcpyAsync(dw.p, w, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    launch_flamin(c->geo, c->nspec, c->cfg.xgdlen, trin, prin, drin, urin, c->d_chem, dv.p, dw.p, c->f.run, c->f.uin,
                  c->f.t, c->f.itn, c->stream);
    CK(cudaGetLastError());
    if (c->f.err) CK(cudaMemsetAsync(c->f.err, 0, (size_t)c->nc * n * sizeof(double), c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int senga_tempin_host(senga_ctx* c, double trin, double* trun, int32_t* itndex, double* prun) {
  if (!c) return fail(SENGA_ERR_ARG, "senga_tempin_host: null context");
  if (!(trin > 0.0)) return fail(SENGA_ERR_ARG, "senga_tempin_host: trin must be a positive temperature");
  return guard([&] {
    const int64_t n = c->geo.n;
    launch_tempin(n, c->nspec, c->f.uin, c->d_chem, trin, c->f.t, c->f.itn, c->f.p, c->d_status, c->stream);
    CK(cudaGetLastError());
    if (trun) CK(cudaMemcpyAsync(trun, c->f.t, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (itndex)
      CK(cudaMemcpyAsync(itndex, c->f.itn, itn_words(c->nspec) * n * sizeof(int32_t), cudaMemcpyDeviceToHost,
                         c->stream));
    if (prun) CK(cudaMemcpyAsync(prun, c->f.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int senga_deriv(senga_ctx* c, int kind, const double* f, double* out) {
  if (!c || !f || !out || kind < 0 || kind > 8) return fail(SENGA_ERR_ARG, "senga_deriv: bad argument");
  return guard([&] {
    launch_deriv(c->geo, kind, f, out, c->stream);
    CK(cudaGetLastError());
  });
}

int senga_deriv_host(senga_ctx* c, int kind, const double* f, double* out) {
  if (!c || !f || !out || kind < 0 || kind > 8) return fail(SENGA_ERR_ARG, "senga_deriv_host: bad argument");
  return guard([&] {
    const size_t bytes = c->geo.n * sizeof(double);
    // the context's rhs scratch holds the operand and the result
    double* din = c->f.rhs;
    double* dout = c->f.rhs + c->geo.n;
    CK(cudaMemcpyAsync(din, f, bytes, cudaMemcpyHostToDevice, c->stream));
    launch_deriv(c->geo, kind, din, dout, c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int senga_deriv_big(senga_ctx* c, int kind, const double* f_big, double* out) {
  if (!c || !f_big || !out || kind < 0 || kind > 8) return fail(SENGA_ERR_ARG, "senga_deriv_big: bad argument");
  return guard([&] {
    launch_deriv_big(c->geo, kind, f_big, out, c->stream);
    CK(cudaGetLastError());
  });
}

int senga_deriv_big_host(senga_ctx* c, int kind, const double* f_big, double* out) {
  if (!c || !f_big || !out || kind < 0 || kind > 8) return fail(SENGA_ERR_ARG, "senga_deriv_big_host: bad argument");
  return guard([&] {
    const Geo& g = c->geo;
    const size_t nbig = (size_t)(g.nx + 10) * (g.ny + 10) * (g.nz + 10);
    // the context's rhs scratch (nc interior arrays) holds operand and
    // result when the halo-extended array fits beside one interior array;
    // thin boxes (a 1D run's 1 x 1 planes) take a temporary buffer
    double* tmp = nullptr;
    double* din = c->f.rhs;
    double* dout = c->f.rhs + nbig;
    if (nbig + (size_t)g.n > (size_t)c->nc * (size_t)g.n) {
      CK(cudaMalloc(&tmp, (nbig + (size_t)g.n) * sizeof(double)));
      din = tmp;
      dout = tmp + nbig;
    }
    cudaError_t e = cudaMemcpyAsync(din, f_big, nbig * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
      launch_deriv_big(g, kind, din, dout, c->stream);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, (size_t)g.n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (tmp) cudaFree(tmp);
    CK(e);
  });
}

int senga_keep_rates(senga_ctx* c, int on) {
  if (!c) return fail(SENGA_ERR_ARG, "senga_keep_rates: null context");
  return guard([&] {
    CK(cudaStreamSynchronize(c->stream));
    if (on && !c->rrte) {
      CK(cudaMalloc(&c->rrte, (size_t)c->nspec * c->geo.n * sizeof(double)));
      CK(cudaMemset(c->rrte, 0, (size_t)c->nspec * c->geo.n * sizeof(double)));
    } else if (!on && c->rrte) {
      cudaFree(c->rrte);
      c->rrte = nullptr;
    }
    if (c->graph) {
      cudaGraphExecDestroy(c->graph);
      c->graph = nullptr;
    }
  });
}

int senga_post_fields_host(senga_ctx* c, double* out) {
  if (!c || !out) return fail(SENGA_ERR_ARG, "senga_post_fields_host: null argument");
  if (!c->rrte) return fail(SENGA_ERR_ARG, "senga_post_fields_host: RRTE needs senga_keep_rates(ctx, 1) before the step");
  return guard([&] {
    const int64_t n = c->geo.n;
    const size_t prim = (size_t)(7 + c->nspec) * n;
    double* d = nullptr;
    CK(cudaMalloc(&d, prim * sizeof(double)));
    launch_post(n, c->nspec, c->f.run, c->f.t, c->f.p, d, c->stream);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, prim * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out + prim, c->rrte, (size_t)c->nspec * n * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d);
    CK(e);
  });
}

int senga_set_transport(senga_ctx* c, int mixw, int mixp, int soret, int dufour, double wmltdr) {
  if (!c) return fail(SENGA_ERR_ARG, "senga_set_transport: null context");
  return guard([&] {
    if ((mixw || mixp || soret || dufour) && !c->diff.flmavt)
      throw Error(SENGA_ERR_ARG, "senga_set_transport: the switches need mixture-averaged transport (diff.dat)");
    CK(cudaStreamSynchronize(c->stream));
    cudaFree(c->mixt_pool);
    c->mixt_pool = nullptr;
    c->mx = MixtParams{};
    c->mixt = false;
    if (c->graph) {
      cudaGraphExecDestroy(c->graph);
      c->graph = nullptr;
    }
    if (!(mixw || mixp || soret || dufour)) return;
    MixtParams m{};
    m.w = mixw ? 1 : 0;
    m.p = mixp ? 1 : 0;
    m.t = (soret || dufour) ? 1 : 0;
    // light species: W_k <= WMLTDR + WMLTOL, WMLTOL = 1e-3 (src/diffin.f:34,390-405)
    for (int k = 0; k < c->nspec; ++k) {
      if (c->chem.wmolar[k] > wmltdr + 1.0e-3) continue;
      if (soret) m.sor |= 1u << k;
      if (dufour) m.duf |= 1u << k;
      if (soret || dufour) m.tdr |= 1u << k;
    }
    const int64_t n = c->geo.n;
    const int nb = m.w + m.p + m.t;
    const int64_t fields = 1 + 5 * (int64_t)nb + (m.tdr ? c->nspec : 0);
    CK(cudaMalloc(&c->mixt_pool, (size_t)(fields * n) * sizeof(double)));
    double* p = c->mixt_pool;
    m.wmix = p;
    p += n;
    const int on[3] = {m.w, m.p, m.t};
    for (int b = 0; b < 3; ++b) {
      if (!on[b]) continue;
      m.lng[b] = p;
      m.g1[b] = p + n;
      m.g2[b] = p + 4 * n;
      p += 5 * n;
    }
    if (m.tdr) m.tdrmix = p;
    c->mx = m;
    c->mixt = true;
  });
}

int senga_set_radiation(senga_ctx* c, const senga_radn* r) {
  if (!c) return fail(SENGA_ERR_ARG, "senga_set_radiation: null context");
  if (!r) {
    c->rad = false;
  } else {
    if (r->nsprad < 0 || r->nsprad > SENGA_NSPCMX) return fail(SENGA_ERR_ARG, "senga_set_radiation: bad nsprad");
    RadParams p{};
    p.nsprad = r->nsprad;
    for (int j = 0; j < r->nsprad; ++j) {
      if (r->nsprid[j] < 1 || r->nsprid[j] > c->nspec || r->nkprad[j] < 1 || r->nkprad[j] > SENGA_NCFRMX)
        return fail(SENGA_ERR_ARG, "senga_set_radiation: bad radiating species record");
      p.id[j] = r->nsprid[j] - 1;
      p.nk[j] = r->nkprad[j];
      for (int k = 0; k < r->nkprad[j]; ++k) p.ak[j][k] = r->akprad[j][k];
      p.rg[j] = c->chem.rgspec[p.id[j]];
    }
    p.foursb = 4.0 * 5.67037321e-08;  // FOUR*STEFBO, src/radcin.f; STEFBO of src/com_senga2.h:222
    p.trfrth = r->trefrn * r->trefrn * r->trefrn * r->trefrn;
    c->rp = p;
    c->rad = true;
  }
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  return SENGA_OK;
}

int senga_set_nscbc(senga_ctx* c, const senga_nscbc* b) {
  if (!c || !b) return fail(SENGA_ERR_ARG, "senga_set_nscbc: null argument");
  auto kind_ok = [](int k) { return k == 11 || k == 12 || k == 13 || k == 14 || k == 21 || k == 31 || k == 32; };
  auto inflow = [](int k) { return k == 11 || k == 12 || k == 13 || k == 14; };
  auto either = [b](int k) { return b->xl == k || b->xr == k; };
  if (!kind_ok(b->xl) || !kind_ok(b->xr) || (inflow(b->xl) && inflow(b->xr)))
    return fail(SENGA_ERR_UNSUPPORTED, "senga_set_nscbc: built face kinds are I1 (11), I2 (12), I3 (13), I4 (14, "
                                       "x-left), O1 (21), W1 (31) and W2 (32), inflow on one x face at most");
  if (b->xr == 14)
    return fail(SENGA_ERR_UNSUPPORTED, "senga_set_nscbc: the I4 inflow is coded for the x-left face only");
  if (b->xl == 14 && !(b->t_in > 0.0)) return fail(SENGA_ERR_ARG, "senga_set_nscbc: an I4 inflow needs t_in > 0");
  if (either(12) && !(b->t_in > 0.0)) return fail(SENGA_ERR_ARG, "senga_set_nscbc: an I2 inflow needs t_in > 0");
  if (c->geo.per[0] || b->xl == 0 || b->xr == 0)
    return fail(SENGA_ERR_ARG, "senga_set_nscbc: needs a bounded x direction and a kind on both x faces");
  if (either(13) && b->rho_in <= 0.0) return fail(SENGA_ERR_ARG, "senga_set_nscbc: an I3 inflow needs rho_in > 0");
  if (either(21) && b->p_inf <= 0.0) return fail(SENGA_ERR_ARG, "senga_set_nscbc: an O1 outflow needs p_inf > 0");
  if ((b->xl == 32 && !(b->t_wall[0] > 0.0)) || (b->xr == 32 && !(b->t_wall[1] > 0.0)))
    return fail(SENGA_ERR_ARG, "senga_set_nscbc: a W2 wall needs its t_wall > 0");
  return guard([&] {
    NscbcParams& p = c->bc;
    p = NscbcParams{};
    p.xl = b->xl;
    p.xr = b->xr;
    p.u_in = b->u_in;
    p.rho_in = b->rho_in;
    for (int s = 0; s < c->nspec; ++s) p.y_in[s] = b->y_in[s];
    p.p_inf = b->p_inf;
    p.cobc = b->sigma * (1.0 - b->eta) / (2.0 * c->cfg.xgdlen);  // COBCXL/COBCXR, src/bcinit.f:309,324
    p.bet = 0.050;                                               // BET default, src/bounds.f:103
    p.xlen = c->cfg.xgdlen;
    p.pio = b->pio;
    p.betloc = b->bet_local;
    p.t_in = b->t_in;
    p.t_wall[0] = b->t_wall[0];
    p.t_wall[1] = b->t_wall[1];
    for (int k = 0; k < 6; ++k) p.nrieta[k] = b->nrieta[k];
    // face-plane flags of src/bcinit.f:299-326,396-407,458-480,560-586,653-666,
    // 702-735,822-855: I1, I4 -> FxxCNV, FxxVSN, every field integrated; I3 ->
    // FxxCNV, FxxVSN, the plane imposed; I2 -> FxxCNV, all but the density
    // imposed; O1 -> FxxCNV, FxxVST, FxxCON, FxxADB, FxxDIF; W1 -> FxxCNV,
    // FxxCON, FxxADB, FxxDIF, FxxCNW, FxxDFW, momentum not integrated; W2
    // -> FxxCNV, FxxDIF, FxxDFW, momentum and energy not integrated
    auto bits = [](int kind) {
      return kind == 11 || kind == 14 ? (BF_VSN | BF_NSCBC)
             : kind == 13 ? (BF_VSN | BF_NSCBC | BF_IMPOSED)
             : kind == 12 ? (BF_NSCBC | BF_IMPOSED_D)
             : kind == 31 ? (BF_CON | BF_DIF | BF_NSCBC | BF_WALL)
             : kind == 32 ? (BF_DIF | BF_NSCBC | BF_WALL)
                          : (BF_VST | BF_CON | BF_DIF | BF_NSCBC);
    };
    c->geo.bxl = bits(b->xl);
    c->geo.bxr = bits(b->xr);
    if (!c->nscbc_pool) {
      const int64_t n = c->geo.n, nyz = (int64_t)c->geo.ny * c->geo.nz;
      CK(cudaMalloc(&c->nscbc_pool, (size_t)(2 * n + 2 * c->nc * nyz) * sizeof(double)));
      CK(cudaMemsetAsync(c->nscbc_pool, 0, (size_t)(2 * n + 2 * c->nc * nyz) * sizeof(double), c->stream));
      c->f.cp = c->nscbc_pool;
      c->f.rmix = c->nscbc_pool + n;
      c->f.face = c->nscbc_pool + 2 * n;
    }
    c->nscbc = true;
    if (c->graph) {
      cudaGraphExecDestroy(c->graph);
      c->graph = nullptr;
    }
    CK(cudaStreamSynchronize(c->stream));
  });
}

int senga_get_tstep(senga_ctx* c, double* tstep, double* errmax, int* inderr) {
  if (!c) return fail(SENGA_ERR_ARG, "senga_get_tstep: null context");
  if (tstep) *tstep = c->tstep;
  if (errmax) *errmax = c->errmax;
  if (inderr) *inderr = c->inderr;
  return SENGA_OK;
}

int senga_filter(senga_ctx* c, int mode) {
  if (!c || mode < 0 || mode > 3) return fail(SENGA_ERR_ARG, "senga_filter: bad argument");
  return guard([&] {
    const FilterCoef cf = filter_coef(mode & 1);
    const int64_t n = c->geo.n;
    double* t1 = c->f.rhs;  // free between steps
    double* t2 = c->f.rhs + n;
    for (int fl = 0; fl < c->nc; ++fl) launch_filter_field(c->geo, c->f.uin + fl * n, c->f.uin + fl * n, t1, t2, cf, c->stream);
    if (mode & 2)
      for (int fl = 0; fl < c->nc; ++fl)
        launch_filter_field(c->geo, c->f.run + fl * n, c->f.run + fl * n, t1, t2, cf, c->stream);
    CK(cudaGetLastError());
  });
}

int senga_filter_field_host(senga_ctx* c, int mode, const double* f, double* out) {
  if (!c || !f || !out || mode < 0 || mode > 3) return fail(SENGA_ERR_ARG, "senga_filter_field_host: bad argument");
  return guard([&] {
    const int64_t n = c->geo.n;
    const size_t bytes = n * sizeof(double);
    double* a = c->f.rhs;
    double* t1 = c->f.rhs + n;
    double* t2 = c->f.rhs + 2 * n;
    CK(cudaMemcpyAsync(a, f, bytes, cudaMemcpyHostToDevice, c->stream));
    launch_filter_field(c->geo, a, a, t1, t2, filter_coef(mode & 1), c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, a, bytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int senga_temper_host(senga_ctx* c, double* trun, double* prun) {
  if (!c) return fail(SENGA_ERR_ARG, "null context");
  return guard([&] {
    launch_thermo(c->geo, thermo_fields(c), c->d_chem, c->d_diff, c->nspec, c->diff.flmavt, c->mech, c->stream);
    CK(cudaGetLastError());
    const int64_t n = c->geo.n;
    if (trun) CK(cudaMemcpyAsync(trun, c->f.t, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (prun) CK(cudaMemcpyAsync(prun, c->f.p, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int senga_chrate_host(senga_ctx* c, double* rate) {
  if (!c || !rate) return fail(SENGA_ERR_ARG, "senga_chrate_host: null argument");
  return guard([&] {
    launch_thermo(c->geo, thermo_fields(c), c->d_chem, c->d_diff, c->nspec, c->diff.flmavt, c->mech, c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(rate, c->f.wdot, (size_t)c->nspec * c->geo.n * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// A box split along z into slabs, one context each (one GPU each, or several
// on one GPU). The stencil kernels of a slab read their z halo straight from
// the neighbouring slabs' registers (peer loads over NVLink between GPUs);
// between the phases that write what the others read, every slab's stream
// waits for the others' events: after TEMPER/CHRATE (T, p, Y, transport read
// in halos), after the species kernel (the flow and species kernels read the
// U register that the RK update then overwrites in place), and after the RK
// update (the next substage reads it).
struct senga_zgroup {
  int nr = 0, nx = 0, ny = 0, nzg = 0, nzl = 0, nc = 0;
  senga_ctx* ctx[kMaxZRanks] = {};
  ZDec zd[kMaxZRanks];
  cudaEvent_t ev[kMaxZRanks] = {};
};

namespace {

// restores the caller's current device when a group call returns
struct DeviceGuard {
  int dev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
  }
  ~DeviceGuard() {
    if (dev >= 0) cudaSetDevice(dev);
  }
};

void zgroup_barrier(senga_zgroup* g) {
  for (int r = 0; r < g->nr; ++r) {
    CK(cudaSetDevice(g->ctx[r]->cfg.device));
    CK(cudaEventRecord(g->ev[r], g->ctx[r]->stream));
  }
  for (int r = 0; r < g->nr; ++r) {
    CK(cudaSetDevice(g->ctx[r]->cfg.device));
    for (int q = 0; q < g->nr; ++q)
      if (q != r) CK(cudaStreamWaitEvent(g->ctx[r]->stream, g->ev[q], 0));
  }
}

void zgroup_destroy(senga_zgroup* g) {
  for (int r = 0; r < g->nr; ++r) {
    if (g->ev[r]) cudaEventDestroy(g->ev[r]);
    senga_ctx_destroy(g->ctx[r]);
  }
  delete g;
}

}  // namespace

int senga_zgroup_create(const senga_config* cfg, const senga_chem* chem, const senga_diff* diff, int nslabs,
                        const int* devices, senga_zgroup** out) {
  if (!cfg || !chem || !diff || !out || nslabs < 1 || nslabs > kMaxZRanks)
    return fail(SENGA_ERR_ARG, "senga_zgroup_create: bad argument (1..16 slabs)");
  // y and z periodic; x periodic, or bounded on both faces with NSCBC face
  // conditions (senga_zgroup_set_nscbc), whose face kernels read only their
  // own slab's face planes
  for (int k = 2; k < 6; ++k)
    if (cfg->nend[k] != SENGA_NPERI)
      return fail(SENGA_ERR_UNSUPPORTED, "senga_zgroup_create: z-split boxes must be periodic in y and z");
  if (!((cfg->nend[0] == SENGA_NPERI && cfg->nend[1] == SENGA_NPERI) ||
        (cfg->nend[0] == SENGA_NBOUND && cfg->nend[1] == SENGA_NBOUND)))
    return fail(SENGA_ERR_UNSUPPORTED, "senga_zgroup_create: x must be periodic or bounded on both faces");
  if (cfg->adaptive) return fail(SENGA_ERR_UNSUPPORTED, "senga_zgroup_create: fixed time step only");
  if (cfg->nz % nslabs != 0) return fail(SENGA_ERR_ARG, "senga_zgroup_create: nz must divide into equal slabs");
  *out = nullptr;
  DeviceGuard dg;
  senga_zgroup* g = new senga_zgroup;
  g->nr = nslabs;
  g->nx = cfg->nx;
  g->ny = cfg->ny;
  g->nzg = cfg->nz;
  g->nzl = cfg->nz / nslabs;
  g->nc = 5 + chem->nspec;
  const int rc = guard([&] {
    for (int r = 0; r < nslabs; ++r) {
      senga_config c = *cfg;
      c.nz = g->nzl;
      c.device = devices ? devices[r] : cfg->device;
      if (senga_ctx_create(&c, chem, diff, &g->ctx[r]) != SENGA_OK) throw Error(SENGA_ERR_CUDA, senga_last_error());
      // z spacing of the whole box, DELTAZ = ZGDLEN/REAL(NZGLBL-1)
      const double delta = cfg->zgdlen / (double)(float)(cfg->nz - 1);
      g->ctx[r]->geo.ovd[2] = 1.0 / delta;
      g->ctx[r]->geo.ovd2[2] = g->ctx[r]->geo.ovd[2] * g->ctx[r]->geo.ovd[2];
      CK(cudaEventCreateWithFlags(&g->ev[r], cudaEventDisableTiming));
    }
    for (int r = 0; r < nslabs; ++r) {  // peer access between distinct GPUs
      const int dr = g->ctx[r]->cfg.device;
      CK(cudaSetDevice(dr));
      for (int q = 0; q < nslabs; ++q) {
        const int dq = g->ctx[q]->cfg.device;
        if (dq == dr) continue;
        int can = 0;
        CK(cudaDeviceCanAccessPeer(&can, dr, dq));
        if (!can) throw Error(SENGA_ERR_UNSUPPORTED, "senga_zgroup_create: no peer access between the GPUs");
        const cudaError_t e = cudaDeviceEnablePeerAccess(dq, 0);
        if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled) CK(e);
        (void)cudaGetLastError();
      }
    }
    for (int r = 0; r < nslabs; ++r) {
      ZDec& z = g->zd[r];
      z.nr = nslabs;
      z.rank = r;
      z.nzg = cfg->nz;
      for (int q = 0; q < nslabs; ++q) {
        const std::ptrdiff_t d =
            reinterpret_cast<const char*>(g->ctx[q]->pool) - reinterpret_cast<const char*>(g->ctx[r]->pool);
        if (d % (std::ptrdiff_t)sizeof(double) != 0) throw Error(SENGA_ERR_CUDA, "senga_zgroup_create: pool alignment");
        z.base[q] = (int64_t)(d / (std::ptrdiff_t)sizeof(double));
      }
    }
  });
  if (rc != SENGA_OK) {
    zgroup_destroy(g);
    return rc;
  }
  *out = g;
  return SENGA_OK;
}

int senga_zgroup_destroy(senga_zgroup* g) {
  if (g) zgroup_destroy(g);
  return SENGA_OK;
}

int senga_zgroup_upload_host(senga_zgroup* g, const double* fields, const double* trun, const int32_t* itn) {
  if (!g || !fields || !trun || !itn) return fail(SENGA_ERR_ARG, "senga_zgroup_upload_host: null argument");
  DeviceGuard dg;
  return guard([&] {
    const int64_t nl = (int64_t)g->nx * g->ny * g->nzl, ng = nl * g->nr;
    for (int r = 0; r < g->nr; ++r) {
      senga_ctx* c = g->ctx[r];
      CK(cudaSetDevice(c->cfg.device));
      for (int fl = 0; fl < g->nc; ++fl)
        CK(cudaMemcpyAsync(c->f.run + fl * nl, fields + fl * ng + r * nl, nl * sizeof(double), cudaMemcpyHostToDevice,
                           c->stream));
      CK(cudaMemcpyAsync(c->f.uin, c->f.run, (size_t)g->nc * nl * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
      CK(cudaMemcpyAsync(c->f.t, trun + r * nl, nl * sizeof(double), cudaMemcpyHostToDevice, c->stream));
      for (int w = 0; w < itn_words(c->nspec); ++w)  // one interior array per ITNDEX word
        CK(cudaMemcpyAsync(c->f.itn + w * nl, itn + w * ng + r * nl, nl * sizeof(int32_t), cudaMemcpyHostToDevice,
                           c->stream));
    }
    for (int r = 0; r < g->nr; ++r) CK(cudaStreamSynchronize(g->ctx[r]->stream));
  });
}

int senga_zgroup_download_host(senga_zgroup* g, double* fields, double* trun, int32_t* itn) {
  if (!g || !fields) return fail(SENGA_ERR_ARG, "senga_zgroup_download_host: null argument");
  DeviceGuard dg;
  return guard([&] {
    const int64_t nl = (int64_t)g->nx * g->ny * g->nzl, ng = nl * g->nr;
    for (int r = 0; r < g->nr; ++r) {
      senga_ctx* c = g->ctx[r];
      CK(cudaSetDevice(c->cfg.device));
      for (int fl = 0; fl < g->nc; ++fl)
        CK(cudaMemcpyAsync(fields + fl * ng + r * nl, c->f.run + fl * nl, nl * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
      if (trun) CK(cudaMemcpyAsync(trun + r * nl, c->f.t, nl * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
      if (itn)
        for (int w = 0; w < itn_words(c->nspec); ++w)
          CK(cudaMemcpyAsync(itn + w * ng + r * nl, c->f.itn + w * nl, nl * sizeof(int32_t), cudaMemcpyDeviceToHost,
                             c->stream));
    }
    for (int r = 0; r < g->nr; ++r) CK(cudaStreamSynchronize(g->ctx[r]->stream));
  });
}

int senga_set_synthetic_inflow(senga_ctx* c, const senga_synth_inflow* p) {
  if (!c || !p) return fail(SENGA_ERR_ARG, "senga_set_synthetic_inflow: null argument");
  if (!c->nscbc || c->bc.xl != 13)
    return fail(SENGA_ERR_UNSUPPORTED, "senga_set_synthetic_inflow: needs an I3 inflow at x-left (senga_set_nscbc)");
  if (!(p->urms >= 0.0) || p->lnx < 1 || p->lny < 1 || p->lnz < 1 || p->nfy < 0 || p->nfz < 0 || p->itime < 1 ||
      !(c->bc.u_in > 0.0))
    return fail(SENGA_ERR_ARG, "senga_set_synthetic_inflow: urms >= 0, lengths >= 1, nfy, nfz >= 0, itime >= 1 "
                               "and a positive inflow velocity");
  return guard([&] {
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    synth_destroy(c->synth);
    c->synth = nullptr;
    c->synth = synth_create(c->geo.ny, c->geo.nz, *p, c->cfg.device);
    if (c->graph) {  // a captured step would bypass the per-step planes
      cudaGraphExecDestroy(c->graph);
      c->graph = nullptr;
    }
  });
}

int senga_zgroup_set_nscbc(senga_zgroup* g, const senga_nscbc* b) {
  if (!g || !b) return fail(SENGA_ERR_ARG, "senga_zgroup_set_nscbc: null argument");
  DeviceGuard dg;
  for (int r = 0; r < g->nr; ++r) {
    if (cudaSetDevice(g->ctx[r]->cfg.device) != cudaSuccess)
      return fail(SENGA_ERR_CUDA, "senga_zgroup_set_nscbc: cudaSetDevice");
    const int rc = senga_set_nscbc(g->ctx[r], b);  // every slab: its ny x nz/nr part of both x faces
    if (rc != SENGA_OK) return rc;
  }
  return SENGA_OK;
}

int senga_zgroup_step(senga_zgroup* g, int nsteps) {
  if (!g || nsteps < 0) return fail(SENGA_ERR_ARG, "senga_zgroup_step: bad argument");
  DeviceGuard dg;
  return guard([&] {
    for (int r = 0; r < g->nr; ++r) require_rhs(g->ctx[r]);
    for (int s = 0; s < nsteps; ++s)
      for (int irk = 1; irk <= 5; ++irk) {
        // the substage sequence of run_substage, with a barrier between the
        // phases that read z halos of what other slabs write
        for (int r = 0; r < g->nr; ++r) {
          senga_ctx* c = g->ctx[r];
          CK(cudaSetDevice(c->cfg.device));
          if (c->nscbc) launch_boundt(c->geo, c->f, c->bc, c->nspec, false, c->d_chem, c->stream);  // BOUNDT
          launch_thermo(c->geo, thermo_fields(c), c->d_chem, c->d_diff, c->nspec, c->diff.flmavt, c->mech, c->stream);
        }
        zgroup_barrier(g);
        for (int r = 0; r < g->nr; ++r) {
          senga_ctx* c = g->ctx[r];
          CK(cudaSetDevice(c->cfg.device));
          // face data + BOUNDS: transverse z derivatives read the neighbouring slabs
          if (c->nscbc) launch_face(c->geo, c->f, c->bc, c->nspec, c->d_chem, c->stream, g->zd[r]);
          launch_flow(c->geo, c->f, c->nspec, c->stream, g->zd[r]);
          launch_species_a(c->geo, c->f, c->nspec, c->stream, g->zd[r]);
          if (c->nscbc) launch_wall_flux(c->geo, c->f, c->bc, c->nspec, c->stream);  // W1 wall diffusion flux
        }
        zgroup_barrier(g);
        for (int r = 0; r < g->nr; ++r) {
          senga_ctx* c = g->ctx[r];
          CK(cudaSetDevice(c->cfg.device));
          RK rk{c->rklhs[irk - 1], c->rkrhs[irk - 1], c->rkerr[irk - 1], irk == 5 ? 1 : 0};
          launch_species_b_rk(c->geo, c->f, c->nspec, rk, c->stream, g->zd[r]);
          if (c->nscbc) launch_wall_fix(c->geo, c->f, c->bc, c->nspec, true, c->stream);  // W1: LINCOM/FINCOM wall Y
          // BOUNTT after the step's last substage (own face planes only)
          if (irk == 5 && c->nscbc) launch_boundt(c->geo, c->f, c->bc, c->nspec, true, c->d_chem, c->stream);
        }
        zgroup_barrier(g);
      }
    CK(cudaGetLastError());
  });
}

int senga_zgroup_sync(senga_zgroup* g) {
  if (!g) return fail(SENGA_ERR_ARG, "senga_zgroup_sync: null group");
  return guard([&] {
    for (int r = 0; r < g->nr; ++r) CK(cudaStreamSynchronize(g->ctx[r]->stream));
  });
}
