// Synthetic turbulent inflow velocity (src/inflow.f, M. Klein's digital
// filter; called once per time step from src/senga2.f:100-103 when
// NXLPRM(1) = 4, consumed by BCUTXL, src/bcutxl.f:476-510) for one context:
// velocity fluctuations only (NXLPRM(2) = 0), USTEAD = 1 and WINF2 = 0 as
// coded, one rank (JFILTSTART = KFILTSTART = 0).
//
// Per step: three random planes over JC = 1-NFY .. NY+NFY, KC = 1-NFZ ..
// NZ+NFZ are drawn on the host with RAN1 (the sequence is serial: it must
// follow the reference's draw order, JC outermost, u, v, w per point) and
// made periodic in y (PERIY; z is not, PERIZ = .FALSE.), copied to the
// device through a page-locked buffer, filtered there with the normalised
// Gaussian kernels AY (over JC) and AZ (over KC), scaled by
// sqrt(URMS^2 (1 - PHI^2)), correlated in time (UINF2 = UFILT + PHI UINF1,
// PHI = 1 - TSTEP/THETA, THETA = LNX DELX / RXLPRM(1)) and stripped of their
// face means. The I3 face kernels then read u = RXLPRM(1) + UINF2 +
// RXLPRM(4), v = VINF2, w = WINF2 and their time derivatives
// (UINF2 - UINF1)/TSTEP.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "senga_gpu.h"
#include "senga_internal.h"

namespace senga {

#define CK(call)                                                                              \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      throw Error(e_ == cudaErrorMemoryAllocation ? SENGA_ERR_NOMEM : SENGA_ERR_CUDA,         \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                        \
  } while (0)

struct SynthInflow {
  senga_synth_inflow p{};
  int ny = 0, nz = 0, wy = 0, wz = 0, device = 0;
  int iv[32] = {}, iy = 0;  // RAN1's saved shuffle table and output
  double* h_rand = nullptr;  // page-locked: u, v, w planes [3][wz][wy]
  double* d_rand = nullptr;
  double* d_fold = nullptr;  // y-filtered planes [3][wz][ny]
  double* d_inf = nullptr;   // uinf1, uinf2, vinf1, vinf2, winf1, winf2 [6][nz][ny]
  double* d_ay = nullptr;    // AY, AZ
  int cur = 0;               // which of each pair holds this step's plane
  cudaEvent_t copied = nullptr;
};

namespace {

// RAN1 of src/inflow.f:448-475: the minimal-standard multiplicative
// congruential generator of Park and Miller (a = 16807, m = 2^31 - 1, by
// Schrage's factorisation) behind the Bays-Durham shuffle of 32 entries, as
// in Numerical Recipes' ran1; single-precision output in [eps, 1 - eps],
// mapped to (2r - 1)/0.577. The state (idum, the table, the last output)
// carries across calls; a positive idum re-seeds only the generator, not
// the table.
float ran1(int& idum, int (&iv)[32], int& iy) {
  constexpr int kA = 16807, kM = 2147483647, kQ = 127773, kR = 2836, kTab = 32, kDiv = 1 + (kM - 1) / kTab;
  const float am = 1.0f / (float)kM, eps = 1.2e-7f, rnmx = 1.0f - eps;
  auto next = [&]() {
    const int k = idum / kQ;
    idum = kA * (idum - k * kQ) - kR * k;
    if (idum < 0) idum += kM;
  };
  if (idum <= 0 || iy == 0) {
    idum = std::max(-idum, 1);
    for (int j = kTab + 8; j >= 1; --j) {
      next();
      if (j <= kTab) iv[j - 1] = idum;
    }
    iy = iv[0];
  }
  next();
  const int j = iy / kDiv;
  iy = iv[j];
  iv[j] = idum;
  float r = std::min(am * (float)iy, rnmx);
  r = (r * 2.0f - 1.0f) / 0.577f;
  return r;
}

constexpr int kSynBlock = 128;

// y filter: fold[f][kc][jc] = sum_j2 rand[f][kc][jc + j2] AY(j2), j2 ascending
__global__ void __launch_bounds__(kSynBlock) k_syn_fold(const double* __restrict__ rnd, double* __restrict__ fold,
                                                        const double* __restrict__ ay, int ny, int wy, int wz,
                                                        int nfy) {
  const int t = blockIdx.x * kSynBlock + threadIdx.x;
  if (t >= ny * wz) return;
  const int j = t % ny, k = t / ny;  // jc = j + 1, plane row k = kc + NFZ - 1
  for (int f = 0; f < 3; ++f) {
    const double* r = rnd + (size_t)f * wy * wz + (size_t)k * wy + j;  // rand(jc - NFY .. )
    double s = 0.0;
    for (int j2 = 0; j2 <= 2 * nfy; ++j2) s = s + r[j2] * ay[j2];
    fold[(size_t)f * ny * wz + t] = s;
  }
}

// z filter, scaling and the temporal correlation: this step's planes into
// the slots of the previous step's (the previous kept as UINF1)
__global__ void __launch_bounds__(kSynBlock) k_syn_filt(const double* __restrict__ fold, const double* __restrict__ az,
                                                        double* __restrict__ inf, int ny, int nz, int nfz, int cur,
                                                        double scale, double phi) {
  const int t = blockIdx.x * kSynBlock + threadIdx.x;
  if (t >= ny * nz) return;
  const int j = t % ny, k = t / ny;
  const size_t m = (size_t)ny * nz;
  for (int f = 0; f < 3; ++f) {
    const double* fo = fold + (size_t)f * ny * (nz + 2 * nfz) + (size_t)k * ny + j;  // fold(jc, kc - NFZ ..)
    double s = 0.0;
    for (int k2 = 0; k2 <= 2 * nfz; ++k2) s = s + fo[(size_t)k2 * ny] * az[k2];
    s = s * scale;
    const double prev = inf[(2 * f + (1 - cur)) * m + t];  // UINF1 = the previous UINF2
    double v = s + phi * prev;
    v = f == 2 ? 0.0 : v * 1.0;  // times USTEAD = 1; WINF2 = 0
    inf[(2 * f + cur) * m + t] = v;
  }
}

// the face means removed, one CTA: sums in a fixed order
__global__ void __launch_bounds__(256) k_syn_mean(double* __restrict__ inf, int m, int cur) {
  __shared__ double part[256];
  for (int f = 0; f < 3; ++f) {
    double* a = inf + (size_t)(2 * f + cur) * m;
    double s = 0.0;
    for (int q = threadIdx.x; q < m; q += 256) s = s + a[q];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) part[threadIdx.x] = part[threadIdx.x] + part[threadIdx.x + w];
      __syncthreads();
    }
    const double mean = part[0] / (double)m;  // DENOM = sum of USTEAD = the face points
    __syncthreads();
    for (int q = threadIdx.x; q < m; q += 256) a[q] = a[q] - mean;
    __syncthreads();
  }
}

}  // namespace

SynthInflow* synth_create(int ny, int nz, const senga_synth_inflow& p, int device) {
  auto* s = new SynthInflow;
  try {
  s->p = p;
  s->ny = ny;
  s->nz = nz;
  s->wy = ny + 2 * p.nfy;
  s->wz = nz + 2 * p.nfz;
  s->device = device;
  const size_t nr = (size_t)3 * s->wy * s->wz, nf = (size_t)3 * ny * s->wz, ni = (size_t)6 * ny * nz;
  CK(cudaMallocHost(&s->h_rand, nr * sizeof(double)));
  CK(cudaMalloc(&s->d_rand, nr * sizeof(double)));
  CK(cudaMalloc(&s->d_fold, nf * sizeof(double)));
  CK(cudaMalloc(&s->d_inf, ni * sizeof(double)));
  CK(cudaMemset(s->d_inf, 0, ni * sizeof(double)));  // UINF1 = UINF2 = 0 (src/indata.f:150-151)
  CK(cudaEventCreateWithFlags(&s->copied, cudaEventDisableTiming));
  // AY, AZ: exp(-pi j^2 / (2 L^2)) normalised to unit sum of squares
  const double pi = 4.0 * std::atan(1.0);
  std::vector<double> ay(2 * p.nfy + 1), az(2 * p.nfz + 1);
  auto kernel = [&](std::vector<double>& a, int nf, int l) {
    double norm = 0.0;
    for (int j = -nf; j <= nf; ++j) {
      a[j + nf] = std::exp(-pi * j * j / (2 * l * l));
      norm = norm + a[j + nf] * a[j + nf];
    }
    norm = std::sqrt(norm);
    for (auto& v : a) v = v / norm;
  };
  kernel(ay, p.nfy, p.lny);
  kernel(az, p.nfz, p.lnz);
  CK(cudaMalloc(&s->d_ay, (ay.size() + az.size()) * sizeof(double)));
  CK(cudaMemcpy(s->d_ay, ay.data(), ay.size() * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(s->d_ay + ay.size(), az.data(), az.size() * sizeof(double), cudaMemcpyHostToDevice));
  } catch (...) {
    synth_destroy(s);
    throw;
  }
  return s;
}

void synth_destroy(SynthInflow* s) {
  if (!s) return;
  if (s->copied) cudaEventSynchronize(s->copied);
  cudaFreeHost(s->h_rand);
  cudaFree(s->d_rand);
  cudaFree(s->d_fold);
  cudaFree(s->d_inf);
  cudaFree(s->d_ay);
  if (s->copied) cudaEventDestroy(s->copied);
  delete s;
}

void synth_step(SynthInflow* s, double xgdlen, int nx, double tstep, NscbcParams& bc, cudaStream_t st) {
  const int ny = s->ny, nz = s->nz, wy = s->wy, wz = s->wz, nfy = s->p.nfy, nfz = s->p.nfz;
  // the last step's copy has left the page-locked buffer
  CK(cudaEventSynchronize(s->copied));
  double* u = s->h_rand;
  double* v = u + (size_t)wy * wz;
  double* w = v + (size_t)wy * wz;
  auto at = [&](int jc, int kc) { return (size_t)(jc + nfy - 1) + (size_t)wy * (size_t)(kc + nfz - 1); };
  int intran = s->p.itime;  // INTRAN = ITIME
  for (int jc = 1 - nfy; jc <= ny + nfy; ++jc)
    for (int kc = 1 - nfz; kc <= nz + nfz; ++kc) {
      u[at(jc, kc)] = ran1(intran, s->iv, s->iy);
      v[at(jc, kc)] = ran1(intran, s->iv, s->iy);
      w[at(jc, kc)] = ran1(intran, s->iv, s->iy);
    }
  for (int jc = 1 - nfy; jc <= 0; ++jc)  // periodic in y, rows in ascending order
    for (int kc = 1 - nfz; kc <= nz + nfz; ++kc) {
      u[at(jc, kc)] = u[at(jc + ny, kc)];
      v[at(jc, kc)] = v[at(jc + ny, kc)];
      w[at(jc, kc)] = w[at(jc + ny, kc)];
    }
  for (int jc = ny + 1; jc <= ny + nfy; ++jc)
    for (int kc = 1 - nfz; kc <= nz + nfz; ++kc) {
      u[at(jc, kc)] = u[at(jc - ny, kc)];
      v[at(jc, kc)] = v[at(jc - ny, kc)];
      w[at(jc, kc)] = w[at(jc - ny, kc)];
    }
  ++s->p.itime;
  CK(cudaMemcpyAsync(s->d_rand, s->h_rand, (size_t)3 * wy * wz * sizeof(double), cudaMemcpyHostToDevice, st));
  CK(cudaEventRecord(s->copied, st));
  const double delx = xgdlen / (double)(float)(nx - 1);  // XGDLEN/REAL(NXGLBL-1)
  const double theta = (double)s->p.lnx * delx / bc.u_in;
  const double phi = 1.0 - tstep / theta;
  const double scale = std::sqrt(s->p.urms * s->p.urms * (1.0 - phi * phi));
  s->cur = 1 - s->cur;
  k_syn_fold<<<(ny * wz + kSynBlock - 1) / kSynBlock, kSynBlock, 0, st>>>(s->d_rand, s->d_fold, s->d_ay, ny, wy, wz,
                                                                          nfy);
  k_syn_filt<<<(ny * nz + kSynBlock - 1) / kSynBlock, kSynBlock, 0, st>>>(s->d_fold, s->d_ay + 2 * nfy + 1,
                                                                          s->d_inf, ny, nz, nfz, s->cur, scale, phi);
  k_syn_mean<<<1, 256, 0, st>>>(s->d_inf, ny * nz, s->cur);
  const size_t m = (size_t)ny * nz;
  bc.uinf2 = s->d_inf + (0 + s->cur) * m;
  bc.uinf1 = s->d_inf + (0 + 1 - s->cur) * m;
  bc.vinf2 = s->d_inf + (2 + s->cur) * m;
  bc.vinf1 = s->d_inf + (2 + 1 - s->cur) * m;
  bc.winf2 = s->d_inf + (4 + s->cur) * m;
  bc.winf1 = s->d_inf + (4 + 1 - s->cur) * m;
  bc.coflow = s->p.coflow;
  bc.tstep = tstep;
}

}  // namespace senga
