// Initial turbulence generator on the device: SENGA2's TURBIN
// (src/turbin.f:76-362) with its inverse transform TURBFT (src/turbft.f,
// src/fftsym.f) and spectrum ESPECT (src/espect.f, parameters from
// src/espini.f:46-50), for one box.
//
//   host    RANINI/RANUNI (src/rndlib): the shuffled three-LCG stream, three
//           draws per point in x-fastest order (sequential by design: each
//           draw depends on the shuffle table's history)
//   k_turb_modes  Rogallo construction of the upper half of wavenumber
//           space: |u(k)|^2 = E(|k|)/(2 pi k^2) split between the two
//           directions normal to k by the azimuth draw, phases from the two
//           other draws; the lower half zero
//   k_turb_lines<DIR>  TURBFT's pencil transforms: x lines of kz > 0 and of
//           kz = 0, ky > 0 as they are, the kz = ky = 0 line made
//           conjugate-symmetric first (FFTSYM: entry N-k = conj(entry k),
//           0 < k < N/2 rounded up, the even-N Nyquist entry zeroed); y lines
//           of kz > 0 as they are, of kz = 0 symmetric; every z line
//           symmetric. The transform is the library's INVRS = -1 one,
//           sum_n x_n exp(-2 pi i j n / N) without scaling, here one CTA per
//           line summing directly from a shared-memory copy of the line and
//           a twiddle table (any N up to 1024, the library's NFTMAX).
// The REAL() conversions of the reference are single precision (its build
// has no -fdefault-real-8), which matters for the random draws.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "senga_gpu.h"
#include "senga_internal.h"

namespace senga {
namespace {

constexpr int kTurbBlock = 256;
constexpr int kMaxLine = 1024;

// src/rndlib/ranini.f, ranuni.f
struct RanStream {
  static constexpr int M1 = 259200, A1 = 7141, C1 = 54773;
  static constexpr int M2 = 134456, A2 = 8121, C2 = 28411;
  static constexpr int M3 = 243000, A3 = 4561, C3 = 51349;
  static constexpr int NSHUFF = 97;
  double table[NSHUFF];
  int x1 = 0, x2 = 0, x3 = 0;
  static double value(int a, int b) { return (double)(((float)a + (float)b / (float)M2) / (float)M1); }
  explicit RanStream(int iseed) {
    x1 = (C1 + iseed) % M1;
    x1 = (A1 * x1 + C1) % M1;
    x2 = x1 % M2;
    x1 = (A1 * x1 + C1) % M1;
    x3 = x1 % M3;
    for (int ic = 0; ic < NSHUFF; ++ic) {
      x1 = (A1 * x1 + C1) % M1;
      x2 = (A2 * x2 + C2) % M2;
      table[ic] = value(x1, x2);
    }
  }
  double next() {
    x1 = (A1 * x1 + C1) % M1;
    x2 = (A2 * x2 + C2) % M2;
    x3 = (A3 * x3 + C3) % M3;
    const int ic = (NSHUFF * x3) / M3;
    const double r = table[ic];
    table[ic] = value(x1, x2);
    return r;
  }
};

struct TurbBox {
  int nx, ny, nz;
  double ovk0, covk0;
  const double* az;  // azimuth draws
  const double* p1;  // phase draws
  const double* p2;
  double* re[3];
  double* im[3];
};

__device__ __forceinline__ int turbin_map(int c, int n) {  // turbin.f:82-90: N/2 maps to -N/2
  const int nodbl = n / 2 - 1 + n % 2;
  return c > nodbl ? c - n : c;
}
__device__ __forceinline__ int turbft_map(int c, int n) {  // turbft.f: N/2 stays +N/2
  return c > n / 2 ? c - n : c;
}

__global__ void __launch_bounds__(kTurbBlock) k_turb_modes(TurbBox b) {
  const int64_t q = (int64_t)blockIdx.x * kTurbBlock + threadIdx.x;
  const int64_t n = (int64_t)b.nx * b.ny * b.nz;
  if (q >= n) return;
  const int i = (int)(q % b.nx), j = (int)((q / b.nx) % b.ny), k = (int)(q / ((int64_t)b.nx * b.ny));
  const int ix = turbin_map(i, b.nx), jx = turbin_map(j, b.ny), kx = turbin_map(k, b.nz);
  const bool up = (kx > 0) || (kx == 0 && jx > 0) || (kx == 0 && jx == 0 && ix >= 0);
  if (!up) {
    for (int c = 0; c < 3; ++c) b.re[c][q] = b.im[c][q] = 0.0;
    return;
  }
  const double pi = 3.141592653589793, twopi = 2.0 * pi, ovtopi = 1.0 / twopi, vectol = 1.0e-5;
  double k1 = (double)ix, k2 = (double)jx, k3 = (double)kx;
  const double vk = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ovk = vk > vectol ? 1.0 / vk : 1.0;
  const double pl = sqrt(k1 * k1 + k2 * k2);
  double ovpl;
  if (pl < vectol) {  // azimuth arbitrary on the kz axis: k1 = 0, k2 = 1 (turbin.f:248-253)
    ovpl = 1.0;
    k1 = 0.0;
    k2 = 1.0;
  } else {
    ovpl = 1.0 / pl;
  }
  double w = vk * b.ovk0;
  w = w * w;
  double vm = b.covk0 * w * w * exp(-2.0 * w);  // ESPECT
  vm = sqrt(vm * ovtopi) * ovk;
  const double a = twopi * b.az[q];
  const double ca = cos(a), sa = sin(a);
  const double f1 = pi * (2.0 * b.p1[q] - 1.0), f2 = pi * (2.0 * b.p2[q] - 1.0);
  const double c1 = cos(f1), s1 = sin(f1), c2 = cos(f2), s2 = sin(f2);
  const double vf = vm * ovk * ovpl;
  double va = vf * vk * k2 * ca, vb = vf * k1 * k3 * sa;
  b.re[0][q] = va * c1 + vb * c2;
  b.im[0][q] = va * s1 + vb * s2;
  va = vf * vk * k1 * ca;
  vb = vf * k2 * k3 * sa;
  b.re[1][q] = vb * c2 - va * c1;
  b.im[1][q] = vb * s2 - va * s1;
  vb = -vf * pl * pl * sa;
  b.re[2][q] = vb * c2;
  b.im[2][q] = vb * s2;
}

// One CTA per pencil along DIR, the three components together.
template <int DIR>
__global__ void __launch_bounds__(kTurbBlock) k_turb_lines(TurbBox b) {
  extern __shared__ double sm[];
  const int n = DIR == 0 ? b.nx : DIR == 1 ? b.ny : b.nz;
  const int na = DIR == 0 ? b.ny : b.nx;  // the two other coordinates of the pencil
  const int a = (int)(blockIdx.x % na), c = (int)(blockIdx.x / na);
  // which pencils TURBFT transforms, and with the symmetric fill
  bool go = true, sym = true;
  if (DIR == 0) {  // a = j, c = k
    const int kx = turbft_map(c, b.nz), jx = turbft_map(a, b.ny);
    go = kx > 0 || (kx == 0 && jx >= 0);
    sym = kx == 0 && jx == 0;
  } else if (DIR == 1) {  // a = i, c = k
    const int kx = turbft_map(c, b.nz);
    go = kx >= 0;
    sym = kx == 0;
  }
  if (!go) return;
  int64_t base, stride;
  if (DIR == 0) {
    base = (int64_t)b.nx * ((int64_t)a + (int64_t)b.ny * c);
    stride = 1;
  } else if (DIR == 1) {
    base = (int64_t)a + (int64_t)b.nx * b.ny * c;
    stride = b.nx;
  } else {
    base = (int64_t)a + (int64_t)b.nx * c;
    stride = (int64_t)b.nx * b.ny;
  }
  double* xr = sm;           // [3][n] real parts
  double* xi = sm + 3 * n;   // [3][n] imaginary parts
  double* tc = sm + 6 * n;   // cos(2 pi m / n)
  double* ts = sm + 7 * n;   // sin(2 pi m / n)
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    double s, co;
    sincospi(2.0 * (double)m / (double)n, &s, &co);
    tc[m] = co;
    ts[m] = s;
    for (int cp = 0; cp < 3; ++cp) {
      xr[cp * n + m] = b.re[cp][base + m * stride];
      xi[cp * n + m] = b.im[cp][base + m * stride];
    }
  }
  __syncthreads();
  if (sym) {  // FFTSYM, NDOSYM = 1
    const int nsymax = n / 2 + n % 2;
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
      for (int cp = 0; cp < 3; ++cp) {
        if (m >= 1 && m < nsymax) {
          xr[cp * n + n - m] = xr[cp * n + m];
          xi[cp * n + n - m] = -xi[cp * n + m];
        }
      }
    }
    __syncthreads();
    if (n % 2 == 0 && threadIdx.x < 3) {
      xr[threadIdx.x * n + n / 2] = 0.0;
      xi[threadIdx.x * n + n / 2] = 0.0;
    }
    __syncthreads();
  }
  // X_j = sum_m x_m exp(-2 pi i j m / n)
  for (int jj = threadIdx.x; jj < n; jj += blockDim.x) {
    double sr[3] = {0.0, 0.0, 0.0}, si[3] = {0.0, 0.0, 0.0};
    int idx = 0;  // (jj * m) mod n
    for (int m = 0; m < n; ++m) {
      const double co = tc[idx], s = -ts[idx];
#pragma unroll
      for (int cp = 0; cp < 3; ++cp) {
        const double r = xr[cp * n + m], ii = xi[cp * n + m];
        sr[cp] = sr[cp] + (r * co - ii * s);
        si[cp] = si[cp] + (r * s + ii * co);
      }
      idx += jj;
      if (idx >= n) idx -= n;
    }
    for (int cp = 0; cp < 3; ++cp) {
      b.re[cp][base + jj * stride] = sr[cp];
      b.im[cp][base + jj * stride] = si[cp];
    }
  }
}

}  // namespace
}  // namespace senga

using namespace senga;

extern "C" int senga_turbin_host(int nx, int ny, int nz, int inseed, double const0, double ck0, double* uvw,
                                 double* imag_max) {
  if (!uvw || nx < 2 || ny < 2 || nz < 2 || nx > kMaxLine || ny > kMaxLine || nz > kMaxLine || !(ck0 > 0.0))
    return fail(SENGA_ERR_ARG, "senga_turbin_host: bad argument (extents 2..1024, ck0 > 0)");
  const int64_t n = (int64_t)nx * ny * nz;
  // turbin.f:128-191: one rank, so the local and global sweeps give the
  // same stream from RANINI(INSEED)
  std::vector<double> draws((size_t)(3 * n));
  {
    RanStream r(inseed);
    for (int64_t q = 0; q < n; ++q) {
      draws[q] = r.next();
      draws[n + q] = r.next();
      draws[2 * n + q] = r.next();
    }
  }
  double* d = nullptr;
  cudaError_t e = cudaMalloc(&d, (size_t)(9 * n) * sizeof(double));
  if (e != cudaSuccess) return fail(SENGA_ERR_CUDA, std::string("senga_turbin_host: ") + cudaGetErrorString(e));
  TurbBox b{nx, ny, nz, 1.0 / ck0, const0 / ck0, d, d + n, d + 2 * n, {d + 3 * n, d + 4 * n, d + 5 * n},
            {d + 6 * n, d + 7 * n, d + 8 * n}};
  const int mx = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
  const size_t smem = (size_t)8 * mx * sizeof(double);
  std::vector<double> im((size_t)(3 * n));
  e = cudaMemcpy(d, draws.data(), (size_t)(3 * n) * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_turb_lines<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_turb_lines<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_turb_lines<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) {
    k_turb_modes<<<(unsigned)((n + kTurbBlock - 1) / kTurbBlock), kTurbBlock>>>(b);
    k_turb_lines<0><<<(unsigned)((int64_t)ny * nz), kTurbBlock, smem>>>(b);
    k_turb_lines<1><<<(unsigned)((int64_t)nx * nz), kTurbBlock, smem>>>(b);
    k_turb_lines<2><<<(unsigned)((int64_t)nx * ny), kTurbBlock, smem>>>(b);
    e = cudaGetLastError();
  }
  for (int c = 0; c < 3 && e == cudaSuccess; ++c)
    e = cudaMemcpy(uvw + c * n, b.re[c], (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
  for (int c = 0; c < 3 && e == cudaSuccess; ++c)
    e = cudaMemcpy(im.data() + c * n, b.im[c], (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(SENGA_ERR_CUDA, std::string("senga_turbin_host: ") + cudaGetErrorString(e));
  if (imag_max) {  // turbin.f:366-383 checks the imaginary parts against TOLIMG
    double mxim = 0.0;
    for (double v : im) mxim = std::fabs(v) > mxim ? std::fabs(v) : mxim;
    *imag_max = mxim;
  }
  return SENGA_OK;
}
