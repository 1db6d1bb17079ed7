// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of SENGA2's initial turbulence generator for one rank, used
// by tests/ to check the device implementation; the product never links it.
// Parity unpinned against outputs of the reference (Fortran, not buildable
// here); pinned instead by closed-form checks in the tests (a real,
// solenoidal, zero-mean field whose shell energies follow the spectrum).
//
// Restated (file:line within the reference project):
//   src/rndlib/ranini.f, src/rndlib/ranuni.f  shuffled three-LCG generator;
//       REAL() there is default (single) precision, as the build has no
//       -fdefault-real-8 (src/Makefile:19)
//   src/espect.f, src/espini.f:46-50  E(k) = C/k0 (k/k0)^4 exp(-2 (k/k0)^2)
//   src/turbin.f:76-192  index maps, seeds, three random numbers per point
//   src/turbin.f:195-320 Rogallo construction in the upper half of k-space
//   src/turbft.f, src/fftsym.f  inverse transform pencil by pencil: x lines
//       of kz > 0 and of kz = 0, ky > 0 as they are, the kz = ky = 0 line made
//       conjugate-symmetric first; y lines of kz > 0 as they are, of kz = 0
//       symmetric; all z lines symmetric. Symmetric: entry N-k = conj(entry
//       k), 0 < k < N/2 (+1 if N odd), the even-N Nyquist entry zeroed. The
//       library transform (src/fftlib, INVRS = -1) is sum_n x_n exp(-2 pi i
//       j n / N) without scaling; here as a direct sum.
#include <cmath>
#include <complex>
#include <cstdint>
#include <vector>

namespace {

struct Ran {
  static constexpr int M1 = 259200, A1 = 7141, C1 = 54773;
  static constexpr int M2 = 134456, A2 = 8121, C2 = 28411;
  static constexpr int M3 = 243000, A3 = 4561, C3 = 51349;
  static constexpr int NSHUFF = 97;
  double shuffl[NSHUFF];
  int x1 = 0, x2 = 0, x3 = 0;
  static double draw(int a, int b) {
    return (double)(((float)a + (float)b / (float)M2) / (float)M1);
  }
  void init(int iseed) {
    x1 = (C1 + iseed) % M1;
    x1 = (A1 * x1 + C1) % M1;
    x2 = x1 % M2;
    x1 = (A1 * x1 + C1) % M1;
    x3 = x1 % M3;
    for (int ic = 0; ic < NSHUFF; ++ic) {
      x1 = (A1 * x1 + C1) % M1;
      x2 = (A2 * x2 + C2) % M2;
      shuffl[ic] = draw(x1, x2);
    }
  }
  double uni() {
    x1 = (A1 * x1 + C1) % M1;
    x2 = (A2 * x2 + C2) % M2;
    x3 = (A3 * x3 + C3) % M3;
    const int ic = (NSHUFF * x3) / M3;
    const double r = shuffl[ic];
    shuffl[ic] = draw(x1, x2);
    return r;
  }
};

using cd = std::complex<double>;

void line_dft(std::vector<cd>& a, bool sym) {
  const int n = (int)a.size();
  if (sym) {
    const int nsymax = n / 2 + n % 2;
    for (int k = 1; k < nsymax; ++k) a[n - k] = std::conj(a[k]);
    if (n % 2 == 0) a[n / 2] = 0.0;
  }
  std::vector<cd> out(n);
  for (int j = 0; j < n; ++j) {
    cd s = 0.0;
    for (int m = 0; m < n; ++m) {
      const double th = -2.0 * M_PI * (double)((int64_t)j * m % n) / n;
      s += a[m] * cd(std::cos(th), std::sin(th));
    }
    out[j] = s;
  }
  a = out;
}

}  // namespace

extern "C" {

// Velocity field of TURBIN for an (nx, ny, nz) box: uvw[3][nz][ny][nx] real
// parts, imag[3][...] the imaginary parts left by the transform.
int oracle_turbin(int nx, int ny, int nz, int inseed, double const0, double ck0, double* uvw, double* imag) {
  const int64_t n = (int64_t)nx * ny * nz;
  auto at = [&](int i, int j, int k) { return (int64_t)i + (int64_t)nx * ((int64_t)j + (int64_t)ny * k); };
  std::vector<double> az(n), p1(n), p2(n);
  Ran r;
  r.init(inseed);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const int64_t q = at(i, j, k);
        az[q] = r.uni();
        p1[q] = r.uni();
        p2[q] = r.uni();
      }
  // turbin.f:82-122
  const int nodblx = nx / 2 - 1 + nx % 2, nodbly = ny / 2 - 1 + ny % 2, nodblz = nz / 2 - 1 + nz % 2;
  const double pi = M_PI, twopi = 2.0 * pi, ovtopi = 1.0 / twopi;
  const double ovk0 = 1.0 / ck0, covk0 = const0 / ck0;
  const double vectol = 1.0e-5;
  auto espect = [&](double k) {
    double w = k * ovk0;
    w = w * w;
    return covk0 * w * w * std::exp(-2.0 * w);
  };
  std::vector<cd> U(n), V(n), W(n);
  for (int k = 0; k < nz; ++k) {
    int kx = k;
    if (kx > nodblz) kx -= nz;
    for (int j = 0; j < ny; ++j) {
      int jx = j;
      if (jx > nodbly) jx -= ny;
      for (int i = 0; i < nx; ++i) {
        int ix = i;
        if (ix > nodblx) ix -= nx;
        const int64_t q = at(i, j, k);
        const bool up = (kx > 0) || (kx == 0 && jx > 0) || (kx == 0 && jx == 0 && ix >= 0);
        if (!up) continue;
        double k1 = (double)(float)ix, k2 = (double)(float)jx, k3 = (double)(float)kx;
        const double vk = std::sqrt(k1 * k1 + k2 * k2 + k3 * k3);
        double ovk = 1.0;
        if (vk > vectol) ovk = 1.0 / vk;
        const double pl = std::sqrt(k1 * k1 + k2 * k2);
        double ovpl;
        if (pl < vectol) {
          ovpl = 1.0;
          k1 = 0.0;
          k2 = 1.0;
        } else {
          ovpl = 1.0 / pl;
        }
        double vm = espect(vk);
        vm = std::sqrt(vm * ovtopi) * ovk;
        const double a = twopi * az[q];
        const double ca = std::cos(a), sa = std::sin(a);
        const double f1 = pi * (2.0 * p1[q] - 1.0), f2 = pi * (2.0 * p2[q] - 1.0);
        const double c1 = std::cos(f1), s1 = std::sin(f1), c2 = std::cos(f2), s2 = std::sin(f2);
        const double vf = vm * ovk * ovpl;
        double va = vf * vk * k2 * ca, vb = vf * k1 * k3 * sa;
        U[q] = cd(va * c1 + vb * c2, va * s1 + vb * s2);
        va = vf * vk * k1 * ca;
        vb = vf * k2 * k3 * sa;
        V[q] = cd(vb * c2 - va * c1, vb * s2 - va * s1);
        vb = -vf * pl * pl * sa;
        W[q] = cd(vb * c2, vb * s2);
      }
    }
  }
  // turbft.f: TURBFT's own wavenumber map, N/2 -> +N/2
  auto tmap = [](int c, int nn) { return c > nn / 2 ? c - nn : c; };
  std::vector<cd>* comp[3] = {&U, &V, &W};
  std::vector<cd> line;
  for (int k = 0; k < nz; ++k)  // x lines
    for (int j = 0; j < ny; ++j) {
      const int kx = tmap(k, nz), jx = tmap(j, ny);
      bool go = false, sym = false;
      if (kx > 0) go = true;
      else if (kx == 0 && jx > 0) go = true;
      else if (kx == 0 && jx == 0) go = sym = true;
      if (!go) continue;
      for (auto* c : comp) {
        line.resize(nx);
        for (int i = 0; i < nx; ++i) line[i] = (*c)[at(i, j, k)];
        line_dft(line, sym);
        for (int i = 0; i < nx; ++i) (*c)[at(i, j, k)] = line[i];
      }
    }
  for (int k = 0; k < nz; ++k)  // y lines
    for (int i = 0; i < nx; ++i) {
      const int kx = tmap(k, nz);
      if (kx < 0) continue;
      const bool sym = kx == 0;
      for (auto* c : comp) {
        line.resize(ny);
        for (int j = 0; j < ny; ++j) line[j] = (*c)[at(i, j, k)];
        line_dft(line, sym);
        for (int j = 0; j < ny; ++j) (*c)[at(i, j, k)] = line[j];
      }
    }
  for (int j = 0; j < ny; ++j)  // z lines
    for (int i = 0; i < nx; ++i)
      for (auto* c : comp) {
        line.resize(nz);
        for (int k = 0; k < nz; ++k) line[k] = (*c)[at(i, j, k)];
        line_dft(line, true);
        for (int k = 0; k < nz; ++k) (*c)[at(i, j, k)] = line[k];
      }
  for (int c = 0; c < 3; ++c)
    for (int64_t q = 0; q < n; ++q) {
      uvw[c * n + q] = (*comp[c])[q].real();
      if (imag) imag[c * n + q] = (*comp[c])[q].imag();
    }
  return 0;
}

// The generator's stream after RANINI(iseed): n draws of RANUNI.
int oracle_ranuni(int iseed, int64_t n, double* out) {
  Ran r;
  r.init(iseed);
  for (int64_t q = 0; q < n; ++q) out[q] = r.uni();
  return 0;
}

}  // extern "C"
