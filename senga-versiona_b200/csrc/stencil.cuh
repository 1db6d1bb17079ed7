// 10th-order explicit finite-difference operators on device.
//
// Coefficients: src/dfinit.f:61-171 (first), :191-301 (second), :326-336
// (mixed). Interior first derivative src/dfbydx.f:67-105 with scaling :234-238;
// one-sided 4th/4th/4th/6th/8th-order closures :116-223. Second derivative
// src/d2fdx2.f:96-111, closures :127-263, scaling :270. Mixed derivative
// interior src/d2fdxy.f:126-141, scaling :1937.
//
// Periodic directions wrap the index (the single-rank halo copy of
// src/parfer.f:840-873 produces exactly those values); bounded directions use
// the one-sided closures on the first/last five points.
#pragma once
#include <cstdint>

#include "senga_internal.h"

namespace senga {

// ---- coefficients (constant-folded exactly as DFINIT computes them) ----
namespace fdc {
constexpr double A = 5.0 / 3.0, B = -2.0e1 / 2.1e1, C = 5.0 / 1.4e1, D = -5.0 / 6.3e1, E = 1.0 / 1.26e2;
constexpr double a1 = A / 2.0, b1 = B / 4.0, c1 = C / 6.0, d1 = D / 8.0, e1 = E / 1.0e1;
constexpr double a2 = A, b2 = B / 4.0, c2 = C / 9.0, d2 = D / 1.6e1, e2 = E / 2.5e1;
constexpr double ax = A / 4.0, bx = B / 4.0 / 4.0, cx = C / 4.0 / 9.0, dx = D / 4.0 / 1.6e1, ex = E / 4.0 / 2.5e1;
// first-derivative closures
constexpr double p1a = 4.0, p1b = -3.0, p1c = 4.0 / 3.0, p1d = -1.0 / 4.0;
constexpr double p2a = -1.0 / 4.0, p2b = 3.0 / 2.0, p2c = -1.0 / 2.0, p2d = 1.0 / 1.2e1;
constexpr double p3a = (4.0 / 3.0) / 2.0, p3b = (-1.0 / 3.0) / 4.0;
constexpr double p4a = (3.0 / 2.0) / 2.0, p4b = (-3.0 / 5.0) / 4.0, p4c = (1.0 / 1.0e1) / 6.0;
constexpr double p5a = (8.0 / 5.0) / 2.0, p5b = (-4.0 / 5.0) / 4.0, p5c = (8.0 / 3.5e1) / 6.0, p5d = (-1.0 / 3.5e1) / 8.0;
// second-derivative closures
constexpr double s1a = -7.7e1 / 6.0, s1b = 1.07e2 / 6.0, s1c = -1.3e1, s1d = 6.1e1 / 1.2e1, s1e = -5.0 / 6.0;
constexpr double s2a = 5.0 / 6.0, s2b = -1.0 / 3.0, s2c = 7.0 / 6.0, s2d = -1.0 / 2.0, s2e = 1.0 / 1.2e1;
constexpr double s3a = 4.0 / 3.0, s3b = (-1.0 / 3.0) / 4.0;
constexpr double s4a = 3.0 / 2.0, s4b = (-3.0 / 5.0) / 4.0, s4c = (1.0 / 1.0e1) / 9.0;
constexpr double s5a = 8.0 / 5.0, s5b = (-4.0 / 5.0) / 4.0, s5c = (8.0 / 3.5e1) / 9.0, s5d = (-1.0 / 3.5e1) / 1.6e1;
}  // namespace fdc

struct Pt {
  int i, j, k;
  int64_t q;
};

template <int DIR>
__device__ __forceinline__ int ext(const Geo& g) {
  return DIR == 0 ? g.nx : DIR == 1 ? g.ny : g.nz;
}
template <int DIR>
__device__ __forceinline__ int64_t strd(const Geo& g) {
  return DIR == 0 ? (int64_t)1 : DIR == 1 ? (int64_t)g.nx : (int64_t)g.nx * g.ny;
}
template <int DIR>
__device__ __forceinline__ int crd(const Pt& p) {
  return DIR == 0 ? p.i : DIR == 1 ? p.j : p.k;
}
// element offset of the point m steps along DIR (periodic wrap)
template <int DIR>
__device__ __forceinline__ int64_t woff(const Geo& g, int c, int m) {
  const int n = ext<DIR>(g);
  int cm = c + m;
  if (n > 5) {
    cm = cm < 0 ? cm + n : (cm >= n ? cm - n : cm);
  } else {  // short periodic extents (a one-point direction of a 1D or 2D box)
    cm %= n;
    if (cm < 0) cm += n;
  }
  return (int64_t)(cm - c) * strd<DIR>(g);
}

// ---- scheme cores -----------------------------------------------------------
// v(m) returns the field m points along the direction from the evaluation
// point; c is the point's coordinate in that direction, n the extent, per the
// periodic flag. Results are unscaled (the caller multiplies by 1/Delta^k).
template <class V>
__device__ __forceinline__ double d1core(const V& v, int c, int n, int per) {
  using namespace fdc;
  // points past the end of a partial tile (never stored) evaluate as the
  // last point, so a closure never reaches outside the staged halo
  if (!per && c > n - 1) c = n - 1;
  if (per || (c >= 5 && c <= n - 6))
    return a1 * (v(1) - v(-1)) + b1 * (v(2) - v(-2)) + c1 * (v(3) - v(-3)) + d1 * (v(4) - v(-4)) +
           e1 * (v(5) - v(-5));
  auto a = [&](int abs0) { return v(abs0 - c); };  // 0-based absolute index
  if (c < 5) {
    switch (c) {
      case 0: return p1a * (a(1) - a(0)) + p1b * (a(2) - a(0)) + p1c * (a(3) - a(0)) + p1d * (a(4) - a(0));
      case 1: return p2a * (a(0) - a(1)) + p2b * (a(2) - a(1)) + p2c * (a(3) - a(1)) + p2d * (a(4) - a(1));
      case 2: return p3a * (a(3) - a(1)) + p3b * (a(4) - a(0));
      case 3: return p4a * (a(4) - a(2)) + p4b * (a(5) - a(1)) + p4c * (a(6) - a(0));
      default: return p5a * (a(5) - a(3)) + p5b * (a(6) - a(2)) + p5c * (a(7) - a(1)) + p5d * (a(8) - a(0));
    }
  }
  const int L = n - 1;
  switch (L - c) {
    case 4: return p5a * (a(L - 3) - a(L - 5)) + p5b * (a(L - 2) - a(L - 6)) + p5c * (a(L - 1) - a(L - 7)) + p5d * (a(L) - a(L - 8));
    case 3: return p4a * (a(L - 2) - a(L - 4)) + p4b * (a(L - 1) - a(L - 5)) + p4c * (a(L) - a(L - 6));
    case 2: return p3a * (a(L - 1) - a(L - 3)) + p3b * (a(L) - a(L - 4));
    case 1: return p2a * (a(L - 1) - a(L)) + p2b * (a(L - 1) - a(L - 2)) + p2c * (a(L - 1) - a(L - 3)) + p2d * (a(L - 1) - a(L - 4));
    default: return p1a * (a(L) - a(L - 1)) + p1b * (a(L) - a(L - 2)) + p1c * (a(L) - a(L - 3)) + p1d * (a(L) - a(L - 4));
  }
}

template <class V>
__device__ __forceinline__ double d2core(const V& v, int c, int n, int per) {
  using namespace fdc;
  if (!per && c > n - 1) c = n - 1;  // see d1core
  if (per || (c >= 5 && c <= n - 6)) {
    const double f0 = v(0);
    return a2 * ((v(1) - f0) - (f0 - v(-1))) + b2 * ((v(2) - f0) - (f0 - v(-2))) +
           c2 * ((v(3) - f0) - (f0 - v(-3))) + d2 * ((v(4) - f0) - (f0 - v(-4))) +
           e2 * ((v(5) - f0) - (f0 - v(-5)));
  }
  auto a = [&](int abs0) { return v(abs0 - c); };
  if (c < 5) {
    switch (c) {
      case 0: return s1a * (a(1) - a(0)) + s1b * (a(2) - a(0)) + s1c * (a(3) - a(0)) + s1d * (a(4) - a(0)) + s1e * (a(5) - a(0));
      case 1: return s2a * (a(0) - a(1)) + s2b * (a(2) - a(1)) + s2c * (a(3) - a(1)) + s2d * (a(4) - a(1)) + s2e * (a(5) - a(1));
      case 2: return s3a * ((a(3) - a(2)) - (a(2) - a(1))) + s3b * ((a(4) - a(2)) - (a(2) - a(0)));
      case 3: return s4a * ((a(4) - a(3)) - (a(3) - a(2))) + s4b * ((a(5) - a(3)) - (a(3) - a(1))) + s4c * ((a(6) - a(3)) - (a(3) - a(0)));
      default: return s5a * ((a(5) - a(4)) - (a(4) - a(3))) + s5b * ((a(6) - a(4)) - (a(4) - a(2))) + s5c * ((a(7) - a(4)) - (a(4) - a(1))) + s5d * ((a(8) - a(4)) - (a(4) - a(0)));
    }
  }
  const int L = n - 1;
  switch (L - c) {
    case 4: return s5a * ((a(L - 3) - a(L - 4)) - (a(L - 4) - a(L - 5))) + s5b * ((a(L - 2) - a(L - 4)) - (a(L - 4) - a(L - 6))) + s5c * ((a(L - 1) - a(L - 4)) - (a(L - 4) - a(L - 7))) + s5d * ((a(L) - a(L - 4)) - (a(L - 4) - a(L - 8)));
    case 3: return s4a * ((a(L - 2) - a(L - 3)) - (a(L - 3) - a(L - 4))) + s4b * ((a(L - 1) - a(L - 3)) - (a(L - 3) - a(L - 5))) + s4c * ((a(L) - a(L - 3)) - (a(L - 3) - a(L - 6)));
    case 2: return s3a * ((a(L - 1) - a(L - 2)) - (a(L - 2) - a(L - 3))) + s3b * ((a(L) - a(L - 2)) - (a(L - 2) - a(L - 4)));
    case 1: return s2a * (a(L) - a(L - 1)) + s2b * (a(L - 2) - a(L - 1)) + s2c * (a(L - 3) - a(L - 1)) + s2d * (a(L - 4) - a(L - 1)) + s2e * (a(L - 5) - a(L - 1));
    default: return s1a * (a(L - 1) - a(L)) + s1b * (a(L - 2) - a(L)) + s1c * (a(L - 3) - a(L)) + s1d * (a(L - 4) - a(L)) + s1e * (a(L - 5) - a(L));
  }
}

// Mixed derivative, interior diagonal scheme; v(ma, mb) is the value ma, mb
// points away along the two directions.
template <class V2>
__device__ __forceinline__ double dmcore(const V2& v) {
  using namespace fdc;
  const double fa = v(1, 1) - v(1, -1) - v(-1, 1) + v(-1, -1);
  const double fb = v(2, 2) - v(2, -2) - v(-2, 2) + v(-2, -2);
  const double fc = v(3, 3) - v(3, -3) - v(-3, 3) + v(-3, -3);
  const double fd = v(4, 4) - v(4, -4) - v(-4, 4) + v(-4, -4);
  const double fe = v(5, 5) - v(5, -5) - v(-5, 5) + v(-5, -5);
  return ax * fa + bx * fb + cx * fc + dx * fd + ex * fe;
}

// Mixed derivative with a bounded first direction and a periodic second one
// (src/d2fdxy.f:151-392, d2fdxz.f likewise): on the first two points the
// one-sided first-derivative rows act on a 4th-order centred difference in
// the second direction (ACOFY1, BCOFY1); points 3-5 from each end use the
// diagonal 4th/6th/8th-order schemes (ACF3XY..DCF5XY); the rest the
// 10th-order interior scheme. c is the point's coordinate along the bounded
// direction, n its extent; v(ma, mb) as for dmcore.
namespace fdc {
constexpr double my1 = (4.0 / 3.0) / 2.0, my2 = (-1.0 / 3.0) / 4.0;
constexpr double m3a = (4.0 / 3.0) / 4.0, m3b = (-1.0 / 3.0) / 4.0 / 4.0;
constexpr double m4a = (3.0 / 2.0) / 4.0, m4b = (-3.0 / 5.0) / 4.0 / 4.0, m4c = (1.0 / 1.0e1) / 4.0 / 9.0;
constexpr double m5a = (8.0 / 5.0) / 4.0, m5b = (-4.0 / 5.0) / 4.0 / 4.0, m5c = (8.0 / 3.5e1) / 4.0 / 9.0,
                 m5d = (-1.0 / 3.5e1) / 4.0 / 1.6e1;
}  // namespace fdc
template <class V2>
__device__ __forceinline__ double dmcore_b(const V2& v, int c, int n) {
  using namespace fdc;
  if (c > n - 1) c = n - 1;  // see d1core
  if (c >= 5 && c <= n - 6) return dmcore(v);
  auto dg = [&](int m) { return v(m, m) - v(m, -m) - v(-m, m) + v(-m, -m); };
  auto g2 = [&](int a, int a0) {  // absolute indices along the bounded direction
    const int da = a - c, d0 = a0 - c;
    return my1 * (v(da, 1) - v(da, -1) - v(d0, 1) + v(d0, -1)) + my2 * (v(da, 2) - v(da, -2) - v(d0, 2) + v(d0, -2));
  };
  const int L = n - 1;
  const int e = c < 5 ? c : L - c;  // distance from the nearer end
  switch (e) {
    case 2: return m3a * dg(1) + m3b * dg(2);
    case 3: return m4a * dg(1) + m4b * dg(2) + m4c * dg(3);
    case 4: return m5a * dg(1) + m5b * dg(2) + m5c * dg(3) + m5d * dg(4);
    default: break;
  }
  if (c == 0) return p1a * g2(1, 0) + p1b * g2(2, 0) + p1c * g2(3, 0) + p1d * g2(4, 0);
  if (c == 1) return p2a * g2(0, 1) + p2b * g2(2, 1) + p2c * g2(3, 1) + p2d * g2(4, 1);
  if (c == L) return p1a * g2(L, L - 1) + p1b * g2(L, L - 2) + p1c * g2(L, L - 3) + p1d * g2(L, L - 4);
  return p2a * g2(L - 1, L) + p2b * g2(L - 1, L - 2) + p2c * g2(L - 1, L - 3) + p2d * g2(L - 1, L - 4);
}

// Mixed derivative with the second direction bounded, or both
// (src/d2fdxy.f:393-1924; d2fdxz.f and d2fdyz.f likewise). ea, eb are the
// point's distances from the nearer bounded end of each direction (a large
// number for a periodic one), ra_a / ra_b whether that end is the right one.
// Classification per point:
//   ea, eb >= 5: interior scheme;
//   ea, eb >= 2: diagonal 4th/6th/8th-order scheme of min(ea, eb) (end
//     sections' third to fifth rows and the corners' inner blocks);
//   ea <= 1 < eb (or the reverse): one-sided first-derivative rows along the
//     near direction on the 4th-order centred difference along the other;
//   ea, eb <= 1: corner point (ACC1XY, :516-528), its diagonal neighbour
//     (ACC2XY, :530-542), the two edge points (first-point rows of
//     second-point differences, :544-626).
// A right end is the mirror image of the left: offsets are taken inward and
// a one-sided result changes sign per mirrored direction. v(ma, mb) as for
// dmcore.
namespace fdc {
constexpr double k1a = p1a, k1b = p1b * 2.0 / 4.0, k1c = p1c * 3.0 / 9.0, k1d = p1d * 4.0 / 1.6e1;  // ACC1XY..
constexpr double k2a = -p2a, k2b = p2b, k2c = p2c * 2.0 / 4.0, k2d = p2d * 3.0 / 9.0;                // ACC2XY..
}  // namespace fdc
template <class V2>
__device__ __forceinline__ double dmcore_ends(const V2& v, int ea, bool ra_a, int eb, bool ra_b) {
  using namespace fdc;
  if (ea >= 5 && eb >= 5) return dmcore(v);
  const int sa = (ea <= 1 && ra_a) ? -1 : 1, sb = (eb <= 1 && ra_b) ? -1 : 1;
  auto w = [&](int ia, int ib) { return v(sa * ia, sb * ib); };
  auto dg = [&](int m) { return w(m, m) - w(m, -m) - w(-m, m) + w(-m, -m); };
  if (ea >= 2 && eb >= 2) {
    switch (ea < eb ? ea : eb) {
      case 2: return m3a * dg(1) + m3b * dg(2);
      case 3: return m4a * dg(1) + m4b * dg(2) + m4c * dg(3);
      default: return m5a * dg(1) + m5b * dg(2) + m5c * dg(3) + m5d * dg(4);
    }
  }
  if (eb >= 2) {  // one-sided along a, centred along b
    auto g = [&](int i1, int i0) {
      return my1 * (w(i1, 1) - w(i1, -1) - w(i0, 1) + w(i0, -1)) + my2 * (w(i1, 2) - w(i1, -2) - w(i0, 2) + w(i0, -2));
    };
    const double r = ea == 0 ? p1a * g(1, 0) + p1b * g(2, 0) + p1c * g(3, 0) + p1d * g(4, 0)
                             : p2a * g(-1, 0) + p2b * g(1, 0) + p2c * g(2, 0) + p2d * g(3, 0);
    return r * sa;
  }
  if (ea >= 2) {  // one-sided along b, centred along a
    auto g = [&](int i1, int i0) {
      return my1 * (w(1, i1) - w(-1, i1) - w(1, i0) + w(-1, i0)) + my2 * (w(2, i1) - w(-2, i1) - w(2, i0) + w(-2, i0));
    };
    const double r = eb == 0 ? p1a * g(1, 0) + p1b * g(2, 0) + p1c * g(3, 0) + p1d * g(4, 0)
                             : p2a * g(-1, 0) + p2b * g(1, 0) + p2c * g(2, 0) + p2d * g(3, 0);
    return r * sb;
  }
  auto q = [&](int ia, int ib) { return w(ia, ib) - w(ia, 0) - w(0, ib) + w(0, 0); };
  double r;
  if (ea == 0 && eb == 0) {
    r = k1a * q(1, 1) + k1b * q(2, 2) + k1c * q(3, 3) + k1d * q(4, 4);
  } else if (ea == 1 && eb == 1) {
    r = k2a * q(-1, -1) + k2b * q(1, 1) + k2c * q(2, 2) + k2d * q(3, 3);
  } else if (ea == 0) {  // eb == 1: first-point rows along a of second-point differences along b
    auto t = [&](int m) { return p2a * q(m, -1) + p2b * q(m, 1) + p2c * q(m, 2) + p2d * q(m, 3); };
    r = p1a * t(1) + p1b * t(2) + p1c * t(3) + p1d * t(4);
  } else {  // ea == 1, eb == 0
    auto t = [&](int m) { return p2a * q(-1, m) + p2b * q(1, m) + p2c * q(2, m) + p2d * q(3, m); };
    r = p1a * t(1) + p1b * t(2) + p1c * t(3) + p1d * t(4);
  }
  return r * (sa * sb);
}

// ---- global-memory forms (operator-level entry points) ----------------------
// Periodic directions wrap the index; bounded ones never leave the domain
// because the closures only read inward.
template <int DIR, class F>
__device__ __forceinline__ double D1(const Geo& g, const Pt& p, const F& f) {
  const int n = ext<DIR>(g), c = crd<DIR>(p);
  auto v = [&](int m) { return f(p.q + woff<DIR>(g, c, m)); };
  return d1core(v, c, n, g.per[DIR]) * g.ovd[DIR];
}
template <int DIR, class F>
__device__ __forceinline__ double D2(const Geo& g, const Pt& p, const F& f) {
  const int n = ext<DIR>(g), c = crd<DIR>(p);
  auto v = [&](int m) { return f(p.q + woff<DIR>(g, c, m)); };
  return d2core(v, c, n, g.per[DIR]) * g.ovd2[DIR];
}
template <int DA, int DB, class F>
__device__ __forceinline__ double DM(const Geo& g, const Pt& p, const F& f) {
  const int ca = crd<DA>(p), cb = crd<DB>(p);
  auto v = [&](int ma, int mb) { return f(p.q + woff<DA>(g, ca, ma) + woff<DB>(g, cb, mb)); };
  if (!g.per[DB]) {
    constexpr int kFar = 1 << 20;
    const int la = g.per[DA] ? kFar : ca, ra = g.per[DA] ? kFar : ext<DA>(g) - 1 - ca;
    const int lb = cb, rb = ext<DB>(g) - 1 - cb;
    return dmcore_ends(v, la < ra ? la : ra, ra < la, lb < rb ? lb : rb, rb < lb) * g.ovd[DA] * g.ovd[DB];
  }
  if (!g.per[DA]) return dmcore_b(v, ca, ext<DA>(g)) * g.ovd[DA] * g.ovd[DB];
  return dmcore(v) * g.ovd[DA] * g.ovd[DB];
}

// ---- accessors ----
// Field loads of the stencil kernels. NC = true: through the read-only data
// path (ld.global.nc), for launches in which no CTA writes the field. The
// persistent batch kernel reads fields that other CTAs of the same launch
// wrote (behind an acquire on a completion counter), so it takes NC = false:
// ordinary (coherent) global loads, cached in L1, which the acquire of the
// completion counter orders after the producers' writes.
template <bool NC>
__device__ __forceinline__ double ldf(const double* p) {
  if constexpr (NC) return __ldg(p);
  else return __ldca(p);  // ld.global.ca: global space, cached in L1, coherent
}
template <bool NC = true>
struct LdT {
  const double* a;
  __device__ __forceinline__ double operator()(int64_t q) const { return ldf<NC>(a + q); }
};
template <bool NC = true>
struct LdMulT {
  const double* a;
  const double* b;
  __device__ __forceinline__ double operator()(int64_t q) const { return ldf<NC>(a + q) * ldf<NC>(b + q); }
};
template <bool NC = true>
struct LdSubT {
  const double* a;
  double c;
  __device__ __forceinline__ double operator()(int64_t q) const { return ldf<NC>(a + q) - c; }
};
using Ld = LdT<true>;
using LdMul = LdMulT<true>;
using LdSub = LdSubT<true>;

__device__ __forceinline__ Pt point_of(const Geo& g, int64_t q) {
  Pt p;
  p.q = q;
  const int64_t nxy = (int64_t)g.nx * g.ny;
  p.k = (int)(q / nxy);
  const int64_t r = q - (int64_t)p.k * nxy;
  p.j = (int)(r / g.nx);
  p.i = (int)(r - (int64_t)p.j * g.nx);
  return p;
}

}  // namespace senga
