// Host-side chemistry / transport table construction.
//
// chem.dat records: src/chemin.f:146-344 (fixed-format Fortran records,
// e.g. '(I5,1PE12.4)'); derived tables: src/chemin.f:822-983.
// diff.dat records: src/diffin.f:100-232 (list-directed); derived tables:
// src/diffin.f:328-405.
// The reference reads on rank 0 and broadcasts (P_BCST); here the host reads
// once and the tables are uploaded to the device with the context.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "senga_gpu.h"
#include "senga_internal.h"

namespace {

constexpr double kRgUniv = 8.3142e3;  // RGUNIV, src/com_senga2.h:119
constexpr double kAlamdc = 2.58e-5, kRlamda = 7.0e-1, kTlamda = 2.98e2;  // :113

class Records {
 public:
  explicit Records(const char* path) : in_(path) {
    if (!in_) throw senga::Error(SENGA_ERR_IO, std::string("cannot open ") + path);
  }
  std::string line() {
    std::string s;
    if (!std::getline(in_, s)) throw senga::Error(SENGA_ERR_IO, "premature end of table file");
    if (!s.empty() && s.back() == '\r') s.pop_back();
    return s;
  }
  void skip(int n = 1) {
    for (int i = 0; i < n; ++i) line();
  }

 private:
  std::ifstream in_;
};

// Fixed-width field [col, col+width) of a record: blank-padded, embedded
// blanks ignored, 'D' exponents accepted (Fortran formatted input rules).
std::string field(const std::string& rec, size_t col, size_t width) {
  std::string out;
  for (size_t i = col; i < col + width && i < rec.size(); ++i) {
    char ch = rec[i];
    if (ch == ' ' || ch == '\t') continue;
    out.push_back(ch == 'D' || ch == 'd' ? 'E' : ch);
  }
  return out;
}
int ifield(const std::string& rec, size_t col, size_t width) {
  std::string s = field(rec, col, width);
  return s.empty() ? 0 : std::atoi(s.c_str());
}
double rfield(const std::string& rec, size_t col, size_t width) {
  std::string s = field(rec, col, width);
  return s.empty() ? 0.0 : std::strtod(s.c_str(), nullptr);
}
// 0-based index of a record field, checked against the table extent.
int at(int v, int extent, const char* what) {
  if (v < 0 || v >= extent) throw senga::Error(SENGA_ERR_ARG, std::string("chem.dat: bad index in ") + what);
  return v;
}
std::vector<double> free_format(const std::string& rec) {
  std::string s = rec;
  for (auto& ch : s) {
    if (ch == ',') ch = ' ';
    if (ch == 'D' || ch == 'd') ch = 'E';
  }
  std::istringstream is(s);
  std::vector<double> v;
  double x;
  while (is >> x) v.push_back(x);
  return v;
}

void load_chem(const char* path, senga_chem& c) {
  std::memset(&c, 0, sizeof(c));
  Records r(path);
  r.skip(5);
  r.skip();
  c.nspec = ifield(r.line(), 0, 5);
  if (c.nspec < 1 || c.nspec > SENGA_NSPCMX) throw senga::Error(SENGA_ERR_ARG, "chem.dat: NSPEC out of range");
  r.skip(c.nspec);
  r.skip();
  c.prefgb = free_format(r.line()).at(0);
  for (int n = 0; n < c.nspec; ++n) {
    std::string rec = r.line();
    int is = ifield(rec, 0, 5) - 1;
    if (is < 0 || is >= c.nspec) throw senga::Error(SENGA_ERR_ARG, "chem.dat: species index");
    c.wmolar[is] = rfield(rec, 5, 12);
    c.clewis[is] = rfield(r.line(), 0, 12);
    c.ntint[is] = ifield(r.line(), 0, 5);
    if (c.ntint[is] < 1 || c.ntint[is] > SENGA_NTINMX) throw senga::Error(SENGA_ERR_ARG, "chem.dat: NTINT");
    for (int it = 0; it < c.ntint[is]; ++it) {
      std::string ri = r.line();
      c.tintlo[is][it] = rfield(ri, 0, 12);
      c.tinthi[is][it] = rfield(ri, 12, 12);
      c.ncofcp[is][it] = ifield(ri, 24, 5);
      if (c.ncofcp[is][it] < 3 || c.ncofcp[is][it] > SENGA_NCOFMX) throw senga::Error(SENGA_ERR_ARG, "chem.dat: NCOFCP");
      for (int icp = 0; icp < c.ncofcp[is][it]; ++icp) c.amolcp[is][it][icp] = rfield(r.line(), 0, 15);
    }
  }
  r.skip();
  c.nstep = ifield(r.line(), 0, 5);
  if (c.nstep < 1 || c.nstep > SENGA_NSTPMX) throw senga::Error(SENGA_ERR_ARG, "chem.dat: NSTEP out of range");
  for (int n = 0; n < c.nstep; ++n) {
    std::string rec = r.line();
    int st = at(ifield(rec, 0, 5) - 1, c.nstep, "step rate data");
    for (int q = 0; q < 3; ++q) c.rparam[st][q] = rfield(rec, 5 + 12 * q, 12);
  }
  auto step_list = [&](int* len, int (*lst)[SENGA_NSSMAX], double (*coef)[SENGA_NSSMAX]) {
    r.skip();
    for (int n = 0; n < c.nstep; ++n) {
      std::string rec = r.line();
      int st = at(ifield(rec, 0, 5) - 1, c.nstep, "step list");
      len[st] = ifield(rec, 5, 5);
      if (len[st] < 0 || len[st] > SENGA_NSSMAX) throw senga::Error(SENGA_ERR_ARG, "chem.dat: list length");
      for (int q = 0; q < len[st]; ++q) {
        std::string e = r.line();
        int st2 = at(ifield(e, 0, 5) - 1, c.nstep, "step list"), slot = at(ifield(e, 5, 5) - 1, SENGA_NSSMAX, "step list");
        lst[st2][slot] = ifield(e, 10, 8);
        if (coef) coef[st2][slot] = rfield(e, 18, 12);
      }
    }
  };
  step_list(c.nsslen, c.nsspec, nullptr);
  step_list(c.nrslen, c.nrspec, nullptr);
  step_list(c.npslen, c.npspec, nullptr);
  step_list(c.nrclen, c.nrcpec, c.crspec);
  step_list(c.npclen, c.npcpec, c.cpspec);
  r.skip();
  for (int st = 0; st < c.nstep; ++st)
    for (int q = 0; q < c.nsslen[st]; ++q) {
      std::string e = r.line();
      c.diffmu[at(ifield(e, 0, 5) - 1, c.nstep, "delta-list")][at(ifield(e, 5, 5) - 1, SENGA_NSSMAX, "delta-list")] =
          rfield(e, 10, 5);
    }
  r.skip();
  c.nbody = ifield(r.line(), 0, 5);
  if (c.nbody < 0 || c.nbody > SENGA_NBDYMX) throw senga::Error(SENGA_ERR_ARG, "chem.dat: NBODY out of range");
  r.skip(c.nbody);
  r.skip();
  if (c.nbody > 0)
    for (int n = 0; n < c.nstep; ++n) {
      std::string e = r.line();
      c.mblist[at(ifield(e, 0, 5) - 1, c.nstep, "third-body step-list")] = ifield(e, 5, 8);
    }
  r.skip();
  for (int b = 0; b < c.nbody; ++b)
    for (int s = 0; s < c.nspec; ++s) {
      std::string e = r.line();
      c.effy3b[at(ifield(e, 0, 5) - 1, c.nbody, "efficiencies")][at(ifield(e, 5, 5) - 1, c.nspec, "efficiencies")] =
          rfield(e, 10, 12);
    }
  auto flag_list = [&](int* count, int* lst) {
    r.skip();
    *count = ifield(r.line(), 0, 5);
    if (*count > 0)
      for (int n = 0; n < c.nstep; ++n) {
        std::string e = r.line();
        lst[at(ifield(e, 0, 5) - 1, c.nstep, "step flag list")] = ifield(e, 5, 8);
      }
  };
  flag_list(&c.ngibb, c.mglist);
  flag_list(&c.nlind, c.mllist);
  r.skip();
  for (int n = 0; n < c.nlind; ++n) {
    std::string e = r.line();
    int il = at(ifield(e, 0, 5) - 1, SENGA_NLLMAX, "Lindemann data");
    for (int q = 0; q < 4; ++q) c.rclind[il][q] = rfield(e, 5 + 12 * q, 12);
  }
  flag_list(&c.ntroe, c.mtlist);
  r.skip();
  for (int n = 0; n < c.ntroe; ++n) {
    std::string e = r.line();
    int it = at(ifield(e, 0, 5) - 1, SENGA_NLLMAX, "Troe data");
    for (int q = 0; q < 6; ++q) c.rctroe[it][q] = rfield(e, 5 + 12 * q, 12);
    e = r.line();
    for (int q = 0; q < 6; ++q) c.rctroe[it][6 + q] = rfield(e, 5 + 12 * q, 12);
  }
  flag_list(&c.nsrif, c.mslist);
  r.skip();
  for (int n = 0; n < c.nsrif; ++n) {
    std::string e = r.line();
    int is = at(ifield(e, 0, 5) - 1, SENGA_NLLMAX, "SRI data");
    for (int q = 0; q < 3; ++q) c.rcsrif[is][q] = rfield(e, 5 + 12 * q, 12);
    e = r.line();
    for (int q = 0; q < 5; ++q) c.rcsrif[is][3 + q] = rfield(e, 5 + 12 * q, 12);
  }

  // every species/step index used by the device kernels must be in range
  auto in_range = [](int v, int lo, int hi, const char* what) {
    if (v < lo || v > hi) throw senga::Error(SENGA_ERR_ARG, std::string("chem.dat: index out of range in ") + what);
  };
  for (int st = 0; st < c.nstep; ++st) {
    for (int q = 0; q < c.nsslen[st]; ++q) in_range(c.nsspec[st][q], 1, c.nspec, "species-list");
    for (int q = 0; q < c.nrslen[st]; ++q) in_range(c.nrspec[st][q], 1, c.nspec, "reactant-list");
    for (int q = 0; q < c.npslen[st]; ++q) in_range(c.npspec[st][q], 1, c.nspec, "product-list");
    for (int q = 0; q < c.nrclen[st]; ++q) in_range(c.nrcpec[st][q], 1, c.nspec, "reactant coefficient-list");
    for (int q = 0; q < c.npclen[st]; ++q) in_range(c.npcpec[st][q], 1, c.nspec, "product coefficient-list");
    in_range(c.mblist[st], 0, c.nbody, "third-body step-list");
    in_range(c.mllist[st], 0, c.nlind, "Lindemann step-list");
    in_range(c.mtlist[st], 0, c.ntroe, "Troe step-list");
    in_range(c.mslist[st], 0, c.nsrif, "SRI step-list");
  }
  in_range(c.nbody, 0, SENGA_NBDYMX, "third-body count");
  in_range(c.nlind, 0, SENGA_NLLMAX, "Lindemann count");
  in_range(c.ntroe, 0, SENGA_NLLMAX, "Troe count");
  in_range(c.nsrif, 0, SENGA_NLLMAX, "SRI count");

  // ---- derived quantities (src/chemin.f:822-983) ----
  for (int st = 0; st < c.nstep; ++st) {
    c.rparam[st][0] = std::log(c.rparam[st][0]);
    c.rparam[st][2] = c.rparam[st][2] / kRgUniv;
  }
  for (int il = 0; il < c.nlind; ++il) {
    c.rclind[il][0] = std::log(c.rclind[il][0]);
    c.rclind[il][2] = c.rclind[il][2] / kRgUniv;
  }
  for (int it = 0; it < c.ntroe; ++it) {
    c.rctroe[it][0] = std::log(c.rctroe[it][0]);
    c.rctroe[it][2] = c.rctroe[it][2] / kRgUniv;
    c.rctroe[it][4] = -1.0 / c.rctroe[it][4];
    c.rctroe[it][6] = -1.0 / c.rctroe[it][6];
  }
  for (int is = 0; is < c.nsrif; ++is) {
    c.rcsrif[is][0] = std::log(c.rcsrif[is][0]);
    c.rcsrif[is][2] = c.rcsrif[is][2] / kRgUniv;
    c.rcsrif[is][4] = -c.rcsrif[is][4];
    c.rcsrif[is][5] = -1.0 / c.rcsrif[is][5];
  }
  for (int st = 0; st < c.nstep; ++st)
    for (int q = 0; q < c.nsslen[st]; ++q) c.diffmw[st][q] = c.diffmu[st][q] * c.wmolar[c.nsspec[st][q] - 1];
  for (int s = 0; s < c.nspec; ++s) {
    c.ovwmol[s] = 1.0 / c.wmolar[s];
    c.rgspec[s] = kRgUniv * c.ovwmol[s];
  }
  for (int s = 0; s < c.nspec; ++s)
    for (int it = 0; it < c.ntint[s]; ++it) {
      c.ncpoly[s][it] = c.ncofcp[s][it] - 2;
      c.ncpom1[s][it] = c.ncpoly[s][it] - 1;
      c.ncenth[s][it] = c.ncofcp[s][it] - 1;
      c.ncenpy[s][it] = c.ncofcp[s][it];
    }
  for (int s = 0; s < c.nspec; ++s)
    for (int it = 0; it < c.ntint[s]; ++it) {
      const int np = c.ncpoly[s][it], nh = c.ncenth[s][it] - 1, ns = c.ncenpy[s][it] - 1;
      double* cp = c.amascp[s][it];
      for (int q = 0; q < c.ncofcp[s][it]; ++q) cp[q] = c.amolcp[s][it][q] * kRgUniv * c.ovwmol[s];
      c.amasct[s][it][0] = cp[0] - c.rgspec[s];
      c.amasch[s][it][0] = cp[0];
      c.amascs[s][it][0] = cp[0];
      for (int q = 2; q <= np; ++q) {
        c.amasct[s][it][q - 1] = cp[q - 1] / (double)q;
        c.amasch[s][it][q - 1] = cp[q - 1] / (double)q;
        c.amascs[s][it][q - 1] = cp[q - 1] / (double)(q - 1);
      }
      c.amasct[s][it][nh] = 0.0;
      c.amasct[s][it][ns] = 0.0;
      c.amasch[s][it][nh] = cp[nh];
      c.amasch[s][it][ns] = 0.0;
      c.amascs[s][it][nh] = 0.0;
      c.amascs[s][it][ns] = cp[ns];
    }
  const double giblet = std::log(c.prefgb / kRgUniv);
  for (int s = 0; s < c.nspec; ++s)
    for (int it = 0; it < c.ntint[s]; ++it) {
      const int np = c.ncpoly[s][it], nh = c.ncenth[s][it] - 1, ns = c.ncenpy[s][it] - 1;
      double* m = c.amolcp[s][it];
      double* g = c.amolgb[s][it];
      g[0] = m[ns] - m[0] + giblet;
      for (int q = 2; q <= np; ++q) g[q - 1] = m[q - 1] / (double)(q * (q - 1));
      g[nh] = m[nh];
      g[ns] = m[0] - 1.0;
    }
  for (int s = 0; s < c.nspec; ++s)
    for (int it = 0; it < c.ntint[s]; ++it)
      for (int q = 0; q < c.ncofcp[s][it]; ++q) c.amolcp[s][it][q] = c.amolcp[s][it][q] * kRgUniv;
  for (int s = 0; s < c.nspec; ++s) c.olewis[s] = 1.0 / c.clewis[s];
  c.alamda = kAlamdc * std::exp(-kRlamda * std::log(kTlamda));
}

void load_diff(const char* path, const senga_chem& c, senga_diff& d) {
  std::memset(&d, 0, sizeof(d));
  if (path == nullptr) return;  // constant-Lewis transport
  Records r(path);
  r.skip(5);
  r.skip();
  int nd = ifield(r.line(), 0, 5);
  if (nd != c.nspec) throw senga::Error(SENGA_ERR_ARG, "diff.dat: species count differs from chem.dat");
  r.skip(c.nspec);
  r.skip();
  {
    auto v = free_format(r.line());
    if (v.size() < 2) throw senga::Error(SENGA_ERR_IO, "diff.dat: reference data");
    d.pdifgb = v[0];
    d.tdifgb = v[1];
  }
  auto values = [&](size_t n) {
    std::vector<double> v;
    while (v.size() < n) {
      auto t = free_format(r.line());
      v.insert(v.end(), t.begin(), t.end());
    }
    return v;
  };
  auto header_count = [&]() {
    auto h = free_format(r.line());
    int n = (int)h.at(1);
    if (n < 1 || n > SENGA_NDCFMX) throw senga::Error(SENGA_ERR_ARG, "diff.dat: coefficient count");
    return n;
  };
  r.skip();
  for (int s = 0; s < c.nspec; ++s) {
    d.ncovis = header_count();
    auto v = values(d.ncovis);
    for (int q = 0; q < d.ncovis; ++q) d.viscco[s][q] = v[q];
  }
  r.skip();
  for (int s = 0; s < c.nspec; ++s) {
    d.ncocon = header_count();
    auto v = values(d.ncocon);
    for (int q = 0; q < d.ncocon; ++q) d.condco[s][q] = v[q];
  }
  r.skip();
  for (int s = 0; s < c.nspec; ++s) {
    d.ncodif = header_count();
    for (int t = 0; t <= s; ++t) {
      auto v = values(1 + d.ncodif);
      for (int q = 0; q < d.ncodif; ++q) d.diffco[s][t][q] = v[1 + q];
    }
  }
  r.skip();
  for (int s = 0; s < c.nspec; ++s) {
    d.ncotdr = header_count();
    for (int t = 0; t < s; ++t) {
      auto v = values(1 + d.ncotdr);
      for (int q = 0; q < d.ncotdr; ++q) d.tdrcco[s][t][q] = v[1 + q];
    }
  }
  // symmetric binary diffusion, antisymmetric thermal diffusion (:331-365)
  for (int s = 0; s < c.nspec; ++s)
    for (int t = s + 1; t < c.nspec; ++t)
      for (int q = 0; q < d.ncodif; ++q) d.diffco[s][t][q] = d.diffco[t][s][q];
  for (int s = 0; s < c.nspec; ++s) {
    for (int q = 0; q < d.ncotdr; ++q) d.tdrcco[s][s][q] = 0.0;
    for (int t = 0; t < s; ++t)
      for (int q = 0; q < d.ncotdr; ++q) d.tdrcco[s][t][q] = -d.tdrcco[s][t][q];
    for (int t = s + 1; t < c.nspec; ++t)
      for (int q = 0; q < d.ncotdr; ++q) d.tdrcco[s][t][q] = d.tdrcco[t][s][q];
  }
  // Wilke combination-rule factors (:370-377); WILKO(JSPEC,ISPEC) -> [is][js]
  for (int s = 0; s < c.nspec; ++s)
    for (int t = 0; t < c.nspec; ++t) {
      double ratio = c.wmolar[s] / c.wmolar[t];
      d.wilko2[s][t] = 1.0 / std::sqrt(std::sqrt(ratio));
      d.wilko1[s][t] = 1.0 / std::sqrt(8.0 * (1.0 + ratio));
    }
  d.flmavt = 1;
}

}  // namespace

extern "C" int senga_chem_load(const char* path, senga_chem* out) {
  if (!path || !out) return senga::fail(SENGA_ERR_ARG, "senga_chem_load: null argument");
  try {
    load_chem(path, *out);
    return SENGA_OK;
  } catch (const senga::Error& e) {
    return senga::fail(e.code, e.what());
  } catch (const std::exception& e) {
    return senga::fail(SENGA_ERR_IO, e.what());
  }
}

extern "C" int senga_diff_load(const char* path, const senga_chem* chem, senga_diff* out) {
  if (!chem || !out) return senga::fail(SENGA_ERR_ARG, "senga_diff_load: null argument");
  try {
    load_diff(path, *chem, *out);
    return SENGA_OK;
  } catch (const senga::Error& e) {
    return senga::fail(e.code, e.what());
  } catch (const std::exception& e) {
    return senga::fail(SENGA_ERR_IO, e.what());
  }
}

// INTEGF (src/integf.f:34-96): trapezoid sums refined by midpoints and
// combined Richardson-style into Simpson estimates (TOLINT=1e-6, INTMAX=20,
// first answer VSMALL). Like the reference, the first refinement samples 4
// midpoints on top of the 1-interval trapezoid (the 15-SEP-2012 change of
// the initial sampling), and a non-converged result is returned with a
// warning status rather than stopping.
extern "C" int senga_integf(senga_integrand f, void* user, double argmin, double argmax, double* answer) {
  if (!f || !answer) return senga::fail(SENGA_ERR_ARG, "senga_integf: null argument");
  const double tolint = 1.0e-6, vsmall = 1.0e-30;
  const int intmax = 20;
  int interv = 4, icount = 1;
  double ans = vsmall;
  double tmp = 0.5 * (argmax - argmin) * (f(argmin, user) + f(argmax, user));
  for (;;) {
    const double oldans = ans, oldtmp = tmp;
    const double delta = (argmax - argmin) / (double)(float)interv;
    double arg = argmin - 0.5 * delta, add = 0.0;
    for (int ic = 1; ic <= interv; ++ic) {
      arg = arg + delta;
      add = add + f(arg, user);
    }
    tmp = 0.5 * (tmp + add * delta);
    ans = (4.0 * tmp - oldtmp) / 3.0;
    if (std::fabs(ans - oldans) > tolint * std::fabs(oldans)) {
      icount = icount + 1;
      if (icount <= intmax) {
        interv = 2 * interv;
        continue;
      }
      *answer = ans;
      return senga::fail(SENGA_ERR_ARG, "senga_integf: integral not converged");
    }
    break;
  }
  *answer = ans;
  return SENGA_OK;
}
