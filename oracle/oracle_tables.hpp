// ORACLE — TEST INFRASTRUCTURE ONLY.
// CPU restatement of the reference's chemistry / transport table set-up.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
// load this code, and only as the checker. The product path never does.
//
// Restates (file:line within the reference project):
//   src/chemin.f:146-344   chem.dat parsing (fixed-format Fortran records)
//   src/chemin.f:822-983   derived thermochemical tables
//   src/diffin.f:100-232   diff.dat parsing (list-directed records)
//   src/diffin.f:328-405   derived transport tables (symmetric DIFFCO,
//                          antisymmetric TDRCCO, Wilke factors)
//   src/com_senga2.h:80-214 table dimensions and physical constants
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

// Dimensions (src/com_senga2.h:80-100)
// NSPCMX and NSTPMX as the reference's largest shipped case compiles them
// (src/casefiles/68step/com_senga2.h:74)
constexpr int NSPCMX = 18, NSTPMX = 68, NTINMX = 2, NCOFMX = 7, NCTMAX = 5;
constexpr int NSPIMX = 15, NTBASE = 4, NINTMX = 2, NBDYMX = 10;
constexpr int NSSMAX = 10, NRSMAX = 10, NLLMAX = 10;
constexpr int NDCFMX = 4, NVCFMX = 4, NCCFMX = 4;
// Constants (src/com_senga2.h:113-119,187)
constexpr double ALAMDC = 2.58e-5, RLAMDA = 7.0e-1, TLAMDA = 2.98e2;
constexpr double PRANTL = 7.0e-1;
constexpr double RGUNIV = 8.3142e3;
constexpr double DFCTOL = 1.0e-12;

// Fortran-style 1-based table with column-major storage.
struct Chem {
  int nspec = 0, nstep = 0, nbody = 0, ngibb = 0, nlind = 0, ntroe = 0, nsrif = 0;
  double prefgb = 0, alamda = 0;
  // [icp][itint][ispec] -> amolcp[(ispec-1)*NTINMX*NCOFMX + (itint-1)*NCOFMX + icp-1]
  double amolcp[NSPCMX * NTINMX * NCOFMX] = {}, amolgb[NSPCMX * NTINMX * NCOFMX] = {};
  double amascp[NSPCMX * NTINMX * NCOFMX] = {}, amasct[NSPCMX * NTINMX * NCOFMX] = {};
  double amasch[NSPCMX * NTINMX * NCOFMX] = {}, amascs[NSPCMX * NTINMX * NCOFMX] = {};
  double tintlo[NSPCMX * NTINMX] = {}, tinthi[NSPCMX * NTINMX] = {};
  double diffmu[NSTPMX * NSSMAX] = {}, diffmw[NSTPMX * NSSMAX] = {};
  double crspec[NSTPMX * NSSMAX] = {}, cpspec[NSTPMX * NSSMAX] = {};
  double effy3b[NBDYMX * NSPCMX] = {};
  double rparam[NSTPMX * 3] = {};
  double rclind[NLLMAX * 4] = {}, rctroe[NLLMAX * 12] = {}, rcsrif[NLLMAX * 8] = {};
  double wmolar[NSPCMX] = {}, ovwmol[NSPCMX] = {}, rgspec[NSPCMX] = {};
  double clewis[NSPCMX] = {}, olewis[NSPCMX] = {};
  int nsspec[NSTPMX * NSSMAX] = {}, nrspec[NSTPMX * NSSMAX] = {}, npspec[NSTPMX * NSSMAX] = {};
  int nrcpec[NSTPMX * NSSMAX] = {}, npcpec[NSTPMX * NSSMAX] = {};
  int ncofcp[NSPCMX * NTINMX] = {}, ncpoly[NSPCMX * NTINMX] = {}, ncpom1[NSPCMX * NTINMX] = {};
  int ncenth[NSPCMX * NTINMX] = {}, ncenpy[NSPCMX * NTINMX] = {};
  int nsslen[NSTPMX] = {}, nrslen[NSTPMX] = {}, npslen[NSTPMX] = {};
  int nrclen[NSTPMX] = {}, npclen[NSTPMX] = {};
  int mblist[NSTPMX] = {}, mglist[NSTPMX] = {}, mllist[NSTPMX] = {};
  int mtlist[NSTPMX] = {}, mslist[NSTPMX] = {};
  int ntint[NSPCMX] = {};

  // 1-based accessors
  static int c3(int icp, int it, int is) { return (is - 1) * NTINMX * NCOFMX + (it - 1) * NCOFMX + (icp - 1); }
  static int c2(int it, int is) { return (is - 1) * NTINMX + (it - 1); }
  static int ss(int isl, int istep) { return (istep - 1) * NSSMAX + (isl - 1); }
};

struct Diff {
  bool flmavt = false, flmixw = false, flmixp = false, flmixt = false;
  int ncodif = 0, ncotdr = 0, ncovis = 0, nccon = 0;
  double pdifgb = 0, tdifgb = 0;
  // DIFFCO(icoeff, jspec, ispec)
  double diffco[NDCFMX * NSPCMX * NSPCMX] = {}, tdrcco[NDCFMX * NSPCMX * NSPCMX] = {};
  double wilko1[NSPCMX * NSPCMX] = {}, wilko2[NSPCMX * NSPCMX] = {};
  double viscco[NVCFMX * NSPCMX] = {}, condco[NCCFMX * NSPCMX] = {};
  static int d3(int ic, int j, int i) { return (i - 1) * NSPCMX * NDCFMX + (j - 1) * NDCFMX + (ic - 1); }
  static int d2(int j, int i) { return (i - 1) * NSPCMX + (j - 1); }
  static int v2(int ic, int is) { return (is - 1) * NVCFMX + (ic - 1); }
};

// ---------------------------------------------------------------------------
// Fortran fixed-format field extraction. A field that is all blanks reads as
// zero (BLANK='NULL' default for formatted input); text beyond the end of a
// record reads as blanks (PAD='YES').
inline std::string fld(const std::string& line, size_t off, size_t w) {
  if (off >= line.size()) return std::string();
  return line.substr(off, w);
}
inline long fint(const std::string& s) {
  std::string t;
  for (char ch : s) if (ch != ' ' && ch != '\r' && ch != '\n') t.push_back(ch);
  if (t.empty()) return 0;
  return std::strtol(t.c_str(), nullptr, 10);
}
inline double freal(const std::string& s) {
  std::string t;
  for (char ch : s) {
    if (ch == ' ' || ch == '\r' || ch == '\n') continue;
    t.push_back((ch == 'D' || ch == 'd') ? 'E' : ch);
  }
  if (t.empty()) return 0.0;
  return std::strtod(t.c_str(), nullptr);
}

struct LineReader {
  std::ifstream in;
  explicit LineReader(const std::string& path) : in(path) {
    if (!in) throw std::runtime_error("cannot open " + path);
  }
  std::string next() {
    std::string l;
    if (!std::getline(in, l)) throw std::runtime_error("unexpected end of file");
    return l;
  }
};

// chem.dat reader: src/chemin.f:146-344 (records), src/chemin.f:822-983 (derived).
inline void read_chem(const std::string& path, Chem& c) {
  LineReader r(path);
  for (int i = 0; i < 5; ++i) r.next();  // header
  r.next();                              // "Species list:"
  c.nspec = (int)fint(fld(r.next(), 0, 5));
  if (c.nspec < 1 || c.nspec > NSPCMX) throw std::runtime_error("NSPEC out of range");
  for (int j = 0; j < c.nspec; ++j) r.next();  // '(I5,3X,A)' symbols
  r.next();                                     // "Species data:"
  c.prefgb = freal(r.next());                   // list-directed
  for (int j = 0; j < c.nspec; ++j) {
    std::string l = r.next();
    int is = (int)fint(fld(l, 0, 5));
    c.wmolar[is - 1] = freal(fld(l, 5, 12));
    c.clewis[is - 1] = freal(fld(r.next(), 0, 12));
    c.ntint[is - 1] = (int)fint(fld(r.next(), 0, 5));
    for (int it = 1; it <= c.ntint[is - 1]; ++it) {
      std::string li = r.next();
      c.tintlo[Chem::c2(it, is)] = freal(fld(li, 0, 12));
      c.tinthi[Chem::c2(it, is)] = freal(fld(li, 12, 12));
      c.ncofcp[Chem::c2(it, is)] = (int)fint(fld(li, 24, 5));
      for (int icp = 1; icp <= c.ncofcp[Chem::c2(it, is)]; ++icp)
        c.amolcp[Chem::c3(icp, it, is)] = freal(fld(r.next(), 0, 15));
    }
  }
  r.next();  // "Step rate data:"
  c.nstep = (int)fint(fld(r.next(), 0, 5));
  if (c.nstep < 1 || c.nstep > NSTPMX) throw std::runtime_error("NSTEP out of range");
  for (int j = 0; j < c.nstep; ++j) {
    std::string l = r.next();
    int ist = (int)fint(fld(l, 0, 5));
    for (int icp = 0; icp < 3; ++icp) c.rparam[(ist - 1) * 3 + icp] = freal(fld(l, 5 + 12 * icp, 12));
  }
  auto read_list = [&](int* len, int* lst, double* coef) {
    r.next();
    for (int j = 0; j < c.nstep; ++j) {
      std::string l = r.next();
      int ist = (int)fint(fld(l, 0, 5));
      len[ist - 1] = (int)fint(fld(l, 5, 5));
      for (int k = 0; k < len[ist - 1]; ++k) {
        std::string lk = r.next();
        int ist2 = (int)fint(fld(lk, 0, 5));
        int isl = (int)fint(fld(lk, 5, 5));
        lst[Chem::ss(isl, ist2)] = (int)fint(fld(lk, 10, 8));
        if (coef) coef[Chem::ss(isl, ist2)] = freal(fld(lk, 18, 12));
      }
    }
  };
  read_list(c.nsslen, c.nsspec, nullptr);
  read_list(c.nrslen, c.nrspec, nullptr);
  read_list(c.npslen, c.npspec, nullptr);
  read_list(c.nrclen, c.nrcpec, c.crspec);
  read_list(c.npclen, c.npcpec, c.cpspec);
  r.next();  // "Species delta-list:"
  for (int js = 1; js <= c.nstep; ++js)
    for (int k = 0; k < c.nsslen[js - 1]; ++k) {
      std::string l = r.next();
      int ist = (int)fint(fld(l, 0, 5));
      int isl = (int)fint(fld(l, 5, 5));
      c.diffmu[Chem::ss(isl, ist)] = freal(fld(l, 10, 5));
    }
  r.next();  // "Third-body list:"
  c.nbody = (int)fint(fld(r.next(), 0, 5));
  for (int j = 0; j < c.nbody; ++j) r.next();
  r.next();  // "Third-body step-list:"
  if (c.nbody > 0)
    for (int j = 0; j < c.nstep; ++j) {
      std::string l = r.next();
      c.mblist[fint(fld(l, 0, 5)) - 1] = (int)fint(fld(l, 5, 8));
    }
  r.next();  // "Third-body efficiencies:"
  for (int jb = 0; jb < c.nbody; ++jb)
    for (int js = 0; js < c.nspec; ++js) {
      std::string l = r.next();
      int ib = (int)fint(fld(l, 0, 5)), is = (int)fint(fld(l, 5, 5));
      c.effy3b[(ib - 1) * NSPCMX + (is - 1)] = freal(fld(l, 10, 12));
    }
  auto read_steplist = [&](int* n, int* lst) {
    r.next();
    *n = (int)fint(fld(r.next(), 0, 5));
    if (*n > 0)
      for (int j = 0; j < c.nstep; ++j) {
        std::string l = r.next();
        lst[fint(fld(l, 0, 5)) - 1] = (int)fint(fld(l, 5, 8));
      }
  };
  read_steplist(&c.ngibb, c.mglist);
  read_steplist(&c.nlind, c.mllist);
  r.next();  // "Lindemann step rate data:"
  for (int j = 0; j < c.nlind; ++j) {
    std::string l = r.next();
    int il = (int)fint(fld(l, 0, 5));
    for (int icp = 0; icp < 4; ++icp) c.rclind[(il - 1) * 4 + icp] = freal(fld(l, 5 + 12 * icp, 12));
  }
  read_steplist(&c.ntroe, c.mtlist);
  r.next();  // "Troe step rate data:"
  for (int j = 0; j < c.ntroe; ++j) {
    std::string l = r.next();
    int it = (int)fint(fld(l, 0, 5));
    for (int icp = 0; icp < 6; ++icp) c.rctroe[(it - 1) * 12 + icp] = freal(fld(l, 5 + 12 * icp, 12));
    l = r.next();
    for (int icp = 0; icp < 6; ++icp) c.rctroe[(it - 1) * 12 + 6 + icp] = freal(fld(l, 5 + 12 * icp, 12));
  }
  read_steplist(&c.nsrif, c.mslist);
  r.next();  // "SRI step rate data:"
  for (int j = 0; j < c.nsrif; ++j) {
    std::string l = r.next();
    int is = (int)fint(fld(l, 0, 5));
    for (int icp = 0; icp < 3; ++icp) c.rcsrif[(is - 1) * 8 + icp] = freal(fld(l, 5 + 12 * icp, 12));
    l = r.next();
    for (int icp = 0; icp < 5; ++icp) c.rcsrif[(is - 1) * 8 + 3 + icp] = freal(fld(l, 5 + 12 * icp, 12));
  }

  // ---- derived quantities: src/chemin.f:822-983 ----
  for (int is = 1; is <= c.nstep; ++is) {
    c.rparam[(is - 1) * 3 + 0] = std::log(c.rparam[(is - 1) * 3 + 0]);
    c.rparam[(is - 1) * 3 + 2] = c.rparam[(is - 1) * 3 + 2] / RGUNIV;
  }
  for (int il = 1; il <= c.nlind; ++il) {
    c.rclind[(il - 1) * 4 + 0] = std::log(c.rclind[(il - 1) * 4 + 0]);
    c.rclind[(il - 1) * 4 + 2] = c.rclind[(il - 1) * 4 + 2] / RGUNIV;
  }
  for (int it = 1; it <= c.ntroe; ++it) {
    double* t = &c.rctroe[(it - 1) * 12];
    t[0] = std::log(t[0]);
    t[2] = t[2] / RGUNIV;
    t[4] = -1.0 / t[4];
    t[6] = -1.0 / t[6];
  }
  for (int is = 1; is <= c.nsrif; ++is) {
    double* t = &c.rcsrif[(is - 1) * 8];
    t[0] = std::log(t[0]);
    t[2] = t[2] / RGUNIV;
    t[4] = -t[4];
    t[5] = -1.0 / t[5];
  }
  for (int ist = 1; ist <= c.nstep; ++ist)
    for (int isl = 1; isl <= c.nsslen[ist - 1]; ++isl) {
      int js = c.nsspec[Chem::ss(isl, ist)];
      c.diffmw[Chem::ss(isl, ist)] = c.diffmu[Chem::ss(isl, ist)] * c.wmolar[js - 1];
    }
  for (int is = 1; is <= c.nspec; ++is) {
    c.ovwmol[is - 1] = 1.0 / c.wmolar[is - 1];
    c.rgspec[is - 1] = RGUNIV * c.ovwmol[is - 1];
  }
  for (int is = 1; is <= c.nspec; ++is)
    for (int it = 1; it <= c.ntint[is - 1]; ++it) {
      int k = Chem::c2(it, is);
      c.ncpoly[k] = c.ncofcp[k] - 2;
      c.ncpom1[k] = c.ncpoly[k] - 1;
      c.ncenth[k] = c.ncofcp[k] - 1;
      c.ncenpy[k] = c.ncofcp[k];
    }
  for (int is = 1; is <= c.nspec; ++is)
    for (int it = 1; it <= c.ntint[is - 1]; ++it)
      for (int icp = 1; icp <= c.ncofcp[Chem::c2(it, is)]; ++icp)
        c.amascp[Chem::c3(icp, it, is)] = c.amolcp[Chem::c3(icp, it, is)] * RGUNIV * c.ovwmol[is - 1];
  for (int is = 1; is <= c.nspec; ++is)
    for (int it = 1; it <= c.ntint[is - 1]; ++it) {
      int k = Chem::c2(it, is);
      c.amasct[Chem::c3(1, it, is)] = c.amascp[Chem::c3(1, it, is)] - c.rgspec[is - 1];
      for (int icp = 2; icp <= c.ncpoly[k]; ++icp)
        c.amasct[Chem::c3(icp, it, is)] = c.amascp[Chem::c3(icp, it, is)] / (double)icp;
      c.amasct[Chem::c3(c.ncenth[k], it, is)] = 0.0;
      c.amasct[Chem::c3(c.ncenpy[k], it, is)] = 0.0;
    }
  for (int is = 1; is <= c.nspec; ++is)
    for (int it = 1; it <= c.ntint[is - 1]; ++it) {
      int k = Chem::c2(it, is);
      c.amasch[Chem::c3(1, it, is)] = c.amascp[Chem::c3(1, it, is)];
      for (int icp = 2; icp <= c.ncpoly[k]; ++icp)
        c.amasch[Chem::c3(icp, it, is)] = c.amascp[Chem::c3(icp, it, is)] / (double)icp;
      c.amasch[Chem::c3(c.ncenth[k], it, is)] = c.amascp[Chem::c3(c.ncenth[k], it, is)];
      c.amasch[Chem::c3(c.ncenpy[k], it, is)] = 0.0;
    }
  for (int is = 1; is <= c.nspec; ++is)
    for (int it = 1; it <= c.ntint[is - 1]; ++it) {
      int k = Chem::c2(it, is);
      c.amascs[Chem::c3(1, it, is)] = c.amascp[Chem::c3(1, it, is)];
      for (int icp = 2; icp <= c.ncpoly[k]; ++icp)
        c.amascs[Chem::c3(icp, it, is)] = c.amascp[Chem::c3(icp, it, is)] / (double)(icp - 1);
      c.amascs[Chem::c3(c.ncenth[k], it, is)] = 0.0;
      c.amascs[Chem::c3(c.ncenpy[k], it, is)] = c.amascp[Chem::c3(c.ncenpy[k], it, is)];
    }
  double giblet = std::log(c.prefgb / RGUNIV);
  for (int is = 1; is <= c.nspec; ++is)
    for (int it = 1; it <= c.ntint[is - 1]; ++it) {
      int k = Chem::c2(it, is);
      c.amolgb[Chem::c3(1, it, is)] =
          c.amolcp[Chem::c3(c.ncenpy[k], it, is)] - c.amolcp[Chem::c3(1, it, is)] + giblet;
      for (int icp = 2; icp <= c.ncpoly[k]; ++icp)
        c.amolgb[Chem::c3(icp, it, is)] = c.amolcp[Chem::c3(icp, it, is)] / (double)(icp * (icp - 1));
      c.amolgb[Chem::c3(c.ncenth[k], it, is)] = c.amolcp[Chem::c3(c.ncenth[k], it, is)];
      c.amolgb[Chem::c3(c.ncenpy[k], it, is)] = c.amolcp[Chem::c3(1, it, is)] - 1.0;
    }
  for (int is = 1; is <= c.nspec; ++is)
    for (int it = 1; it <= c.ntint[is - 1]; ++it)
      for (int icp = 1; icp <= c.ncofcp[Chem::c2(it, is)]; ++icp)
        c.amolcp[Chem::c3(icp, it, is)] = c.amolcp[Chem::c3(icp, it, is)] * RGUNIV;
  for (int is = 1; is <= c.nspec; ++is) c.olewis[is - 1] = 1.0 / c.clewis[is - 1];
  c.alamda = ALAMDC * std::exp(-RLAMDA * std::log(TLAMDA));
}

// List-directed numeric tokens of one record.
inline std::vector<double> ld_tokens(const std::string& l) {
  std::vector<double> v;
  std::string s = l;
  for (char& ch : s)
    if (ch == ',') ch = ' ';
  std::istringstream is(s);
  std::string tok;
  while (is >> tok) v.push_back(freal(tok));
  return v;
}

// diff.dat reader: src/diffin.f:100-232 (records), src/diffin.f:328-405 (derived).
inline void read_diff(const std::string& path, const Chem& c, Diff& d) {
  LineReader r(path);
  for (int i = 0; i < 5; ++i) r.next();
  r.next();
  int ndspec = (int)fint(fld(r.next(), 0, 5));
  if (ndspec != c.nspec) std::fprintf(stderr, "oracle: diff.dat species count mismatch\n");
  for (int j = 0; j < c.nspec; ++j) r.next();
  r.next();
  {
    auto t = ld_tokens(r.next());
    d.pdifgb = t.at(0);
    d.tdifgb = t.at(1);
  }
  // list-directed READ of N values may span records; gather tokens until N read
  auto read_n = [&](int n) {
    std::vector<double> v;
    while ((int)v.size() < n) {
      auto t = ld_tokens(r.next());
      v.insert(v.end(), t.begin(), t.end());
    }
    return v;
  };
  r.next();  // Viscosity
  for (int is = 1; is <= c.nspec; ++is) {
    auto h = ld_tokens(r.next());
    d.ncovis = (int)h.at(1);
    auto v = read_n(d.ncovis);
    for (int ic = 1; ic <= d.ncovis; ++ic) d.viscco[Diff::v2(ic, is)] = v[ic - 1];
  }
  r.next();  // Thermal conductivity
  for (int is = 1; is <= c.nspec; ++is) {
    auto h = ld_tokens(r.next());
    d.nccon = (int)h.at(1);
    auto v = read_n(d.nccon);
    for (int ic = 1; ic <= d.nccon; ++ic) d.condco[Diff::v2(ic, is)] = v[ic - 1];
  }
  r.next();  // Binary diffusion
  for (int is = 1; is <= c.nspec; ++is) {
    auto h = ld_tokens(r.next());
    d.ncodif = (int)h.at(1);
    for (int js = 1; js <= is; ++js) {
      auto v = read_n(1 + d.ncodif);
      for (int ic = 1; ic <= d.ncodif; ++ic) d.diffco[Diff::d3(ic, js, is)] = v[ic];
    }
  }
  r.next();  // Thermal diffusion
  for (int is = 1; is <= c.nspec; ++is) {
    auto h = ld_tokens(r.next());
    d.ncotdr = (int)h.at(1);
    for (int js = 1; js <= is - 1; ++js) {
      auto v = read_n(1 + d.ncotdr);
      for (int ic = 1; ic <= d.ncotdr; ++ic) d.tdrcco[Diff::d3(ic, js, is)] = v[ic];
    }
  }
  // derived (src/diffin.f:331-368)
  for (int is = 1; is <= c.nspec; ++is)
    for (int js = is + 1; js <= c.nspec; ++js)
      for (int ic = 1; ic <= d.ncodif; ++ic) d.diffco[Diff::d3(ic, js, is)] = d.diffco[Diff::d3(ic, is, js)];
  for (int is = 1; is <= c.nspec; ++is) {
    for (int ic = 1; ic <= d.ncotdr; ++ic) d.tdrcco[Diff::d3(ic, is, is)] = 0.0;
    for (int js = 1; js <= is - 1; ++js)
      for (int ic = 1; ic <= d.ncotdr; ++ic) d.tdrcco[Diff::d3(ic, js, is)] = -d.tdrcco[Diff::d3(ic, js, is)];
    for (int js = is + 1; js <= c.nspec; ++js)
      for (int ic = 1; ic <= d.ncotdr; ++ic) d.tdrcco[Diff::d3(ic, js, is)] = d.tdrcco[Diff::d3(ic, is, js)];
  }
  for (int is = 1; is <= c.nspec; ++is)
    for (int js = 1; js <= c.nspec; ++js) {
      double f = c.wmolar[is - 1] / c.wmolar[js - 1];
      d.wilko2[Diff::d2(js, is)] = 1.0 / std::sqrt(std::sqrt(f));
      f = 8.0 * (1.0 + f);
      d.wilko1[Diff::d2(js, is)] = 1.0 / std::sqrt(f);
    }
  d.flmavt = true;
}

// radn.dat reader: src/radcin.f:80-113 (records) and :210-220 (derived).
// Five header records, the "Species list:" record, NRDSPC '(I5)', NSPEC
// species records, a comment record, NSPRAD, then per radiating species a
// record "JSPEC NKPRAD" and the NKPRAD coefficients read list-directed (the
// read continues onto following records until it has them all).
constexpr int NCFRMX = 6;
struct Radn {
  int nsprad = 0;
  int nsprid[NSPCMX] = {};
  int nkprad[NSPCMX] = {};
  double akprad[NSPCMX][NCFRMX] = {};
  double foursb = 0.0, trfrth = 0.0;
};
inline void read_radn(const std::string& path, const Chem& c, double trefrn, Radn& r) {
  LineReader rd(path);
  for (int i = 0; i < 6; ++i) rd.next();
  rd.next();  // NRDSPC: only compared with NSPEC
  for (int j = 0; j < c.nspec; ++j) rd.next();
  rd.next();  // "Planck mean absorption coefficient data"
  std::istringstream n0(rd.next());
  if (!(n0 >> r.nsprad) || r.nsprad < 0 || r.nsprad > NSPCMX) throw std::runtime_error("NSPRAD out of range");
  for (int j = 0; j < r.nsprad; ++j) {
    std::istringstream h(rd.next());
    if (!(h >> r.nsprid[j] >> r.nkprad[j]) || r.nsprid[j] < 1 || r.nsprid[j] > c.nspec || r.nkprad[j] < 1 ||
        r.nkprad[j] > NCFRMX)
      throw std::runtime_error("bad radiating species record");
    int got = 0;
    while (got < r.nkprad[j]) {
      std::istringstream v(rd.next());
      std::string tok;
      while (got < r.nkprad[j] && v >> tok) r.akprad[j][got++] = freal(tok);
    }
  }
  r.foursb = 4.0 * 5.67037321e-08;  // FOUR*STEFBO; STEFBO from src/com_senga2.h:222
  r.trfrth = trefrn * trefrn * trefrn * trefrn;
}

}  // namespace orc
