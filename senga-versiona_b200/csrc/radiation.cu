// Optically thin radiation heat loss (RADCAL, src/radcal.f:45-119; data
// from RADCIN, src/radcin.f:57-200; called at src/rhscal.f:810 when the
// cont.dat radiation switch is on):
//   ERHS -= 4 sigma * sum_j a_j(T) p_j * (T^4 - T_ref^4),
// a_j the Planck-mean absorption polynomial of radiating species j in T and
// p_j = rho Y_j R_j T its partial pressure. Pointwise; applied as one pass
// after the flow kernel has written the energy right-hand side (the species
// kernel then adds to it), with T from the thermochemistry kernel and rho Y
// from the U register, as in the reference (YRHS is still rho Y there).
#include <cuda_runtime.h>

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "senga_gpu.h"
#include "senga_internal.h"

namespace senga {
namespace {

constexpr int kRadBlock = 256;

__global__ void __launch_bounds__(kRadBlock) k_radcal(Geo g, Fields f, RadParams r) {
  const int64_t q = (int64_t)blockIdx.x * kRadBlock + threadIdx.x;
  if (q >= g.n) return;
  const int64_t n = g.n;
  const double T = f.t[q];
  double s1 = 0.0;
  for (int j = 0; j < r.nsprad; ++j) {
    double pl = r.ak[j][r.nk[j] - 1];
    for (int icp = r.nk[j] - 2; icp >= 0; --icp) pl = pl * T + r.ak[j][icp];
    const double fornow = f.uin[(int64_t)(5 + r.id[j]) * n + q] * r.rg[j] * T;
    s1 = s1 + pl * fornow;
  }
  const double t4 = T * T * T * T;
  f.rhs[4 * n + q] = f.rhs[4 * n + q] - r.foursb * s1 * (t4 - r.trfrth);
}

}  // namespace

void launch_radcal(const Geo& g, const Fields& f, const RadParams& r, cudaStream_t s) {
  k_radcal<<<(unsigned)((g.n + kRadBlock - 1) / kRadBlock), kRadBlock, 0, s>>>(g, f, r);
}

}  // namespace senga

using namespace senga;

// Restatement of RADCIN's reading of radn.dat (src/radcin.f:64-113): six
// header lines, the species count (I5) and NSPEC species lines, one comment
// line, NSPRAD,
// then per radiating species its index and coefficient count and the
// coefficients (list-directed, D exponents allowed).
extern "C" int senga_radn_load(const char* path, const senga_chem* chem, double trefrn, senga_radn* out) {
  if (!path || !chem || !out) return fail(SENGA_ERR_ARG, "senga_radn_load: null argument");
  std::ifstream in(path);
  if (!in) return fail(SENGA_ERR_IO, std::string("senga_radn_load: cannot read ") + path);
  std::vector<std::string> lines;
  for (std::string l; std::getline(in, l);) lines.push_back(l);
  size_t k = 6;
  if (lines.size() <= k) return fail(SENGA_ERR_IO, "senga_radn_load: file too short");
  // the count NRDSPC is only compared with NSPEC (a warning there); the list
  // read takes NSPEC lines, as RADCIN's loop does
  k += 1;
  if (k + (size_t)chem->nspec + 1 > lines.size()) return fail(SENGA_ERR_IO, "senga_radn_load: bad species list");
  k += (size_t)chem->nspec + 1;  // species lines and the comment line
  std::string rest;
  for (; k < lines.size(); ++k) rest += lines[k] + " ";
  for (char& c : rest)
    if (c == 'D' || c == 'd') c = 'E';
  std::istringstream ss(rest);
  senga_radn r{};
  r.trefrn = trefrn;
  if (!(ss >> r.nsprad) || r.nsprad < 0 || r.nsprad > SENGA_NSPCMX)
    return fail(SENGA_ERR_IO, "senga_radn_load: bad count of radiating species");
  for (int j = 0; j < r.nsprad; ++j) {
    int js = 0, nk = 0;
    if (!(ss >> js >> nk) || js < 1 || js > chem->nspec || nk < 1 || nk > SENGA_NCFRMX)
      return fail(SENGA_ERR_IO, "senga_radn_load: bad radiating species record");
    r.nsprid[j] = js;
    r.nkprad[j] = nk;
    for (int c = 0; c < nk; ++c)
      if (!(ss >> r.akprad[j][c])) return fail(SENGA_ERR_IO, "senga_radn_load: missing absorption coefficients");
  }
  *out = r;
  return SENGA_OK;
}
