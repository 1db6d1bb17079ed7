// Restart dump files in the reference's two layouts, and the
// post-processing record (host code).
//
// Writer: src/output.f:296-322 (NDOFMT = 0 unformatted, 1 formatted);
// reader: src/indata.f:1405-1436 (NDIFMT likewise). One record / one file
// per rank holds
//   NXNODE, NYNODE, NZNODE, NSPEC              (4 default integers)
//   DRUN, URUN, VRUN, WRUN, ERUN               (nx*ny*nz doubles each)
//   YRUN                                       (nx*ny*nz*NSPCMX doubles:
//                                               the whole COMMON array, also
//                                               the slots past NSPEC)
//   ETIME, TSTEP, ERROLD, ERRLDR               (doubles)
// Unformatted: one sequential record with 4-byte length markers before and
// after, split into sub-records with negative continuation markers when it
// exceeds 2^31-1 bytes (the layout of gfortran's sequential files).
// Formatted: list-directed text, the four sizes, then per point
// D U V W E Y_1..Y_NSPEC, then the four scalars; the reader takes the values
// as a stream of blank-separated items, as READ(*) does, including r*c
// repeat counts.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "senga_gpu.h"
#include "senga_internal.h"

namespace senga {
namespace {

constexpr int64_t kMaxSub = 2147483639;  // largest sub-record gfortran writes

bool write_unformatted(const std::string& path, const std::vector<char>& rec) {
  std::FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) return false;
  int64_t left = (int64_t)rec.size(), off = 0;
  bool ok = true;
  do {
    const int64_t chunk = left > kMaxSub ? kMaxSub : left;
    const bool more = left > kMaxSub;
    // the marker of a sub-record followed by another one is negative
    const int32_t head = (int32_t)(more ? -chunk : chunk);
    const int32_t tail = (int32_t)(off > 0 ? -chunk : chunk);
    ok = ok && std::fwrite(&head, 4, 1, fp) == 1;
    ok = ok && (chunk == 0 || std::fwrite(rec.data() + off, 1, (size_t)chunk, fp) == (size_t)chunk);
    ok = ok && std::fwrite(&tail, 4, 1, fp) == 1;
    off += chunk;
    left -= chunk;
  } while (left > 0 && ok);
  return std::fclose(fp) == 0 && ok;
}

bool read_unformatted(const std::string& path, std::vector<char>& rec) {
  std::FILE* fp = std::fopen(path.c_str(), "rb");
  if (!fp) return false;
  rec.clear();
  bool ok = true, more = true;
  while (more && ok) {
    int32_t head = 0, tail = 0;
    ok = std::fread(&head, 4, 1, fp) == 1;
    if (!ok) break;
    const int64_t chunk = head < 0 ? -(int64_t)head : head;
    more = head < 0;
    const size_t at = rec.size();
    rec.resize(at + (size_t)chunk);
    ok = chunk == 0 || std::fread(rec.data() + at, 1, (size_t)chunk, fp) == (size_t)chunk;
    ok = ok && std::fread(&tail, 4, 1, fp) == 1;
    ok = ok && (tail == head || tail == -head);
  }
  std::fclose(fp);
  return ok;
}

// Fortran list-directed items: blank/comma separated, r*c repeats, D exponents
struct Items {
  std::vector<std::string> tok;
  size_t pos = 0;
  std::string pending;
  long repeat = 0;
  bool next(std::string& out) {
    if (repeat > 0) {
      --repeat;
      out = pending;
      return true;
    }
    if (pos >= tok.size()) return false;
    std::string t = tok[pos++];
    const size_t star = t.find('*');
    if (star != std::string::npos) {
      repeat = std::strtol(t.substr(0, star).c_str(), nullptr, 10) - 1;
      pending = t.substr(star + 1);
      out = pending;
      return repeat >= 0;
    }
    out = t;
    return true;
  }
  bool real(double& v) {
    std::string s;
    if (!next(s)) return false;
    for (char& c : s)
      if (c == 'D' || c == 'd') c = 'E';
    char* end = nullptr;
    errno = 0;
    v = std::strtod(s.c_str(), &end);
    return end && *end == '\0' && errno == 0;
  }
  bool integer(int& v) {
    double d;
    if (!real(d) || d != std::floor(d)) return false;
    v = (int)d;
    return true;
  }
};

}  // namespace
}  // namespace senga

using namespace senga;

extern "C" int senga_dump_write(const char* path, int formatted, int nx, int ny, int nz, int nspec, int nspcmx,
                                const double* fields, const double* scalars) {
  if (!path || !fields || !scalars || nx < 1 || ny < 1 || nz < 1 || nspec < 1 || nspcmx < nspec)
    return fail(SENGA_ERR_ARG, "senga_dump_write: bad argument");
  const int64_t n = (int64_t)nx * ny * nz;
  if (!formatted) {
    const int64_t bytes = 16 + (int64_t)(5 + nspcmx) * n * 8 + 32;
    std::vector<char> rec((size_t)bytes, 0);
    const int32_t sz[4] = {nx, ny, nz, nspec};
    std::memcpy(rec.data(), sz, 16);
    std::memcpy(rec.data() + 16, fields, (size_t)(5 + nspec) * n * 8);  // YRUN slots past NSPEC stay zero
    std::memcpy(rec.data() + 16 + (size_t)(5 + nspcmx) * n * 8, scalars, 32);
    if (!write_unformatted(path, rec)) return fail(SENGA_ERR_IO, std::string("senga_dump_write: cannot write ") + path);
    return SENGA_OK;
  }
  std::FILE* fp = std::fopen(path, "w");
  if (!fp) return fail(SENGA_ERR_IO, std::string("senga_dump_write: cannot write ") + path);
  std::fprintf(fp, " %11d %11d %11d %11d\n", nx, ny, nz, nspec);
  for (int64_t q = 0; q < n; ++q) {
    for (int fl = 0; fl < 5 + nspec; ++fl) std::fprintf(fp, " %25.17E", fields[fl * n + q]);
    std::fputc('\n', fp);
  }
  std::fprintf(fp, " %25.17E %25.17E %25.17E %25.17E\n", scalars[0], scalars[1], scalars[2], scalars[3]);
  if (std::fclose(fp) != 0) return fail(SENGA_ERR_IO, std::string("senga_dump_write: cannot write ") + path);
  return SENGA_OK;
}

// Post-processing record (src/output.f:240-265): D, u, v, w, E, T, p,
// Y_1..Y_NSPEC, RRTE(..., 1..NSPCMX) (slots past NSPEC zero), ETIME; one
// sequential unformatted record, no size header.
extern "C" int senga_post_write(const char* path, int nx, int ny, int nz, int nspec, int nspcmx, const double* post,
                                double etime) {
  if (!path || !post || nx < 1 || ny < 1 || nz < 1 || nspec < 1 || nspcmx < nspec)
    return fail(SENGA_ERR_ARG, "senga_post_write: bad argument");
  const int64_t n = (int64_t)nx * ny * nz;
  std::vector<char> rec((size_t)((7 + nspec + nspcmx) * n + 1) * 8, 0);
  std::memcpy(rec.data(), post, (size_t)(7 + 2 * nspec) * n * 8);
  std::memcpy(rec.data() + (size_t)(7 + nspec + nspcmx) * n * 8, &etime, 8);
  if (!write_unformatted(path, rec)) return fail(SENGA_ERR_IO, std::string("senga_post_write: cannot write ") + path);
  return SENGA_OK;
}

extern "C" int senga_post_read(const char* path, int nx, int ny, int nz, int nspec, int nspcmx, double* post,
                               double* etime) {
  if (!path || !post || nx < 1 || ny < 1 || nz < 1 || nspec < 1 || nspcmx < nspec)
    return fail(SENGA_ERR_ARG, "senga_post_read: bad argument");
  std::vector<char> rec;
  if (!read_unformatted(path, rec)) return fail(SENGA_ERR_IO, std::string("senga_post_read: cannot read ") + path);
  const int64_t n = (int64_t)nx * ny * nz;
  if ((int64_t)rec.size() != ((7 + nspec + nspcmx) * n + 1) * 8)
    return fail(SENGA_ERR_IO, "senga_post_read: record size does not match the sizes given");
  std::memcpy(post, rec.data(), (size_t)(7 + 2 * nspec) * n * 8);
  if (etime) std::memcpy(etime, rec.data() + (size_t)(7 + nspec + nspcmx) * n * 8, 8);
  return SENGA_OK;
}

extern "C" int senga_dump_read(const char* path, int formatted, int nspcmx, int* dims, double* fields, int64_t capacity,
                               double* scalars) {
  if (!path || !dims || nspcmx < 1) return fail(SENGA_ERR_ARG, "senga_dump_read: bad argument");
  if (!formatted) {
    std::vector<char> rec;
    if (!read_unformatted(path, rec) || rec.size() < 16)
      return fail(SENGA_ERR_IO, std::string("senga_dump_read: cannot read ") + path);
    int32_t sz[4];
    std::memcpy(sz, rec.data(), 16);
    for (int i = 0; i < 4; ++i) dims[i] = sz[i];
    const int64_t n = (int64_t)sz[0] * sz[1] * sz[2];
    if (sz[0] < 1 || sz[1] < 1 || sz[2] < 1 || sz[3] < 1) return fail(SENGA_ERR_IO, "senga_dump_read: bad header");
    if (!fields) return SENGA_OK;  // size query
    if (sz[3] > nspcmx || (int64_t)rec.size() != 16 + (int64_t)(5 + nspcmx) * n * 8 + 32)
      return fail(SENGA_ERR_IO, "senga_dump_read: record size does not match the header and NSPCMX");
    if (capacity < (int64_t)(5 + sz[3]) * n) return fail(SENGA_ERR_ARG, "senga_dump_read: fields too small");
    std::memcpy(fields, rec.data() + 16, (size_t)(5 + sz[3]) * n * 8);
    if (scalars) std::memcpy(scalars, rec.data() + 16 + (size_t)(5 + nspcmx) * n * 8, 32);
    return SENGA_OK;
  }
  std::ifstream in(path);
  if (!in) return fail(SENGA_ERR_IO, std::string("senga_dump_read: cannot read ") + path);
  Items it;
  std::string w;
  while (in >> w) {
    std::replace(w.begin(), w.end(), ',', ' ');
    std::istringstream ss(w);
    std::string t;
    while (ss >> t) it.tok.push_back(t);
  }
  for (int i = 0; i < 4; ++i)
    if (!it.integer(dims[i]) || dims[i] < 1) return fail(SENGA_ERR_IO, "senga_dump_read: bad size line");
  if (!fields) return SENGA_OK;
  const int64_t n = (int64_t)dims[0] * dims[1] * dims[2];
  const int nc = 5 + dims[3];
  if (capacity < (int64_t)nc * n) return fail(SENGA_ERR_ARG, "senga_dump_read: fields too small");
  for (int64_t q = 0; q < n; ++q)
    for (int fl = 0; fl < nc; ++fl)
      if (!it.real(fields[fl * n + q])) return fail(SENGA_ERR_IO, "senga_dump_read: short or malformed point data");
  double sc[4];
  for (int i = 0; i < 4; ++i)
    if (!it.real(sc[i])) return fail(SENGA_ERR_IO, "senga_dump_read: missing ETIME/TSTEP/ERROLD/ERRLDR");
  if (scalars) std::memcpy(scalars, sc, sizeof(sc));
  return SENGA_OK;
}
