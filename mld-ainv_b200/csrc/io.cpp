// Factor interchange for the solver types.
//
//  * MatrixMarket load: the files `dump` writes, which are the files of the
//    reference's dump (mld_d_base_ainv_solver_dmp,
//    src/impl/mld_d_base_ainv_solver_dmp.f90:82-108): <prefix>_wmat.mtx
//    (sv%w, i.e. W^T, coordinate format), <prefix>_diag.mtx (sv%d, array
//    format) and <prefix>_zmat.mtx (sv%z).  A dump of a real MLD2P4 run
//    loads with its full prefix (e.g. "dump_ainv_d_p000_l001").
//  * Binary cache: the host factors and the settings in one file with a
//    checksum, for reloading large factors without rebuilding them.
#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "solver_impl.h"

namespace ainv {
namespace {

struct File {
  FILE *f = nullptr;
  explicit File(const std::string &name, const char *mode) : f(std::fopen(name.c_str(), mode)) {}
  ~File() {
    if (f) std::fclose(f);
  }
};

// Next non-comment, non-blank line; false at end of file.
bool next_line(FILE *f, std::string &line) {
  char buf[512];
  while (std::fgets(buf, sizeof buf, f)) {
    line = buf;
    size_t b = 0;
    while (b < line.size() && (line[b] == ' ' || line[b] == '\t')) b++;
    if (b == line.size() || line[b] == '\n' || line[b] == '\r' || line[b] == '%') continue;
    return true;
  }
  return false;
}

int read_coo(const std::string &name, HostCsr &out) {
  File fh(name, "r");
  if (!fh.f) {
    set_error("load: cannot open %s (%s)", name.c_str(), std::strerror(errno));
    return AINV_ERR_ARG;
  }
  char hdr[256] = {0};
  if (!std::fgets(hdr, sizeof hdr, fh.f) || std::strncmp(hdr, "%%MatrixMarket matrix coordinate", 32)) {
    set_error("load: %s is not a MatrixMarket coordinate file", name.c_str());
    return AINV_ERR_ARG;
  }
  std::string line;
  long long nr = 0, nc = 0, nz = 0;
  if (!next_line(fh.f, line) || std::sscanf(line.c_str(), "%lld %lld %lld", &nr, &nc, &nz) != 3 ||
      nr <= 0 || nr != nc || nz < 0 || nr > 0x7fffffffLL || nz > 0x7fffffffLL) {
    set_error("load: bad size line in %s", name.c_str());
    return AINV_ERR_ARG;
  }
  const int n = (int)nr;
  std::vector<int> ri((size_t)nz), ci((size_t)nz);
  std::vector<double> v((size_t)nz);
  for (long long k = 0; k < nz; k++) {
    long long i, j;
    double x;
    if (!next_line(fh.f, line) || std::sscanf(line.c_str(), "%lld %lld %lf", &i, &j, &x) != 3 ||
        i < 1 || i > n || j < 1 || j > n) {
      set_error("load: bad entry %lld in %s", k + 1, name.c_str());
      return AINV_ERR_ARG;
    }
    ri[(size_t)k] = (int)(i - 1);
    ci[(size_t)k] = (int)(j - 1);
    v[(size_t)k] = x;
  }
  // CSR by counting sort on rows, then columns sorted within each row
  out = HostCsr{};
  out.n = n;
  out.irp.assign((size_t)n + 1, 0);
  for (int r : ri) out.irp[(size_t)r + 1]++;
  for (int r = 0; r < n; r++) out.irp[(size_t)r + 1] += out.irp[(size_t)r];
  out.ja.resize((size_t)nz);
  out.val.resize((size_t)nz);
  std::vector<int> pos(out.irp.begin(), out.irp.end() - 1);
  for (long long k = 0; k < nz; k++) {
    const int at = pos[(size_t)ri[(size_t)k]]++;
    out.ja[(size_t)at] = ci[(size_t)k];
    out.val[(size_t)at] = v[(size_t)k];
  }
  std::vector<std::pair<int, double>> row;
  for (int r = 0; r < n; r++) {
    const int b = out.irp[(size_t)r], e = out.irp[(size_t)r + 1];
    row.clear();
    for (int k = b; k < e; k++) row.push_back({out.ja[(size_t)k], out.val[(size_t)k]});
    std::sort(row.begin(), row.end(),
              [](const std::pair<int, double> &a, const std::pair<int, double> &c) {
                return a.first < c.first;
              });
    for (int k = b; k < e; k++) {
      const auto &p = row[(size_t)(k - b)];
      if (k > b && p.first == out.ja[(size_t)k - 1]) {
        set_error("load: duplicate entry (%d, %d) in %s", r + 1, p.first + 1, name.c_str());
        return AINV_ERR_ARG;
      }
      out.ja[(size_t)k] = p.first;
      out.val[(size_t)k] = p.second;
    }
  }
  return AINV_SUCCESS;
}

int read_array(const std::string &name, std::vector<double> &d) {
  File fh(name, "r");
  if (!fh.f) {
    set_error("load: cannot open %s (%s)", name.c_str(), std::strerror(errno));
    return AINV_ERR_ARG;
  }
  char hdr[256] = {0};
  if (!std::fgets(hdr, sizeof hdr, fh.f) || std::strncmp(hdr, "%%MatrixMarket matrix array", 27)) {
    set_error("load: %s is not a MatrixMarket array file", name.c_str());
    return AINV_ERR_ARG;
  }
  std::string line;
  long long nr = 0, nc = 0;
  if (!next_line(fh.f, line) || std::sscanf(line.c_str(), "%lld %lld", &nr, &nc) != 2 ||
      nr <= 0 || nc != 1 || nr > 0x7fffffffLL) {
    set_error("load: bad size line in %s", name.c_str());
    return AINV_ERR_ARG;
  }
  d.resize((size_t)nr);
  for (long long k = 0; k < nr; k++) {
    if (!next_line(fh.f, line) || std::sscanf(line.c_str(), "%lf", &d[(size_t)k]) != 1) {
      set_error("load: bad value %lld in %s", k + 1, name.c_str());
      return AINV_ERR_ARG;
    }
  }
  return AINV_SUCCESS;
}

// FNV-1a over the payload bytes.
uint64_t fnv1a(const void *p, size_t n, uint64_t h) {
  const unsigned char *b = static_cast<const unsigned char *>(p);
  for (size_t i = 0; i < n; i++) {
    h ^= b[i];
    h *= 1099511628211ull;
  }
  return h;
}

constexpr char kMagic[8] = {'A', 'I', 'N', 'V', 'B', '2', '0', '0'};
constexpr uint32_t kVersion = 1;

struct CacheHeader {
  char magic[8];
  uint32_t version;
  int32_t kind, alg, fill_in, inv_fill, n;
  double thresh, inv_thresh;
  int64_t nnz_wt, nnz_z;
};

template <class T>
bool put(FILE *f, const std::vector<T> &v, uint64_t &h) {
  h = fnv1a(v.data(), sizeof(T) * v.size(), h);
  return std::fwrite(v.data(), sizeof(T), v.size(), f) == v.size();
}
template <class T>
bool get(FILE *f, std::vector<T> &v, size_t n, uint64_t &h) {
  v.resize(n);
  if (std::fread(v.data(), sizeof(T), n, f) != n) return false;
  h = fnv1a(v.data(), sizeof(T) * n, h);
  return true;
}

}  // namespace

int load_matrix_market(mld_d_solver *sv, const std::string &prefix) {
  HostCsr wt, z;
  std::vector<double> d;
  AINV_TRY(read_coo(prefix + "_wmat.mtx", wt));
  AINV_TRY(read_coo(prefix + "_zmat.mtx", z));
  AINV_TRY(read_array(prefix + "_diag.mtx", d));
  if (wt.n != z.n || (int)d.size() != wt.n) {
    set_error("load: sizes differ (W^T %d, Z %d, d %zu)", wt.n, z.n, d.size());
    return AINV_ERR_ARG;
  }
  return install_factors(sv, std::move(wt), std::move(z), std::move(d));
}

int save_cache(const mld_d_solver *sv, const std::string &path) {
  if (!sv->built) {
    set_error("save: solver not built");
    return AINV_ERR_NOT_BUILT;
  }
  File fh(path, "wb");
  if (!fh.f) {
    set_error("save: cannot open %s (%s)", path.c_str(), std::strerror(errno));
    return AINV_ERR_ARG;
  }
  CacheHeader hd{};
  std::memcpy(hd.magic, kMagic, sizeof kMagic);
  hd.version = kVersion;
  hd.kind = sv->kind;
  hd.alg = sv->alg;
  hd.fill_in = sv->fill_in;
  hd.inv_fill = sv->inv_fill;
  hd.n = sv->wt.n;
  hd.thresh = sv->thresh;
  hd.inv_thresh = sv->inv_thresh;
  hd.nnz_wt = sv->wt.nnz();
  hd.nnz_z = sv->z.nnz();
  uint64_t h = fnv1a(&hd, sizeof hd, 1469598103934665603ull);
  bool ok = std::fwrite(&hd, sizeof hd, 1, fh.f) == 1;
  ok = ok && put(fh.f, sv->wt.irp, h) && put(fh.f, sv->wt.ja, h) && put(fh.f, sv->wt.val, h);
  ok = ok && put(fh.f, sv->z.irp, h) && put(fh.f, sv->z.ja, h) && put(fh.f, sv->z.val, h);
  ok = ok && put(fh.f, sv->d, h);
  ok = ok && std::fwrite(&h, sizeof h, 1, fh.f) == 1;
  if (!ok) {
    set_error("save: write to %s failed", path.c_str());
    return AINV_ERR_INTERNAL;
  }
  return AINV_SUCCESS;
}

int load_cache(mld_d_solver *sv, const std::string &path) {
  File fh(path, "rb");
  if (!fh.f) {
    set_error("restore: cannot open %s (%s)", path.c_str(), std::strerror(errno));
    return AINV_ERR_ARG;
  }
  CacheHeader hd{};
  if (std::fread(&hd, sizeof hd, 1, fh.f) != 1 || std::memcmp(hd.magic, kMagic, sizeof kMagic) ||
      hd.version != kVersion || hd.n < 1 || hd.nnz_wt < 0 || hd.nnz_z < 0) {
    set_error("restore: %s is not a factor cache of this library", path.c_str());
    return AINV_ERR_ARG;
  }
  if (hd.kind != sv->kind) {
    set_error("restore: %s holds factors of another solver type", path.c_str());
    return AINV_ERR_ARG;
  }
  uint64_t h = fnv1a(&hd, sizeof hd, 1469598103934665603ull), stored = 0;
  HostCsr wt, z;
  std::vector<double> d;
  wt.n = z.n = hd.n;
  const size_t n1 = (size_t)hd.n + 1;
  bool ok = get(fh.f, wt.irp, n1, h) && get(fh.f, wt.ja, (size_t)hd.nnz_wt, h) &&
            get(fh.f, wt.val, (size_t)hd.nnz_wt, h) && get(fh.f, z.irp, n1, h) &&
            get(fh.f, z.ja, (size_t)hd.nnz_z, h) && get(fh.f, z.val, (size_t)hd.nnz_z, h) &&
            get(fh.f, d, (size_t)hd.n, h);
  ok = ok && std::fread(&stored, sizeof stored, 1, fh.f) == 1;
  if (!ok || stored != h) {
    set_error("restore: %s is truncated or corrupt (checksum)", path.c_str());
    return AINV_ERR_ARG;
  }
  // structural checks before the arrays are trusted
  HostCsr wt2, z2;
  AINV_TRY(import_csr(wt.n, wt.irp.data(), wt.ja.data(), wt.val.data(), 0, wt2, "W^T"));
  AINV_TRY(import_csr(z.n, z.irp.data(), z.ja.data(), z.val.data(), 0, z2, "Z"));
  sv->alg = hd.alg;
  sv->fill_in = hd.fill_in;
  sv->inv_fill = hd.inv_fill;
  sv->thresh = hd.thresh;
  sv->inv_thresh = hd.inv_thresh;
  return install_factors(sv, std::move(wt2), std::move(z2), std::move(d));
}

}  // namespace ainv
