// Host factor construction for the INVK and INVT solvers: an incomplete LDU
// factorisation followed by the sparse approximate inverse of each
// triangular factor, producing W^T ~ L^-1, Z ~ U^-1 and d = D^-1 for the
// same device apply as AINV.
//
//   INVK: mld_d_invk_bld (src/impl/mld_d_invk_bld.f90:104-125)
//         ILU(fill1) of A, then mld_sparse_invk(fill2) on U and on L^T.
//   INVT: mld_d_invt_bld (src/impl/mld_d_invt_bld.f90:108-136)
//         ILUT(fillin, thresh) of A with maxval scaling, then
//         mld_sparse_invt(invfill, invthresh) on U and on L^T.
//
// The incomplete factorisations are MLD2P4's mld_iluk_fact / mld_ilut_fact
// (MLD2P4 >= 2.1.1, not part of the plugin's sources), restated from the
// published row-by-row IKJ form those routines use: a min-heap of column
// indices drives the elimination in ascending column order, U rows are
// stored scaled by the inverted pivot, L and U hold no diagonal (unit
// triangles) and d holds the inverted pivots.  ILU(k) tracks levels of fill
// (lev(i,j) = min(lev(i,j), lev(i,k) + lev(k,j) + 1)); ILUT drops by the
// 2-norm of the scaled input row and keeps, per triangle, the row's original
// entry count plus `fill` largest entries, always keeping the largest
// original upper entry.
//
// The sparse inverses follow the plugin's own routines line for line:
//   mld_dsparse_invk (src/impl/mld_dsparse_invk.f90:88-146) with
//     invk_copyin (src/impl/mld_d_invk_copyin.f90:85-110),
//     invk_inv (src/impl/mld_d_invk_inv.f90:80-137),
//     invk_copyout (src/impl/mld_d_invk_copyout.f90:98-133);
//   mld_dsparse_invt (src/impl/mld_dsparse_invt.f90:96-144) with
//     invt_copyin (src/impl/mld_d_invt_copyin.f90:90-130),
//     invt_inv (src/impl/mld_d_invt_inv.f90:85-145),
//     invt_copyout (src/impl/mld_d_invt_copyout.f90:100-297, the branch
//     the reference enables).
// Each row of an inverse depends only on the (read-only) triangular factor,
// so rows are computed on several threads; every row's arithmetic is
// sequential and in the reference's order, so the result does not depend on
// the thread count.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <limits>
#include <queue>
#include <thread>
#include <vector>

#include "host_build.h"

namespace ainv {
namespace {

constexpr double kEpsTol = 1.1e-16;  // PSBLAS d_epstol (pivot guard)

using MinQueue = std::priority_queue<int, std::vector<int>, std::greater<int>>;

void clear_queue(MinQueue &q) {
  while (!q.empty()) q.pop();
}

// Magnitude-ordered heap with the pop order of PSBLAS psb_d_idx_heap in
// psb_asort_down_ mode (the same order the AINV sparsifier uses): 1-based
// binary heap, an inserted key rises while strictly larger in magnitude
// than its parent, the root's replacement sinks toward the larger child
// (left on ties, or when it is the last element) while strictly smaller.
class MagnitudeHeap {
 public:
  void clear() {
    key_.resize(1);
    idx_.resize(1);
  }
  void push(double k, int i) {
    key_.push_back(k);
    idx_.push_back(i);
    size_t c = key_.size() - 1;
    while (c > 1) {
      const size_t p = c / 2;
      if (std::fabs(key_[c]) <= std::fabs(key_[p])) break;
      std::swap(key_[c], key_[p]);
      std::swap(idx_[c], idx_[p]);
      c = p;
    }
  }
  void pop(double &k, int &i) {
    k = key_[1];
    i = idx_[1];
    key_[1] = key_.back();
    idx_[1] = idx_.back();
    key_.pop_back();
    idx_.pop_back();
    const size_t last = key_.size() - 1;
    size_t c = 1;
    while (c <= last / 2) {
      const size_t l = 2 * c;
      const size_t j = (l == last || std::fabs(key_[l]) > std::fabs(key_[l + 1])) ? l : l + 1;
      if (!(std::fabs(key_[c]) < std::fabs(key_[j]))) break;
      std::swap(key_[c], key_[j]);
      std::swap(idx_[c], idx_[j]);
      c = j;
    }
  }

 private:
  std::vector<double> key_{0.0};
  std::vector<int> idx_{0};
};

// Euclidean norm by the scaled sum of squares of the reference BLAS dnrm2
// (Hammarling's one-pass form), which the ILUT row norms call.
double dnrm2(const double *x, int n) {
  double scale = 0.0, ssq = 1.0;
  for (int k = 0; k < n; k++) {
    if (x[k] == 0.0) continue;
    const double ax = std::fabs(x[k]);
    if (scale < ax) {
      const double r = scale / ax;
      ssq = 1.0 + ssq * (r * r);
      scale = ax;
    } else {
      const double r = ax / scale;
      ssq = ssq + r * r;
    }
  }
  return scale * std::sqrt(ssq);
}

// The entries kept for one output row, sorted by column (psb_msort on the
// column indices, which are distinct).
void sort_by_column(std::vector<std::pair<int, double>> &v) {
  std::sort(v.begin(), v.end(),
            [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
              return a.first < b.first;
            });
}

int pivot_error(const char *who, int i, double p) {
  set_error("%s: pivot too small at row %d (%.17g)", who, i + 1, p);
  return AINV_ERR_BREAKDOWN;
}

// ---------------------------------------------------------------------------
// ILU(k)
// ---------------------------------------------------------------------------
int iluk_factor(const HostCsr &a, int fill, HostCsr &l, HostCsr &u, std::vector<double> &d) {
  const int n = a.n;
  const int unset = -(n + 1);
  std::vector<double> row((size_t)n, 0.0);
  std::vector<int> lev((size_t)n, unset), idxs;
  std::vector<int> uplev;
  l = HostCsr{};
  u = HostCsr{};
  l.n = u.n = n;
  l.irp.assign((size_t)n + 1, 0);
  u.irp.assign((size_t)n + 1, 0);
  d.assign((size_t)n, 0.0);
  MinQueue heap;
  for (int i = 0; i < n; i++) {
    // copyin: the row of A, level 0
    clear_queue(heap);
    for (int p = a.irp[i]; p < a.irp[i + 1]; p++) {
      const int k = a.ja[p];
      row[k] = a.val[p];
      lev[k] = 0;
      heap.push(k);
    }
    // elimination in ascending column order
    idxs.clear();
    int lastk = -1;
    while (!heap.empty()) {
      const int k = heap.top();
      heap.pop();
      if (k == lastk) continue;
      lastk = k;
      idxs.push_back(k);
      if (row[k] != 0.0 && lev[k] <= fill && k < i) {
        // U is stored scaled by 1/pivot, so the unscaled row entry is the
        // coefficient of the update; the L multiplier is row(k) * d(k).
        const double rwk = row[k];
        const int lrwk = lev[k];
        row[k] = row[k] * d[k];
        for (int jj = u.irp[k]; jj < u.irp[k + 1]; jj++) {
          const int j = u.ja[jj];
          if (lev[j] < 0) {
            heap.push(j);
            lev[j] = -lev[j];
          }
          row[j] = row[j] - rwk * u.val[jj];
          lev[j] = std::min(lev[j], lrwk + uplev[jj] + 1);
        }
      }
    }
    // copyout: L (j < i), the pivot (j == i), U (j > i) with its levels
    double piv = 0.0;
    for (int j : idxs) {
      if (j < i) {
        if (lev[j] <= fill) {
          l.ja.push_back(j);
          l.val.push_back(row[j]);
        }
      } else if (j == i) {
        piv = row[j];
      } else if (lev[j] <= fill) {
        u.ja.push_back(j);
        u.val.push_back(row[j]);
        uplev.push_back(lev[j]);
      }
      row[j] = 0.0;
      lev[j] = unset;
    }
    l.irp[(size_t)i + 1] = (int)l.ja.size();
    u.irp[(size_t)i + 1] = (int)u.ja.size();
    if (std::fabs(piv) < kEpsTol) return pivot_error("ILU(k)", i, piv);
    d[i] = 1.0 / piv;
    for (int p = u.irp[i]; p < u.irp[i + 1]; p++) u.val[p] = d[i] * u.val[p];
  }
  return AINV_SUCCESS;
}

// ---------------------------------------------------------------------------
// ILUT(fill, thresh) with maxval scaling
// ---------------------------------------------------------------------------
int ilut_factor(const HostCsr &a, int fill, double thresh, HostCsr &l, HostCsr &u,
                std::vector<double> &d) {
  const int n = a.n;
  double mx = 0.0;
  for (double v : a.val) mx = std::max(mx, std::fabs(v));
  if (!(mx > 0.0)) {
    set_error("INVT build: matrix has no nonzero entries");
    return AINV_ERR_ARG;
  }
  const double weight = 1.0 / mx;
  std::vector<double> row((size_t)n, 0.0), scaled;
  std::vector<int> idxs;
  std::vector<std::pair<int, double>> kept;
  l = HostCsr{};
  u = HostCsr{};
  l.n = u.n = n;
  l.irp.assign((size_t)n + 1, 0);
  u.irp.assign((size_t)n + 1, 0);
  d.assign((size_t)n, 0.0);
  MinQueue heap;
  MagnitudeHeap mheap;
  for (int i = 0; i < n; i++) {
    // copyin: scaled row, counts of the lower / upper entries, the column
    // of the largest upper entry, and the row's 2-norm
    clear_queue(heap);
    int nlw = 0, nup = 0, jmaxup = -1;
    double dmaxup = 0.0;
    scaled.clear();
    for (int p = a.irp[i]; p < a.irp[i + 1]; p++) {
      const int k = a.ja[p];
      row[k] = weight * a.val[p];
      scaled.push_back(row[k]);
      heap.push(k);
      if (k < i) nlw++;
      if (k > i) {
        nup++;
        if (std::fabs(row[k]) > dmaxup) {
          jmaxup = k;
          dmaxup = std::fabs(row[k]);
        }
      }
    }
    const double tol = thresh * dnrm2(scaled.data(), (int)scaled.size());
    // elimination; a column enters the heap when its value is zero, so an
    // entry that cancels to zero may be queued twice (skipped via lastk)
    idxs.clear();
    int lastk = -1;
    while (!heap.empty()) {
      const int k = heap.top();
      heap.pop();
      if (k == lastk) continue;
      lastk = k;
      idxs.push_back(k);
      if (k < i) {
        const double rwk = row[k];
        row[k] = row[k] * d[k];
        if (std::fabs(row[k]) < tol) {
          row[k] = 0.0;
          continue;
        }
        for (int jj = u.irp[k]; jj < u.irp[k + 1]; jj++) {
          const int j = u.ja[jj];
          if (row[j] == 0.0) heap.push(j);
          row[j] = row[j] - rwk * u.val[jj];
        }
      }
    }
    // copyout, lower part: at most nlw + fill largest entries above tol
    size_t ip = 0;
    mheap.clear();
    kept.clear();
    for (; ip < idxs.size() && idxs[ip] < i; ip++) {
      const int j = idxs[ip];
      if (std::fabs(row[j]) < tol) continue;
      kept.push_back({j, row[j]});
      mheap.push(row[j], j);
    }
    if ((int)kept.size() > nlw + fill) {
      kept.resize((size_t)(nlw + fill));
      for (auto &e : kept) mheap.pop(e.second, e.first);
    }
    sort_by_column(kept);
    for (const auto &e : kept) {
      l.ja.push_back(e.first);
      l.val.push_back(e.second);
    }
    l.irp[(size_t)i + 1] = (int)l.ja.size();
    // the pivot
    if (ip >= idxs.size() || idxs[ip] != i) return pivot_error("ILUT", i, 0.0);
    const double piv = row[i];
    if (std::fabs(piv) < kEpsTol) return pivot_error("ILUT", i, piv);
    d[i] = 1.0 / piv;
    ip++;
    // upper part: at most nup + fill largest entries above tol, always
    // including the largest original upper entry (jmaxup)
    mheap.clear();
    kept.clear();
    for (; ip < idxs.size(); ip++) {
      const int j = idxs[ip];
      if (j != jmaxup && std::fabs(row[j]) < tol) continue;
      kept.push_back({j, row[j]});
      mheap.push(row[j], j);
    }
    if ((int)kept.size() > nup + fill) {
      const size_t cap = (size_t)(nup + fill);
      bool found = false;
      kept.resize(cap);
      for (auto &e : kept) {
        mheap.pop(e.second, e.first);
        found = found || e.first == jmaxup;
      }
      if (!found && jmaxup > i && cap > 0) kept[cap - 1] = {jmaxup, row[jmaxup]};
    }
    sort_by_column(kept);
    for (const auto &e : kept) {
      u.ja.push_back(e.first);
      u.val.push_back(d[i] * e.second);
    }
    u.irp[(size_t)i + 1] = (int)u.ja.size();
    for (int j : idxs) row[j] = 0.0;
  }
  // pivots of the scaled matrix -> inverted pivots of A
  for (double &v : d) v = v * weight;
  return AINV_SUCCESS;
}

// ---------------------------------------------------------------------------
// Sparse approximate inverse of a unit upper triangle (no stored diagonal),
// row by row; the result stores its diagonal.
// ---------------------------------------------------------------------------
struct RowsOut {
  std::vector<int> cnt, ja;
  std::vector<double> val;
};

class InvkRows {
 public:
  InvkRows(const HostCsr &u, int fill)
      : u_(u), fill_(fill), row_((size_t)u.n, 0.0), lev_((size_t)u.n, -(u.n + 1)) {}

  int run(int i, RowsOut &out) {
    const int n = u_.n;
    // copyin with sign -1, levels 0
    clear_queue(heap_);
    for (int p = u_.irp[i]; p < u_.irp[i + 1]; p++) {
      const int k = u_.ja[p];
      row_[k] = -1.0 * u_.val[p];
      lev_[k] = 0;
      heap_.push(k);
    }
    row_[i] = 1.0;
    lev_[i] = 0;
    // inv
    idxs_.clear();
    idxs_.push_back(i);
    int lastk = i;
    while (!heap_.empty()) {
      const int k = heap_.top();
      heap_.pop();
      if (k == lastk) continue;
      lastk = k;
      idxs_.push_back(k);
      if (row_[k] != 0.0 && lev_[k] <= fill_) {
        const double rwk = row_[k];
        const int lrwk = lev_[k];
        for (int jj = u_.irp[k]; jj < u_.irp[k + 1]; jj++) {
          const int j = u_.ja[jj];
          if (j <= k) return bad_factor(i);
          if (lev_[j] < 0) {
            heap_.push(j);
            lev_[j] = -lev_[j];
          }
          row_[j] = row_[j] - rwk * u_.val[jj];
          lev_[j] = std::min(lev_[j], lrwk + 1);  // the input's levels are all 0
        }
      }
    }
    // copyout
    int c = 0;
    for (int j : idxs_) {
      if (j >= i) {
        if (lev_[j] <= fill_) {
          out.ja.push_back(j);
          out.val.push_back(row_[j]);
          c++;
        }
        row_[j] = 0.0;
        lev_[j] = -(n + 1);
      }
    }
    out.cnt.push_back(c);
    return AINV_SUCCESS;
  }

 private:
  int bad_factor(int i) {
    set_error("INVK: factor row %d is not strictly upper triangular", i + 1);
    return AINV_ERR_INTERNAL;
  }
  const HostCsr &u_;
  const int fill_;
  std::vector<double> row_;
  std::vector<int> lev_, idxs_;
  MinQueue heap_;
};

class InvtRows {
 public:
  InvtRows(const HostCsr &u, int fill, double thresh)
      : u_(u), fill_(fill), thresh_(thresh), row_((size_t)u.n, 0.0), in_row_((size_t)u.n, 0) {}

  int run(int i, RowsOut &out) {
    // copyin with sign -1; nup = upper entries of the row; the norm is
    // taken over the stored values
    clear_queue(heap_);
    const int p0 = u_.irp[i], p1 = u_.irp[i + 1];
    int nup = 0;
    for (int p = p0; p < p1; p++) {
      const int k = u_.ja[p];
      row_[k] = -1.0 * u_.val[p];
      heap_.push(k);
      in_row_[k] = 1;
      if (k > i) nup++;
    }
    double nrmi = dnrm2(u_.val.data() + p0, p1 - p0);
    row_[i] = 1.0;
    // norm of the row with its unit diagonal, without overflow
    if (nrmi < 1.0)
      nrmi = std::sqrt(1.0 + nrmi * nrmi);
    else
      nrmi = nrmi * std::sqrt(1.0 + 1.0 / (nrmi * nrmi));
    const double tol = thresh_ * nrmi;
    // inv
    idxs_.clear();
    idxs_.push_back(i);
    int lastk = i;
    in_row_[i] = 1;
    while (!heap_.empty()) {
      const int k = heap_.top();
      heap_.pop();
      if (k == lastk) continue;
      lastk = k;
      const double rwk = row_[k];
      if (std::fabs(rwk) < tol) {
        row_[k] = 0.0;
        in_row_[k] = 0;
        continue;
      }
      for (int jj = u_.irp[k]; jj < u_.irp[k + 1]; jj++) {
        const int j = u_.ja[jj];
        if (j <= k) return bad_factor(i);
        row_[j] = row_[j] - rwk * u_.val[jj];
        if (!in_row_[j]) {
          if (std::fabs(row_[j]) < tol) {
            row_[j] = 0.0;
          } else {
            heap_.push(j);
            in_row_[j] = 1;
          }
        }
      }
      idxs_.push_back(k);
      in_row_[k] = 0;
    }
    in_row_[i] = 0;
    // copyout: the diagonal and the entries above tol, offered in idxs
    // order; past nup + fill accepted entries, only those at least as large
    // as the smallest accepted so far; then the nup + fill largest
    const int cap = nup + fill_;
    kept_.clear();
    heapm_.clear();
    double wmin = std::numeric_limits<double>::max();  // HUGE(wmin)
    for (int j : idxs_) {
      const double w = row_[j];
      if (j != i && std::fabs(w) < tol) continue;
      if ((int)kept_.size() > cap && std::fabs(w) < wmin) continue;
      wmin = std::min(std::fabs(w), wmin);
      kept_.push_back({j, w});
      heapm_.push(w, j);
    }
    if ((int)kept_.size() > cap) {
      kept_.resize((size_t)cap);
      for (auto &e : kept_) heapm_.pop(e.second, e.first);
    }
    sort_by_column(kept_);
    for (const auto &e : kept_) {
      out.ja.push_back(e.first);
      out.val.push_back(e.second);
    }
    out.cnt.push_back((int)kept_.size());
    for (int j : idxs_) row_[j] = 0.0;
    return AINV_SUCCESS;
  }

 private:
  int bad_factor(int i) {
    set_error("INVT: factor row %d is not strictly upper triangular", i + 1);
    return AINV_ERR_INTERNAL;
  }
  const HostCsr &u_;
  const int fill_;
  const double thresh_;
  std::vector<double> row_;
  std::vector<char> in_row_;
  std::vector<int> idxs_;
  std::vector<std::pair<int, double>> kept_;
  MinQueue heap_;
  MagnitudeHeap heapm_;
};

int host_threads() {
  if (const char *e = std::getenv("AINV_BUILD_THREADS")) {
    const int v = std::atoi(e);
    if (v > 0) return v;
  }
  const unsigned hc = std::thread::hardware_concurrency();
  // each worker holds dense row work arrays of n entries
  return (int)std::max(1u, std::min(hc, 16u));
}

// Rows 0..n-2 through `Rows`, in contiguous blocks per thread; the last row
// is the unit diagonal (src/impl/mld_dsparse_invk.f90:137-142).
template <class Rows, class... Args>
int sparse_inverse(const HostCsr &u, HostCsr &z, Args... args) {
  const int n = u.n;
  z = HostCsr{};
  z.n = n;
  z.irp.assign((size_t)n + 1, 0);
  if (n == 0) return AINV_SUCCESS;
  const int rows = n - 1;
  const int nt = std::max(1, std::min(host_threads(), rows / 4096 + 1));
  std::vector<RowsOut> parts((size_t)nt);
  std::vector<int> rc((size_t)nt, AINV_SUCCESS);
  auto work = [&](int t) {
    Rows r(u, args...);
    const int b = (int)((long long)rows * t / nt), e = (int)((long long)rows * (t + 1) / nt);
    for (int i = b; i < e && rc[(size_t)t] == AINV_SUCCESS; i++)
      rc[(size_t)t] = r.run(i, parts[(size_t)t]);
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; t++) th.emplace_back(work, t);
  work(0);
  for (auto &x : th) x.join();
  for (int v : rc)
    if (v != AINV_SUCCESS) return v;
  size_t total = 1;
  for (const auto &p : parts) total += p.ja.size();
  z.ja.reserve(total);
  z.val.reserve(total);
  int i = 0;
  for (const auto &p : parts) {
    for (int c : p.cnt) {
      z.irp[(size_t)i + 1] = z.irp[(size_t)i] + c;
      i++;
    }
    z.ja.insert(z.ja.end(), p.ja.begin(), p.ja.end());
    z.val.insert(z.val.end(), p.val.begin(), p.val.end());
  }
  z.ja.push_back(n - 1);
  z.val.push_back(1.0);
  z.irp[(size_t)n] = (int)z.ja.size();
  return AINV_SUCCESS;
}

// The factor pair (L, U) -> (W^T, Z): Z ~ U^-1, W^T ~ L^-1 through L^T.
template <class Rows, class... Args>
int invert_factors(const HostCsr &l, const HostCsr &u, HostCsr &wt, HostCsr &z, Args... args) {
  AINV_TRY((sparse_inverse<Rows>(u, z, args...)));
  HostCsr zl;
  AINV_TRY((sparse_inverse<Rows>(transpose(l), zl, args...)));
  wt = transpose(zl);
  return AINV_SUCCESS;
}

}  // namespace

int invk_build(const HostCsr &a, int fill1, int fill2, HostCsr &wt, HostCsr &z,
               std::vector<double> &d) {
  if (fill1 < 0 || fill2 < 0) {
    set_error("INVK build: fill levels must be >= 0 (got %d, %d)", fill1, fill2);
    return AINV_ERR_ARG;
  }
  HostCsr l, u;
  AINV_TRY(iluk_factor(a, fill1, l, u, d));
  return invert_factors<InvkRows>(l, u, wt, z, fill2);
}

int invt_build(const HostCsr &a, int fill, double thresh, int invfill, double invthresh,
               HostCsr &wt, HostCsr &z, std::vector<double> &d) {
  if (fill < 0 || invfill < 0 || !(thresh >= 0.0) || !(invthresh >= 0.0)) {
    set_error("INVT build: fill levels and thresholds must be >= 0");
    return AINV_ERR_ARG;
  }
  HostCsr l, u;
  AINV_TRY(ilut_factor(a, fill, thresh, l, u, d));
  return invert_factors<InvtRows>(l, u, wt, z, invfill, invthresh);
}

}  // namespace ainv
