// Host factor construction for the AINV solver (sparse left-looking
// biconjugation), producing the Z / W^T patterns the device apply consumes.
//
// Algorithm: mld_d_ainv_bld (src/impl/mld_d_ainv_bld.F90:35-194) with the
// maxval scaling the solver always requests (src/impl/mld_d_ainv_solver_bld.f90:68-69),
// the left-looking biconjugation of src/impl/mld_dsparse_biconjg_llk.F90:35-366
// (plus the SYM-LLK, no-alpha-test, stabilised STAB-LLK and list-based MLK
// variants), and the column
// sparsification of src/impl/mld_d_sparsify.f90:35-149.  Floating-point
// operations happen in the reference's order with one rounding per
// operation, so the factors are bit-identical to the reference algorithm.
// (STAB-LLK also multiplies A by sparse columns of Z and W; the order of
// those sums is documented at SparseProduct.)
//
// In LLK the Z and W halves only share read-only data (A and its
// transpose), so they run on two threads.  STAB-LLK interleaves them.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <queue>
#include <thread>
#include <vector>

#include "host_build.h"

namespace ainv {
namespace {

constexpr double kEpsTol = 1.1e-16;  // PSBLAS d_epstol
constexpr double kTinyPivot = 1.0e-3;

// Magnitude-ordered heap with the exact pop order of PSBLAS psb_d_idx_heap
// in psb_asort_down_ mode: 1-based binary heap; an inserted key rises while
// strictly larger in magnitude than its parent; the root's replacement sinks
// toward the larger child (the left one only when strictly larger or when
// it is the last element, so the right one on ties) while strictly smaller
// than it.  This order decides which
// equal-magnitude entries survive the fill cap.
class MagnitudeHeap {
 public:
  void clear() {
    key_.resize(1);
    idx_.resize(1);
  }
  bool empty() const { return key_.size() <= 1; }
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

// PSBLAS psb_hsort(x, ix, dir=psb_asort_down_) on m entries: a heap with
// the smallest magnitude at the root (1-based; an inserted key rises while
// strictly smaller in magnitude than its parent; the root's replacement
// sinks toward the smaller child -- the left one only when strictly smaller
// or when it is the last element -- while strictly larger than it) takes
// the entries in order; then the root is taken out m-1 times and stored
// from the last position backwards, and the first position keeps the last
// root.  The result is descending in magnitude; this fixes the order of
// equal magnitudes.
void hsort_abs_down(double *x, int *ix, int m) {
  std::vector<double> k(1);
  std::vector<int> v(1);
  for (int j = 0; j < m; j++) {
    k.push_back(x[j]);
    v.push_back(ix[j]);
    size_t c = k.size() - 1;
    while (c > 1 && std::fabs(k[c]) < std::fabs(k[c / 2])) {
      std::swap(k[c], k[c / 2]);
      std::swap(v[c], v[c / 2]);
      c /= 2;
    }
  }
  for (int j = m - 1; j >= 1; j--) {
    x[j] = k[1];
    ix[j] = v[1];
    k[1] = k.back();
    v[1] = v.back();
    k.pop_back();
    v.pop_back();
    const size_t last = k.size() - 1;
    size_t c = 1;
    while (c <= last / 2) {
      const size_t l = 2 * c;
      const size_t ch = (l == last || std::fabs(k[l]) < std::fabs(k[l + 1])) ? l : l + 1;
      if (!(std::fabs(k[c]) > std::fabs(k[ch]))) break;
      std::swap(k[c], k[ch]);
      std::swap(v[c], v[ch]);
      c = ch;
    }
  }
  if (m > 0) {
    x[0] = k[1];
    ix[0] = v[1];
  }
}

using MinQueue = std::priority_queue<int, std::vector<int>, std::greater<int>>;

// Column-by-column builder of one unit upper triangular factor (Z, or W).
// `dots` gives the sparse vector whose dot with the working column yields
// the biconjugation coefficient for step j (rows of A for Z, columns of A
// for W); `touch` maps a position kr to the steps j whose dot vector has a
// nonzero at kr (columns of A for Z, rows of A for W).
class HalfBuilder {
 public:
  // list_sparsify: MLK's mld_d_sparsify_list instead of mld_d_sparsify.
  HalfBuilder(const HostCsr &dots, const HostCsr &touch, int cap, double thresh,
              bool alpha_test, bool list_sparsify = false)
      : dots_(dots), touch_(touch), n_(dots.n), cap_(cap), thresh_(thresh),
        alpha_test_(alpha_test), list_sparsify_(list_sparsify) {}

  // piv receives the pivots; out gets the factor as CSC columns.
  void run(double piv0, std::vector<double> &piv, HostCsr &out) {
    start(out);
    piv.assign((size_t)n_, 0.0);
    piv[0] = piv0;
    for (int i = 1; i < n_; i++) {
      update(i, piv, out, [&](int j) { return dot_with(j); });
      double p = dot_with(i);
      if (std::fabs(p) < kEpsTol) p = kTinyPivot;
      piv[i] = p;
      keep_column(i, out);
    }
  }

  // Column 0 of the factor (e_0) and empty work state.
  void start(HostCsr &out) {
    out.n = n_;
    out.irp.assign((size_t)n_ + 1, 0);
    out.ja.clear();
    out.val.clear();
    out.ja.reserve((size_t)n_ * 4);
    out.val.reserve((size_t)n_ * 4);
    work_.assign((size_t)n_, 0.0);
    in_col_.assign((size_t)n_, 0);
    queued_.assign((size_t)n_, 0);
    out.ja.push_back(0);
    out.val.push_back(1.0);
    out.irp[1] = 1;
  }

  // Work column i = e_i updated by the earlier columns j < i of out whose
  // coefficient -dot(j)/piv[j] passes the alpha test; dot(j) sees the work
  // column through work().
  template <class Dot>
  void update(int i, const std::vector<double> &piv, const HostCsr &out, Dot &&dot) {
    nz_.clear();
    work_[i] = 1.0;
    in_col_[i] = 1;
    nz_.push_back(i);
    MinQueue steps;
    for (int k = touch_.irp[i]; k < touch_.irp[i + 1]; k++) {
      const int j = touch_.ja[k];
      if (j < i) {
        steps.push(j);
        queued_[j] = 1;
      }
    }
    int lastj = -1;
    while (!steps.empty()) {
      const int j = steps.top();
      steps.pop();
      if (j <= lastj) continue;  // repeated entry
      lastj = j;
      queued_[j] = 0;
      if (j >= i) continue;
      const double alpha = -dot(j) / piv[j];
      if (alpha_test_ && !(std::fabs(alpha) > thresh_)) continue;
      for (int k = out.irp[j]; k < out.irp[j + 1]; k++) {
        const int kr = out.ja[k];
        work_[kr] = work_[kr] + alpha * out.val[k];
        if (!in_col_[kr]) {
          in_col_[kr] = 1;
          nz_.push_back(kr);
          for (int kc = touch_.irp[kr]; kc < touch_.irp[kr + 1]; kc++) {
            const int nj = touch_.ja[kc];
            if (!queued_[nj] && nj > j && nj < i) {
              steps.push(nj);
              queued_[nj] = 1;
            }
          }
        }
      }
    }
  }

  const std::vector<double> &work() const { return work_; }

  // mld_d_sparsify_list (src/impl/mld_d_sparsify.f90:152-230): the column's
  // entries in index order, the diagonal swapped into the first slot (the
  // entry it displaces takes the diagonal's place); the rest sorted by
  // descending magnitude (psb_hsort); cut at the first entry below thresh
  // and at cap entries; survivors sorted by index.
  void keep_column_list(int i, HostCsr &out) {
    std::sort(nz_.begin(), nz_.end());
    lw_.clear();
    li_.clear();
    for (int r : nz_) {
      lw_.push_back(work_[r]);
      li_.push_back(r);
      if (r == i) {
        std::swap(lw_.front(), lw_.back());
        std::swap(li_.front(), li_.back());
      }
      work_[r] = 0.0;
      in_col_[r] = 0;
    }
    const int m = (int)lw_.size();
    if (m > 2) hsort_abs_down(lw_.data() + 1, li_.data() + 1, m - 1);
    int k = 1;
    while (k < m && !(std::fabs(lw_[k]) < thresh_)) k++;
    const int keep = std::max(1, std::min(k, cap_));
    kept_.clear();
    for (int e = 0; e < keep; e++) kept_.push_back({li_[e], lw_[e]});
    std::sort(kept_.begin(), kept_.end(),
              [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
                return a.first < b.first;
              });
    for (const auto &e : kept_) {
      out.ja.push_back(e.first);
      out.val.push_back(e.second);
    }
    out.irp[(size_t)i + 1] = (int)out.ja.size();
  }

  // Diagonal plus at most cap-1 entries of largest magnitude >= thresh,
  // offered to the heap in ascending index order; survivors sorted by index.
  void keep_column(int i, HostCsr &out) {
    if (list_sparsify_) {
      keep_column_list(i, out);
      return;
    }
    std::sort(nz_.begin(), nz_.end());
    heap_.clear();
    double diag = 0.0;
    for (int r : nz_) {
      if (r == i)
        diag = work_[r];
      else if (std::fabs(work_[r]) >= thresh_)
        heap_.push(work_[r], r);
      work_[r] = 0.0;
      in_col_[r] = 0;
    }
    kept_.clear();
    kept_.push_back({i, diag});
    while ((int)kept_.size() < cap_ && !heap_.empty()) {
      double v;
      int r;
      heap_.pop(v, r);
      kept_.push_back({r, v});
    }
    std::sort(kept_.begin(), kept_.end(),
              [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
                return a.first < b.first;
              });
    for (const auto &e : kept_) {
      out.ja.push_back(e.first);
      out.val.push_back(e.second);
    }
    out.irp[(size_t)i + 1] = (int)out.ja.size();
  }

 private:
  double dot_with(int j) const {
    double s = 0.0;
    for (int k = dots_.irp[j]; k < dots_.irp[j + 1]; k++) s = s + work_[dots_.ja[k]] * dots_.val[k];
    return s;
  }

  const HostCsr &dots_;
  const HostCsr &touch_;
  const int n_, cap_;
  const double thresh_;
  const bool alpha_test_, list_sparsify_;
  std::vector<double> work_, lw_;
  std::vector<int> li_;
  std::vector<char> in_col_, queued_;
  std::vector<int> nz_;  // positions set in work_, in insertion order
  MagnitudeHeap heap_;
  std::vector<std::pair<int, double>> kept_;
};

// y = x^T M for a sparse x (an index-sorted column of Z or W) and M in CSR:
// psb_d_spvspm (M = A) and psb_d_spmspv (M = A^T, i.e. A's CSC arrays, giving
// A x) of src/mld_d_biconjg_mod.F90:145-296.  Those take x's entries in
// order and merge (1*x_k) * M(k, :) into the running result with PSBLAS's
// sorted sparse axpby psb_nspaxpby (y_c = x_k*m + y_c, two roundings), so
// the result is index-sorted and each sum runs in x's order, as here.
class SparseProduct {
 public:
  explicit SparseProduct(int n) : acc_((size_t)n, 0.0), seen_((size_t)n, 0) {}
  void run(const HostCsr &x, int col, const HostCsr &m) {
    idx_.clear();
    for (int k = x.irp[col]; k < x.irp[col + 1]; k++) {
      const int r = x.ja[k];
      const double xv = x.val[k];
      for (int e = m.irp[r]; e < m.irp[r + 1]; e++) {
        const int c = m.ja[e];
        if (!seen_[c]) {
          seen_[c] = 1;
          acc_[c] = 0.0;
          idx_.push_back(c);
        }
        acc_[c] = acc_[c] + xv * m.val[e];
      }
    }
    std::sort(idx_.begin(), idx_.end());
    val_.resize(idx_.size());
    for (size_t m2 = 0; m2 < idx_.size(); m2++) {
      val_[m2] = acc_[idx_[m2]];
      seen_[idx_[m2]] = 0;
    }
  }
  // psb_spge_dot: sum of y_k * w[idx_k] in index order, from zero
  double dot_dense(const std::vector<double> &w) const {
    double s = 0.0;
    for (size_t m = 0; m < idx_.size(); m++) s = s + val_[m] * w[(size_t)idx_[m]];
    return s;
  }
  // psb_spdot_srtd: merge with an index-sorted column of f
  double dot_sorted(const HostCsr &f, int col) const {
    double s = 0.0;
    size_t a = 0;
    int b = f.irp[col];
    while (a < idx_.size() && b < f.irp[col + 1]) {
      if (idx_[a] < f.ja[b]) {
        a++;
      } else if (idx_[a] > f.ja[b]) {
        b++;
      } else {
        s = s + val_[a] * f.val[b];
        a++;
        b++;
      }
    }
    return s;
  }

 private:
  std::vector<double> acc_;
  std::vector<char> seen_;
  std::vector<int> idx_;
  std::vector<double> val_;
};

// Stabilised left-looking biconjugation (STAB-LLK,
// src/impl/mld_dsparse_biconjg_s_ft_llk.F90:35-414).  For each i, column i
// of Z and then column i of W: the Z step j uses p_i = (w_j^T A) . z
// (:164-169), the W step j uses q_i = (A z_j) . w (:297-304), both divided by
// the common pivot of column j; the pivot of column i is then
// (A z_i) . w_i over the kept entries (:381-389) with the 1e-3 guard
// (:402-406), psb_spdot_srtd being a merge of two index-sorted sparse
// vectors.  Candidate steps come from A's columns (Z) and rows (W) as in
// LLK.  The halves depend on each other column by column, so they run in
// turn on one thread.
void stab_llk(const HostCsr &a, const HostCsr &at, int cap, double thresh, double piv0,
              std::vector<double> &piv, HostCsr &zc, HostCsr &wc) {
  const int n = a.n;
  HalfBuilder zb(a, at, cap, thresh, true), wb(at, a, cap, thresh, true);
  zb.start(zc);
  wb.start(wc);
  piv.assign((size_t)n, 0.0);
  piv[0] = piv0;
  SparseProduct y(n);
  for (int i = 1; i < n; i++) {
    zb.update(i, piv, zc, [&](int j) {
      y.run(wc, j, a);  // w_j^T A
      return y.dot_dense(zb.work());
    });
    zb.keep_column(i, zc);
    wb.update(i, piv, wc, [&](int j) {
      y.run(zc, j, at);  // A z_j
      return y.dot_dense(wb.work());
    });
    wb.keep_column(i, wc);
    y.run(zc, i, at);  // A z_i
    double q = y.dot_sorted(wc, i);
    if (std::fabs(q) < kEpsTol) q = kTinyPivot;
    piv[(size_t)i] = q;
  }
}

}  // namespace

int ainv_biconjg_build(const HostCsr &a_in, int alg, int fill_in, double thresh,
                       HostCsr &wt, HostCsr &z, std::vector<double> &d) {
  if (fill_in < 1) {
    set_error("AINV build: fill_in must be >= 1 (got %d)", fill_in);
    return AINV_ERR_ARG;
  }
  if (alg != kAlgLLK && alg != kAlgSymLLK && alg != kAlgLLKNoth && alg != kAlgStabLLK &&
      alg != kAlgMLK) {
    set_error("AINV build: Invalid alg %d", alg);
    return AINV_ERR_ARG;
  }
  const int n = a_in.n;
  // clip to the local n x n block and scale by 1/max|a_ij|
  HostCsr a;
  a.n = n;
  a.irp.assign((size_t)n + 1, 0);
  for (int r = 0; r < n; r++) {
    for (int k = a_in.irp[r]; k < a_in.irp[r + 1]; k++)
      if (a_in.ja[k] >= 0 && a_in.ja[k] < n) {
        a.ja.push_back(a_in.ja[k]);
        a.val.push_back(a_in.val[k]);
      }
    a.irp[(size_t)r + 1] = (int)a.ja.size();
  }
  double mx = 0.0;
  for (double v : a.val) mx = std::max(mx, std::fabs(v));
  if (!(mx > 0.0)) {
    set_error("AINV build: matrix has no nonzero entries");
    return AINV_ERR_ARG;
  }
  const double weight = 1.0 / mx;
  for (double &v : a.val) v = v * weight;
  const HostCsr at = transpose(a);

  double a11 = 0.0;
  for (int k = a.irp[0]; k < a.irp[1]; k++)
    if (a.ja[k] == 0) {
      a11 = a.val[k];
      break;
    }
  if (std::fabs(a11) < kEpsTol) a11 = kTinyPivot;

  const bool alpha_test = alg != kAlgLLKNoth;
  std::vector<double> p, q;
  HostCsr zc, wc;
  // MLK (src/impl/mld_dsparse_biconjg_mlk.F90) keeps its candidate steps and
  // nonzero positions in sorted linked lists merged by hlmerge (:444-487)
  // instead of heaps.  Those visit the same steps in the same ascending order
  // as LLK's heaps, so only its list form of sparsify differs.
  const bool mlk = alg == kAlgMLK;
  HalfBuilder zb(a, at, fill_in, thresh, alpha_test, mlk);   // dots: rows of A
  if (alg == kAlgSymLLK) {
    zb.run(a11, p, zc);
    wc = zc;  // W = Z (src/impl/mld_dsparse_biconjg_s_llk.F90:246)
  } else if (alg == kAlgStabLLK) {
    stab_llk(a, at, fill_in, thresh, a11, p, zc, wc);
  } else {
    HalfBuilder wb(at, a, fill_in, thresh, alpha_test, mlk);  // dots: columns of A
    std::thread th([&] { wb.run(a11, q, wc); });
    zb.run(a11, p, zc);
    th.join();
  }
  // W is held by columns; its CSC arrays are the CSR arrays of W^T
  // (src/mld_d_biconjg_mod.F90:133-135).  Z goes CSC -> CSR (:131-132).
  wt = std::move(wc);
  z = transpose(zc);
  d.resize((size_t)n);
  for (int i = 0; i < n; i++) {
    const double inv = (std::fabs(p[i]) < kEpsTol) ? 1.0 : 1.0 / p[i];
    d[i] = inv * weight;  // src/impl/mld_d_ainv_bld.F90:161-173
  }
  return AINV_SUCCESS;
}

}  // namespace ainv
