// C-ABI entry points: device factors (create / apply / destroy) and the
// device operator A.  The Krylov loop lives in krylov.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <new>
#include <vector>

#include "internal.h"

namespace ainv {
const char *last_error();
}

using ainv::DevSell;
using ainv::HostCsr;

namespace {

void destroy_handle(ainv_handle *h) {
  if (!h) return;
  ainv::free_sell(h->wt);
  ainv::free_sell(h->z);
  ainv::free_sell(h->zt);
  ainv::free_sell(h->w);
  if (h->d) cudaFree(h->d);
  if (h->t) cudaFree(h->t);
  if (h->xs) cudaFree(h->xs);
  if (h->ys) cudaFree(h->ys);
  if (h->status) cudaFree(h->status);
  ainv::destroy_host_pipe(h->pipe);
  for (cudaStream_t st : h->hs)
    if (st) cudaStreamDestroy(st);
  for (cudaEvent_t e : h->hev) cudaEventDestroy(e);
  delete h;
}

// ---- host-array apply, pipelined over row chunks ----------------------------
// With page-locked x and y the copies overlap the sweeps chunk by chunk:
// chunk j of x is copied in while earlier chunks are swept, and rows of y
// go out as soon as their second sweep is done.  PCIe carries both
// directions at once, so a large apply costs little more than one transfer
// of x.  Sweep 1 over chunk c needs the input chunks up to the one holding
// the largest column its rows read (W^T and Z^T are lower triangular: chunk
// c itself).  Sweep 2 (Z or W, upper triangular) is split per chunk into the
// rows whose columns stay in the chunk, finished as soon as the chunk is in,
// and the remaining rows (the band reaching into later chunks).  Chunks ramp
// up from 1/8 of the nominal size at the start and back down at the end,
// which shortens the wait before the first rows of y and the tail after the
// last chunk of x.  Two forms run this schedule:
//  * fused (hostpipe.cu): copies of x plus one persistent kernel that polls
//    per-chunk flags and writes y straight into the caller's array;
//  * streams (below, when the two sweeps differ in pack width or y is not
//    device-mapped): per-chunk kernels and copies on three streams linked by
//    events.  Under PCIe load each event wait takes tens of microseconds to
//    resolve, which makes this form slower.
// The arithmetic per row is that of the whole-vector sweeps.

// Events of the stream pipeline: [0] orders it after the legacy stream; then
// one per chunk copied in and one per unit swept.
constexpr int kPipeEvents = 1;

// Nominal slices per chunk: about n/8 rows and at least 128K rows (1 MB per
// copy), a multiple of 4 slices.  AINV_HOST_CHUNK_ROWS sets the rows instead.
// (At n = 8M: 13 chunks after the ramps.  Each chunk costs about 20-30 us
// of PCIe time under bidirectional load; n/16 and n/4 measured slower.)
int host_chunk_slices(int n) {
  long long rows = std::max<long long>(131072, ((long long)n + 7) / 8);
  if (const char *e = std::getenv("AINV_HOST_CHUNK_ROWS")) {
    const long long v = std::atoll(e);
    if (v > 0) rows = v;
  }
  const long long sl = ((rows + ainv::kSlice - 1) / ainv::kSlice + 3) / 4 * 4;
  return (int)std::min<long long>(sl, 1 << 28);
}

bool page_locked(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Chunk bounds over ns slices: ramp cs/8, cs/4, cs/2, then chunks of about
// cs, then the ramp reversed; plain chunks of about cs when ns is too small.
std::vector<int> chunk_bounds(int ns, int cs) {
  auto r4 = [](long long v) { return (int)std::max<long long>(4, v / 4 * 4); };
  std::vector<int> ramp;
  for (int r = cs / 8; r < cs && r >= 4; r *= 2) ramp.push_back(r4(r));
  long long rs = 0;
  for (int r : ramp) rs += 2LL * r;
  if (ns < rs + 2LL * cs) {
    ramp.clear();
    rs = 0;
  }
  // sizes over ns rounded up to 4 slices, so every bound but the last one is
  // a multiple of 4; the last chunk ends at ns
  std::vector<int> sizes(ramp.begin(), ramp.end());
  const long long mid = (ns + 3LL) / 4 * 4 - rs;
  const long long cm = std::max<long long>(1, (mid + cs - 1) / cs);
  const int each = r4((mid + cm - 1) / cm + 3);
  for (long long left = mid; left > 0;) {
    const int sz = (int)std::min<long long>(each, left);
    sizes.push_back(sz);
    left -= sz;
  }
  sizes.insert(sizes.end(), ramp.rbegin(), ramp.rend());
  std::vector<int> bound(1, 0);
  for (int sz : sizes) bound.push_back(bound.back() + sz);
  bound.back() = ns;
  return bound;
}

// Chunk holding slice s.
int chunk_of(const std::vector<int> &bound, int s) {
  return (int)(std::upper_bound(bound.begin(), bound.end(), s) - bound.begin()) - 1;
}

// Last input chunk read by the rows of slices [s0, s1) of m (-1: none).
int needs(const DevSell &m, const std::vector<int> &bound, int s0, int s1) {
  int mc = -1;
  for (int s = s0; s < s1; s++) mc = std::max(mc, m.slice_maxcol[(size_t)s]);
  return mc < 0 ? -1 : chunk_of(bound, mc / ainv::kSlice);
}

void make_plan(const DevSell &m1, const DevSell &m2, int cs, ainv::HostPlan &p) {
  p = ainv::HostPlan{};
  p.cs = cs;
  p.bound = chunk_bounds(m1.nslices, cs);
  const int C = (int)p.bound.size() - 1;
  for (int c = 0; c < C; c++) {
    const int b0 = p.bound[(size_t)c], b1 = p.bound[(size_t)c + 1];
    p.need1.push_back(needs(m1, p.bound, b0, b1));
    // leading slices (a multiple of 4) whose rows read t of chunks <= c only
    const long long end_row = (long long)b1 * ainv::kSlice;
    int q = b0;
    while (q < b1 && m2.slice_maxcol[(size_t)q] < end_row) q++;
    q = std::max(b0, q / 4 * 4);
    for (int part = 0; part < 2; part++) {
      const int lo = part == 0 ? b0 : q, hi = part == 0 ? q : b1;
      if (lo == hi) continue;
      p.u0.push_back(lo);
      p.u1.push_back(hi);
      p.need2.push_back(needs(m2, p.bound, lo, hi));
    }
  }
}

// Enqueue the pipeline on si (copies in), sc (sweeps) and so (copies out);
// the three streams must already be ordered after whatever comes before.
int enqueue_pipeline(ainv_handle *h, bool tr, double alpha, const double *x, double beta,
                     double *y) {
  const DevSell &m1 = tr ? h->zt : h->wt, &m2 = tr ? h->w : h->z;
  const ainv::HostPlan &p = h->hplan[tr];
  const int C = (int)p.bound.size() - 1, U = (int)p.u0.size();
  cudaStream_t si = h->hs[0], sc = h->hs[1], so = h->hs[2];
  cudaEvent_t *ein = &h->hev[kPipeEvents], *eout = ein + C;
  const size_t n = (size_t)h->n;
  auto span = [&](int s0, int s1, size_t &r0, size_t &nb) {
    r0 = (size_t)s0 * ainv::kSlice;
    nb = sizeof(double) * (std::min(n, (size_t)s1 * ainv::kSlice) - r0);
  };
  int rc = AINV_SUCCESS;
  auto cuda = [&](cudaError_t e, const char *what) {
    if (rc == AINV_SUCCESS && e != cudaSuccess) {
      ainv::set_error("host apply: %s failed: %s", what, cudaGetErrorString(e));
      rc = AINV_ERR_CUDA;
    }
    return rc == AINV_SUCCESS;
  };
  bool ok = true;
  for (int c = 0; ok && c < C; c++) {
    size_t r0, nb;
    span(p.bound[(size_t)c], p.bound[(size_t)c + 1], r0, nb);
    ok = cuda(cudaMemcpyAsync(h->xs + r0, x + r0, nb, cudaMemcpyHostToDevice, si), "copy in");
    if (ok && beta != 0.0)
      ok = cuda(cudaMemcpyAsync(h->ys + r0, y + r0, nb, cudaMemcpyHostToDevice, si), "copy in");
    ok = ok && cuda(cudaEventRecord(ein[c], si), "event record");
  }
  for (int i = 0, u = 0; ok && i < C; i++) {
    const int need = p.need1[(size_t)i];
    if (need >= 0) ok = cuda(cudaStreamWaitEvent(sc, ein[need], 0), "stream wait");
    if (ok) {
      rc = ainv::launch_sweep_dscale_slices(m1, h->d, h->xs, h->t, p.bound[(size_t)i],
                                            p.bound[(size_t)i + 1], sc);
      ok = rc == AINV_SUCCESS;
    }
    for (; ok && u < U && p.need2[(size_t)u] <= i; u++) {
      const int a = p.u0[(size_t)u], b = p.u1[(size_t)u];
      // the y rows of a unit (inside one chunk) came in with that chunk
      if (beta != 0.0) ok = cuda(cudaStreamWaitEvent(sc, ein[chunk_of(p.bound, a)], 0), "stream wait");
      if (ok) {
        rc = ainv::launch_sweep_axpby_slices(m2, h->t, alpha, beta, h->ys, a, b, sc);
        ok = rc == AINV_SUCCESS;
      }
      size_t r0, nb;
      span(a, b, r0, nb);
      ok = ok && cuda(cudaEventRecord(eout[u], sc), "event record") &&
           cuda(cudaStreamWaitEvent(so, eout[u], 0), "stream wait") &&
           cuda(cudaMemcpyAsync(y + r0, h->ys + r0, nb, cudaMemcpyDeviceToHost, so), "copy out");
    }
  }
  return rc;
}

int apply_host_chunked(ainv_handle *h, bool tr, int cs, double alpha, const double *x,
                       double beta, double *y) {
  ainv::HostPlan &p = h->hplan[tr];
  if (p.cs != cs) make_plan(tr ? h->zt : h->wt, tr ? h->w : h->z, cs, p);
  for (cudaStream_t &st : h->hs)
    if (!st) AINV_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  const int C = (int)p.bound.size() - 1, U = (int)p.u0.size();
  while ((int)h->hev.size() < kPipeEvents + C + U) {
    cudaEvent_t e;
    AINV_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    h->hev.push_back(e);
  }
  cudaEvent_t e0 = h->hev[0];
  // ordered after earlier work on the legacy stream, as the serial form is
  AINV_CUDA_TRY(cudaEventRecord(e0, 0));
  for (cudaStream_t st : h->hs) AINV_CUDA_TRY(cudaStreamWaitEvent(st, e0, 0));
  const bool fused = ainv::host_pipe_usable(h, tr, y);
  int rc = fused ? ainv::host_pipe_apply(h, tr, p, alpha, x, beta, y, h->hs[0], h->hs[1])
                 : enqueue_pipeline(h, tr, alpha, x, beta, y);
  // every copy touching the caller's arrays is done before returning
  for (cudaStream_t st : h->hs) {
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess && rc == AINV_SUCCESS) {
      ainv::set_error("host apply: synchronize failed: %s", cudaGetErrorString(e));
      rc = AINV_ERR_CUDA;
    }
  }
  if (rc == AINV_SUCCESS && fused) rc = ainv::host_pipe_status(h);
  return rc;
}

int check_unit_triangle(const HostCsr &m, bool lower, const char *what) {
  // W^T is unit lower, Z unit upper (src/impl/mld_dsparse_biconjg_llk.F90:97-110,
  // diag kept by sparsify).  A violation means the caller swapped the factors.
  for (int i = 0; i < m.n; i++)
    for (int k = m.irp[i]; k < m.irp[i + 1]; k++)
      if (lower ? (m.ja[k] > i) : (m.ja[k] < i)) {
        ainv::set_error("%s is not %s triangular (row %d, column %d)", what,
                        lower ? "lower" : "upper", i, m.ja[k]);
        return AINV_ERR_ARG;
      }
  return AINV_SUCCESS;
}

}  // namespace

extern "C" {

const char *ainv_last_error(void) { return ainv::last_error(); }
const char *ainv_version(void) { return "ainv_b200 0.1 (sm_100a)"; }

int ainv_gpu_create(ainv_handle **hp, int n, const int *wt_irp, const int *wt_ja,
                    const double *wt_val, const int *z_irp, const int *z_ja,
                    const double *z_val, const double *dinv, int prec, int one_based) {
  if (!hp) {
    ainv::set_error("ainv_gpu_create: null handle pointer");
    return AINV_ERR_ARG;
  }
  *hp = nullptr;
  if (ainv::prec_size(prec) == 0) {
    ainv::set_error("ainv_gpu_create: unknown precision %d", prec);
    return AINV_ERR_ARG;
  }
  if (!dinv) {
    ainv::set_error("ainv_gpu_create: null diagonal");
    return AINV_ERR_ARG;
  }
  HostCsr wt, z;
  AINV_TRY(ainv::import_csr(n, wt_irp, wt_ja, wt_val, one_based, wt, "W^T"));
  AINV_TRY(ainv::import_csr(n, z_irp, z_ja, z_val, one_based, z, "Z"));
  AINV_TRY(check_unit_triangle(wt, true, "W^T"));
  AINV_TRY(check_unit_triangle(z, false, "Z"));

  ainv_handle *h = new (std::nothrow) ainv_handle;
  if (!h) {
    ainv::set_error("ainv_gpu_create: host allocation failed");
    return AINV_ERR_ALLOC;
  }
  h->serial = ainv::next_serial();
  h->n = n;
  h->prec = prec;
  int rc = ainv::upload_sell(wt, prec, h->wt);
  if (rc == AINV_SUCCESS) rc = ainv::upload_sell(z, prec, h->z);
  if (rc == AINV_SUCCESS) rc = ainv::upload_sell(ainv::transpose(z), prec, h->zt);
  if (rc == AINV_SUCCESS) rc = ainv::upload_sell(ainv::transpose(wt), prec, h->w);
  if (rc == AINV_SUCCESS) rc = ainv::upload_values(dinv, (size_t)n, prec, &h->d);
  if (rc == AINV_SUCCESS) {
    const size_t ts = (prec == AINV_PREC_FP32 || prec == AINV_PREC_BF16) ? 4 : 8;
    cudaError_t e = cudaMalloc(&h->t, ts * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&h->status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(h->status, 0, sizeof(int));
    if (e != cudaSuccess) {
      ainv::set_error("ainv_gpu_create: scratch allocation failed: %s", cudaGetErrorString(e));
      rc = AINV_ERR_ALLOC;
    }
  }
  if (rc != AINV_SUCCESS) {
    destroy_handle(h);
    return rc;
  }
  *hp = h;
  return AINV_SUCCESS;
}

int ainv_gpu_apply(ainv_handle *h, char trans, double alpha, const double *x_dev,
                   double beta, double *y_dev, void *stream) {
  if (!h || !x_dev || !y_dev) {
    ainv::set_error("ainv_gpu_apply: null argument");
    return AINV_ERR_ARG;
  }
  return ainv::ainv_apply_async(h, trans, alpha, x_dev, beta, y_dev, (cudaStream_t)stream);
}

int ainv_gpu_apply_stage(ainv_handle *h, char trans, int stage, double alpha,
                         const double *x_dev, double beta, double *y_dev, void *stream) {
  if (!h || (stage == 1 && !x_dev) || (stage == 2 && !y_dev) || (stage != 1 && stage != 2)) {
    ainv::set_error("ainv_gpu_apply_stage: invalid argument");
    return AINV_ERR_ARG;
  }
  const bool tr = (trans == 'T' || trans == 't' || trans == 'C' || trans == 'c');
  if (!tr && trans != 'N' && trans != 'n') {
    ainv::set_error("ainv_gpu_apply_stage: invalid trans '%c'", trans);
    return AINV_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (stage == 1)
    return ainv::launch_sweep_dscale(tr ? h->zt : h->wt, h->d, x_dev, h->t, s, nullptr, h->status);
  return ainv::launch_sweep_axpby(tr ? h->w : h->z, h->t, alpha, beta, y_dev, s, nullptr,
                                  h->status);
}

int ainv_gpu_apply_host(ainv_handle *h, char trans, double alpha, const double *x,
                        double beta, double *y) {
  if (!h || !x || !y) {
    ainv::set_error("ainv_gpu_apply_host: null argument");
    return AINV_ERR_ARG;
  }
  const size_t bytes = sizeof(double) * (size_t)h->n;
  if (!h->xs) {
    AINV_CUDA_TRY(cudaMalloc(&h->xs, bytes));
    AINV_CUDA_TRY(cudaMalloc(&h->ys, bytes));
  }
  const bool tr = (trans == 'T' || trans == 't' || trans == 'C' || trans == 'c');
  const int cs = host_chunk_slices(h->n);
  // The pipelined forms write y while later chunks of x are still being read,
  // so arrays that overlap take the serial form (copy all of x first).
  const bool overlap = x < y + h->n && y < x + h->n;
  if ((tr || trans == 'N' || trans == 'n') && h->wt.nslices > cs && !overlap &&
      page_locked(x) && page_locked(y))
    return apply_host_chunked(h, tr, cs, alpha, x, beta, y);
  AINV_CUDA_TRY(cudaMemcpyAsync(h->xs, x, bytes, cudaMemcpyHostToDevice, 0));
  if (beta != 0.0) AINV_CUDA_TRY(cudaMemcpyAsync(h->ys, y, bytes, cudaMemcpyHostToDevice, 0));
  AINV_TRY(ainv_gpu_apply(h, trans, alpha, h->xs, beta, h->ys, nullptr));
  AINV_CUDA_TRY(cudaMemcpyAsync(y, h->ys, bytes, cudaMemcpyDeviceToHost, 0));
  AINV_CUDA_TRY(cudaStreamSynchronize(0));
  return AINV_SUCCESS;
}

int ainv_gpu_destroy(ainv_handle *h) {
  destroy_handle(h);
  return AINV_SUCCESS;
}

size_t ainv_gpu_sizeof(const ainv_handle *h) {
  if (!h) return 0;
  size_t b = sizeof(*h) + h->wt.bytes() + h->z.bytes() + h->zt.bytes() + h->w.bytes();
  b += ainv::prec_size(h->prec) * (size_t)h->n;                    // D^-1
  b += (h->prec == AINV_PREC_FP32 || h->prec == AINV_PREC_BF16 ? 4 : 8) * (size_t)h->n;  // t
  if (h->xs) b += 2 * sizeof(double) * (size_t)h->n;
  return b;
}

long long ainv_gpu_get_nzeros(const ainv_handle *h) {
  // dv rows + nnz(W^T) + nnz(Z), as d_base_ainv_get_nzeros counts them.
  return h ? (long long)h->n + h->wt.nnz + h->z.nnz : 0;
}

int ainv_gpu_get_n(const ainv_handle *h) { return h ? h->n : 0; }
int ainv_gpu_get_prec(const ainv_handle *h) { return h ? h->prec : -1; }

int ainv_gpu_layout_info(const ainv_handle *h, int which, long long *nnz, long long *slots,
                         long long *nidx, int *nslices, int *offset_slices) {
  if (!h || which < 0 || which > 3) {
    ainv::set_error("ainv_gpu_layout_info: invalid argument");
    return AINV_ERR_ARG;
  }
  const DevSell &m = which == 0 ? h->wt : which == 1 ? h->z : which == 2 ? h->zt : h->w;
  if (nnz) *nnz = m.nnz;
  if (slots) *slots = m.slots;
  if (nidx) *nidx = m.nidx;
  if (nslices) *nslices = m.nslices;
  if (offset_slices) *offset_slices = m.offset_slices;
  return AINV_SUCCESS;
}

// Streaming kernels record a timed-out wait in the object's status word;
// reading it synchronises the device and clears it.
static int read_status(int *word, const char *what) {
  if (!word) return AINV_SUCCESS;
  int v = 0;
  AINV_CUDA_TRY(cudaMemcpy(&v, word, sizeof(int), cudaMemcpyDeviceToHost));
  if (v != 0) {
    AINV_CUDA_TRY(cudaMemset(word, 0, sizeof(int)));
    ainv::set_error("%s: a device wait ran past its time limit; results are incomplete", what);
    return AINV_ERR_TIMEOUT;
  }
  return AINV_SUCCESS;
}

int ainv_gpu_check(const ainv_handle *h) {
  if (!h) return AINV_ERR_ARG;
  return read_status(h->status, "ainv_gpu_check");
}

int ainv_csr_check(const ainv_csr *a) {
  if (!a) return AINV_ERR_ARG;
  return read_status(a->status, "ainv_csr_check");
}

int ainv_csr_create(ainv_csr **ap, int n, const int *irp, const int *ja, const double *val,
                    int one_based) {
  if (!ap) {
    ainv::set_error("ainv_csr_create: null pointer");
    return AINV_ERR_ARG;
  }
  *ap = nullptr;
  HostCsr a;
  AINV_TRY(ainv::import_csr(n, irp, ja, val, one_based, a, "A"));
  ainv_csr *m = new (std::nothrow) ainv_csr;
  if (!m) {
    ainv::set_error("ainv_csr_create: host allocation failed");
    return AINV_ERR_ALLOC;
  }
  m->n = n;
  int rc = ainv::upload_sell(a, AINV_PREC_FP64, m->a);
  if (rc == AINV_SUCCESS) {
    cudaError_t e = cudaMalloc(&m->status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(m->status, 0, sizeof(int));
    if (e != cudaSuccess) {
      ainv::set_error("ainv_csr_create: status allocation failed: %s", cudaGetErrorString(e));
      rc = AINV_ERR_ALLOC;
    }
  }
  if (rc != AINV_SUCCESS) {
    ainv::free_sell(m->a);
    if (m->status) cudaFree(m->status);
    delete m;
    return rc;
  }
  *ap = m;
  return AINV_SUCCESS;
}

int ainv_csr_spmv(const ainv_csr *a, double alpha, const double *x_dev, double beta,
                  double *y_dev, void *stream) {
  if (!a || !x_dev || !y_dev) {
    ainv::set_error("ainv_csr_spmv: null argument");
    return AINV_ERR_ARG;
  }
  return ainv::launch_spmv(a->a, alpha, x_dev, beta, y_dev, (cudaStream_t)stream, a->status);
}

int ainv_csr_destroy(ainv_csr *a) {
  if (a) {
    ainv::destroy_ws(a->ws);
    ainv::destroy_mws(a->mws);
    ainv::free_sell(a->a);
    if (a->status) cudaFree(a->status);
    delete a;
  }
  return AINV_SUCCESS;
}

}  // extern "C"
