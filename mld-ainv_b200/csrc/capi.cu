// C-ABI entry points: device factors (create / apply / destroy) and the
// device operator A.  The Krylov loop lives in krylov.cu.
#include <cuda_runtime.h>

#include <cstdio>
#include <new>

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
  delete h;
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
