// sm_100a kernels for the factor sweeps of the AINV apply and the A SpMV.
//
// Layout: SELL-32 (see internal.h).  One warp owns one slice of 32 rows,
// one lane one row; slot k of a slice is a 32-wide contiguous run, so each
// value/index load of the warp is one coalesced 256 B / 128 B request.
// Factor values and indices are read exactly once per apply and use the
// streaming (evict-first) hint, so the gathered vectors (x and t: 64 MB at
// n = 8M, inside the 126 MB L2) stay resident between the two sweeps.
//
// Epilogues are fused: sweep 1 writes t = D^-1 .* (W^T x), sweep 2 writes
// y = alpha*Z t + beta*y, so the reference's three passes
// (src/impl/mld_d_base_ainv_solver_apply_vect.f90:114-119) become two.
// `stop` (optional) is a device flag set by the Krylov loop once it has
// converged; kernels launched after that return immediately.
#include "sell_device.cuh"

namespace ainv {
namespace {

using namespace dev;

template <class V, class T>
__global__ void __launch_bounds__(kBlock)
    k_sweep_dscale(int n, int nslices, const int *__restrict__ sptr,
                   const int *__restrict__ col, const V *__restrict__ val,
                   const double *__restrict__ x, const V *__restrict__ d,
                   T *__restrict__ t, const int *__restrict__ stop) {
  if (stop && *stop) return;
  SliceCtx c;
  if (!slice_ctx(nslices, sptr, c)) return;
  const auto acc = row_dot(col + c.beg + c.lane, val + c.beg + c.lane, x, c.w);
  if (c.row < n) t[c.row] = (T)(ldd(d + c.row) * acc);
}

template <class V, class T>
__global__ void __launch_bounds__(kBlock)
    k_sweep_axpby(int n, int nslices, const int *__restrict__ sptr,
                  const int *__restrict__ col, const V *__restrict__ val,
                  const T *__restrict__ t, double alpha, double beta,
                  double *__restrict__ y, const int *__restrict__ stop) {
  if (stop && *stop) return;
  SliceCtx c;
  if (!slice_ctx(nslices, sptr, c)) return;
  const auto acc = row_dot(col + c.beg + c.lane, val + c.beg + c.lane, t, c.w);
  if (c.row < n) {
    const double r = alpha * (double)acc;
    y[c.row] = (beta == 0.0) ? r : r + beta * y[c.row];
  }
}

inline int check_launch(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s launch failed: %s", what, cudaGetErrorString(e));
    return AINV_ERR_CUDA;
  }
  return AINV_SUCCESS;
}

}  // namespace

int launch_sweep_dscale(const DevSell &m, const void *d, const double *x, void *t,
                        cudaStream_t s, const int *stop) {
  if (m.nslices == 0) return AINV_SUCCESS;
  const int g = grid_for(m.nslices);
  switch (m.prec) {
    case AINV_PREC_FP64:
      k_sweep_dscale<double, double><<<g, kBlock, 0, s>>>(
          m.n, m.nslices, m.sptr, m.col, (const double *)m.val, x, (const double *)d,
          (double *)t, stop);
      break;
    case AINV_PREC_FP32:
      k_sweep_dscale<float, float><<<g, kBlock, 0, s>>>(
          m.n, m.nslices, m.sptr, m.col, (const float *)m.val, x, (const float *)d,
          (float *)t, stop);
      break;
    case AINV_PREC_BF16:
      k_sweep_dscale<__nv_bfloat16, float><<<g, kBlock, 0, s>>>(
          m.n, m.nslices, m.sptr, m.col, (const __nv_bfloat16 *)m.val, x,
          (const __nv_bfloat16 *)d, (float *)t, stop);
      break;
    default:
      set_error("unknown precision %d", m.prec);
      return AINV_ERR_ARG;
  }
  return check_launch("sweep_dscale");
}

int launch_sweep_axpby(const DevSell &m, const void *t, double alpha, double beta,
                       double *y, cudaStream_t s, const int *stop) {
  if (m.nslices == 0) return AINV_SUCCESS;
  const int g = grid_for(m.nslices);
  switch (m.prec) {
    case AINV_PREC_FP64:
      k_sweep_axpby<double, double><<<g, kBlock, 0, s>>>(
          m.n, m.nslices, m.sptr, m.col, (const double *)m.val, (const double *)t, alpha,
          beta, y, stop);
      break;
    case AINV_PREC_FP32:
      k_sweep_axpby<float, float><<<g, kBlock, 0, s>>>(
          m.n, m.nslices, m.sptr, m.col, (const float *)m.val, (const float *)t, alpha,
          beta, y, stop);
      break;
    case AINV_PREC_BF16:
      k_sweep_axpby<__nv_bfloat16, float><<<g, kBlock, 0, s>>>(
          m.n, m.nslices, m.sptr, m.col, (const __nv_bfloat16 *)m.val, (const float *)t,
          alpha, beta, y, stop);
      break;
    default:
      set_error("unknown precision %d", m.prec);
      return AINV_ERR_ARG;
  }
  return check_launch("sweep_axpby");
}

int launch_spmv(const DevSell &a, double alpha, const double *x, double beta, double *y,
                cudaStream_t s) {
  if (a.prec != AINV_PREC_FP64) {
    set_error("operator A must be stored in FP64");
    return AINV_ERR_ARG;
  }
  if (a.nslices == 0) return AINV_SUCCESS;
  k_sweep_axpby<double, double><<<grid_for(a.nslices), kBlock, 0, s>>>(
      a.n, a.nslices, a.sptr, a.col, (const double *)a.val, x, alpha, beta, y, nullptr);
  return check_launch("spmv");
}

int ainv_apply_async(const ainv_handle *h, char trans, double alpha, const double *x,
                     double beta, double *y, cudaStream_t s, const int *stop) {
  switch (trans) {
    case 'N': case 'n':
      AINV_TRY(launch_sweep_dscale(h->wt, h->d, x, h->t, s, stop));
      return launch_sweep_axpby(h->z, h->t, alpha, beta, y, s, stop);
    case 'T': case 't': case 'C': case 'c':
      AINV_TRY(launch_sweep_dscale(h->zt, h->d, x, h->t, s, stop));
      return launch_sweep_axpby(h->w, h->t, alpha, beta, y, s, stop);
    default:
      // psb_err_iarg_invalid_i_ (src/impl/mld_d_base_ainv_solver_apply_vect.f90:64-71)
      set_error("invalid trans '%c'", trans);
      return AINV_ERR_ARG;
  }
}

}  // namespace ainv
