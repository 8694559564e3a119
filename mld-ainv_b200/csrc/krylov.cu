// Krylov loop on the device: preconditioned CG and BiCGSTAB in the form of
// PSBLAS psb_dcg / psb_dbicgstab with istop=2 (stop when ||r|| <= eps*||b||),
// as driven at tests/pdegen/ppde3d.f90:280-281.
//
// Every scalar of the recurrence (rho, alpha, omega, beta, norms, status)
// lives in device memory and is produced by the last block of the kernel
// that computes the corresponding reduction, so one iteration is a fixed
// sequence of launches with no host round trip.  Reductions are
// deterministic: per-block partials are folded in block order.  Iterations
// are issued in chunks captured once into a CUDA graph; when the loop has
// converged (or broken down) a device flag makes every later kernel of the
// chunk return at once, and the host inspects the state once per chunk.
//
// Fused steps: the A product and the dots that consume it (p.q, rt.v, t.t
// and t.s) share one kernel; the Z sweep of the preconditioner and the CG
// dot r.z share one kernel; x/r updates and the residual norm (plus rt.r
// for BiCGSTAB) share one kernel.
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <new>

#include "sell_device.cuh"

namespace ainv {

struct KState {
  double rho, rho_old, alpha, beta, omega, rn2, bn2, eps;
  int iter, itmax, done, status, replace_every, method;
  unsigned ticket[4];
};

namespace {

using namespace dev;

enum { kCgSigma = 0, kBicgSigma = 1, kBicgOmega = 2, kReplace = 3, kInit = 4 };
constexpr int kChunk = 8;  // iterations per captured graph launch

__device__ __forceinline__ void finish_iteration(KState *st, double rn2) {
  st->rn2 = rn2;
  st->iter += 1;
  const double err = sqrt(rn2) / st->bn2;
  if (!isfinite(rn2)) {
    st->status = AINV_ERR_NONFINITE;
    st->done = 1;
  } else if (err <= st->eps) {
    st->status = AINV_SUCCESS;
    st->done = 1;
  } else if (st->iter >= st->itmax) {
    st->status = AINV_ERR_NOCONV;
    st->done = 1;
  }
}

// BiCGSTAB: start the next iteration's scalars from rho = rt.r.
__device__ __forceinline__ void bicg_next_rho(KState *st, double rr) {
  if (st->done) return;
  st->rho_old = st->rho;
  st->rho = rr;
  if (rr == 0.0) {
    st->status = AINV_ERR_BREAKDOWN;
    st->done = 1;
  } else {
    st->beta = (st->rho / st->rho_old) * (st->alpha / st->omega);
  }
}

// ||b||_2 (istop=2 denominator).
__global__ void __launch_bounds__(kBlock)
    k_bnorm(int n, const double *__restrict__ b, KState *st, double *partials) {
  const int i = blockIdx.x * kBlock + threadIdx.x;
  double pr[1] = {0.0};
  if (i < n) pr[0] = b[i] * b[i];
  if (grid_sum<1>(pr, partials, &st->ticket[0]) && threadIdx.x == 0) {
    const double bn = sqrt(pr[0]);
    st->bn2 = (bn == 0.0) ? 1.0 : bn;
  }
}

// y = A x with the reductions each caller needs (see MODE):
//   kCgSigma:   sigma = x.y, alpha = rho/sigma               (q = A p)
//   kBicgSigma: sigma = w1.y, alpha = rho/sigma              (v = A f, w1 = rt)
//   kBicgOmega: omega = (y.w1)/(y.y)                         (t = A z, w1 = s)
//   kReplace:   y = w1 - A x (true residual, w1 = b), every replace_every its
//   kInit:      y = w1 - A x, optional copy into w2 (rt), initial norm/rho
template <int MODE>
__global__ void __launch_bounds__(kBlock)
    k_spmv_dots(int n, int nslices, const int *__restrict__ sptr,
                const int *__restrict__ col, const double *__restrict__ val,
                const double *__restrict__ x, double *__restrict__ y,
                const double *__restrict__ w1, double *__restrict__ w2, KState *st,
                double *partials) {
  if (st->done) return;
  if (MODE == kReplace &&
      (st->replace_every <= 0 || st->iter == 0 || st->iter % st->replace_every != 0))
    return;
  SliceCtx c;
  double pr[2] = {0.0, 0.0};
  if (slice_ctx(nslices, sptr, c)) {
    const double acc = row_dot(col + c.beg + c.lane, val + c.beg + c.lane, x, c.w);
    if (c.row < n) {
      const int i = c.row;
      if (MODE == kReplace || MODE == kInit) {
        const double ri = w1[i] - acc;
        y[i] = ri;
        pr[0] = ri * ri;
        if (w2) {
          if (MODE == kInit) {
            w2[i] = ri;
            pr[1] = ri * ri;
          } else {
            pr[1] = w2[i] * ri;
          }
        }
      } else {
        y[i] = acc;
        if (MODE == kCgSigma) pr[0] = x[i] * acc;
        if (MODE == kBicgSigma) pr[0] = w1[i] * acc;
        if (MODE == kBicgOmega) {
          pr[0] = acc * acc;
          pr[1] = acc * w1[i];
        }
      }
    }
  }
  if (grid_sum<2>(pr, partials, &st->ticket[1]) && threadIdx.x == 0) {
    if (MODE == kCgSigma || MODE == kBicgSigma) {
      if (pr[0] == 0.0) {
        st->status = AINV_ERR_BREAKDOWN;
        st->done = 1;
      } else {
        st->alpha = st->rho / pr[0];
      }
    } else if (MODE == kBicgOmega) {
      const double om = (pr[0] == 0.0) ? 0.0 : pr[1] / pr[0];
      if (pr[0] == 0.0 || om == 0.0) {
        st->status = AINV_ERR_BREAKDOWN;
        st->done = 1;
      } else {
        st->omega = om;
      }
    } else {  // kReplace / kInit: convergence on the true residual
      st->rn2 = pr[0];
      const double err = sqrt(pr[0]) / st->bn2;
      if (!isfinite(pr[0])) {
        st->status = AINV_ERR_NONFINITE;
        st->done = 1;
      } else if (err <= st->eps) {
        st->status = AINV_SUCCESS;
        st->done = 1;
      }
      if (MODE == kInit) {
        st->rho = pr[1];
        if (!st->done && st->itmax <= 0) {
          st->status = AINV_ERR_NOCONV;
          st->done = 1;
        }
      } else if (w2 && !st->done) {
        // rho for the coming iteration follows the replaced residual
        st->rho = pr[1];
        if (pr[1] == 0.0) {
          st->status = AINV_ERR_BREAKDOWN;
          st->done = 1;
        } else {
          st->beta = (st->rho / st->rho_old) * (st->alpha / st->omega);
        }
      }
    }
  }
}

// CG: z = Z t (sweep 2 of the AINV apply) fused with rho = r.z, then beta.
template <class V, class T>
__global__ void __launch_bounds__(kBlock)
    k_cg_sweep2(int n, int nslices, const int *__restrict__ sptr, const int *__restrict__ col,
                const V *__restrict__ val, const T *__restrict__ t,
                const double *__restrict__ r, double *__restrict__ z, KState *st,
                double *partials) {
  if (st->done) return;
  SliceCtx c;
  double pr[1] = {0.0};
  if (slice_ctx(nslices, sptr, c)) {
    const auto acc = row_dot(col + c.beg + c.lane, val + c.beg + c.lane, t, c.w);
    if (c.row < n) {
      const double zi = (double)acc;
      z[c.row] = zi;
      pr[0] = r[c.row] * zi;
    }
  }
  if (grid_sum<1>(pr, partials, &st->ticket[0]) && threadIdx.x == 0) {
    st->rho_old = st->rho;
    st->rho = pr[0];
    if (st->iter > 0) {
      if (st->rho_old == 0.0) {
        st->status = AINV_ERR_BREAKDOWN;
        st->done = 1;
      } else {
        st->beta = st->rho / st->rho_old;
      }
    }
  }
}

// CG without preconditioner: z = r, rho = r.r.
__global__ void __launch_bounds__(kBlock)
    k_cg_ident(int n, const double *__restrict__ r, double *__restrict__ z, KState *st,
               double *partials) {
  if (st->done) return;
  const int i = blockIdx.x * kBlock + threadIdx.x;
  double pr[1] = {0.0};
  if (i < n) {
    z[i] = r[i];
    pr[0] = r[i] * r[i];
  }
  if (grid_sum<1>(pr, partials, &st->ticket[0]) && threadIdx.x == 0) {
    st->rho_old = st->rho;
    st->rho = pr[0];
    if (st->iter > 0) {
      if (st->rho_old == 0.0) {
        st->status = AINV_ERR_BREAKDOWN;
        st->done = 1;
      } else {
        st->beta = st->rho / st->rho_old;
      }
    }
  }
}

// CG: p = z (first iteration) or p = z + beta p.
__global__ void __launch_bounds__(kBlock)
    k_cg_p(int n, const double *__restrict__ z, double *__restrict__ p, const KState *st) {
  if (st->done) return;
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  p[i] = (st->iter == 0) ? z[i] : z[i] + st->beta * p[i];
}

// CG: x += alpha p, r -= alpha q, rn2 = r.r, convergence.
__global__ void __launch_bounds__(kBlock)
    k_cg_xr(int n, const double *__restrict__ p, const double *__restrict__ q,
            double *__restrict__ x, double *__restrict__ r, KState *st, double *partials) {
  if (st->done) return;
  const int i = blockIdx.x * kBlock + threadIdx.x;
  const double alpha = st->alpha;
  double pr[1] = {0.0};
  if (i < n) {
    x[i] = x[i] + alpha * p[i];
    const double ri = r[i] - alpha * q[i];
    r[i] = ri;
    pr[0] = ri * ri;
  }
  if (grid_sum<1>(pr, partials, &st->ticket[2]) && threadIdx.x == 0)
    finish_iteration(st, pr[0]);
}

// BiCGSTAB: p = r (first iteration) or p = r + beta (p - omega v).
__global__ void __launch_bounds__(kBlock)
    k_bicg_p(int n, const double *__restrict__ r, const double *__restrict__ v,
             double *__restrict__ p, const KState *st) {
  if (st->done) return;
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  p[i] = (st->iter == 0) ? r[i] : r[i] + st->beta * (p[i] - st->omega * v[i]);
}

// BiCGSTAB: s = r - alpha v.
__global__ void __launch_bounds__(kBlock)
    k_bicg_s(int n, const double *__restrict__ r, const double *__restrict__ v,
             double *__restrict__ s, const KState *st) {
  if (st->done) return;
  const int i = blockIdx.x * kBlock + threadIdx.x;
  if (i >= n) return;
  s[i] = r[i] - st->alpha * v[i];
}

// BiCGSTAB: x += alpha f + omega z, r = s - omega t, rn2 = r.r, rho' = rt.r.
__global__ void __launch_bounds__(kBlock)
    k_bicg_xr(int n, const double *__restrict__ f, const double *__restrict__ z,
              const double *__restrict__ s, const double *__restrict__ t,
              const double *__restrict__ rt, double *__restrict__ x,
              double *__restrict__ r, KState *st, double *partials) {
  if (st->done) return;
  const int i = blockIdx.x * kBlock + threadIdx.x;
  const double alpha = st->alpha, omega = st->omega;
  double pr[2] = {0.0, 0.0};
  if (i < n) {
    x[i] = (x[i] + alpha * f[i]) + omega * z[i];
    const double ri = s[i] - omega * t[i];
    r[i] = ri;
    pr[0] = ri * ri;
    pr[1] = rt[i] * ri;
  }
  if (grid_sum<2>(pr, partials, &st->ticket[2]) && threadIdx.x == 0) {
    finish_iteration(st, pr[0]);
    bicg_next_rho(st, pr[1]);
  }
}

template <class V, class T>
void launch_cg_sweep2(const DevSell &m, const void *t, const double *r, double *z,
                      KState *st, double *partials, cudaStream_t s) {
  k_cg_sweep2<V, T><<<grid_for(m.nslices), kBlock, 0, s>>>(
      m.n, m.nslices, m.sptr, m.col, (const V *)m.val, (const T *)t, r, z, st, partials);
}

std::atomic<unsigned long long> g_serial{1};

}  // namespace

unsigned long long next_serial() { return g_serial.fetch_add(1); }

// ------------------------------------------------------------ workspace --
struct KrylovWs {
  int n = 0, G = 0;
  double *vec = nullptr;  // 10 vectors of n
  double *partials = nullptr;
  KState *st = nullptr;
  KState *hst = nullptr;  // pinned mirror
  cudaStream_t s = nullptr;
  cudaEvent_t ev = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long key_serial = 0;
  int key_method = -1, key_replace = -1;
  double *v(int i) const { return vec + (size_t)i * (size_t)n; }
};

void destroy_ws(KrylovWs *w) {
  if (!w) return;
  if (w->exec) cudaGraphExecDestroy(w->exec);
  if (w->vec) cudaFree(w->vec);
  if (w->partials) cudaFree(w->partials);
  if (w->st) cudaFree(w->st);
  if (w->hst) cudaFreeHost(w->hst);
  if (w->ev) cudaEventDestroy(w->ev);
  if (w->s) cudaStreamDestroy(w->s);
  delete w;
}

namespace {

enum { XW = 0, BW, R, RT, P, V, F, S, Z, T };

int get_ws(ainv_csr *a, KrylovWs **out) {
  if (a->ws) {
    *out = a->ws;
    return AINV_SUCCESS;
  }
  KrylovWs *w = new (std::nothrow) KrylovWs;
  if (!w) {
    set_error("krylov workspace: host allocation failed");
    return AINV_ERR_ALLOC;
  }
  w->n = a->n;
  w->G = (a->n + kBlock - 1) / kBlock;
  cudaError_t e = cudaMalloc(&w->vec, sizeof(double) * 10 * (size_t)a->n);
  if (e == cudaSuccess) e = cudaMalloc(&w->partials, sizeof(double) * 4 * (size_t)w->G);
  if (e == cudaSuccess) e = cudaMalloc(&w->st, sizeof(KState));
  if (e == cudaSuccess) e = cudaMallocHost(&w->hst, sizeof(KState));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&w->s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w->ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMemset(w->vec, 0, sizeof(double) * 10 * (size_t)a->n);
  if (e != cudaSuccess) {
    destroy_ws(w);
    set_error("krylov workspace allocation failed: %s", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? AINV_ERR_ALLOC : AINV_ERR_CUDA;
  }
  a->ws = w;
  *out = w;
  return AINV_SUCCESS;
}

void precond_sweep2_cg(const ainv_handle *h, const double *r, double *z, KState *st,
                       double *partials, cudaStream_t s) {
  switch (h->prec) {
    case AINV_PREC_FP64: launch_cg_sweep2<double, double>(h->z, h->t, r, z, st, partials, s); break;
    case AINV_PREC_FP32: launch_cg_sweep2<float, float>(h->z, h->t, r, z, st, partials, s); break;
    default: launch_cg_sweep2<__nv_bfloat16, float>(h->z, h->t, r, z, st, partials, s); break;
  }
}

// One iteration, enqueued on ws->s.
int enqueue_iteration(KrylovWs *w, const ainv_handle *h, const ainv_csr *a, int method) {
  const int n = w->n, G = w->G;
  const DevSell &A = a->a;
  const int gA = grid_for(A.nslices);
  KState *st = w->st;
  double *pp = w->partials;
  cudaStream_t s = w->s;
  const int *stop = &st->done;
  if (method == AINV_KRYLOV_CG) {
    double *r = w->v(R), *z = w->v(Z), *p = w->v(P), *q = w->v(V), *x = w->v(XW);
    if (h) {
      AINV_TRY(launch_sweep_dscale(h->wt, h->d, r, h->t, s, stop));
      precond_sweep2_cg(h, r, z, st, pp, s);
    } else {
      k_cg_ident<<<G, kBlock, 0, s>>>(n, r, z, st, pp);
    }
    k_cg_p<<<G, kBlock, 0, s>>>(n, z, p, st);
    k_spmv_dots<kCgSigma><<<gA, kBlock, 0, s>>>(n, A.nslices, A.sptr, A.col,
                                                (const double *)A.val, p, q, nullptr,
                                                nullptr, st, pp);
    k_cg_xr<<<G, kBlock, 0, s>>>(n, p, q, x, r, st, pp);
    k_spmv_dots<kReplace><<<gA, kBlock, 0, s>>>(n, A.nslices, A.sptr, A.col,
                                                (const double *)A.val, x, r, w->v(BW),
                                                nullptr, st, pp);
  } else {
    double *r = w->v(R), *rt = w->v(RT), *p = w->v(P), *v = w->v(V), *f = w->v(F),
           *sv = w->v(S), *z = w->v(Z), *t = w->v(T), *x = w->v(XW);
    k_bicg_p<<<G, kBlock, 0, s>>>(n, r, v, p, st);
    if (h) {
      AINV_TRY(ainv_apply_async(h, 'N', 1.0, p, 0.0, f, s, stop));
    } else {
      AINV_CUDA_TRY(cudaMemcpyAsync(f, p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    }
    k_spmv_dots<kBicgSigma><<<gA, kBlock, 0, s>>>(n, A.nslices, A.sptr, A.col,
                                                  (const double *)A.val, f, v, rt, nullptr,
                                                  st, pp);
    k_bicg_s<<<G, kBlock, 0, s>>>(n, r, v, sv, st);
    if (h) {
      AINV_TRY(ainv_apply_async(h, 'N', 1.0, sv, 0.0, z, s, stop));
    } else {
      AINV_CUDA_TRY(cudaMemcpyAsync(z, sv, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    }
    k_spmv_dots<kBicgOmega><<<gA, kBlock, 0, s>>>(n, A.nslices, A.sptr, A.col,
                                                  (const double *)A.val, z, t, sv, nullptr,
                                                  st, pp);
    k_bicg_xr<<<G, kBlock, 0, s>>>(n, f, z, sv, t, rt, x, r, st, pp);
    k_spmv_dots<kReplace><<<gA, kBlock, 0, s>>>(n, A.nslices, A.sptr, A.col,
                                                (const double *)A.val, x, r, w->v(BW), rt,
                                                st, pp);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("krylov launch failed: %s", cudaGetErrorString(e));
    return AINV_ERR_CUDA;
  }
  return AINV_SUCCESS;
}

int ensure_graph(KrylovWs *w, const ainv_handle *h, const ainv_csr *a, int method,
                 int replace) {
  const unsigned long long key = h ? h->serial : 0ull;
  if (w->exec && w->key_serial == key && w->key_method == method &&
      w->key_replace == replace)
    return AINV_SUCCESS;
  if (w->exec) {
    cudaGraphExecDestroy(w->exec);
    w->exec = nullptr;
  }
  AINV_CUDA_TRY(cudaStreamBeginCapture(w->s, cudaStreamCaptureModeThreadLocal));
  int rc = AINV_SUCCESS;
  for (int k = 0; k < kChunk && rc == AINV_SUCCESS; k++) rc = enqueue_iteration(w, h, a, method);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(w->s, &g);
  if (rc != AINV_SUCCESS) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) {
    set_error("graph capture failed: %s", cudaGetErrorString(e));
    return AINV_ERR_CUDA;
  }
  e = cudaGraphInstantiate(&w->exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    w->exec = nullptr;
    set_error("graph instantiate failed: %s", cudaGetErrorString(e));
    return AINV_ERR_CUDA;
  }
  w->key_serial = key;
  w->key_method = method;
  w->key_replace = replace;
  return AINV_SUCCESS;
}

}  // namespace

int krylov_solve(const ainv_handle *h, ainv_csr *a, const double *b, double *x, int method,
                 double eps, int itmax, int replace_every, int *iter, double *err,
                 cudaStream_t user) {
  KrylovWs *w = nullptr;
  AINV_TRY(get_ws(a, &w));
  const int n = w->n;
  const size_t bytes = sizeof(double) * (size_t)n;
  // order after the caller's stream
  AINV_CUDA_TRY(cudaEventRecord(w->ev, user));
  AINV_CUDA_TRY(cudaStreamWaitEvent(w->s, w->ev, 0));
  AINV_CUDA_TRY(cudaMemcpyAsync(w->v(XW), x, bytes, cudaMemcpyDeviceToDevice, w->s));
  AINV_CUDA_TRY(cudaMemcpyAsync(w->v(BW), b, bytes, cudaMemcpyDeviceToDevice, w->s));
  KState init{};
  init.eps = eps;
  init.itmax = itmax;
  init.replace_every = replace_every;
  init.method = method;
  *w->hst = init;
  AINV_CUDA_TRY(cudaMemcpyAsync(w->st, w->hst, sizeof(KState), cudaMemcpyHostToDevice, w->s));
  const DevSell &A = a->a;
  k_bnorm<<<w->G, kBlock, 0, w->s>>>(n, w->v(BW), w->st, w->partials);
  k_spmv_dots<kInit><<<grid_for(A.nslices), kBlock, 0, w->s>>>(
      n, A.nslices, A.sptr, A.col, (const double *)A.val, w->v(XW), w->v(R), w->v(BW),
      method == AINV_KRYLOV_BICGSTAB ? w->v(RT) : nullptr, w->st, w->partials);
  AINV_CUDA_TRY(cudaGetLastError());

  const bool use_graph = getenv("AINV_NO_GRAPH") == nullptr;
  if (use_graph) AINV_TRY(ensure_graph(w, h, a, method, replace_every));
  const long max_chunks = (long)itmax / kChunk + 2;
  for (long c = 0; c < max_chunks; c++) {
    AINV_CUDA_TRY(cudaMemcpyAsync(w->hst, w->st, sizeof(KState), cudaMemcpyDeviceToHost, w->s));
    AINV_CUDA_TRY(cudaStreamSynchronize(w->s));
    if (w->hst->done) break;
    if (use_graph) {
      AINV_CUDA_TRY(cudaGraphLaunch(w->exec, w->s));
    } else {
      for (int k = 0; k < kChunk; k++) AINV_TRY(enqueue_iteration(w, h, a, method));
    }
  }
  AINV_CUDA_TRY(cudaMemcpyAsync(x, w->v(XW), bytes, cudaMemcpyDeviceToDevice, w->s));
  AINV_CUDA_TRY(cudaMemcpyAsync(w->hst, w->st, sizeof(KState), cudaMemcpyDeviceToHost, w->s));
  AINV_CUDA_TRY(cudaStreamSynchronize(w->s));
  AINV_CUDA_TRY(cudaEventRecord(w->ev, w->s));
  AINV_CUDA_TRY(cudaStreamWaitEvent(user, w->ev, 0));
  const KState &f = *w->hst;
  if (iter) *iter = f.iter;
  if (err) *err = sqrt(f.rn2) / f.bn2;
  if (!f.done) {
    set_error("krylov loop did not terminate");
    return AINV_ERR_INTERNAL;
  }
  if (f.status != AINV_SUCCESS) {
    switch (f.status) {
      case AINV_ERR_NOCONV: set_error("itmax (%d) reached, err %.3e", itmax, sqrt(f.rn2) / f.bn2); break;
      case AINV_ERR_BREAKDOWN: set_error("Krylov breakdown at iteration %d", f.iter); break;
      default: set_error("non-finite residual at iteration %d", f.iter); break;
    }
  }
  return f.status;
}

}  // namespace ainv

extern "C" int ainv_gpu_solve(ainv_handle *h, const ainv_csr *a, const double *b_dev,
                              double *x_dev, int method, double eps, int itmax, int *iter,
                              double *err, void *stream) {
  if (!a || !b_dev || !x_dev) {
    ainv::set_error("ainv_gpu_solve: null argument");
    return AINV_ERR_ARG;
  }
  if (method != AINV_KRYLOV_CG && method != AINV_KRYLOV_BICGSTAB) {
    ainv::set_error("ainv_gpu_solve: unknown method %d", method);
    return AINV_ERR_ARG;
  }
  if (h && h->n != a->n) {
    ainv::set_error("ainv_gpu_solve: preconditioner size %d != operator size %d", h->n, a->n);
    return AINV_ERR_ARG;
  }
  if (!(eps > 0.0) || itmax < 0) {
    ainv::set_error("ainv_gpu_solve: invalid eps/itmax");
    return AINV_ERR_ARG;
  }
  // Mixed-precision factors: true-residual replacement every 50 iterations.
  const int replace = (h && h->prec != AINV_PREC_FP64) ? 50 : 0;
  return ainv::krylov_solve(h, const_cast<ainv_csr *>(a), b_dev, x_dev, method, eps, itmax,
                            replace, iter, err, (cudaStream_t)stream);
}
