// The host-array apply (mld_d_base_ainv_solver_apply, the array form:
// src/impl/mld_d_base_ainv_solver_apply.f90:35-152) as copy-engine transfers
// of x plus ONE persistent kernel.
//
// PCIe is full duplex, so the floor of an apply on host arrays is about one
// transfer of the larger vector.  Splitting the sweeps into per-chunk
// kernels that wait on copy events does not get near it: on B200 a
// cross-stream event wait takes 20-170 us to resolve while copies run, and
// the sweeps fall behind the copies.  So nothing here waits on an event:
//
//  * stream si copies x (and y when beta != 0) chunk by chunk into device
//    staging; after each chunk a stream memory write (cuStreamWriteValue32,
//    else a 4-byte copy) puts the call's epoch into that chunk's flag, so the
//    flag turns over exactly when the chunk (and every chunk before it) is in;
//  * one kernel on stream sc walks a list of work items, taken in order
//    from an atomic counter: sweep 1 over a slice range of W^T (or Z^T) once
//    the flag of the last chunk it reads shows the epoch, and sweep 2 over a
//    slice range of Z (or W) once every chunk of t it reads is complete
//    (per-chunk counters of finished sweep-1 items);
//  * sweep 2 writes y straight into the caller's page-locked array (device-
//    mapped), so y leaves over PCIe while x is still coming in.
//
// An item waits only on the copy engine or on items with smaller indices,
// which blocks already running took before it, so the kernel cannot
// deadlock whatever the number of resident blocks.  Every wait is bounded
// (2 s); a timeout sets an abort word that ends all other waits and a
// status word the host reads.  The arithmetic per row is that of the
// whole-vector sweeps (same slot order and epilogues).
#include <cuda.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <new>
#include <vector>

#include "stream.cuh"

namespace ainv {

// Device state of the pipeline, owned by a handle (see ainv_handle::pipe).
struct HostPipe {
  int cap = 0;                 // chunks the buffers below hold
  int *ctr = nullptr;          // [0] next item, [1] abort, [2..2+cap) finished sweep-1 items
  unsigned *flags = nullptr;   // cap chunk flags (the epoch of the last copy in)
  unsigned *epoch_h = nullptr; // page-locked source word of the flag copies
  int *status_h = nullptr;     // page-locked, device-mapped: 1 after a timeout
  int *status_d = nullptr;     // its device address
  unsigned epoch = 0;
  struct Items {
    int cs = -1;               // plan the items were made for
    int nitems = 0, C = 0;
    int4 *items = nullptr;     // (kind | chunk << 1, s0, s1, dep)
    int *pieces1 = nullptr;    // sweep-1 items per chunk
  } it[2];
};

namespace {

using namespace dev;

constexpr int kPieceSlices = 128;  // slices per work item (4096 rows)

__device__ __forceinline__ bool wait_until(const volatile unsigned *w, unsigned want, bool ge,
                                           volatile int *abort, int *status_h) {
  const unsigned long long t0 = global_ns();
  for (;;) {
    const unsigned v = *w;
    if (ge ? (int)v >= (int)want : v == want) return true;
    if (*abort) return false;
    if (global_ns() - t0 > kWaitNs) {
      *abort = 1;
      *(volatile int *)status_h = 1;
      return false;
    }
    __nanosleep(256);
  }
}

template <class V, class T>
struct PipeArgs {
  SellView<V> m1, m2;
  const V *d;
  const double *xs;  // device copy of x
  T *t;
  const double *ys;  // device copy of y (beta != 0)
  double *y;         // the caller's page-locked y, device-mapped
  double alpha, beta;
  const int4 *items;
  int nitems;
  const int *pieces1;
  const unsigned *flags;
  unsigned epoch;
  int *ctr;
  int *status_h;
};

template <class V, class T, int P>
__global__ void __launch_bounds__(kBlock) k_host_pipe(PipeArgs<V, T> a) {
  constexpr int S = 2;
  __shared__ int s_item, s_ok;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  volatile int *abort = a.ctr + 1;
  int *done1 = a.ctr + 2;
  for (;;) {
    if (threadIdx.x == 0) {
      const int it = atomicAdd(a.ctr, 1);
      int ok = 1;
      if (it < a.nitems) {
        const int4 w = a.items[it];
        const int chunk = w.x >> 1;
        if ((w.x & 1) == 0) {
          if (w.w >= 0) ok = wait_until(a.flags + w.w, a.epoch, false, abort, a.status_h);
        } else {
          for (int c = 0; ok && c <= w.w; c++)
            ok = wait_until((const volatile unsigned *)(done1 + c), (unsigned)a.pieces1[c], true,
                            abort, a.status_h);
          if (ok && a.beta != 0.0)
            ok = wait_until(a.flags + chunk, a.epoch, false, abort, a.status_h);
        }
        __threadfence();
      }
      s_item = it;
      s_ok = ok;
    }
    __syncthreads();
    const int it = s_item;
    if (it >= a.nitems) return;
    const int4 w = a.items[it];
    if (s_ok) {
      const int g0 = w.y / S, g1 = (w.z + S - 1) / S;
      if ((w.x & 1) == 0) {
        for (int g = g0 + warp; g < g1; g += kSlicesPerBlock) {
          GroupCtx<S> c;
          group_ctx(a.m1, g, c);
          typename Acc<V>::type acc[S];
          group_dot<P, 4, false>(a.m1, c, g, a.xs, acc);
#pragma unroll
          for (int q = 0; q < S; q++) {
            const int row = (g * S + q) * kSlice + lane;
            if (row < a.m1.n) a.t[row] = (T)(ldd(a.d + row) * acc[q]);
          }
        }
      } else {
        for (int g = g0 + warp; g < g1; g += kSlicesPerBlock) {
          GroupCtx<S> c;
          group_ctx(a.m2, g, c);
          typename Acc<V>::type acc[S];
          group_dot<P, 4, false>(a.m2, c, g, a.t, acc);
#pragma unroll
          for (int q = 0; q < S; q++) {
            const int row = (g * S + q) * kSlice + lane;
            if (row < a.m2.n)
              a.y[row] = axpby_row(a.alpha, (double)acc[q], a.beta,
                                   a.beta == 0.0 ? 0.0 : __ldcg(a.ys + row));
          }
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && (w.x & 1) == 0) {
      __threadfence();
      atomicAdd(done1 + (w.x >> 1), 1);
    }
  }
}

// Work items in the order of the chunk plan: the sweep-1 pieces of chunk i,
// then the sweep-2 pieces of every unit whose t is complete with chunk i.
void build_items(const HostPlan &p, std::vector<int4> &items, std::vector<int> &pieces1) {
  const int C = (int)p.bound.size() - 1, U = (int)p.u0.size();
  items.clear();
  pieces1.assign((size_t)C, 0);
  auto pieces = [&](int kind, int chunk, int a, int b, int dep) {
    int n = 0;
    for (int s = a; s < b; s += kPieceSlices, n++)
      items.push_back(make_int4(kind | (chunk << 1), s, std::min(b, s + kPieceSlices), dep));
    return n;
  };
  for (int i = 0, u = 0; i < C; i++) {
    pieces1[(size_t)i] = pieces(0, i, p.bound[(size_t)i], p.bound[(size_t)i + 1], p.need1[(size_t)i]);
    for (; u < U && p.need2[(size_t)u] <= i; u++) {
      const int a = p.u0[(size_t)u];
      const int chunk = (int)(std::upper_bound(p.bound.begin(), p.bound.end(), a) - p.bound.begin()) - 1;
      pieces(1, chunk, a, p.u1[(size_t)u], p.need2[(size_t)u]);
    }
  }
}

template <class V, class T>
struct PipeLaunch {
  PipeArgs<V, T> a;
  int grid;
  cudaStream_t s;
  template <int S, int P>
  void run() const {
    k_host_pipe<V, T, P><<<grid, kBlock, 0, s>>>(a);
  }
};

template <class V, class T>
void launch_pipe(const DevSell &m1, const DevSell &m2, const PipeArgs<V, T> &a, int grid,
                 cudaStream_t s) {
  with_pack<V, 1>(m1.pack, PipeLaunch<V, T>{a, grid, s});
}

template <class V_, class T_>
struct Types {
  using V = V_;
  using T = T_;
};
// f(Types<V, T>) for the storage type V and intermediate type T of prec.
template <class F>
int by_prec_pipe(int prec, F &&f) {
  switch (prec) {
    case AINV_PREC_FP64: f(Types<double, double>()); break;
    case AINV_PREC_FP32: f(Types<float, float>()); break;
    case AINV_PREC_BF16: f(Types<__nv_bfloat16, float>()); break;
    case AINV_PREC_FP32_ACC64: f(Types<f32w, double>()); break;
    case AINV_PREC_BF16_ACC64: f(Types<b16w, double>()); break;
    default:
      set_error("unknown precision %d", prec);
      return AINV_ERR_ARG;
  }
  return AINV_SUCCESS;
}

// cuStreamWriteValue32, resolved through the runtime (no link-time libcuda
// dependency): the flag write is a stream memory operation, ordered after
// the chunk's copy, and costs the copy stream about 5 us under load against
// about 10 us for a 4-byte copy.  Null when the driver does not offer it.
using WriteValue32 = CUresult (*)(CUstream, CUdeviceptr, cuuint32_t, unsigned int);
WriteValue32 write_value32() {
  static WriteValue32 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuStreamWriteValue32", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<WriteValue32>(p);
    cudaGetLastError();
  });
  return fn;
}

}  // namespace

void destroy_host_pipe(HostPipe *hp) {
  if (!hp) return;
  if (hp->ctr) cudaFree(hp->ctr);
  if (hp->flags) cudaFree(hp->flags);
  if (hp->epoch_h) cudaFreeHost(hp->epoch_h);
  if (hp->status_h) cudaFreeHost(hp->status_h);
  for (auto &it : hp->it) {
    if (it.items) cudaFree(it.items);
    if (it.pieces1) cudaFree(it.pieces1);
  }
  delete hp;
}

bool host_pipe_usable(const ainv_handle *h, bool tr, const double *y) {
  // AINV_HOST_FUSED=0 selects the event-driven stream pipeline instead
  if (const char *e = std::getenv("AINV_HOST_FUSED"))
    if (std::atoi(e) == 0) return false;
  const DevSell &m1 = tr ? h->zt : h->wt, &m2 = tr ? h->w : h->z;
  if (m1.pack != m2.pack) return false;
  void *yd = nullptr;
  if (cudaHostGetDevicePointer(&yd, (void *)y, 0) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  // the kernel stores into y, so y must not be registered read-only (a
  // contract of every form, which all write y from the device); where the
  // runtime reports the flags, such a y is sent to the other forms
  unsigned flags = 0;
  if (cudaHostGetFlags(&flags, (void *)y) == cudaSuccess) {
    if (flags & cudaHostRegisterReadOnly) return false;
  } else {
    cudaGetLastError();
  }
  return true;
}

int host_pipe_apply(ainv_handle *h, bool tr, const HostPlan &p, double alpha, const double *x,
                    double beta, double *y, cudaStream_t si, cudaStream_t sc) {
  const DevSell &m1 = tr ? h->zt : h->wt, &m2 = tr ? h->w : h->z;
  const int C = (int)p.bound.size() - 1;
  if (!h->pipe) {
    h->pipe = new (std::nothrow) HostPipe;
    if (!h->pipe) {
      set_error("host apply: host allocation failed");
      return AINV_ERR_ALLOC;
    }
    AINV_CUDA_TRY(cudaHostAlloc((void **)&h->pipe->epoch_h, 64, cudaHostAllocDefault));
    AINV_CUDA_TRY(cudaHostAlloc((void **)&h->pipe->status_h, 64, cudaHostAllocMapped));
    AINV_CUDA_TRY(cudaHostGetDevicePointer((void **)&h->pipe->status_d, h->pipe->status_h, 0));
  }
  HostPipe &hp = *h->pipe;
  if (hp.cap < C) {
    if (hp.ctr) cudaFree(hp.ctr);
    if (hp.flags) cudaFree(hp.flags);
    hp.ctr = nullptr;
    hp.flags = nullptr;
    hp.cap = 0;
    AINV_CUDA_TRY(cudaMalloc(&hp.ctr, sizeof(int) * (size_t)(C + 2)));
    AINV_CUDA_TRY(cudaMalloc(&hp.flags, sizeof(unsigned) * (size_t)C));
    AINV_CUDA_TRY(cudaMemset(hp.flags, 0, sizeof(unsigned) * (size_t)C));
    hp.cap = C;
    hp.epoch = 0;
  }
  HostPipe::Items &it = hp.it[tr];
  if (it.cs != p.cs || it.C != C) {
    std::vector<int4> items;
    std::vector<int> pieces1;
    build_items(p, items, pieces1);
    if (it.items) cudaFree(it.items);
    if (it.pieces1) cudaFree(it.pieces1);
    it = HostPipe::Items{};
    AINV_CUDA_TRY(cudaMalloc(&it.items, sizeof(int4) * items.size()));
    AINV_CUDA_TRY(cudaMalloc(&it.pieces1, sizeof(int) * pieces1.size()));
    AINV_CUDA_TRY(cudaMemcpy(it.items, items.data(), sizeof(int4) * items.size(),
                             cudaMemcpyHostToDevice));
    AINV_CUDA_TRY(cudaMemcpy(it.pieces1, pieces1.data(), sizeof(int) * pieces1.size(),
                             cudaMemcpyHostToDevice));
    it.nitems = (int)items.size();
    it.C = C;
    it.cs = p.cs;
  }
  double *yd = nullptr;
  AINV_CUDA_TRY(cudaHostGetDevicePointer((void **)&yd, y, 0));
  // a new epoch per call (never 0, the flags' initial value)
  if (++hp.epoch == 0) hp.epoch = 1;
  *hp.epoch_h = hp.epoch;
  *(volatile int *)hp.status_h = 0;
  const size_t n = (size_t)h->n;
  // The copies are enqueued before the kernel: a tool that runs each kernel
  // to completion before the host goes on (a profiler) then still finds
  // every chunk on its way instead of a kernel waiting for copies that are
  // not enqueued yet.
  AINV_CUDA_TRY(cudaMemsetAsync(hp.ctr, 0, sizeof(int) * (size_t)(C + 2), sc));
  // si: the chunks of x (and y), each followed by its flag
  for (int c = 0; c < C; c++) {
    const size_t r0 = (size_t)p.bound[(size_t)c] * kSlice;
    const size_t nb = sizeof(double) * (std::min(n, (size_t)p.bound[(size_t)c + 1] * kSlice) - r0);
    AINV_CUDA_TRY(cudaMemcpyAsync(h->xs + r0, x + r0, nb, cudaMemcpyHostToDevice, si));
    if (beta != 0.0)
      AINV_CUDA_TRY(cudaMemcpyAsync(h->ys + r0, y + r0, nb, cudaMemcpyHostToDevice, si));
    if (WriteValue32 wv = write_value32()) {
      if (wv((CUstream)si, (CUdeviceptr)(uintptr_t)(hp.flags + c), hp.epoch, 0) != CUDA_SUCCESS) {
        set_error("host apply: flag write failed");
        return AINV_ERR_CUDA;
      }
    } else {
      AINV_CUDA_TRY(cudaMemcpyAsync(hp.flags + c, hp.epoch_h, sizeof(unsigned),
                                    cudaMemcpyHostToDevice, si));
    }
  }
  // sc: the kernel, after the counters are reset
  int dev = 0, sms = 0;
  AINV_CUDA_TRY(cudaGetDevice(&dev));
  AINV_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int grid = std::max(1, std::min(it.nitems, 2 * sms));
  int rc = by_prec_pipe(h->prec, [&](auto ty) {
    using V = typename decltype(ty)::V;
    using T = typename decltype(ty)::T;
    PipeArgs<V, T> a{view<V>(m1), view<V>(m2), (const V *)h->d, h->xs, (T *)h->t, h->ys, yd,
                     alpha, beta, it.items, it.nitems, it.pieces1, hp.flags, hp.epoch, hp.ctr,
                     hp.status_d};
    launch_pipe(m1, m2, a, grid, sc);
  });
  if (rc != AINV_SUCCESS) return rc;
  AINV_CUDA_TRY(cudaGetLastError());
  return AINV_SUCCESS;
}

int host_pipe_status(const ainv_handle *h) {
  if (h->pipe && *(volatile int *)h->pipe->status_h) {
    set_error("host apply: a wait of the pipeline kernel timed out");
    return AINV_ERR_TIMEOUT;
  }
  return AINV_SUCCESS;
}

}  // namespace ainv
