// Device helpers shared by the SELL-32 kernels (apply sweeps, A SpMV and
// the fused Krylov kernels).
#pragma once

#include <cuda_bf16.h>

#include "internal.h"

namespace ainv {
namespace dev {

constexpr int kBlock = 256;  // 8 slices (warps) per block
constexpr int kSlicesPerBlock = kBlock / kSlice;
constexpr int kWarps = kBlock / 32;
constexpr int kUnroll = 4;

template <class V>
struct Acc { using type = float; };
template <>
struct Acc<double> { using type = double; };

// Streaming loads (read once, evict first) for factor values / indices.
__device__ __forceinline__ double ldv(const double *p) { return __ldcs(p); }
__device__ __forceinline__ float ldv(const float *p) { return __ldcs(p); }
__device__ __forceinline__ float ldv(const __nv_bfloat16 *p) {
  unsigned short u = __ldcs(reinterpret_cast<const unsigned short *>(p));
  return __uint_as_float(((unsigned)u) << 16);
}
// Cached loads for per-row vectors (D^-1).
__device__ __forceinline__ double ldd(const double *p) { return __ldg(p); }
__device__ __forceinline__ float ldd(const float *p) { return __ldg(p); }
__device__ __forceinline__ float ldd(const __nv_bfloat16 *p) {
  unsigned short u = __ldg(reinterpret_cast<const unsigned short *>(p));
  return __uint_as_float(((unsigned)u) << 16);
}

// Sequential (slot-ordered) dot of one SELL row with a gathered vector.
// Indices and values for kUnroll slots are issued before the dependent
// gathers so each lane keeps several independent requests in flight.
template <class V, class X>
__device__ __forceinline__ typename Acc<V>::type row_dot(const int *__restrict__ col,
                                                         const V *__restrict__ val,
                                                         const X *__restrict__ x, int w) {
  using A = typename Acc<V>::type;
  A acc = A(0);
  int k = 0;
  for (; k + kUnroll <= w; k += kUnroll) {
    int c[kUnroll];
    A v[kUnroll], xv[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; u++) {
      c[u] = __ldcs(col + (k + u) * kSlice);
      v[u] = (A)ldv(val + (k + u) * kSlice);
    }
#pragma unroll
    for (int u = 0; u < kUnroll; u++) xv[u] = (A)__ldg(x + c[u]);
#pragma unroll
    for (int u = 0; u < kUnroll; u++) acc = fma(v[u], xv[u], acc);
  }
  for (; k < w; k++) {
    const int c = __ldcs(col + k * kSlice);
    acc = fma((A)ldv(val + k * kSlice), (A)__ldg(x + c), acc);
  }
  return acc;
}

// Slice geometry for the calling thread: returns false when the warp has no
// slice.  row may be >= n for the tail lanes of the last slice.
struct SliceCtx {
  int beg, w, row, lane;
};
__device__ __forceinline__ bool slice_ctx(int nslices, const int *__restrict__ sptr,
                                          SliceCtx &c) {
  const int s = blockIdx.x * kSlicesPerBlock + (threadIdx.x >> 5);
  if (s >= nslices) return false;
  c.lane = threadIdx.x & (kSlice - 1);
  c.beg = __ldg(sptr + s);
  c.w = (__ldg(sptr + s + 1) - c.beg) / kSlice;
  c.row = s * kSlice + c.lane;
  return true;
}

inline int grid_for(int nslices) { return (nslices + kSlicesPerBlock - 1) / kSlicesPerBlock; }

// ---- deterministic block reduction --------------------------------------
// Fixed shuffle tree inside each warp, then warp 0 folds the kWarps
// partials in index order.  The result is valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double sh[NV][kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; i++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) sh[i][warp] = v[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double s = 0.0;
      for (int w = 0; w < kWarps; w++) s += sh[i][w];
      v[i] = s;
    }
  }
  __syncthreads();
}

// Grid-wide deterministic sum: every block stores its partials, the last
// block to arrive (ticket) folds all partials in block order.  Returns true
// in the last block, where thread 0 holds the totals in v.  The ticket is
// reset by the last block so the slot can be reused by the next launch.
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double *__restrict__ partials,
                                         unsigned *__restrict__ ticket) {
  __shared__ bool is_last;
  block_sum<NV>(v);
  const int G = gridDim.x;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) partials[i * G + blockIdx.x] = v[i];
    __threadfence();
    const unsigned t = atomicAdd(ticket, 1u);
    is_last = (t == (unsigned)G - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
#pragma unroll
  for (int i = 0; i < NV; i++) {
    double s = 0.0;
    for (int b = threadIdx.x; b < G; b += kBlock) s += __ldcg(partials + i * G + b);
    v[i] = s;
  }
  block_sum<NV>(v);
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

}  // namespace dev
}  // namespace ainv
