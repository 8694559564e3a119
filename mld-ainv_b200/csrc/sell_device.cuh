// Device helpers shared by the sliced-layout kernels (apply sweeps, A SpMV
// and the fused Krylov kernels).
#pragma once

#include <cuda_bf16.h>

#include <type_traits>
#include <utility>

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

// c + a*b of the row accumulations.  In FP64 the product and the sum each
// round once, with no fused multiply-add: the arithmetic of the reference's
// CSR product compiled for a target without FMA, so an FP64 row sum here
// equals the oracle's bit for bit (same operations, same column order).
// FP32 accumulation keeps the fused form.
__device__ __forceinline__ double madd(double a, double b, double c) {
  return __dadd_rn(c, __dmul_rn(a, b));
}
__device__ __forceinline__ float madd(float a, float b, float c) { return fmaf(a, b, c); }

// Sweep-2 epilogue of a row: y = alpha*acc + beta*y as the reference's CSR
// product forms it (src/impl/mld_d_base_ainv_solver_apply_vect.f90:117-119
// through psb_spmm), each product and the sum rounded once; y is not read
// when beta is zero.
__device__ __forceinline__ double axpby_row(double alpha, double acc, double beta, double y) {
  const double r = __dmul_rn(alpha, acc);
  return (beta == 0.0) ? r : __dadd_rn(r, __dmul_rn(beta, y));
}

// Storage types of the FP64-accumulating modes (AINV_PREC_FP32_ACC64,
// AINV_PREC_BF16_ACC64): FP32 / BF16 values whose loads yield FP64, so the
// products, sums and the intermediate are those of the FP64 apply.
struct f32w {
  float v;
  f32w() = default;
  __host__ __device__ explicit f32w(double x) : v((float)x) {}
};
struct b16w {
  unsigned short v;
  b16w() = default;
  __host__ __device__ explicit b16w(double x)
      : v(__bfloat16_as_ushort(__double2bfloat16(x))) {}
};
template <>
struct Acc<f32w> { using type = double; };
template <>
struct Acc<b16w> { using type = double; };
__device__ __forceinline__ double ldv(const f32w *p) { return (double)__ldcs(&p->v); }
__device__ __forceinline__ double ldv(const b16w *p) {
  return (double)__uint_as_float(((unsigned)__ldcs(&p->v)) << 16);
}
__device__ __forceinline__ double ldd(const f32w *p) { return (double)__ldg(&p->v); }
__device__ __forceinline__ double ldd(const b16w *p) {
  return (double)__uint_as_float(((unsigned)__ldg(&p->v)) << 16);
}
template <class V>
constexpr bool is_acc64() { return std::is_same<V, f32w>::value || std::is_same<V, b16w>::value; }

// Kernel-side view of a DevSell with typed values.
template <class V>
struct SellView {
  int n, nslices;
  const int *__restrict__ sptr;
  const int *__restrict__ iptr;
  const int *__restrict__ idx;
  const V *__restrict__ val;
};
template <class V>
inline SellView<V> view(const DevSell &m) {
  return SellView<V>{m.n, m.nslices, m.sptr, m.iptr, m.idx, (const V *)m.val};
}

// ---- packed loads: P adjacent slots of one lane in one vector load --------
// EF (evict first): values read once per pass stream through with the
// evict-first hint; EF = false keeps them cached, for kernels in which
// several right-hand sides read the same slice back to back.
template <bool EF, class T>
__device__ __forceinline__ T ldp(const T *p) {
  if constexpr (EF) return __ldcs(p);
  else return __ldg(p);
}
__device__ __forceinline__ float bf16lo(unsigned w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16hi(unsigned w) { return __uint_as_float(w & 0xffff0000u); }

template <class V, int P>
struct Pack;
template <>
struct Pack<double, 1> {
  template <bool EF = true>
  static __device__ __forceinline__ void load(const double *p, double (&o)[1]) { o[0] = ldp<EF>(p); }
};
template <>
struct Pack<double, 2> {
  template <bool EF = true>
  static __device__ __forceinline__ void load(const double *p, double (&o)[2]) {
    const double2 v = ldp<EF>(reinterpret_cast<const double2 *>(p));
    o[0] = v.x;
    o[1] = v.y;
  }
};
template <>
struct Pack<float, 1> {
  template <bool EF = true>
  static __device__ __forceinline__ void load(const float *p, float (&o)[1]) { o[0] = ldp<EF>(p); }
};
template <>
struct Pack<float, 2> {
  template <bool EF = true>
  static __device__ __forceinline__ void load(const float *p, float (&o)[2]) {
    const float2 v = ldp<EF>(reinterpret_cast<const float2 *>(p));
    o[0] = v.x;
    o[1] = v.y;
  }
};
template <>
struct Pack<float, 4> {
  template <bool EF = true>
  static __device__ __forceinline__ void load(const float *p, float (&o)[4]) {
    const float4 v = ldp<EF>(reinterpret_cast<const float4 *>(p));
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
  }
};
template <>
struct Pack<__nv_bfloat16, 1> {
  template <bool EF = true>
  static __device__ __forceinline__ void load(const __nv_bfloat16 *p, float (&o)[1]) {
    o[0] = bf16lo(ldp<EF>(reinterpret_cast<const unsigned short *>(p)));
  }
};
template <>
struct Pack<__nv_bfloat16, 2> {
  template <bool EF = true>
  static __device__ __forceinline__ void load(const __nv_bfloat16 *p, float (&o)[2]) {
    const unsigned v = ldp<EF>(reinterpret_cast<const unsigned *>(p));
    o[0] = bf16lo(v);
    o[1] = bf16hi(v);
  }
};
template <>
struct Pack<__nv_bfloat16, 4> {
  template <bool EF = true>
  static __device__ __forceinline__ void load(const __nv_bfloat16 *p, float (&o)[4]) {
    const uint2 v = ldp<EF>(reinterpret_cast<const uint2 *>(p));
    o[0] = bf16lo(v.x);
    o[1] = bf16hi(v.x);
    o[2] = bf16lo(v.y);
    o[3] = bf16hi(v.y);
  }
};
template <>
struct Pack<__nv_bfloat16, 8> {
  template <bool EF = true>
  static __device__ __forceinline__ void load(const __nv_bfloat16 *p, float (&o)[8]) {
    const uint4 v = ldp<EF>(reinterpret_cast<const uint4 *>(p));
    o[0] = bf16lo(v.x);
    o[1] = bf16hi(v.x);
    o[2] = bf16lo(v.y);
    o[3] = bf16hi(v.y);
    o[4] = bf16lo(v.z);
    o[5] = bf16hi(v.z);
    o[6] = bf16lo(v.w);
    o[7] = bf16hi(v.w);
  }
};

template <int P>
struct Pack<f32w, P> {
  template <bool EF = true>
  static __device__ __forceinline__ void load(const f32w *p, double (&o)[P]) {
    float f[P];
    Pack<float, P>::template load<EF>(reinterpret_cast<const float *>(p), f);
#pragma unroll
    for (int e = 0; e < P; e++) o[e] = (double)f[e];
  }
};
template <int P>
struct Pack<b16w, P> {
  template <bool EF = true>
  static __device__ __forceinline__ void load(const b16w *p, double (&o)[P]) {
    float f[P];
    Pack<__nv_bfloat16, P>::template load<EF>(reinterpret_cast<const __nv_bfloat16 *>(p), f);
#pragma unroll
    for (int e = 0; e < P; e++) o[e] = (double)f[e];
  }
};

// P adjacent int32 words: streaming (per-slot columns) or cached (offsets).
template <int P, bool STREAM>
__device__ __forceinline__ void load_ints(const int *p, int (&o)[P]) {
  if constexpr (P == 1) {
    o[0] = STREAM ? __ldcs(p) : __ldg(p);
  } else if constexpr (P == 2) {
    const int2 v = STREAM ? __ldcs(reinterpret_cast<const int2 *>(p))
                          : __ldg(reinterpret_cast<const int2 *>(p));
    o[0] = v.x;
    o[1] = v.y;
  } else {
#pragma unroll
    for (int h = 0; h < P / 4; h++) {
      const int4 v = STREAM ? __ldcs(reinterpret_cast<const int4 *>(p) + h)
                            : __ldg(reinterpret_cast<const int4 *>(p) + h);
      o[4 * h] = v.x;
      o[4 * h + 1] = v.y;
      o[4 * h + 2] = v.z;
      o[4 * h + 3] = v.w;
    }
  }
}

// Packs a value type can use (at most 16 bytes per load).
template <class V, int P>
constexpr bool pack_ok() {
  return P == 1 || (P * (int)sizeof(V) <= 16 && (P == 2 || P == 4 || P == 8));
}

// Call f.template run<S, P>() for the runtime S (1, 2, 4) and P.
template <class V, int S, class F>
inline bool with_pack(int P, const F &f) {
  switch (P) {
    case 1: f.template run<S, 1>(); return true;
    case 2: if constexpr (pack_ok<V, 2>()) { f.template run<S, 2>(); return true; } break;
    case 4: if constexpr (pack_ok<V, 4>()) { f.template run<S, 4>(); return true; } break;
    case 8: if constexpr (pack_ok<V, 8>()) { f.template run<S, 8>(); return true; } break;
  }
  return false;
}
template <class V, class F>
inline bool with_group_pack(int S, int P, const F &f) {
  switch (S) {
    case 1: return with_pack<V, 1>(P, f);
    case 4: return with_pack<V, 4>(P, f);
    default: return with_pack<V, 2>(P, f);
  }
}

// Warp-level slice loop: warp w of block b takes slices b*8+w, then every
// gridDim.x*8-th slice after it.
__device__ __forceinline__ int first_slice() {
  return blockIdx.x * kSlicesPerBlock + (threadIdx.x >> 5);
}
__device__ __forceinline__ int slice_stride() { return gridDim.x * kSlicesPerBlock; }

// ---- groups of S slices per warp ------------------------------------------
// A warp walks its slices S at a time: the S+1 slice pointers come from one
// lane-parallel load, and every value / offset load of the S slices (kUnroll
// slots each) is issued before the first dependent gather, so a warp keeps
// S*kUnroll independent 256 B requests in flight instead of waiting for
// three dependent round trips per slice.
template <int S>
struct GroupCtx {
  int vb[S], ib[S], w[S];
  bool om[S];
  int maxw;
};

template <class V, int S>
__device__ __forceinline__ void group_ctx(const SellView<V> &m, int g, GroupCtx<S> &c) {
  const int lane = threadIdx.x & 31;
  int sp = 0, ip = 0;
  if (lane <= S) {
    const int s = min(g * S + lane, m.nslices);
    sp = __ldg(m.sptr + s);
    ip = __ldg(m.iptr + s);
  }
  c.maxw = 0;
#pragma unroll
  for (int q = 0; q < S; q++) {
    const int vb = __shfl_sync(0xffffffffu, sp, q), ve = __shfl_sync(0xffffffffu, sp, q + 1);
    const int ib = __shfl_sync(0xffffffffu, ip, q), ie = __shfl_sync(0xffffffffu, ip, q + 1);
    c.vb[q] = vb;
    c.ib[q] = ib;
    c.w[q] = (ve - vb) / kSlice;
    c.om[q] = (ie - ib) == c.w[q];
    c.maxw = max(c.maxw, c.w[q]);
  }
}

// Packs per loop step: K slots (K = 4 or 8), at least one pack.
template <int P, int K = 4>
struct Step { static constexpr int kPacks = P >= K ? 1 : K / P; };

// Slots [k0, k0 + kPacks*P) of the S slices of a group, all in the same
// index encoding (OM: shared offsets; else per-slot columns).  Loads are
// predicated per pack (w is a multiple of P), so all value / index loads of
// the step are in flight before the first dependent gather; the FMAs then
// run in slot order, which is the row's column order.
template <bool OM, int P, int K, bool NC = true, bool EF = true, class V, class X, int S>
__device__ __forceinline__ void group_slots(const SellView<V> &m, const GroupCtx<S> &c,
                                            const int (&row)[S], int k0,
                                            const X *__restrict__ x,
                                            typename Acc<V>::type (&acc)[S]) {
  using A = typename Acc<V>::type;
  constexpr int J = Step<P, K>::kPacks;
  const int lane = threadIdx.x & 31;
  int col[S][J][P];
  A vv[S][J][P];
#pragma unroll
  for (int q = 0; q < S; q++) {
#pragma unroll
    for (int j = 0; j < J; j++) {
      const int k = k0 + j * P;
      const bool ok = k < c.w[q];
      const size_t pos = (size_t)(k / P) * (kSlice * P) + (size_t)lane * P;
      if (ok) {
        Pack<V, P>::template load<EF>(m.val + c.vb[q] + pos, vv[q][j]);
        if (OM) {
          load_ints<P, false>(m.idx + c.ib[q] + k, col[q][j]);
#pragma unroll
          for (int e = 0; e < P; e++) col[q][j][e] += row[q];
        } else {
          load_ints<P, EF>(m.idx + c.ib[q] + pos, col[q][j]);
        }
      } else {
#pragma unroll
        for (int e = 0; e < P; e++) {
          vv[q][j][e] = A(0);
          col[q][j][e] = 0;
        }
      }
    }
  }
  A xv[S][J][P];
#pragma unroll
  for (int q = 0; q < S; q++)
#pragma unroll
    for (int j = 0; j < J; j++)
#pragma unroll
      for (int e = 0; e < P; e++)
        xv[q][j][e] = (vv[q][j][e] != A(0) && (unsigned)col[q][j][e] < (unsigned)m.n)
                          ? (A)(NC ? __ldg(x + col[q][j][e]) : __ldcg(x + col[q][j][e]))
                          : A(0);
#pragma unroll
  for (int q = 0; q < S; q++)
#pragma unroll
    for (int j = 0; j < J; j++)
#pragma unroll
      for (int e = 0; e < P; e++) acc[q] = madd(vv[q][j][e], xv[q][j][e], acc[q]);
}

// acc[q] = row (g*S+q)*32+lane of M dotted with x.  The encoding test is
// warp-uniform and sits outside the slot loop; a group mixing both
// encodings is walked one slice at a time.
template <int P, int K = 4, bool NC = true, bool EF = true, class V, class X, int S>
__device__ __forceinline__ void group_dot(const SellView<V> &m, const GroupCtx<S> &c, int g,
                                          const X *__restrict__ x,
                                          typename Acc<V>::type (&acc)[S]) {
  using A = typename Acc<V>::type;
  constexpr int KS = Step<P, K>::kPacks * P;
  const int lane = threadIdx.x & 31;
  int row[S];
  bool all_om = true, all_col = true;
#pragma unroll
  for (int q = 0; q < S; q++) {
    acc[q] = A(0);
    row[q] = (g * S + q) * kSlice + lane;
    if (c.w[q] > 0) {
      all_om = all_om && c.om[q];
      all_col = all_col && !c.om[q];
    }
  }
  if (all_om) {
    for (int k0 = 0; k0 < c.maxw; k0 += KS) group_slots<true, P, K, NC, EF>(m, c, row, k0, x, acc);
  } else if (all_col) {
    for (int k0 = 0; k0 < c.maxw; k0 += KS) group_slots<false, P, K, NC, EF>(m, c, row, k0, x, acc);
  } else {
#pragma unroll
    for (int q = 0; q < S; q++) {
      GroupCtx<1> c1;
      c1.vb[0] = c.vb[q];
      c1.ib[0] = c.ib[q];
      c1.w[0] = c.w[q];
      c1.om[0] = c.om[q];
      c1.maxw = c.w[q];
      const int r1[1] = {row[q]};
      A a1[1] = {A(0)};
      if (c.om[q]) {
        for (int k0 = 0; k0 < c1.maxw; k0 += KS) group_slots<true, P, K, NC, EF>(m, c1, r1, k0, x, a1);
      } else {
        for (int k0 = 0; k0 < c1.maxw; k0 += KS) group_slots<false, P, K, NC, EF>(m, c1, r1, k0, x, a1);
      }
      acc[q] = a1[0];
    }
  }
}

// Visit every row of M: epi(row, acc) for rows < n, S slices per warp step,
// warps striding over the grid.  [g0, g1) restricts the walk to those groups
// of S slices (rows stay absolute).
template <int S, int P, int K = 4, class V, class X, class Epi>
__device__ __forceinline__ void for_each_row(const SellView<V> &m, const X *__restrict__ x,
                                             Epi &&epi, int g0 = 0, int g1 = 0x7fffffff) {
  const int ngroups = min((m.nslices + S - 1) / S, g1);
  const int lane = threadIdx.x & 31;
  for (int g = g0 + first_slice(); g < ngroups; g += slice_stride()) {
    GroupCtx<S> c;
    group_ctx(m, g, c);
    typename Acc<V>::type acc[S];
    group_dot<P, K>(m, c, g, x, acc);
#pragma unroll
    for (int q = 0; q < S; q++) {
      const int row = (g * S + q) * kSlice + lane;
      if (row < m.n) epi(row, acc[q]);
    }
  }
}

// ---- canonical reduction order of the Krylov dots ---------------------------
// A dot of two n-vectors is summed in one fixed order whatever the grid, the
// kernel or the device, and the oracle's ordered dot restates that order:
//   1. slice sums: the 32 products of slice s (rows 32s..32s+31, zero past
//      n) go through the warp tree below (lane l adds lane l+16, then l+8,
//      4, 2, 1; lane 0's value);
//   2. group sums: the slice sums of slices [8g, 8g+8) added in slice order
//      from zero;
//   3. range sums: groups [256j, 256j+256) folded by 256 threads (thread t
//      takes group t), then the warp tree over each warp's 32 values and the
//      8 warp sums added from zero in warp order (block_sum);
//   4. the total: the range sums folded the same way (thread t adds ranges
//      t, t+256, ... in order from zero).
// The kernels that compute the products store the slice sums (SliceSums);
// a small fold kernel does steps 2-4.
constexpr int kGroupSlices = 8;   // slices per group
constexpr int kFoldThreads = 256;
constexpr int kFoldRange = 256;   // groups per range

__device__ __forceinline__ double warp_tree(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Per-slice sums of NV dots.  Each lane sets v[k] to its row's product;
// end(s), called by the whole warp, stores the slice's warp tree at
// sp[k*ld + s] and clears v for the next slice (lanes past n keep zero).
template <int NV>
struct SliceSums {
  double *__restrict__ sp;
  int ld;
  double v[NV];
  __device__ __forceinline__ void end(int s) {
#pragma unroll
    for (int k = 0; k < NV; k++) {
      const double t = warp_tree(v[k]);
      if ((threadIdx.x & 31) == 0) sp[(size_t)k * ld + s] = t;
      v[k] = 0.0;
    }
  }
};

// Visit every slice (warps striding over groups of S slices): epi(row, acc)
// for each lane whose row is < n, then, with the whole warp, end(slice).
template <int S, int P, int K = 4, class V, class X, class Epi, class End>
__device__ __forceinline__ void for_each_row_sliced(const SellView<V> &m,
                                                    const X *__restrict__ x, Epi &&epi,
                                                    End &&end) {
  const int ngroups = (m.nslices + S - 1) / S;
  const int lane = threadIdx.x & 31;
  for (int g = first_slice(); g < ngroups; g += slice_stride()) {
    GroupCtx<S> c;
    group_ctx(m, g, c);
    typename Acc<V>::type acc[S];
    group_dot<P, K>(m, c, g, x, acc);
#pragma unroll
    for (int q = 0; q < S; q++) {
      const int s = g * S + q;
      if (s < m.nslices) {
        const int row = s * kSlice + lane;
        if (row < m.n) epi(row, acc[q]);
        end(s);
      }
    }
  }
}

// k<<<g, b, smem, s>>>(args...) through cudaLaunchKernelEx.  (Launching the
// apply and Krylov kernels with programmatic dependent launch was measured
// and dropped: the Krylov iteration did not change, and the early-scheduled
// blocks of a sweep's successor took shared memory from the persistent
// streaming sweep, so FP32 and INVK applies lost 20%.)
template <class... P, class... A>
inline void launch(void (*k)(P...), dim3 g, dim3 b, size_t smem, cudaStream_t s, A &&...a) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = g;
  cfg.blockDim = b;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchKernelEx(&cfg, k, std::forward<A>(a)...);
}

inline int grid_for(int nslices) { return (nslices + kSlicesPerBlock - 1) / kSlicesPerBlock; }

// Slices per warp step (S of group_dot) for a value type; the default can
// be overridden with AINV_SLICES_PER_WARP=1|2|4 for tuning.
int group_size(int prec);
inline int grid_for_groups(int nslices, int S) {
  return grid_for((nslices + S - 1) / S);
}

// Blocks for kernels that end in a grid-wide reduction: at most one resident
// wave (8 blocks of 256 threads per SM) so the last block folds few
// partials; never more blocks than units of 256 rows.
int reduction_grid(long long rows);
// Blocks of one full resident wave of `kernel` (256 threads, occupancy from
// its registers and shared memory), at most one per 256 rows: the grid of a
// grid-stride kernel, so no partial second wave runs alone.
int wave_grid(const void *kernel, long long rows);

// ---- deterministic block reduction --------------------------------------
// Fixed shuffle tree inside each warp, then thread 0 folds the per-warp
// partials of every warp of the block in index order.  Works for any block
// size up to 1024 threads; the result is valid in thread 0.
constexpr int kMaxWarps = 32;
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double sh[NV][kMaxWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
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
      for (int w = 0; w < nwarps; w++) s += sh[i][w];
      v[i] = s;
    }
  }
  __syncthreads();
}

// Steps 2-3 of the canonical order for range r (a block of kFoldThreads
// threads): thread t forms group 256r + t's sum from its 8 slice sums (all
// loaded before the first add), then block_sum folds the block's groups.
// The range sums are valid in thread 0.
template <int NV>
__device__ __forceinline__ void fold_range(const double *__restrict__ sp, int ld, int ns, int ng,
                                           int r, double (&v)[NV]) {
  static_assert(kFoldRange == kFoldThreads, "one group per thread");
  const int g0 = r * kFoldRange, g1 = min(ng, g0 + kFoldRange);
  double raw[NV][kGroupSlices];
  const int g = g0 + (int)threadIdx.x;
#pragma unroll
  for (int k = 0; k < NV; k++)
#pragma unroll
    for (int j = 0; j < kGroupSlices; j++) {
      const int sl = g * kGroupSlices + j;
      raw[k][j] = (g < g1 && sl < ns) ? __ldg(sp + (size_t)k * ld + sl) : 0.0;
    }
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double gsum = 0.0;
#pragma unroll
    for (int j = 0; j < kGroupSlices; j++) {
      const int sl = g * kGroupSlices + j;
      if (g < g1 && sl < ns) gsum = __dadd_rn(gsum, raw[k][j]);
    }
    v[k] = __dadd_rn(0.0, gsum);  // the thread's running sum, from zero
  }
  block_sum<NV>(v);
}

// Step 4: the nr range sums (rs[k*ldr + r]) folded the same way; totals in
// thread 0.
template <int NV>
__device__ __forceinline__ void fold_total(const double *rs, int ldr, int nr, double (&v)[NV]) {
#pragma unroll
  for (int k = 0; k < NV; k++) {
    double a = 0.0;
    for (int r = threadIdx.x; r < nr; r += kFoldThreads)
      a = __dadd_rn(a, __ldcg(rs + (size_t)k * ldr + r));
    v[k] = a;
  }
  block_sum<NV>(v);
}

}  // namespace dev
}  // namespace ainv
