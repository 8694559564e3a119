// Multi-right-hand-side preconditioned CG: up to 32 systems A x_l = b_l
// solved together, every matrix pass shared by all of them.
//
// Multivectors are row-interleaved with a stride of 32 columns: entry
// (row, l) at v[row * 32 + l], so the 32 values of one row are one 256-byte
// line.  Every product is an SpMM over the sliced layout: a warp walks one
// 32-row slice four rows at a time, 8 lanes per row, each lane owning 4
// columns, so every matrix entry is loaded once and multiplies a whole
// gathered row of the input multivector (8 lanes x 32 bytes = one 256-byte
// line).  The matrix streams once per iteration for all columns instead of
// once per column.
//
// Each column follows the PSBLAS CG recurrence (psb_dcg, istop=2, as driven
// at tests/pdegen/ppde3d.f90:280-281) with its own scalars: the column-wise
// form of block CG, so every column iterates exactly as a single-vector solve
// would (the per-row products accumulate in the same order as the
// single-vector kernels) and stops on its own criterion; converged columns
// stay frozen while the others continue.  The preconditioner runs in the
// factors' precision (FP32 multivector intermediate for FP32/BF16 factors),
// A, the recurrence, dots and norms in FP64, with the true-residual checks of
// the single-vector loop.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <new>

#include "kstate.cuh"
#include "sell_device.cuh"

namespace ainv {
namespace mrhs {

using namespace dev;
using namespace kstate;

constexpr int kCols = 32;    // multivector stride (columns per row)
constexpr int kChunk = 8;    // iterations per captured graph launch
constexpr int kRecheck = 50; // true-residual period for FP32/BF16 factors
// Resident blocks per SM asked of the gathering kernels (SpMM and sweeps):
// 4 (64 registers) measured 0.489 s per 128^3 x 32 block solve, 5 (48
// registers, a few spills) 0.500 s, 6 (40) and an uncapped build (72-96
// registers) 0.54 s.
#ifndef AINV_MRHS_BLOCKS
#define AINV_MRHS_BLOCKS 4
#endif
constexpr int kGatherBlocks = AINV_MRHS_BLOCKS;

struct MState {
  KState col[kCols];
  int m;
  int alldone;  // every column finished (converged and confirmed, or failed)
  unsigned ticket;
  int pad;
};

// ---------------------------------------------------------------- device --
// Lane map of the SpMM kernels: a warp works on 4 rows of a slice at a time,
// lane = 8 q + g takes row q of the four and columns 4g .. 4g+3, so the 8
// lanes of a row read its 32 columns as one 256-byte line (32 bytes each).
constexpr int kColsPerLane = 4;
constexpr int kRowsPerStep = kSlice / 8;  // 4
constexpr int kSlotBatch = 4;

__device__ __forceinline__ void ldg4(const double *p, double (&o)[4]) {
  const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
  const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
  o[0] = a.x;
  o[1] = a.y;
  o[2] = b.x;
  o[3] = b.y;
}
__device__ __forceinline__ void ldg4(const float *p, float (&o)[4]) {
  const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
  o[0] = a.x;
  o[1] = a.y;
  o[2] = a.z;
  o[3] = a.w;
}
__device__ __forceinline__ void ld4(const double *p, double (&o)[4]) {
  const double2 a = reinterpret_cast<const double2 *>(p)[0];
  const double2 b = reinterpret_cast<const double2 *>(p)[1];
  o[0] = a.x;
  o[1] = a.y;
  o[2] = b.x;
  o[3] = b.y;
}
__device__ __forceinline__ void st4(double *p, const double (&v)[4]) {
  reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}
__device__ __forceinline__ void st4(float *p, const float (&v)[4]) {
  *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
// Evict-first stores for the products' multivector outputs (Q, T, Z): they
// are larger than L2 and read back only by a later kernel, so they should
// not displace the gathered input's rows that the next slices reuse.
__device__ __forceinline__ void st4cs(double *p, const double (&v)[4]) {
  __stcs(reinterpret_cast<double2 *>(p), make_double2(v[0], v[1]));
  __stcs(reinterpret_cast<double2 *>(p) + 1, make_double2(v[2], v[3]));
}
__device__ __forceinline__ void st4cs(float *p, const float (&v)[4]) {
  __stcs(reinterpret_cast<float4 *>(p), make_float4(v[0], v[1], v[2], v[3]));
}

// acc[e] = row `row` (slice-local rs) of M times column c0 + e of x.  Slots
// are taken kSlotBatch at a time: their values and index words load
// together, then the batch's gathers (skipped where the value is 0) are all
// in flight before the first fma.  Slot order and fma sequence per (row,
// column) are those of the single-vector kernels.
template <class V, class X, class A>
__device__ __forceinline__ void row_mm(const SellView<V> &m, int pack, int vb, int ib, int w,
                                       bool om, int row, int rs, const X *__restrict__ x, int c0,
                                       A (&acc)[kColsPerLane]) {
#pragma unroll
  for (int e = 0; e < kColsPerLane; e++) acc[e] = A(0);
  for (int k0 = 0; k0 < w; k0 += kSlotBatch) {
    A v[kSlotBatch];
    int c[kSlotBatch];
#pragma unroll
    for (int j = 0; j < kSlotBatch; j++) {
      const int k = k0 + j;
      if (k < w) {
        const int pos = (k / pack) * (kSlice * pack) + rs * pack + (k % pack);
        v[j] = (A)ldv(m.val + vb + pos);
        c[j] = om ? row + __ldg(m.idx + ib + k) : __ldcs(m.idx + ib + pos);
      } else {
        v[j] = A(0);
        c[j] = 0;
      }
    }
    A xv[kSlotBatch][kColsPerLane];
#pragma unroll
    for (int j = 0; j < kSlotBatch; j++) {
      if (v[j] != A(0) && (unsigned)c[j] < (unsigned)m.n) {
        X t[kColsPerLane];
        ldg4(x + (size_t)c[j] * kCols + c0, t);
#pragma unroll
        for (int e = 0; e < kColsPerLane; e++) xv[j][e] = (A)t[e];
      } else {
#pragma unroll
        for (int e = 0; e < kColsPerLane; e++) xv[j][e] = A(0);
      }
    }
#pragma unroll
    for (int j = 0; j < kSlotBatch; j++)
#pragma unroll
      for (int e = 0; e < kColsPerLane; e++) acc[e] = madd(v[j], xv[j][e], acc[e]);
  }
}

// Visit every row of M (warps striding over slices): epi(row, c0, acc) with
// the thread's 4 columns; each thread's rows come in ascending order.  (A
// contiguous run of slices per warp, which spreads the warps' fronts over
// the matrix, measured slower at 128^3 x 32: 0.604 against 0.497 s per
// block solve.)
template <class V, class X, class Epi>
__device__ __forceinline__ void for_each_slice(const SellView<V> &m, int pack,
                                               const X *__restrict__ x, Epi &&epi) {
  using A = typename Acc<V>::type;
  const int lane = threadIdx.x & 31;
  const int q = lane >> 3, c0 = (lane & 7) * kColsPerLane;
  for (int s = first_slice(); s < m.nslices; s += slice_stride()) {
    const int vb = __ldg(m.sptr + s), ve = __ldg(m.sptr + s + 1);
    const int ib = __ldg(m.iptr + s), ie = __ldg(m.iptr + s + 1);
    const int w = (ve - vb) / kSlice;
    const bool om = (ie - ib) == w;
#pragma unroll 2
    for (int t = 0; t < kSlice / kRowsPerStep; t++) {
      const int rs = t * kRowsPerStep + q;
      const int row = s * kSlice + rs;
      A acc[kColsPerLane];
      row_mm(m, pack, vb, ib, w, om, row, rs, x, c0, acc);
      if (row < m.n) epi(row, c0, acc);
    }
  }
}

// Last-block fold shared by the per-column sums: block partials
// partials[(i*32 + c)*G + b], warp w taking blocks w, w+8, ... then the
// warps combined in order; totals in warp 0, lane = column.
template <int NV>
__device__ __forceinline__ bool fold_last(double (&tot)[NV], double *__restrict__ partials,
                                          unsigned *ticket, double (&sh)[NV][kWarps][kCols]) {
  __shared__ bool is_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int G = gridDim.x;
  __syncthreads();
  if (threadIdx.x == 0) is_last = atomicAdd(ticket, 1u) == (unsigned)G - 1;
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
#pragma unroll
  for (int i = 0; i < NV; i++) {
    double s = 0.0;
    for (int b = warp; b < G; b += kWarps) s += __ldcg(partials + ((size_t)i * kCols + lane) * G + b);
    sh[i][warp][lane] = s;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double s = 0.0;
      for (int w = 0; w < kWarps; w++) s += sh[i][w][lane];
      tot[i] = s;
    }
    if (lane == 0) *ticket = 0u;
  }
  return true;
}

// Per-column grid sums for the vector kernels: each thread holds partials
// for column (threadIdx.x & 31).  Blocks fold their warps in order and store
// one partial per column; the last block folds the blocks in order.
template <int NV>
__device__ __forceinline__ bool col_sum(double (&v)[NV], double *__restrict__ partials,
                                        unsigned *ticket) {
  __shared__ double sh[NV][kWarps][kCols];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int G = gridDim.x;
#pragma unroll
  for (int i = 0; i < NV; i++) sh[i][warp][lane] = v[i];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double s = 0.0;
      for (int w = 0; w < kWarps; w++) s += sh[i][w][lane];
      partials[((size_t)i * kCols + lane) * G + blockIdx.x] = s;
    }
    __threadfence();
  }
  return fold_last<NV>(v, partials, ticket, sh);
}

// The same for the SpMM kernels, whose threads hold partials for their 4
// columns: the block's 32 row-lanes per column are folded in (warp, row)
// order.
template <int NV>
__device__ __forceinline__ bool col_sum4(const double (&v)[NV][kColsPerLane], double (&tot)[NV],
                                         double *__restrict__ partials, unsigned *ticket) {
  __shared__ double part[NV][kCols][kWarps * kRowsPerStep + 1];
  __shared__ double sh[NV][kWarps][kCols];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = warp * kRowsPerStep + (lane >> 3), c0 = (lane & 7) * kColsPerLane;
  const int G = gridDim.x;
#pragma unroll
  for (int i = 0; i < NV; i++)
#pragma unroll
    for (int e = 0; e < kColsPerLane; e++) part[i][c0 + e][slot] = v[i][e];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double s = 0.0;
      for (int k = 0; k < kWarps * kRowsPerStep; k++) s += part[i][lane][k];
      partials[((size_t)i * kCols + lane) * G + blockIdx.x] = s;
    }
    __threadfence();
  }
  return fold_last<NV>(tot, partials, ticket, sh);
}

__device__ __forceinline__ bool finished(const KState &c) {
  return c.done && (c.verified || c.status != AINV_SUCCESS);
}

// Called by warp 0 of a last block after its per-column updates.
__device__ __forceinline__ void update_alldone(MState *ms) {
  const int lane = threadIdx.x & 31;
  const bool f = lane >= ms->m || finished(ms->col[lane]);
  const bool all = __all_sync(0xffffffffu, f);
  if (lane == 0) ms->alldone = all ? 1 : 0;
}

// R = B - A X, ||b_l||, ||r_l|| (initial state of every column).
__global__ void __launch_bounds__(kBlock)
    k_mv_init(SellView<double> a, int apack, const double *__restrict__ X,
              const double *__restrict__ B, double *__restrict__ R, MState *ms,
              double *partials) {
  const int lane = threadIdx.x & 31;
  double pr[2][kColsPerLane] = {};
  for_each_slice(a, apack, X, [&](int row, int c0, const double (&acc)[kColsPerLane]) {
    const size_t e0 = (size_t)row * kCols + c0;
    double b[kColsPerLane], r[kColsPerLane];
    ldg4(B + e0, b);
#pragma unroll
    for (int e = 0; e < kColsPerLane; e++) {
      r[e] = b[e] - acc[e];
      pr[0][e] += r[e] * r[e];
      pr[1][e] += b[e] * b[e];
    }
    st4(R + e0, r);
  });
  double tot[2];
  if (col_sum4<2>(pr, tot, partials, &ms->ticket) && threadIdx.x < 32) {
    if (lane < ms->m) {
      KState *st = &ms->col[lane];
      const double bn = sqrt(tot[1]);
      st->bn2 = (bn == 0.0) ? 1.0 : bn;
      const double p3[3] = {tot[0], 0.0, 0.0};
      finish_dots<kInit>(st, p3, false, nullptr);
    }
    update_alldone(ms);
  }
}

// Sweep 1 of the apply on all columns: T = D^-1 .* (W^T R).
template <class V, class T>
__global__ void __launch_bounds__(kBlock, kGatherBlocks)
    k_mv_sweep1(SellView<V> m, int pack, const double *__restrict__ R, const V *__restrict__ d,
                T *__restrict__ Tm, const MState *ms) {
  if (ms->alldone) return;
  using A = typename Acc<V>::type;
  for_each_slice(m, pack, R, [&](int row, int c0, const A (&acc)[kColsPerLane]) {
    const A dr = ldd(d + row);
    T t[kColsPerLane];
#pragma unroll
    for (int e = 0; e < kColsPerLane; e++) t[e] = (T)(dr * acc[e]);
    st4cs(Tm + (size_t)row * kCols + c0, t);
  });
}

// Sweep 2 on all columns: Zv = Z T, with rho_l = r_l . z_l and beta_l.
template <class V, class T>
__global__ void __launch_bounds__(kBlock, kGatherBlocks)
    k_mv_sweep2(SellView<V> m, int pack, const T *__restrict__ Tm, const double *__restrict__ R,
                double *__restrict__ Zv, MState *ms, double *partials) {
  if (ms->alldone) return;
  using A = typename Acc<V>::type;
  const int lane = threadIdx.x & 31;
  double pr[1][kColsPerLane] = {};
  for_each_slice(m, pack, Tm, [&](int row, int c0, const A (&acc)[kColsPerLane]) {
    const size_t e0 = (size_t)row * kCols + c0;
    double r[kColsPerLane], z[kColsPerLane];
    ldg4(R + e0, r);
#pragma unroll
    for (int e = 0; e < kColsPerLane; e++) {
      z[e] = (double)acc[e];
      pr[0][e] += r[e] * z[e];
    }
    st4cs(Zv + e0, z);
  });
  double tot[1];
  if (col_sum4<1>(pr, tot, partials, &ms->ticket) && threadIdx.x < 32) {
    if (lane < ms->m && !ms->col[lane].done) cg_take_rho(&ms->col[lane], tot[0]);
    update_alldone(ms);
  }
}

// Unpreconditioned: Zv = R, rho = r.r.
__global__ void __launch_bounds__(kBlock)
    k_mv_ident(long long ne, const double *__restrict__ R, double *__restrict__ Zv, MState *ms,
               double *partials) {
  if (ms->alldone) return;
  double pr[1] = {0.0};
  for (long long e = (long long)blockIdx.x * kBlock + threadIdx.x; e < ne;
       e += (long long)gridDim.x * kBlock) {
    Zv[e] = R[e];
    pr[0] += R[e] * R[e];
  }
  const int lane = threadIdx.x & 31;
  if (col_sum<1>(pr, partials, &ms->ticket) && threadIdx.x < 32) {
    if (lane < ms->m && !ms->col[lane].done) cg_take_rho(&ms->col[lane], pr[0]);
    update_alldone(ms);
  }
}

// P = Zv (first iteration of the column) or Zv + beta_l P.
__global__ void __launch_bounds__(kBlock)
    k_mv_p(long long ne, const double *__restrict__ Zv, double *__restrict__ P,
           const MState *ms) {
  if (ms->alldone) return;
  const int lane = threadIdx.x & 31;  // element e has column e % 32 = lane
  const KState &c = ms->col[lane];
  if (lane >= ms->m || c.done) return;
  const bool first = c.iter == 0;
  const double beta = c.beta;
  for (long long e = (long long)blockIdx.x * kBlock + threadIdx.x; e < ne;
       e += (long long)gridDim.x * kBlock)
    P[e] = first ? Zv[e] : Zv[e] + beta * P[e];
}

// Q = A P with sigma_l = p_l . q_l, alpha_l = rho_l / sigma_l.
__global__ void __launch_bounds__(kBlock, kGatherBlocks)
    k_mv_spmm_sigma(SellView<double> a, int apack, const double *__restrict__ P,
                    double *__restrict__ Q, MState *ms, double *partials) {
  if (ms->alldone) return;
  const int lane = threadIdx.x & 31;
  double pr[1][kColsPerLane] = {};
  for_each_slice(a, apack, P, [&](int row, int c0, const double (&acc)[kColsPerLane]) {
    const size_t e0 = (size_t)row * kCols + c0;
    double p[kColsPerLane];
    ldg4(P + e0, p);
#pragma unroll
    for (int e = 0; e < kColsPerLane; e++) pr[0][e] += p[e] * acc[e];
    st4cs(Q + e0, acc);
  });
  double tot[1];
  if (col_sum4<1>(pr, tot, partials, &ms->ticket) && threadIdx.x < 32) {
    if (lane < ms->m && !ms->col[lane].done) {
      const double p3[3] = {tot[0], 0.0, 0.0};
      finish_dots<kCgSigma>(&ms->col[lane], p3, false, nullptr);
    }
    update_alldone(ms);
  }
}

// X += alpha_l P, R -= alpha_l Q, ||r_l||^2 and the convergence test.
__global__ void __launch_bounds__(kBlock)
    k_mv_xr(long long ne, const double *__restrict__ P, const double *__restrict__ Q,
            double *__restrict__ X, double *__restrict__ R, MState *ms, double *partials) {
  if (ms->alldone) return;
  const int lane = threadIdx.x & 31;
  const bool live = lane < ms->m && !ms->col[lane].done;
  const double alpha = ms->col[lane].alpha;
  double pr[1] = {0.0};
  if (live) {
    for (long long e = (long long)blockIdx.x * kBlock + threadIdx.x; e < ne;
         e += (long long)gridDim.x * kBlock) {
      X[e] = X[e] + alpha * P[e];
      const double ri = R[e] - alpha * Q[e];
      R[e] = ri;
      pr[0] += ri * ri;
    }
  }
  if (col_sum<1>(pr, partials, &ms->ticket) && threadIdx.x < 32) {
    if (live) finish_iteration(&ms->col[lane], pr[0]);
    update_alldone(ms);
  }
}

// Which columns take a true-residual pass this iteration (as the
// single-vector kTrueRes kernel decides per solve).
__device__ __forceinline__ bool col_verify(const KState &c) {
  return c.done && c.status == AINV_SUCCESS && !c.verified;
}
__device__ __forceinline__ bool col_periodic(const KState &c) {
  return !c.done && c.check_every > 0 && c.iter > 0 && c.iter % c.check_every == 0;
}

// Rt = B - A X against R for the columns that need a check; decides
// confirmation / replacement per column (finish_dots<kTrueRes>).
__global__ void __launch_bounds__(kBlock)
    k_mv_trueres(SellView<double> a, int apack, const double *__restrict__ X,
                 const double *__restrict__ B, const double *__restrict__ R,
                 double *__restrict__ Rt, MState *ms, double *partials) {
  if (ms->alldone) return;
  const int lane = threadIdx.x & 31;
  const KState &c = ms->col[lane];
  const bool mine = lane < ms->m && (col_verify(c) || col_periodic(c));
  const bool verify = lane < ms->m && col_verify(c);
  if (!__syncthreads_or(mine)) return;  // no column needs a check
  double pr[3][kColsPerLane] = {};
  for_each_slice(a, apack, X, [&](int row, int c0, const double (&acc)[kColsPerLane]) {
    const size_t e0 = (size_t)row * kCols + c0;
    double b[kColsPerLane], r[kColsPerLane], rt[kColsPerLane];
    ldg4(B + e0, b);
    ldg4(R + e0, r);
#pragma unroll
    for (int e = 0; e < kColsPerLane; e++) {
      rt[e] = b[e] - acc[e];
      pr[0][e] += rt[e] * rt[e];
      const double g = rt[e] - r[e];
      pr[1][e] += g * g;
    }
    st4(Rt + e0, rt);
  });
  double tot[3];
  if (col_sum4<3>(pr, tot, partials, &ms->ticket) && threadIdx.x < 32) {
    if (mine) finish_dots<kTrueRes>(&ms->col[lane], tot, verify, nullptr);
    update_alldone(ms);
  }
}

// R := Rt for the columns whose check asked for a replacement.
__global__ void __launch_bounds__(kBlock)
    k_mv_replace(long long ne, const double *__restrict__ Rt, double *__restrict__ R,
                 const MState *ms) {
  const int lane = threadIdx.x & 31;
  if (lane >= ms->m || !ms->col[lane].replace) return;
  for (long long e = (long long)blockIdx.x * kBlock + threadIdx.x; e < ne;
       e += (long long)gridDim.x * kBlock)
    R[e] = Rt[e];
}

// Caller layout (n x m, leading dimension ld) <-> stride-32 multivector.
__global__ void __launch_bounds__(kBlock)
    k_mv_gather(int n, int m, int ld, const double *__restrict__ src, double *__restrict__ dst) {
  const long long ne = (long long)n * kCols;
  for (long long e = (long long)blockIdx.x * kBlock + threadIdx.x; e < ne;
       e += (long long)gridDim.x * kBlock) {
    const int l = (int)(e & (kCols - 1));
    const long long row = e >> 5;
    dst[e] = l < m ? src[row * ld + l] : 0.0;
  }
}
__global__ void __launch_bounds__(kBlock)
    k_mv_scatter(int n, int m, int ld, const double *__restrict__ src, double *__restrict__ dst) {
  const long long ne = (long long)n * kCols;
  for (long long e = (long long)blockIdx.x * kBlock + threadIdx.x; e < ne;
       e += (long long)gridDim.x * kBlock) {
    const int l = (int)(e & (kCols - 1));
    if (l < m) dst[(e >> 5) * ld + l] = src[e];
  }
}

// ------------------------------------------------------------------ host --
enum { MX = 0, MB, MR, MZ, MP, MQ, MRT, kNumMv };

}  // namespace mrhs

struct MrhsWs {
  int n = 0, G = 0;
  size_t stride = 0;       // doubles per multivector (n * 32)
  double *mv = nullptr;    // 7 FP64 multivectors
  void *t = nullptr;       // apply intermediate (n * 32 of double or float)
  double *partials = nullptr;
  mrhs::MState *st = nullptr, *hst = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t ev = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long key_serial = ~0ull;
  double *v(int i) const { return mv + (size_t)i * stride; }
};

void destroy_mws(MrhsWs *w) {
  if (!w) return;
  if (w->exec) cudaGraphExecDestroy(w->exec);
  if (w->mv) cudaFree(w->mv);
  if (w->t) cudaFree(w->t);
  if (w->partials) cudaFree(w->partials);
  if (w->st) cudaFree(w->st);
  if (w->hst) cudaFreeHost(w->hst);
  if (w->ev) cudaEventDestroy(w->ev);
  if (w->s) cudaStreamDestroy(w->s);
  delete w;
}

namespace mrhs {
namespace {

int get_ws(ainv_csr *a, MrhsWs **out) {
  if (a->mws) {
    *out = a->mws;
    return AINV_SUCCESS;
  }
  MrhsWs *w = new (std::nothrow) MrhsWs;
  if (!w) {
    set_error("block solve workspace: host allocation failed");
    return AINV_ERR_ALLOC;
  }
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  w->n = a->n;
  w->stride = (size_t)a->n * kCols;
  w->G = 8 * sms;  // partials capacity: the largest resident wave (8 blocks per SM)
  cudaError_t e = cudaMalloc(&w->mv, sizeof(double) * kNumMv * w->stride);
  if (e == cudaSuccess) e = cudaMalloc(&w->t, sizeof(double) * w->stride);
  if (e == cudaSuccess) e = cudaMalloc(&w->partials, sizeof(double) * 3 * kCols * (size_t)w->G);
  if (e == cudaSuccess) e = cudaMalloc(&w->st, sizeof(MState));
  if (e == cudaSuccess) e = cudaMallocHost(&w->hst, sizeof(MState));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&w->s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&w->ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMemset(w->mv, 0, sizeof(double) * kNumMv * w->stride);
  if (e != cudaSuccess) {
    destroy_mws(w);
    set_error("block solve workspace allocation failed: %s", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? AINV_ERR_ALLOC : AINV_ERR_CUDA;
  }
  a->mws = w;
  *out = w;
  return AINV_SUCCESS;
}

template <class V, class T>
void launch_precond(const MrhsWs *w, const ainv_handle *h, cudaStream_t s) {
  const SellView<V> wt = view<V>(h->wt), z = view<V>(h->z);
  const int g1 = wave_grid((const void *)k_mv_sweep1<V, T>, w->n);
  const int g2 = wave_grid((const void *)k_mv_sweep2<V, T>, w->n);
  k_mv_sweep1<V, T><<<g1, kBlock, 0, s>>>(wt, h->wt.pack, w->v(MR), (const V *)h->d, (T *)w->t,
                                         w->st);
  k_mv_sweep2<V, T><<<g2, kBlock, 0, s>>>(z, h->z.pack, (const T *)w->t, w->v(MR), w->v(MZ),
                                         w->st, w->partials);
}

int enqueue_iteration(const MrhsWs *w, const ainv_handle *h, const ainv_csr *a) {
  const cudaStream_t s = w->s;
  const long long ne = (long long)w->stride;
  const SellView<double> A = view<double>(a->a);
  auto gv = [&](const void *k) { return wave_grid(k, ne); };
  auto gm = [&](const void *k) { return wave_grid(k, w->n); };
  if (h) {
    switch (h->prec) {
      case AINV_PREC_FP64: launch_precond<double, double>(w, h, s); break;
      case AINV_PREC_FP32: launch_precond<float, float>(w, h, s); break;
      case AINV_PREC_FP32_ACC64: launch_precond<f32w, double>(w, h, s); break;
      case AINV_PREC_BF16_ACC64: launch_precond<b16w, double>(w, h, s); break;
      default: launch_precond<__nv_bfloat16, float>(w, h, s); break;
    }
  } else {
    k_mv_ident<<<gv((const void *)k_mv_ident), kBlock, 0, s>>>(ne, w->v(MR), w->v(MZ), w->st,
                                                               w->partials);
  }
  k_mv_p<<<gv((const void *)k_mv_p), kBlock, 0, s>>>(ne, w->v(MZ), w->v(MP), w->st);
  k_mv_spmm_sigma<<<gm((const void *)k_mv_spmm_sigma), kBlock, 0, s>>>(
      A, a->a.pack, w->v(MP), w->v(MQ), w->st, w->partials);
  k_mv_xr<<<gv((const void *)k_mv_xr), kBlock, 0, s>>>(ne, w->v(MP), w->v(MQ), w->v(MX), w->v(MR),
                                                       w->st, w->partials);
  k_mv_trueres<<<gm((const void *)k_mv_trueres), kBlock, 0, s>>>(
      A, a->a.pack, w->v(MX), w->v(MB), w->v(MR), w->v(MRT), w->st, w->partials);
  k_mv_replace<<<gv((const void *)k_mv_replace), kBlock, 0, s>>>(ne, w->v(MRT), w->v(MR), w->st);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("block solve launch failed: %s", cudaGetErrorString(e));
    return AINV_ERR_CUDA;
  }
  return AINV_SUCCESS;
}

int ensure_graph(MrhsWs *w, const ainv_handle *h, const ainv_csr *a) {
  const unsigned long long key = h ? h->serial : 0ull;
  if (w->exec && w->key_serial == key) return AINV_SUCCESS;
  if (w->exec) {
    cudaGraphExecDestroy(w->exec);
    w->exec = nullptr;
  }
  AINV_CUDA_TRY(cudaStreamBeginCapture(w->s, cudaStreamCaptureModeThreadLocal));
  int rc = AINV_SUCCESS;
  for (int k = 0; k < kChunk && rc == AINV_SUCCESS; k++) rc = enqueue_iteration(w, h, a);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(w->s, &g);
  if (rc != AINV_SUCCESS || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    if (rc == AINV_SUCCESS) set_error("block solve capture failed: %s", cudaGetErrorString(e));
    return rc != AINV_SUCCESS ? rc : AINV_ERR_CUDA;
  }
  const cudaError_t ei = cudaGraphInstantiate(&w->exec, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    w->exec = nullptr;
    set_error("block solve graph instantiate failed: %s", cudaGetErrorString(ei));
    return AINV_ERR_CUDA;
  }
  w->key_serial = key;
  return AINV_SUCCESS;
}

}  // namespace
}  // namespace mrhs
}  // namespace ainv

extern "C" int ainv_gpu_block_solve(ainv_handle *h, const ainv_csr *ac, int m, const double *B,
                                    int ldb, double *X, int ldx, double eps, int itmax,
                                    int *iters, double *errs, int *status, void *stream) {
  using namespace ainv;
  using namespace ainv::mrhs;
  ainv_csr *a = const_cast<ainv_csr *>(ac);
  if (!a || !B || !X || m < 1 || m > kCols || ldb < m || ldx < m) {
    set_error("ainv_gpu_block_solve: invalid arguments (m must be 1..%d, ld >= m)", kCols);
    return AINV_ERR_ARG;
  }
  if (h && h->n != a->n) {
    set_error("ainv_gpu_block_solve: preconditioner size %d != operator size %d", h->n, a->n);
    return AINV_ERR_ARG;
  }
  if (!(eps > 0.0) || itmax < 0) {
    set_error("ainv_gpu_block_solve: invalid eps/itmax");
    return AINV_ERR_ARG;
  }
  MrhsWs *w = nullptr;
  AINV_TRY(get_ws(a, &w));
  const cudaStream_t user = (cudaStream_t)stream;
  const int n = a->n;
  const int Gc = wave_grid((const void *)k_mv_gather, (long long)n * kCols);
  AINV_CUDA_TRY(cudaEventRecord(w->ev, user));
  AINV_CUDA_TRY(cudaStreamWaitEvent(w->s, w->ev, 0));
  k_mv_gather<<<Gc, kBlock, 0, w->s>>>(n, m, ldb, B, w->v(MB));
  k_mv_gather<<<Gc, kBlock, 0, w->s>>>(n, m, ldx, X, w->v(MX));
  MState init{};
  init.m = m;
  for (int l = 0; l < kCols; l++) {
    KState &c = init.col[l];
    c.eps = eps;
    c.itmax = itmax;
    c.method = AINV_KRYLOV_CG;
    c.check_every = (h && h->prec != AINV_PREC_FP64) ? kRecheck : 0;
    if (l >= m) {  // unused lanes: finished from the start
      c.done = 1;
      c.verified = 1;
    }
  }
  *w->hst = init;
  AINV_CUDA_TRY(cudaMemcpyAsync(w->st, w->hst, sizeof(MState), cudaMemcpyHostToDevice, w->s));
  k_mv_init<<<wave_grid((const void *)k_mv_init, n), kBlock, 0, w->s>>>(
      view<double>(a->a), a->a.pack, w->v(MX), w->v(MB), w->v(MR), w->st, w->partials);
  AINV_CUDA_TRY(cudaGetLastError());
  const bool use_graph = getenv("AINV_NO_GRAPH") == nullptr;
  const long max_chunks = (long)itmax / kChunk + 2 + 4 * kMaxVerifyFails;
  for (long c = 0; c < max_chunks; c++) {
    AINV_CUDA_TRY(cudaMemcpyAsync(w->hst, w->st, sizeof(MState), cudaMemcpyDeviceToHost, w->s));
    AINV_CUDA_TRY(cudaStreamSynchronize(w->s));
    if (w->hst->alldone) break;
    if (use_graph && c > 0) {
      AINV_TRY(ensure_graph(w, h, a));
      AINV_CUDA_TRY(cudaGraphLaunch(w->exec, w->s));
    } else {
      for (int k = 0; k < kChunk; k++) AINV_TRY(enqueue_iteration(w, h, a));
    }
  }
  k_mv_scatter<<<Gc, kBlock, 0, w->s>>>(n, m, ldx, w->v(MX), X);
  AINV_CUDA_TRY(cudaMemcpyAsync(w->hst, w->st, sizeof(MState), cudaMemcpyDeviceToHost, w->s));
  AINV_CUDA_TRY(cudaStreamSynchronize(w->s));
  AINV_CUDA_TRY(cudaEventRecord(w->ev, w->s));
  AINV_CUDA_TRY(cudaStreamWaitEvent(user, w->ev, 0));
  const MState &f = *w->hst;
  int rc = AINV_SUCCESS;
  for (int l = 0; l < m; l++) {
    const KState &c = f.col[l];
    if (iters) iters[l] = c.iter;
    if (errs) errs[l] = sqrt(c.rn2) / c.bn2;
    const int sl = c.done ? c.status : AINV_ERR_INTERNAL;
    if (status) status[l] = sl;
    if (sl != AINV_SUCCESS && rc == AINV_SUCCESS) rc = sl;
  }
  if (!f.alldone) {
    set_error("block solve did not terminate");
    return AINV_ERR_INTERNAL;
  }
  if (rc != AINV_SUCCESS) set_error("block solve: a column ended with status %d", rc);
  return rc;
}
