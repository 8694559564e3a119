// Streaming sliced SpMV: a persistent kernel feeds shared memory with bulk
// asynchronous copies (cp.async.bulk, the TMA engine's linear mode) so the
// bytes in flight do not occupy registers.
//
// Each block walks stages j0, j0 + stride, ... (by default blockIdx.x and
// gridDim.x; a caller that splits the grid among several vectors passes
// its own walk).  A stage
// (StageDesc) is m.stage_slices consecutive slices.  Its buffer receives, by
// bulk copies: the descriptor, the stage's chunks of the slice pointers,
// its values, its index words and -- for uniform stages, whose slices share
// one offset list -- the windows x[r0+o, r1+o) of the gathered vector for
// every offset o.  The block is warp-specialised: one producer warp keeps D
// stage buffers in flight (a "full" mbarrier per buffer completes when its
// copies land, an "empty" mbarrier when all consumer warps are done with
// it); each of the kConsumerSlices consumer warps computes R consecutive
// slices of every stage from shared memory (one row per lane and slice).
// Consumers know their rows from the stage index alone, load their
// epilogue operands one stage ahead, and never wait on global memory except
// in non-uniform stages' gathers.  No block-wide barrier sits inside the
// stage loop.
//
// Every wait is bounded (kWaitNs of device time).  On a timeout the block
// records it in *status, waits (again bounded) for its own copies in flight
// and returns; nothing spins without a limit.
#pragma once

#include "sell_device.cuh"

namespace ainv {
namespace dev {

constexpr int kConsumerWarps = kConsumerSlices;
constexpr int kStreamThreads = (kConsumerWarps + 1) * 32;  // + the producer warp
// Blocks a streaming kernel must fit per SM: the register budget of a
// thread is capped at 65536 / (4 * kStreamThreads) = 56, so that four
// producers per SM keep their copies in flight.
constexpr int kStreamMinBlocks = 4;
// Stage-buffer header: descriptor, then the sptr and iptr chunks (the
// stage's slice pointers, copied from 16-byte-aligned starts), then the
// stage's derived words (StageDerived), written by the producer warp.
constexpr int kDescBytes = 64;
constexpr int kPtrChunkBytes = ((kMaxStageSlices + 1) * 4 + 24 + 15) / 16 * 16;
constexpr int kDerivedOfs = kDescBytes + 2 * kPtrChunkBytes;
constexpr int kDerivedBytes = 64;
constexpr int kHeaderBytes = kDerivedOfs + kDerivedBytes;
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Add bytes to the barrier's expected transactions without arriving.
__device__ __forceinline__ void mbar_add_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// 16-byte aligned source and destination, size a positive multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes,
                                         unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of a barrier: false after kWaitNs.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned it = 1; it < (1u << 30); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63u) == 0 && global_ns() - t0 > kWaitNs) return false;
  }
  return false;
}

// 16-byte granules in elements of an es-byte type (es in {2, 4, 8}).
__device__ __forceinline__ int granule(int es) { return 16 / es; }

// Shared-memory arrangement of one launch (bytes; computed on the host).
// Buffer: [header | values (vb) | index words (ib) | nwin windows of xw |
//          nrv row-operand areas of rw].
struct StreamLayout {
  int D;      // stage buffers
  int vb;     // value area per buffer
  int ib;     // index area per buffer
  int xw;     // one gathered-vector window
  int nwin;   // windows per buffer (offset clusters)
  int rw;     // one row-operand area (the stage's rows of an epilogue vector)
  int nrv;    // row-operand areas per buffer
  int stage;  // bytes per buffer
  int R;      // slices per consumer warp and stage
};

// Row operands of an epilogue: up to kMaxRowVecs vectors indexed by row
// (element sizes es[i]); null pointers are skipped.  The producer copies a
// stage's rows of each into the buffer; rows whose 16-byte-rounded copy
// would pass the end of the vector are read from global memory instead.
constexpr int kMaxRowVecs = 3;
struct RowVecs {
  const void *p[kMaxRowVecs];
  int es[kMaxRowVecs];
};
static_assert(kMaxRowVecs == 3, "RowVecs initialisers list three vectors");

// Per-stage words the producer derives from the descriptor while it issues
// the copies, so that no consumer warp recomputes them: element k of a row
// of a uniform stage sits at window-area index row + wofs[k] (for k past the
// stage's offsets, an index inside window 0, never read: those slots hold
// zeros), and the stage's first nrows[i] rows of row operand i are staged.
struct __align__(16) StageDerived {
  int wofs[kStageMaxOffsets];
  int nrows[kMaxRowVecs];
  int pad;
};
static_assert(sizeof(StageDerived) <= kDerivedBytes, "derived words overflow the header");
static_assert(kDerivedOfs % 16 == 0, "derived words are read as 16-byte words");

// Rows [r0, ce) of a row vector with es-byte elements are copied: r1
// rounded up to a whole 16-byte granule if that stays inside the n-element
// vector, else rounded down (the rest is read from global memory).
__device__ __forceinline__ int row_copy_end(int r0, int r1, int n, int es) {
  const int g = granule(es);
  const int up = (r1 + g - 1) & ~(g - 1);
  const int ce = up <= n ? up : (r1 & ~(g - 1));
  return ce < r0 ? r0 : ce;
}

// Reader of the staged row operands of one stage (i is a compile-time
// constant at every call site, so everything stays in registers).
struct StagedRows {
  const unsigned char *area;  // first row-operand area of the buffer
  int rw;
  int r0;
  int nrows[kMaxRowVecs];
  const void *p[kMaxRowVecs];
  template <class T>
  __device__ __forceinline__ T get(int i, int row) const {
    const int lr = row - r0;
    if (lr < nrows[i]) return reinterpret_cast<const T *>(area + i * rw)[lr];
    return reinterpret_cast<const T *>(p[i])[row];
  }
};

// Accumulation-type value of a staged operand element.
template <class V>
__device__ __forceinline__ typename Acc<V>::type to_acc(V v) { return v; }
template <>
__device__ __forceinline__ double to_acc<f32w>(f32w v) {
  return (double)v.v;
}
template <>
__device__ __forceinline__ double to_acc<b16w>(b16w v) {
  return (double)__uint_as_float(((unsigned)v.v) << 16);
}
template <>
__device__ __forceinline__ float to_acc<__nv_bfloat16>(__nv_bfloat16 v) {
  return __uint_as_float(((unsigned)__bfloat16_as_ushort(v)) << 16);
}

// Element t of a small register array selected by a runtime index without
// dynamic indexing (which would move the array to local memory).
template <class T, int N>
__device__ __forceinline__ T pick(const T (&a)[N], int t) {
  T v = a[0];
#pragma unroll
  for (int q = 1; q < N; q++)
    if (t == q) v = a[q];
  return v;
}

// Plain vector loads of P adjacent slots from shared memory.
template <class V, int P>
struct SPack;
template <int P>
struct SPack<double, P> {
  static __device__ __forceinline__ void load(const double *p, double (&o)[P]) {
    if constexpr (P == 2) {
      const double2 v = *reinterpret_cast<const double2 *>(p);
      o[0] = v.x;
      o[1] = v.y;
    } else {
#pragma unroll
      for (int e = 0; e < P; e++) o[e] = p[e];
    }
  }
};
template <int P>
struct SPack<float, P> {
  static __device__ __forceinline__ void load(const float *p, float (&o)[P]) {
    if constexpr (P == 4) {
      const float4 v = *reinterpret_cast<const float4 *>(p);
      o[0] = v.x;
      o[1] = v.y;
      o[2] = v.z;
      o[3] = v.w;
    } else if constexpr (P == 2) {
      const float2 v = *reinterpret_cast<const float2 *>(p);
      o[0] = v.x;
      o[1] = v.y;
    } else {
      o[0] = p[0];
    }
  }
};
template <int P>
struct SPack<__nv_bfloat16, P> {
  static __device__ __forceinline__ void load(const __nv_bfloat16 *p, float (&o)[P]) {
    const unsigned short *u = reinterpret_cast<const unsigned short *>(p);
    if constexpr (P == 8) {
      const uint4 v = *reinterpret_cast<const uint4 *>(u);
      const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int h = 0; h < 4; h++) {
        o[2 * h] = bf16lo(w[h]);
        o[2 * h + 1] = bf16hi(w[h]);
      }
    } else if constexpr (P == 4) {
      const uint2 v = *reinterpret_cast<const uint2 *>(u);
      o[0] = bf16lo(v.x);
      o[1] = bf16hi(v.x);
      o[2] = bf16lo(v.y);
      o[3] = bf16hi(v.y);
    } else if constexpr (P == 2) {
      const unsigned v = *reinterpret_cast<const unsigned *>(u);
      o[0] = bf16lo(v);
      o[1] = bf16hi(v);
    } else {
      o[0] = bf16lo(u[0]);
    }
  }
};
template <int P>
struct SPack<f32w, P> {
  static __device__ __forceinline__ void load(const f32w *p, double (&o)[P]) {
    float f[P];
    SPack<float, P>::load(reinterpret_cast<const float *>(p), f);
#pragma unroll
    for (int e = 0; e < P; e++) o[e] = (double)f[e];
  }
};
template <int P>
struct SPack<b16w, P> {
  static __device__ __forceinline__ void load(const b16w *p, double (&o)[P]) {
    float f[P];
    SPack<__nv_bfloat16, P>::load(reinterpret_cast<const __nv_bfloat16 *>(p), f);
#pragma unroll
    for (int e = 0; e < P; e++) o[e] = (double)f[e];
  }
};

// Element range [a, e) of the window of an offset cluster [o0, o1] for rows
// [r0, r1) of an n-element vector: the rows' columns, widened to whole
// 16-byte granules.
template <class X>
__device__ __forceinline__ void window_range(int r0, int r1, int o0, int o1, int n, int &a,
                                             int &e) {
  const int g = granule((int)sizeof(X));
  int lo = r0 + o0, hi = r1 + o1;
  lo = lo < 0 ? 0 : lo;
  hi = hi > n ? n : hi;
  a = lo & ~(g - 1);
  e = (hi + g - 1) & ~(g - 1);
}

// Issue the copies of stage st (descriptor d, in every lane's registers)
// into buffer `buf`: one copy per lane (descriptor, slice pointers, values,
// index words, windows, row operands), each lane adding its bytes to the
// barrier's expected transactions; lane 0 then arrives.  Called by the whole
// producer warp.
template <class V, class X>
__device__ __forceinline__ void issue_stage(const SellView<V> &m,
                                            const StageDesc *__restrict__ stages, int st,
                                            const StageDesc &d, const X *__restrict__ x,
                                            const RowVecs &rv, const StreamLayout &L,
                                            unsigned char *buf, unsigned long long *bar) {
  const int lane = threadIdx.x & 31;
  const int r0 = d.s0 * kSlice, r1 = min(m.n, d.s1 * kSlice);
  const unsigned char *src = nullptr;
  unsigned char *dst = nullptr;
  int bytes = 0;
  StageDerived *dv = reinterpret_cast<StageDerived *>(buf + kDerivedOfs);
  if (lane == 0) {
    src = reinterpret_cast<const unsigned char *>(stages + st);
    dst = buf;
    bytes = kDescBytes;
  } else if (lane <= 2) {
    const int pa = d.s0 & ~3, pe = (d.s1 + 1 + 3) & ~3;
    src = reinterpret_cast<const unsigned char *>(lane == 1 ? m.sptr : m.iptr) + pa * 4;
    dst = buf + kDescBytes + (lane - 1) * kPtrChunkBytes;
    bytes = (pe - pa) * 4;
  } else if (lane == 3) {
    src = reinterpret_cast<const unsigned char *>(m.val) + (size_t)d.vstart * sizeof(V);
    dst = buf + kHeaderBytes;
    bytes = d.vbytes;
  } else if (lane == 4) {
    src = reinterpret_cast<const unsigned char *>(m.idx) + d.ibyte0;
    dst = buf + kHeaderBytes + L.vb;
    bytes = d.ibytes;
  } else if (lane < 5 + kStageMaxOffsets) {
    // offset k's window cluster c (first offset o0, last o1); the cluster's
    // first offset copies the window into area c
    const int k = lane - 5;
    const int noff = d.noff & 0xff;
    int wofs = -r0;
    if (k < noff) {
      // cluster leaders (bit q: offset q starts a cluster); k's cluster runs
      // from the last leader <= k to before the next leader
      const unsigned lead = ((unsigned)d.noff >> 8) & 0xffu;
      const unsigned upto = lead & ((2u << k) - 1u);
      const int kc = __popc(upto) - 1, k0 = 31 - __clz(upto);
      const unsigned after = lead & ~((2u << k) - 1u);
      const int k1 = after ? __ffs(after) - 2 : noff - 1;
      const int o = pick(d.off, k), o0 = pick(d.off, k0), o1 = pick(d.off, k1);
      int a, e;
      window_range<X>(r0, r1, o0, o1, m.n, a, e);
      if (k == k0) {
        src = reinterpret_cast<const unsigned char *>(x + a);
        dst = buf + kHeaderBytes + L.vb + L.ib + kc * L.xw;
        bytes = (e - a) * (int)sizeof(X);
      }
      wofs = kc * (L.xw / (int)sizeof(X)) + o - a;
    }
    dv->wofs[k] = wofs;
  } else if (lane < 5 + kStageMaxOffsets + kMaxRowVecs) {
    const int i = lane - 5 - kStageMaxOffsets;
    const void *p = pick(rv.p, i);
    const int es = pick(rv.es, i);
    int nrows = 0;
    if (i < L.nrv && p) {
      const int ce = row_copy_end(r0, r1, m.n, es);
      src = reinterpret_cast<const unsigned char *>(p) + (size_t)r0 * es;
      dst = buf + kHeaderBytes + L.vb + L.ib + L.nwin * L.xw + i * L.rw;
      bytes = (ce - r0) * es;
      nrows = ce - r0;
    }
    dv->nrows[i] = nrows;
  }
  if (bytes > 0) {
    mbar_add_tx(bar, (unsigned)bytes);
    bulk_g2s(dst, src, (unsigned)bytes, bar);
  }
  // the derived words are plain shared-memory stores: the warp barrier
  // orders them before lane 0's arrive, whose release the consumers'
  // acquiring wait on the full barrier pairs with
  __syncwarp();
  if (lane == 0) mbar_arrive(bar);
}

// A descriptor travels as four int4 words (layout of StageDesc):
// {s0, s1, vstart, vbytes}, {ibyte0 lo, ibyte0 hi, ibytes, noff}, off[0..3], off[4..7].
__device__ __forceinline__ int4 shfl4(const int4 &v, int src) {
  return make_int4(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
                   __shfl_sync(0xffffffffu, v.z, src), __shfl_sync(0xffffffffu, v.w, src));
}
__device__ __forceinline__ StageDesc desc_from(const int4 &a, const int4 &b, const int4 &c,
                                               const int4 &e) {
  StageDesc d;
  d.s0 = a.x;
  d.s1 = a.y;
  d.vstart = a.z;
  d.vbytes = a.w;
  d.ibyte0 = (long long)(unsigned)b.x | ((long long)b.y << 32);
  d.ibytes = b.z;
  d.noff = b.w;
  d.off[0] = c.x;
  d.off[1] = c.y;
  d.off[2] = c.z;
  d.off[3] = c.w;
  d.off[4] = e.x;
  d.off[5] = e.y;
  d.off[6] = e.z;
  d.off[7] = e.w;
  return d;
}

// Per-stage constants of a uniform stage, held in registers for the row
// loop: element k of a row lives at window-area index row + wofs[k].
struct UniformStage {
  int noff;
  int wofs[kStageMaxOffsets];
};
__device__ __forceinline__ void uniform_stage(const StageDesc &d, const StageDerived &dv,
                                              UniformStage &u) {
  u.noff = d.noff & 0xff;
  static_assert(kStageMaxOffsets == 8, "the offsets' shifts are read as two 16-byte words");
  const int4 a = *reinterpret_cast<const int4 *>(dv.wofs);
  const int4 b = *reinterpret_cast<const int4 *>(dv.wofs + 4);
  u.wofs[0] = a.x;
  u.wofs[1] = a.y;
  u.wofs[2] = a.z;
  u.wofs[3] = a.w;
  u.wofs[4] = b.x;
  u.wofs[5] = b.y;
  u.wofs[6] = b.z;
  u.wofs[7] = b.w;
}

// Dot of the lane's row of slice s with x, everything read from the stage
// buffer `buf` (d: the descriptor copy in shared memory).
template <int P, class V, class X>
__device__ __forceinline__ typename Acc<V>::type stream_row_dot(const SellView<V> &m,
                                                                const StageDesc &d,
                                                                const UniformStage &u, int s,
                                                                const unsigned char *buf,
                                                                const StreamLayout &L,
                                                                const X *__restrict__ x) {
  using A = typename Acc<V>::type;
  const int lane = threadIdx.x & 31;
  const int row = s * kSlice + lane;
  const int *spc = reinterpret_cast<const int *>(buf + kDescBytes) + (d.s0 & 3);
  const int *ipc = reinterpret_cast<const int *>(buf + kDescBytes + kPtrChunkBytes) + (d.s0 & 3);
  const int sp0 = spc[s - d.s0], sp1 = spc[s - d.s0 + 1];
  const int w = (sp1 - sp0) / kSlice;
  const V *sv = reinterpret_cast<const V *>(buf + kHeaderBytes) + (sp0 - d.vstart) + lane * P;
  A acc = A(0);
  if (u.noff > 0) {
    // uniform stage: slot k <-> offset k of the stage; windows in shared
    // memory.  w <= kStageMaxOffsets rounded up to P: the loop unrolls.
    const X *win = reinterpret_cast<const X *>(buf + kHeaderBytes + L.vb + L.ib) + row;
#pragma unroll
    for (int k0 = 0; k0 < kStageMaxOffsets; k0 += P) {
      if (k0 < w) {
        A v[P];
        SPack<V, P>::load(sv + (k0 / P) * (kSlice * P), v);
#pragma unroll
        for (int e = 0; e < P; e++) {
          // slots past the stage's offsets hold zeros and are skipped
          const int k = k0 + e;
          if (k < kStageMaxOffsets && v[e] != A(0))
            acc = madd(v[e], (A)win[u.wofs[k < kStageMaxOffsets ? k : 0]], acc);
        }
      }
    }
  } else {
    const int ip0 = ipc[s - d.s0], ip1 = ipc[s - d.s0 + 1];
    const int *si = reinterpret_cast<const int *>(buf + kHeaderBytes + L.vb) +
                    (int)(((long long)ip0 * 4 - d.ibyte0) / 4);
    if (ip1 - ip0 == w) {
      // offset mode, offsets from shared memory, gathers from global
      for (int k0 = 0; k0 < w; k0 += P) {
        A v[P];
        SPack<V, P>::load(sv + (k0 / P) * (kSlice * P), v);
        A xv[P];
#pragma unroll
        for (int e = 0; e < P; e++) {
          const int c = row + si[k0 + e];
          xv[e] = (v[e] != A(0) && (unsigned)c < (unsigned)m.n) ? (A)__ldg(x + c) : A(0);
        }
#pragma unroll
        for (int e = 0; e < P; e++) acc = madd(v[e], xv[e], acc);
      }
    } else {
      // per-slot columns from shared memory, gathers from global
      const int *sc = si + lane * P;
      for (int k0 = 0; k0 < w; k0 += P) {
        A v[P];
        SPack<V, P>::load(sv + (k0 / P) * (kSlice * P), v);
        A xv[P];
#pragma unroll
        for (int e = 0; e < P; e++) {
          const int c = sc[(k0 / P) * (kSlice * P) + e];
          xv[e] = (v[e] != A(0) && (unsigned)c < (unsigned)m.n) ? (A)__ldg(x + c) : A(0);
        }
#pragma unroll
        for (int e = 0; e < P; e++) acc = madd(v[e], xv[e], acc);
      }
    }
  }
  return acc;
}

// Epilogues that reduce per slice (SliceSums) define end_slice(s); it runs
// with the whole warp once slice s is done.  Others have nothing to do.
template <class E>
__device__ __forceinline__ auto slice_end_impl(E &e, int s, int) -> decltype(e.end_slice(s), void()) {
  e.end_slice(s);
}
template <class E>
__device__ __forceinline__ void slice_end_impl(E &, int, long) {}
template <class E>
__device__ __forceinline__ void slice_end(E &e, int s) { slice_end_impl(e, s, 0); }

// Persistent streaming traversal: for every row r < n of M,
// epi.post(r, acc, rows) with acc = (M x)[r] and `rows` the reader of the
// staged row operands epi.row_vecs().  Must be called by all kStreamThreads
// threads; the last warp produces, the others consume.  RMAX bounds L.R
// (slices per consumer warp and stage).  The block takes stages j0,
// j0 + jstride, ... (j0 < 0: blockIdx.x and gridDim.x).  Returns false (and
// sets *status) if a wait ran past its limit.
template <int P, int RMAX, class V, class X, class Epi>
__device__ __forceinline__ bool stream_rows(const SellView<V> &m,
                                            const StageDesc *__restrict__ stages, int nstages,
                                            const X *__restrict__ x, const StreamLayout &L,
                                            Epi &epi, int *status, int j0 = -1,
                                            int jstride = 0) {
  const RowVecs rv = epi.row_vecs();
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned long long *full = reinterpret_cast<unsigned long long *>(smem);
  unsigned long long *empty = full + 8;
  unsigned char *base = smem + 128;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (j0 < 0) {
    j0 = (int)blockIdx.x;
    jstride = (int)gridDim.x;
  }
  const int G = jstride;
  const int mine = (j0 < nstages) ? (nstages - j0 + G - 1) / G : 0;
  const int stage_slices = kConsumerWarps * L.R;
  if (tid == 0) {
    for (int b = 0; b < L.D; b++) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], kConsumerWarps);
    }
    fence_mbar_init();
  }
  __syncthreads();
  bool ok = true;
  if (warp == kConsumerWarps) {
    // producer: the warp loads the next 32 descriptors (one per lane), lane
    // 0 issues each stage's copies as soon as its buffer is free
    int j = 0;
    for (int jb = 0; jb < mine && ok; jb += 32) {
      int4 q0 = make_int4(0, 0, 0, 0), q1 = q0, q2 = q0, q3 = q0;
      const int jl = jb + lane;
      if (jl < mine) {
        const int4 *src = reinterpret_cast<const int4 *>(stages + j0 + jl * G);
        q0 = __ldg(src);
        q1 = __ldg(src + 1);
        q2 = __ldg(src + 2);
        q3 = __ldg(src + 3);
      }
      const int nb = min(32, mine - jb);
      for (int jj = 0; jj < nb; jj++) {
        const StageDesc d = desc_from(shfl4(q0, jj), shfl4(q1, jj), shfl4(q2, jj), shfl4(q3, jj));
        j = jb + jj;
        const int b = j % L.D;
        int go = 1;
        if (lane == 0 && j >= L.D && !mbar_wait(&empty[b], (unsigned)(((j / L.D) - 1) & 1)))
          go = 0;
        go = __shfl_sync(0xffffffffu, go, 0);
        if (!go) {
          ok = false;
          break;
        }
        issue_stage(m, stages, j0 + j * G, d, x, rv, L, base + (size_t)b * L.stage,
                    &full[b]);
        j++;
      }
    }
    if (!ok && lane == 0) {
      atomicExch(status, 1);
      // j: first stage not issued; wait (bounded) for the copies already issued
      for (int k = (j > L.D ? j - L.D : 0); k < j; k++)
        mbar_wait(&full[k % L.D], (unsigned)((k / L.D) & 1));
    }
    __syncwarp();
  } else {
    for (int j = 0; j < mine; j++) {
      const int b = j % L.D;
      if (!mbar_wait(&full[b], (unsigned)((j / L.D) & 1))) {
        if (lane == 0) atomicExch(status, 1);
        ok = false;
        break;
      }
      const unsigned char *buf = base + (size_t)b * L.stage;
      const StageDesc &d = *reinterpret_cast<const StageDesc *>(buf);
      const StageDerived &dv = *reinterpret_cast<const StageDerived *>(buf + kDerivedOfs);
      UniformStage u;
      uniform_stage(d, dv, u);
      StagedRows sr;
      sr.area = buf + kHeaderBytes + L.vb + L.ib + L.nwin * L.xw;
      sr.rw = L.rw;
      sr.r0 = d.s0 * kSlice;
      {
        static_assert(kMaxRowVecs == 3, "staged row counts are read as one 16-byte word");
        const int4 c = *reinterpret_cast<const int4 *>(dv.nrows);
        sr.nrows[0] = c.x;
        sr.nrows[1] = c.y;
        sr.nrows[2] = c.z;
#pragma unroll
        for (int i = 0; i < kMaxRowVecs; i++) sr.p[i] = rv.p[i];
      }
      const int sfirst = d.s0 + warp * L.R;
#pragma unroll
      for (int r = 0; r < RMAX; r++) {
        const int s = sfirst + r;
        if (r < L.R && s < d.s1) {
          const auto acc = stream_row_dot<P>(m, d, u, s, buf, L, x);
          const int row = s * kSlice + lane;
          if (row < m.n) epi.post(row, acc, sr);
          slice_end(epi, s);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[b]);
    }
  }
  __syncthreads();
  return ok;
}

// Epilogues of the apply's two sweeps: t = D^-1 .* acc (D staged as a row
// operand) and y = alpha*acc + beta*y (y staged when beta != 0).
template <class V, class T>
struct EpiDscale {
  const V *__restrict__ d;
  T *__restrict__ t;
  static constexpr int kRowVecs = 1;
  __device__ __forceinline__ RowVecs row_vecs() const {
    return RowVecs{{d, nullptr, nullptr}, {(int)sizeof(V), 0, 0}};
  }
  template <class A>
  __device__ __forceinline__ void post(int row, A acc, const StagedRows &r) const {
    t[row] = (T)(to_acc(r.get<V>(0, row)) * acc);
  }
};

struct EpiAxpby {
  double alpha, beta;
  double *__restrict__ y;
  static constexpr int kRowVecs = 1;
  __device__ __forceinline__ RowVecs row_vecs() const {
    return RowVecs{{beta == 0.0 ? nullptr : y, nullptr, nullptr}, {8, 0, 0}};
  }
  template <class A>
  __device__ __forceinline__ void post(int row, A acc, const StagedRows &r) const {
    y[row] = axpby_row(alpha, (double)acc, beta, beta == 0.0 ? 0.0 : r.get<double>(0, row));
  }
};

// Shared-memory budgets (bytes): one stage buffer at most, per block target,
// per block maximum (opt-in carve-out) and per SM.
constexpr int kStreamStageMax = 64 * 1024;
constexpr int kStreamBlockBudget = 52 * 1024;
constexpr int kStreamSmemMax = 227 * 1024;
constexpr long long kStreamSmemSM = 228 * 1024;

// Launch geometry for a streaming kernel whose gathered vector has elements
// of xs bytes: fills L and returns the grid (0 if the matrix is not
// streamable).
// nrv: row-operand vectors the epilogue stages (elements of at most 8 bytes).
int stream_plan(const DevSell &m, int xs, int nrv, StreamLayout &L, size_t &smem_bytes);
// Slices per consumer warp and stage for a value type (RMAX of stream_rows).
template <class V>
constexpr int stream_rmax() { return sizeof(V) >= 8 ? 1 : (int)(8 / sizeof(V)); }
bool stream_enabled(int prec);
bool stream_enabled_sweep1(int prec);  // sweep 1 (t = D^-1 M x) of the apply
int sm_count();
// A persistent grid of at most `grid` blocks, capped at the blocks of
// `kernel` that can be resident at once (registers and shared memory), so
// a kernel that needs more registers never runs a second partial wave.
int occupancy_grid(const void *kernel, int threads, size_t smem, int grid);
// Allow `bytes` of dynamic shared memory for kernel; false if refused.
bool set_smem_attr(const void *kernel, size_t bytes);

}  // namespace dev
}  // namespace ainv
