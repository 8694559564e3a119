// Continuous-batching solve server: many BiCGSTAB solves, on different
// resident operators and of different sizes, advance together through one
// captured CUDA graph of batched kernels.
//
// Each request occupies a slot.  A device table describes every slot (its
// operator A, its AINV / INVK / INVT factors, its vectors) and maps each
// block of a fixed launch grid to a slot; every batched kernel starts by
// looking up its block's slot there, so one graph serves any mix of
// requests and admitting or retiring a request only rewrites the table
// between graph launches.  One graph launch advances every active slot by
// `iters` iterations of the same recurrence as the single-solve loop
// (psb_dbicgstab with istop=2; true-residual replacement every 50
// iterations for FP32/BF16 factors; convergence confirmed on b - A x).
//
// Results do not depend on the mix: every reduction is computed over fixed
// 512-row chunks, each chunk summed by one block in a fixed order, and the
// chunk sums folded in chunk order; which block handles which chunk, and how
// many blocks a slot gets, changes nothing.  A request's iterates are thus
// bit-identical whether it runs alone or beside others.
//
// Requests on the same operator share its reads.  Active slots are grouped
// by operator (up to kMaxMembers per group); the kernels that read A or the
// factors (the two sweeps and the three A products) walk the group's
// chunks, and for each chunk compute the rows of every member in turn, so a
// chunk's values and indices come from HBM once and from the cache for the
// other members.  The per-member arithmetic is that of a slot alone.
//
// The host side is an engine thread: requests queue on submit, are admitted
// first-come first-served while a slot is free and their vectors fit in the
// server's device arena (sized from free HBM at creation), are launched
// together, and are retired (x copied back, slot and memory released) as
// soon as their state reports completion.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "kstate.cuh"
#include "sell_device.cuh"

namespace ainv {
namespace srv {

using namespace dev;
using namespace kstate;

constexpr int kMaxSlots = 64;
constexpr int kMaxMembers = 8;  // slots per operator group
constexpr int kMaxGrid = 4096;
constexpr int kGroupS = 2;                    // slices per warp in one chunk
constexpr int kChunkRows = kBlock * kGroupS;  // 512 rows: 8 warps x 2 slices
constexpr int kRecheck = 50;                  // true-residual period for FP32/BF16 factors

enum Vec { VX = 0, VB, VR, VRT, VP, VV, VF, VS, VZ, VT, VRTRUE, kNumVec };
enum Phase { kIdle = 0, kInitPhase = 1, kRun = 2 };

struct Mat {
  int n, nslices, pack, prec;
  const int *sptr, *iptr, *idx;
  const void *val;
};

struct SlotDesc {
  int b0, nb;  // launch blocks [b0, b0 + nb)
  int n, nchunks;
  Mat A, wt, z;
  const void *d;  // D^-1 in the factors' precision
  void *t;        // apply intermediate: double (FP64 factors) or float
  double *vec[kNumVec];
  double *partials;  // 3 * nchunks
};

// Slots on one operator, served together by the operator kernels.
struct GroupDesc {
  int b0, nb;  // launch blocks [b0, b0 + nb)
  int nchunks, nmem;
  short mem[kMaxMembers];
};

struct Table {
  SlotDesc slot[kMaxSlots];
  GroupDesc group[kMaxSlots];
  short block_slot[kMaxGrid];   // vector kernels: the block's slot, -1 idle
  short block_group[kMaxGrid];  // operator kernels: the block's group, -1 idle
};

struct SlotState {
  KState k;
  int phase;
  int pad[3];
};

inline Mat mat_of(const DevSell &m) {
  return Mat{m.n, m.nslices, m.pack, m.prec, m.sptr, m.iptr, m.idx, m.val};
}

// ---------------------------------------------------------------- device --
template <class V>
__device__ __forceinline__ SellView<V> sview(const Mat &m) {
  return SellView<V>{m.n, m.nslices, m.sptr, m.iptr, m.idx, (const V *)m.val};
}

// Rows of chunk c of M (warp w takes slice group 8c + w), epi(row, acc).
// Values and indices stay cached (a group's members read them in turn).
template <class V, int P, class X, class Epi>
__device__ __forceinline__ void chunk_rows_p(const Mat &mm, int c, const X *__restrict__ x,
                                             Epi &epi) {
  const SellView<V> m = sview<V>(mm);
  const int g = c * kWarps + (threadIdx.x >> 5);
  const int ngroups = (m.nslices + kGroupS - 1) / kGroupS;
  if (g >= ngroups) return;  // warp-uniform
  GroupCtx<kGroupS> ctx;
  group_ctx(m, g, ctx);
  typename Acc<V>::type acc[kGroupS];
  group_dot<P, 4, true, false>(m, ctx, g, x, acc);
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < kGroupS; q++) {
    const int row = (g * kGroupS + q) * kSlice + lane;
    if (row < m.n) epi(row, acc[q]);
  }
}

template <class V, class X, class Epi>
__device__ __forceinline__ void chunk_rows(const Mat &m, int c, const X *__restrict__ x,
                                           Epi &epi) {
  if constexpr (pack_ok<V, 2>()) {
    if (m.pack == 2) return chunk_rows_p<V, 2>(m, c, x, epi);
  }
  if constexpr (pack_ok<V, 4>()) {
    if (m.pack == 4) return chunk_rows_p<V, 4>(m, c, x, epi);
  }
  if constexpr (pack_ok<V, 8>()) {
    if (m.pack == 8) return chunk_rows_p<V, 8>(m, c, x, epi);
  }
  chunk_rows_p<V, 1>(m, c, x, epi);
}

// Per-chunk sums: the block's fixed tree, stored at partials[i*nchunks + c].
template <int NV>
__device__ __forceinline__ void chunk_store(double (&v)[NV], double *__restrict__ partials,
                                            int nchunks, int c) {
  block_sum<NV>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) partials[i * nchunks + c] = v[i];
  }
}

// The block's chunks lb, lb+nb, ... in batches of kChunkBatch: body(c, pr)
// accumulates chunk c's NV sums in pr; each warp folds its lanes (fixed
// shuffle tree) into a shared slot without waiting, and one barrier per
// batch lets the block fold its warps in order and store the chunk sums at
// partials[i*nchunks + c] -- the same values chunk_store gives.
constexpr int kChunkBatch = 4;
template <int NV, class Body>
__device__ __forceinline__ void for_chunks(int lb, int nb, int nchunks,
                                           double *__restrict__ partials, Body &&body) {
  __shared__ double sh[kChunkBatch][NV][kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c0 = lb; c0 < nchunks; c0 += kChunkBatch * nb) {
#pragma unroll
    for (int q = 0; q < kChunkBatch; q++) {
      const int c = c0 + q * nb;
      if (c >= nchunks) break;  // block-uniform
      double pr[NV];
#pragma unroll
      for (int i = 0; i < NV; i++) pr[i] = 0.0;
      body(c, pr);
#pragma unroll
      for (int i = 0; i < NV; i++) {
        double v = pr[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) sh[q][i][warp] = v;
      }
    }
    __syncthreads();
    if (threadIdx.x < kChunkBatch * NV) {
      const int q = threadIdx.x / NV, i = threadIdx.x % NV, c = c0 + q * nb;
      if (c < nchunks) {
        double s = 0.0;
        for (int w = 0; w < kWarps; w++) s += sh[q][i][w];
        partials[i * nchunks + c] = s;
      }
    }
    __syncthreads();
  }
}

// for_chunks for the members of a group: body(c, i, pr) accumulates member
// i's NV sums of chunk c; the chunk sums of member i go to its slot's
// partials, folded exactly as for_chunks folds them.
template <int NV, class Body>
__device__ __forceinline__ void for_chunks_group(const Table *tab, const GroupDesc &gd,
                                                 unsigned act, int lb, Body &&body) {
  __shared__ double sh[kChunkBatch][kMaxMembers][NV][kWarps];
  __shared__ double *part[kMaxMembers];
  if ((int)threadIdx.x < gd.nmem) part[threadIdx.x] = tab->slot[gd.mem[threadIdx.x]].partials;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nb = gd.nb, nchunks = gd.nchunks;
  for (int c0 = lb; c0 < nchunks; c0 += kChunkBatch * nb) {
#pragma unroll
    for (int q = 0; q < kChunkBatch; q++) {
      const int c = c0 + q * nb;
      if (c >= nchunks) break;  // block-uniform
      for (int i = 0; i < gd.nmem; i++) {
        if (!((act >> i) & 1u)) continue;
        double pr[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) pr[k] = 0.0;
        body(c, i, pr);
#pragma unroll
        for (int k = 0; k < NV; k++) {
          double v = pr[k];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
          if (lane == 0) sh[q][i][k][warp] = v;
        }
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kChunkBatch * kMaxMembers * NV; e += blockDim.x) {
      const int q = e / (kMaxMembers * NV), i = (e / NV) % kMaxMembers, k = e % NV;
      const int c = c0 + q * nb;
      if (c < nchunks && i < gd.nmem && ((act >> i) & 1u)) {
        double sum = 0.0;
        for (int w = 0; w < kWarps; w++) sum += sh[q][i][k][w];
        part[i][k * nchunks + c] = sum;
      }
    }
    __syncthreads();
  }
}

// The slot's last block (atomic ticket, no waiting) folds the chunk sums in
// chunk order; true in that block, totals in thread 0.
template <int NV>
__device__ __forceinline__ bool slot_fold(double (&v)[NV], const double *partials, int nchunks,
                                          int nb, unsigned *ticket) {
  __shared__ bool is_last;
  if (threadIdx.x == 0) {
    __threadfence();
    is_last = atomicAdd(ticket, 1u) == (unsigned)nb - 1;
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
#pragma unroll
  for (int i = 0; i < NV; i++) {
    double s = 0.0;
    for (int c = threadIdx.x; c < nchunks; c += blockDim.x) s += __ldcg(partials + i * nchunks + c);
    v[i] = s;
  }
  block_sum<NV>(v);
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

// Block prologue: the block's slot, or -1.  `need` decides from the slot's
// state whether this kernel acts on it; it is evaluated identically by
// every block of the slot (the state changes only in the slot's last block,
// after all blocks have passed this point).
#define SRV_PROLOGUE(need)                                        \
  const int slot = tab->block_slot[blockIdx.x];                   \
  if (slot < 0) return;                                           \
  SlotState *ss = sts + slot;                                     \
  KState *st = &ss->k;                                            \
  if (!(need)) return;                                            \
  const SlotDesc &sd = tab->slot[slot];                           \
  const int lb = blockIdx.x - sd.b0, nb = sd.nb, n = sd.n;        \
  (void)n;                                                        \
  (void)lb;

#define SRV_RUNNING (ss->phase == kRun && !st->done)

// Prologue of the operator kernels: the block's group (copied out of the
// table, so that the stores of the inner loops cannot force reloads), or
// return.
#define SRV_GROUP_PROLOGUE                                         \
  const int grp = tab->block_group[blockIdx.x];                   \
  if (grp < 0) return;                                            \
  const GroupDesc gd = tab->group[grp];                           \
  const int lb = blockIdx.x - gd.b0;

// The members' vector pointers an operator kernel needs (up to 5 each),
// staged once per block in shared memory; the operator (A, W^T, Z, D^-1)
// is the same for every member and is read from member 0.
constexpr int kMemberVecs = 5;
struct MemberVecs {
  void *p[kMaxMembers][kMemberVecs];
};
template <class F>
__device__ __forceinline__ void stage_members(const Table *tab, const GroupDesc &gd,
                                              MemberVecs &mv, F &&pick) {
  if ((int)threadIdx.x < gd.nmem) pick(tab->slot[gd.mem[threadIdx.x]], mv.p[threadIdx.x]);
  __syncthreads();
}

__device__ __forceinline__ bool slot_running(const SlotState *ss) {
  return ss->phase == kRun && !ss->k.done;
}

// r = rt = b, x = p = v = 0, ||b||; the first rho = r.r (x0 = 0).
__global__ void __launch_bounds__(kBlock) k_srv_init(const Table *tab, SlotState *sts) {
  SRV_PROLOGUE(ss->phase == kInitPhase)
  double *x = sd.vec[VX], *r = sd.vec[VR], *rt = sd.vec[VRT], *p = sd.vec[VP], *v = sd.vec[VV];
  const double *b = sd.vec[VB];
  for_chunks<1>(lb, nb, sd.nchunks, sd.partials, [&](int c, double (&pr)[1]) {
#pragma unroll
    for (int h = 0; h < kGroupS; h++) {
      const int i = c * kChunkRows + h * kBlock + threadIdx.x;
      if (i < n) {
        const double bi = b[i];
        x[i] = 0.0;
        r[i] = bi;
        rt[i] = bi;
        p[i] = 0.0;
        v[i] = 0.0;
        pr[0] += bi * bi;
      }
    }
  });
  double tot[1] = {0.0};
  if (slot_fold<1>(tot, sd.partials, sd.nchunks, nb, &st->ticket[0]) && threadIdx.x == 0) {
    const double bn = sqrt(tot[0]);
    st->bn2 = (bn == 0.0) ? 1.0 : bn;
    const double pr3[3] = {tot[0], tot[0], 0.0};
    finish_dots<kInit>(st, pr3, false, nullptr);
    ss->phase = kRun;
  }
}

// p = r (first iteration) or p = r + beta (p - omega v).
__global__ void __launch_bounds__(kBlock) k_srv_p(const Table *tab, SlotState *sts) {
  SRV_PROLOGUE(SRV_RUNNING)
  const double *r = sd.vec[VR], *v = sd.vec[VV];
  double *p = sd.vec[VP];
  const bool first = st->iter == 0;
  const double beta = st->beta, omega = st->omega;
  for (int i = lb * kBlock + threadIdx.x; i < n; i += nb * kBlock)
    p[i] = first ? r[i] : r[i] + beta * (p[i] - omega * v[i]);
}

// s = r - alpha v.
__global__ void __launch_bounds__(kBlock) k_srv_s(const Table *tab, SlotState *sts) {
  SRV_PROLOGUE(SRV_RUNNING)
  const double *r = sd.vec[VR], *v = sd.vec[VV];
  double *s = sd.vec[VS];
  const double alpha = st->alpha;
  for (int i = lb * kBlock + threadIdx.x; i < n; i += nb * kBlock) s[i] = r[i] - alpha * v[i];
}

// Sweep 1 of the apply for the active members of a group:
// t = D^-1 .* (W^T src), chunk by chunk, every member in turn.
template <class V, class T>
__device__ __forceinline__ void sweep1_group(const Mat &wt, const V *__restrict__ d,
                                             const GroupDesc &gd, const MemberVecs &mv,
                                             unsigned act, int lb) {
  for (int c = lb; c < gd.nchunks; c += gd.nb)
    for (int i = 0; i < gd.nmem; i++) {
      if (!((act >> i) & 1u)) continue;
      const double *src = (const double *)mv.p[i][0];
      T *__restrict__ t = (T *)mv.p[i][1];
      auto epi = [&](int row, auto acc) { t[row] = (T)(ldd(d + row) * acc); };
      chunk_rows<V>(wt, c, src, epi);
    }
}

// Factor precisions come in two kernel families, so each kernel's register
// budget is that of its own value types: FP64 / FP32 / BF16 (ACC = false)
// and the FP64-accumulating FP32 / BF16 storage (ACC = true).
__host__ __device__ inline bool acc64_prec(int prec) {
  return prec == AINV_PREC_FP32_ACC64 || prec == AINV_PREC_BF16_ACC64;
}

// Members of the group that run the sweeps of family ACC (all members share
// the operator, hence its precision).
template <bool ACC>
__device__ __forceinline__ unsigned sweep_members(const Table *tab, const SlotState *sts,
                                                  const GroupDesc &gd, int prec) {
  if (acc64_prec(prec) != ACC) return 0u;
  unsigned act = 0u;
  for (int i = 0; i < gd.nmem; i++)
    if (slot_running(sts + gd.mem[i])) act |= 1u << i;
  return act;
}

template <bool ACC>
__global__ void __launch_bounds__(kBlock) k_srv_sweep1(const Table *tab, SlotState *sts,
                                                       int src) {
  SRV_GROUP_PROLOGUE
  const Mat wt = tab->slot[gd.mem[0]].wt;
  const void *d = tab->slot[gd.mem[0]].d;
  const unsigned act = sweep_members<ACC>(tab, sts, gd, wt.prec);
  if (!act) return;
  __shared__ MemberVecs mv;
  stage_members(tab, gd, mv, [&](const SlotDesc &sd, void *(&p)[kMemberVecs]) {
    p[0] = sd.vec[src];
    p[1] = sd.t;
  });
  if constexpr (ACC) {
    if (wt.prec == AINV_PREC_FP32_ACC64)
      sweep1_group<f32w, double>(wt, (const f32w *)d, gd, mv, act, lb);
    else
      sweep1_group<b16w, double>(wt, (const b16w *)d, gd, mv, act, lb);
  } else {
    switch (wt.prec) {
      case AINV_PREC_FP64: sweep1_group<double, double>(wt, (const double *)d, gd, mv, act, lb); break;
      case AINV_PREC_FP32: sweep1_group<float, float>(wt, (const float *)d, gd, mv, act, lb); break;
      default:
        sweep1_group<__nv_bfloat16, float>(wt, (const __nv_bfloat16 *)d, gd, mv, act, lb);
        break;
    }
  }
}

// Sweep 2 of the apply for the active members: dst = Z t.
template <class V, class T>
__device__ __forceinline__ void sweep2_group(const Mat &z, const GroupDesc &gd,
                                             const MemberVecs &mv, unsigned act, int lb) {
  for (int c = lb; c < gd.nchunks; c += gd.nb)
    for (int i = 0; i < gd.nmem; i++) {
      if (!((act >> i) & 1u)) continue;
      const T *t = (const T *)mv.p[i][0];
      double *__restrict__ y = (double *)mv.p[i][1];
      auto epi = [&](int row, auto acc) { y[row] = 1.0 * (double)acc; };
      chunk_rows<V>(z, c, t, epi);
    }
}

template <bool ACC>
__global__ void __launch_bounds__(kBlock) k_srv_sweep2(const Table *tab, SlotState *sts,
                                                       int dst) {
  SRV_GROUP_PROLOGUE
  const Mat z = tab->slot[gd.mem[0]].z;
  const unsigned act = sweep_members<ACC>(tab, sts, gd, z.prec);
  if (!act) return;
  __shared__ MemberVecs mv;
  stage_members(tab, gd, mv, [&](const SlotDesc &sd, void *(&p)[kMemberVecs]) {
    p[0] = sd.t;
    p[1] = sd.vec[dst];
  });
  if constexpr (ACC) {
    if (z.prec == AINV_PREC_FP32_ACC64)
      sweep2_group<f32w, double>(z, gd, mv, act, lb);
    else
      sweep2_group<b16w, double>(z, gd, mv, act, lb);
  } else {
    switch (z.prec) {
      case AINV_PREC_FP64: sweep2_group<double, double>(z, gd, mv, act, lb); break;
      case AINV_PREC_FP32: sweep2_group<float, float>(z, gd, mv, act, lb); break;
      default: sweep2_group<__nv_bfloat16, float>(z, gd, mv, act, lb); break;
    }
  }
}

// y = A x with the dots of MODE, as the single-solve SpMV kernels:
//   kBicgSigma: v = A f, sigma = rt.v, alpha = rho/sigma
//   kBicgOmega: t = A z, omega = (t.s)/(t.t)
//   kTrueRes:   rtrue = b - A x against r (periodic, and on a convergence claim)
template <int MODE>
__device__ __forceinline__ bool srv_spmv_active(const SlotState *ss, bool *verify) {
  const KState *st = &ss->k;
  *verify = false;
  if (ss->phase != kRun) return false;
  if (MODE == kTrueRes) {
    *verify = st->done && st->status == AINV_SUCCESS && !st->verified;
    const bool periodic = !st->done && st->check_every > 0 && st->iter > 0 &&
                          st->iter % st->check_every == 0;
    return *verify || periodic;
  }
  return !st->done;
}

template <int MODE>
__global__ void __launch_bounds__(kBlock, 4) k_srv_spmv(const Table *tab, SlotState *sts) {
  SRV_GROUP_PROLOGUE
  unsigned act = 0u, ver = 0u;
  for (int i = 0; i < gd.nmem; i++) {
    bool v;
    if (srv_spmv_active<MODE>(sts + gd.mem[i], &v)) {
      act |= 1u << i;
      if (v) ver |= 1u << i;
    }
  }
  if (!act) return;
  const Mat A = tab->slot[gd.mem[0]].A;
  __shared__ MemberVecs mv;
  stage_members(tab, gd, mv, [&](const SlotDesc &sd, void *(&p)[kMemberVecs]) {
    if (MODE == kBicgSigma) {
      p[0] = sd.vec[VF];
      p[1] = sd.vec[VV];
      p[2] = sd.vec[VRT];
    } else if (MODE == kBicgOmega) {
      p[0] = sd.vec[VZ];
      p[1] = sd.vec[VT];
      p[2] = sd.vec[VS];
    } else {
      p[0] = sd.vec[VX];
      p[1] = sd.vec[VRTRUE];
      p[2] = sd.vec[VB];
      p[3] = sd.vec[VRT];
      p[4] = sd.vec[VR];
    }
  });
  for_chunks_group<3>(tab, gd, act, lb, [&](int c, int m, double (&pr)[3]) {
    const double *x = (const double *)mv.p[m][0];
    double *y = (double *)mv.p[m][1];
    const double *w1 = (const double *)mv.p[m][2];
    const double *w2 = (const double *)mv.p[m][3];
    const double *w3 = (const double *)mv.p[m][4];
    auto epi = [&](int i, double acc) {
      if (MODE == kTrueRes) {
        const double ri = w1[i] - acc;
        y[i] = ri;
        pr[0] += ri * ri;
        const double g = ri - w3[i];
        pr[1] += g * g;
        pr[2] += w2[i] * ri;
      } else {
        y[i] = acc;
        if (MODE == kBicgSigma) pr[0] += w1[i] * acc;
        if (MODE == kBicgOmega) {
          pr[0] += acc * acc;
          pr[1] += acc * w1[i];
        }
      }
    };
    chunk_rows<double>(A, c, x, epi);
  });
  for (int m = 0; m < gd.nmem; m++) {
    if (!((act >> m) & 1u)) continue;
    const int sl = gd.mem[m];
    const SlotDesc &sd = tab->slot[sl];
    KState *st = &sts[sl].k;
    double tot[3] = {0.0, 0.0, 0.0};
    if (slot_fold<3>(tot, sd.partials, gd.nchunks, gd.nb, &st->ticket[0]) && threadIdx.x == 0)
      finish_dots<MODE>(st, tot, (ver >> m) & 1u, MODE == kTrueRes ? sd.vec[VRT] : nullptr);
    __syncthreads();  // slot_fold's shared flag is reused by the next member
  }
}

// x += alpha f + omega z, r = s - omega t, rn2 = r.r, rho' = rt.r.
__global__ void __launch_bounds__(kBlock) k_srv_xr(const Table *tab, SlotState *sts) {
  SRV_PROLOGUE(SRV_RUNNING)
  const double *f = sd.vec[VF], *z = sd.vec[VZ], *s = sd.vec[VS], *t = sd.vec[VT],
               *rt = sd.vec[VRT];
  double *x = sd.vec[VX], *r = sd.vec[VR];
  const double alpha = st->alpha, omega = st->omega;
  for_chunks<2>(lb, nb, sd.nchunks, sd.partials, [&](int c, double (&pr)[2]) {
#pragma unroll
    for (int h = 0; h < kGroupS; h++) {
      const int i = c * kChunkRows + h * kBlock + threadIdx.x;
      if (i < n) {
        x[i] = (x[i] + alpha * f[i]) + omega * z[i];
        const double ri = s[i] - omega * t[i];
        r[i] = ri;
        pr[0] += ri * ri;
        pr[1] += rt[i] * ri;
      }
    }
  });
  double tot[2] = {0.0, 0.0};
  if (slot_fold<2>(tot, sd.partials, sd.nchunks, nb, &st->ticket[0]) && threadIdx.x == 0) {
    finish_iteration(st, tot[0]);
    bicg_next_rho(st, tot[1]);
  }
}

// r := b - A x when the last true-residual check asked for it.
__global__ void __launch_bounds__(kBlock) k_srv_replace(const Table *tab, SlotState *sts) {
  SRV_PROLOGUE(ss->phase == kRun && st->replace)
  const double *rtrue = sd.vec[VRTRUE];
  double *r = sd.vec[VR];
  for (int i = lb * kBlock + threadIdx.x; i < n; i += nb * kBlock) r[i] = rtrue[i];
}

enum Family { kFamStd = 1, kFamAcc64 = 2 };

void sweeps(const Table *tab, SlotState *sts, int grid, cudaStream_t s, int fam, int src,
            int dst) {
  if (fam & kFamStd) k_srv_sweep1<false><<<grid, kBlock, 0, s>>>(tab, sts, src);
  if (fam & kFamAcc64) k_srv_sweep1<true><<<grid, kBlock, 0, s>>>(tab, sts, src);
  if (fam & kFamStd) k_srv_sweep2<false><<<grid, kBlock, 0, s>>>(tab, sts, dst);
  if (fam & kFamAcc64) k_srv_sweep2<true><<<grid, kBlock, 0, s>>>(tab, sts, dst);
}

// One batched iteration on stream s (11 launches over the whole grid, plus
// the second family's two sweeps when both families are registered).
cudaError_t enqueue_iteration(const Table *tab, SlotState *sts, int grid, cudaStream_t s,
                              int fam) {
  k_srv_p<<<grid, kBlock, 0, s>>>(tab, sts);
  sweeps(tab, sts, grid, s, fam, VP, VF);
  k_srv_spmv<kBicgSigma><<<grid, kBlock, 0, s>>>(tab, sts);
  k_srv_s<<<grid, kBlock, 0, s>>>(tab, sts);
  sweeps(tab, sts, grid, s, fam, VS, VZ);
  k_srv_spmv<kBicgOmega><<<grid, kBlock, 0, s>>>(tab, sts);
  k_srv_xr<<<grid, kBlock, 0, s>>>(tab, sts);
  k_srv_spmv<kTrueRes><<<grid, kBlock, 0, s>>>(tab, sts);
  k_srv_replace<<<grid, kBlock, 0, s>>>(tab, sts);
  return cudaGetLastError();
}

constexpr int kLaunchesPerIteration = 11;

// ------------------------------------------------------------------ host --
size_t round256(size_t b) { return (b + 255) / 256 * 256; }
size_t vec_stride(int n) { return ((size_t)n + 31) / 32 * 32; }  // doubles
int chunks_of(int n) { return (n + kChunkRows - 1) / kChunkRows; }

// Device bytes of one request's vectors: 11 FP64 vectors, the apply
// intermediate and the chunk partials.
size_t request_bytes(int n) {
  const size_t st = vec_stride(n) * sizeof(double);
  return round256(kNumVec * st + st + 3 * sizeof(double) * (size_t)chunks_of(n));  // t: <= 8 B/row
}

// First-fit allocator over the server's device arena (offsets only).
class Arena {
 public:
  void reset(size_t bytes) {
    free_.clear();
    if (bytes) free_[0] = bytes;
    size_ = bytes;
    used_ = peak_ = 0;
  }
  bool alloc(size_t bytes, size_t *off) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      *off = it->first;
      const size_t rest = it->second - bytes;
      const size_t at = it->first + bytes;
      free_.erase(it);
      if (rest) free_[at] = rest;
      used_ += bytes;
      peak_ = std::max(peak_, used_);
      return true;
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
    used_ -= bytes;
  }
  size_t size() const { return size_; }
  size_t used() const { return used_; }
  size_t peak() const { return peak_; }

 private:
  std::map<size_t, size_t> free_;
  size_t size_ = 0, used_ = 0, peak_ = 0;
};

struct Operator {
  const ainv_csr *a = nullptr;
  const ainv_handle *h = nullptr;
};

struct Request {
  long long id = 0;
  int op = 0, n = 0;
  Operator opd;  // the operator's objects, captured at submit
  const double *b = nullptr;
  double *x = nullptr;
  double eps = 0.0;
  int itmax = 0;
  size_t bytes = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  int status = AINV_SUCCESS, iter = 0;
  double err = 0.0;
  bool complete = false;
};

struct SlotHost {
  Request *req = nullptr;
  size_t off = 0;
};

}  // namespace srv
}  // namespace ainv

struct ainv_server {
  int device = 0, grid = 0, max_slots = 0, iters = 4;
  cudaStream_t s = nullptr;
  cudaGraphExec_t exec = nullptr;
  ainv::srv::Table *tab_d = nullptr, *tab_h = nullptr;
  ainv::srv::Table *tab_empty_d = nullptr;  // all blocks idle: settles new kernels
  int fam = 0, graph_fam = 0;               // kernel families registered / in the graph
  ainv::srv::SlotState *st_d = nullptr, *st_h = nullptr;
  char *arena_d = nullptr;
  ainv::srv::Arena arena;
  std::vector<ainv::srv::Operator> ops;
  std::vector<ainv::srv::SlotHost> slots;
  std::mutex mu;
  std::condition_variable cv_in, cv_out;
  std::deque<ainv::srv::Request *> queue;
  std::unordered_map<long long, ainv::srv::Request *> reqs;
  long long next_id = 1;
  std::thread engine;
  bool running = false, stopping = false;
  int error = AINV_SUCCESS;
  std::string error_msg;
  std::chrono::steady_clock::time_point t0;
  // statistics
  long long submitted = 0, completed = 0, launches = 0;
  int active = 0, peak_active = 0;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace ainv {
namespace srv {
namespace {

// Capture (or re-capture) the step graph for the kernel families `fam`: the
// init kernel and `iters` batched iterations.  Every kernel of the graph is
// first launched once on an all-idle table, so nothing loads during capture
// and no admitted request is advanced.
cudaError_t capture_graph(ainv_server *srv, int fam) {
  k_srv_init<<<srv->grid, kBlock, 0, srv->s>>>(srv->tab_empty_d, srv->st_d);
  cudaError_t e = enqueue_iteration(srv->tab_empty_d, srv->st_d, srv->grid, srv->s, fam);
  if (e == cudaSuccess) e = cudaStreamSynchronize(srv->s);
  if (e != cudaSuccess) return e;
  e = cudaStreamBeginCapture(srv->s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  k_srv_init<<<srv->grid, kBlock, 0, srv->s>>>(srv->tab_d, srv->st_d);
  cudaError_t ce = cudaGetLastError();
  for (int k = 0; k < srv->iters && ce == cudaSuccess; k++)
    ce = enqueue_iteration(srv->tab_d, srv->st_d, srv->grid, srv->s, fam);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(srv->s, &g);
  if (ce != cudaSuccess || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return ce != cudaSuccess ? ce : e;
  }
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return e;
  if (srv->exec) cudaGraphExecDestroy(srv->exec);
  srv->exec = exec;
  srv->graph_fam = fam;
  return cudaSuccess;
}

// Blocks for n units (slots, or operator groups): shares of the grid in
// proportion to weight[k], at least one block and at most cap[k] each,
// contiguous ranges [b0[k], b0[k] + nb[k]).
int plan_weighted(int nslots, const long long *weight, const int *cap, int grid, int *b0,
                  int *nb) {
  if (nslots < 0 || grid < 1 || nslots > grid) {
    set_error("server block plan: %d slots for a grid of %d blocks", nslots, grid);
    return AINV_ERR_ARG;
  }
  long long total = 0;
  for (int k = 0; k < nslots; k++) total += std::max(1LL, weight[k]);
  int used = 0;
  for (int k = 0; k < nslots; k++) {
    const long long w = std::max(1LL, weight[k]);
    int v = (int)((long long)grid * w / std::max(1LL, total));
    nb[k] = std::min(std::max(1, cap[k]), std::max(1, v));
    used += nb[k];
  }
  // rounding up to one block each may overshoot: trim the largest shares
  while (used > grid) {
    int big = 0;
    for (int k = 1; k < nslots; k++)
      if (nb[k] > nb[big]) big = k;
    nb[big]--;
    used--;
  }
  int at = 0;
  for (int k = 0; k < nslots; k++) {
    b0[k] = at;
    at += nb[k];
  }
  return AINV_SUCCESS;
}

// Slots: shares in proportion to their chunks, at most one block per chunk.
int plan(int nslots, const int *nchunks, int grid, int *b0, int *nb) {
  std::vector<long long> w((size_t)std::max(nslots, 0));
  for (int k = 0; k < nslots; k++) w[(size_t)k] = std::max(1, nchunks[k]);
  return plan_weighted(nslots, w.data(), nchunks, grid, b0, nb);
}

void fail_all(ainv_server *srv, int code, const std::string &msg) {
  std::lock_guard<std::mutex> lk(srv->mu);
  srv->error = code;
  srv->error_msg = msg;
  for (auto &sl : srv->slots)
    if (sl.req) {
      sl.req->status = code;
      sl.req->complete = true;
      sl.req->t_done = srv->now();
      sl.req = nullptr;
    }
  for (Request *r : srv->queue) {
    r->status = code;
    r->complete = true;
    r->t_done = srv->now();
  }
  srv->queue.clear();
  srv->active = 0;
  srv->cv_out.notify_all();
}

#define ENG_TRY(expr)                                                                 \
  do {                                                                                \
    cudaError_t e_ = (expr);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      fail_all(srv, AINV_ERR_CUDA, std::string(#expr " failed: ") + cudaGetErrorString(e_)); \
      return;                                                                         \
    }                                                                                 \
  } while (0)

void fill_slot(ainv_server *srv, int k, const Request *r, size_t off) {
  const Operator &op = r->opd;
  SlotDesc &d = srv->tab_h->slot[k];
  std::memset(&d, 0, sizeof(d));
  d.n = r->n;
  d.nchunks = chunks_of(r->n);
  d.A = mat_of(op.a->a);
  d.wt = mat_of(op.h->wt);
  d.z = mat_of(op.h->z);
  d.d = op.h->d;
  const size_t st = vec_stride(r->n);
  double *base = reinterpret_cast<double *>(srv->arena_d + off);
  for (int v = 0; v < kNumVec; v++) d.vec[v] = base + (size_t)v * st;
  d.t = base + (size_t)kNumVec * st;
  d.partials = base + (size_t)(kNumVec + 1) * st;
  SlotState &s = srv->st_h[k];
  std::memset(&s, 0, sizeof(s));
  s.k.eps = r->eps;
  s.k.itmax = r->itmax;
  s.k.method = AINV_KRYLOV_BICGSTAB;
  s.k.check_every = op.h->prec == AINV_PREC_FP64 ? 0 : kRecheck;
  s.phase = kInitPhase;
}

void engine_loop(ainv_server *srv) {
  cudaSetDevice(srv->device);
  const int S = srv->max_slots;
  std::vector<int> order, nch, b0(S), nb(S);
  bool dirty = true;
  for (;;) {
    std::vector<int> admitted;
    {
      std::unique_lock<std::mutex> lk(srv->mu);
      if (srv->active == 0)
        srv->cv_in.wait(lk, [&] { return srv->stopping || !srv->queue.empty(); });
      if (srv->active == 0 && srv->queue.empty() && srv->stopping) return;
      // first come, first served: the head waits for a slot and for memory
      while (!srv->queue.empty()) {
        int k = 0;
        while (k < S && srv->slots[(size_t)k].req) k++;
        if (k == S) break;
        Request *r = srv->queue.front();
        size_t off = 0;
        if (!srv->arena.alloc(r->bytes, &off)) break;
        srv->queue.pop_front();
        r->t_admit = srv->now();
        srv->slots[(size_t)k] = SlotHost{r, off};
        srv->active++;
        srv->peak_active = std::max(srv->peak_active, srv->active);
        admitted.push_back(k);
      }
    }
    if (srv->active == 0) continue;
    for (int k : admitted) {
      const Request *r = srv->slots[(size_t)k].req;
      fill_slot(srv, k, r, srv->slots[(size_t)k].off);
      ENG_TRY(cudaMemcpyAsync(srv->tab_h->slot[k].vec[VB], r->b, sizeof(double) * (size_t)r->n,
                              cudaMemcpyHostToDevice, srv->s));
      ENG_TRY(cudaMemcpyAsync(srv->st_d + k, srv->st_h + k, sizeof(SlotState),
                              cudaMemcpyHostToDevice, srv->s));
    }
    if (!admitted.empty() || dirty) {
      order.clear();
      nch.clear();
      for (int k = 0; k < S; k++)
        if (srv->slots[(size_t)k].req) {
          order.push_back(k);
          nch.push_back(srv->tab_h->slot[k].nchunks);
        }
      if (plan((int)order.size(), nch.data(), srv->grid, b0.data(), nb.data()) != AINV_SUCCESS) {
        fail_all(srv, AINV_ERR_INTERNAL, "server block plan failed");
        return;
      }
      std::fill(srv->tab_h->block_slot, srv->tab_h->block_slot + kMaxGrid, (short)-1);
      for (size_t q = 0; q < order.size(); q++) {
        SlotDesc &d = srv->tab_h->slot[order[q]];
        d.b0 = b0[q];
        d.nb = nb[q];
        for (int b = d.b0; b < d.b0 + d.nb; b++) srv->tab_h->block_slot[b] = (short)order[q];
      }
      // operator groups: active slots on one operator, in slot order, up to
      // kMaxMembers each; blocks in proportion to chunks x members
      int ng = 0;
      std::vector<int> gop;
      for (int k : order) {
        const int op = srv->slots[(size_t)k].req->op;
        int g = ng - 1;
        while (g >= 0 && !(gop[(size_t)g] == op && srv->tab_h->group[g].nmem < kMaxMembers)) g--;
        if (g < 0) {
          g = ng++;
          gop.push_back(op);
          GroupDesc &gd = srv->tab_h->group[g];
          std::memset(&gd, 0, sizeof(gd));
          gd.nchunks = srv->tab_h->slot[k].nchunks;
        }
        GroupDesc &gd = srv->tab_h->group[g];
        gd.mem[gd.nmem++] = (short)k;
      }
      std::vector<long long> gw((size_t)ng);
      std::vector<int> gcap((size_t)ng), gb0((size_t)ng), gnb((size_t)ng);
      for (int g = 0; g < ng; g++) {
        gw[(size_t)g] = (long long)srv->tab_h->group[g].nchunks * srv->tab_h->group[g].nmem;
        gcap[(size_t)g] = srv->tab_h->group[g].nchunks;
      }
      if (plan_weighted(ng, gw.data(), gcap.data(), srv->grid, gb0.data(), gnb.data()) !=
          AINV_SUCCESS) {
        fail_all(srv, AINV_ERR_INTERNAL, "server group plan failed");
        return;
      }
      std::fill(srv->tab_h->block_group, srv->tab_h->block_group + kMaxGrid, (short)-1);
      for (int g = 0; g < ng; g++) {
        GroupDesc &gd = srv->tab_h->group[g];
        gd.b0 = gb0[(size_t)g];
        gd.nb = gnb[(size_t)g];
        for (int b = gd.b0; b < gd.b0 + gd.nb; b++) srv->tab_h->block_group[b] = (short)g;
      }
      ENG_TRY(cudaMemcpyAsync(srv->tab_d, srv->tab_h, sizeof(Table), cudaMemcpyHostToDevice,
                              srv->s));
      dirty = false;
    }
    int fam;
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      fam = srv->fam;
    }
    if (fam != 0 && fam != srv->graph_fam) ENG_TRY(capture_graph(srv, fam));  // new family
    ENG_TRY(cudaGraphLaunch(srv->exec, srv->s));
    ENG_TRY(cudaMemcpyAsync(srv->st_h, srv->st_d, sizeof(SlotState) * (size_t)S,
                            cudaMemcpyDeviceToHost, srv->s));
    ENG_TRY(cudaStreamSynchronize(srv->s));
    srv->launches++;
    std::vector<int> done;
    for (int k = 0; k < S; k++) {
      const SlotHost &sl = srv->slots[(size_t)k];
      if (sl.req && srv->st_h[k].phase == kRun && srv->st_h[k].k.done) {
        done.push_back(k);
        ENG_TRY(cudaMemcpyAsync(sl.req->x, srv->tab_h->slot[k].vec[VX],
                                sizeof(double) * (size_t)sl.req->n, cudaMemcpyDeviceToHost,
                                srv->s));
      }
    }
    if (done.empty()) continue;
    ENG_TRY(cudaStreamSynchronize(srv->s));
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      const double t = srv->now();
      for (int k : done) {
        SlotHost &sl = srv->slots[(size_t)k];
        const KState &f = srv->st_h[k].k;
        Request *r = sl.req;
        r->iter = f.iter;
        r->err = sqrt(f.rn2) / f.bn2;
        r->status = f.status;
        r->t_done = t;
        r->complete = true;
        srv->arena.release(sl.off, r->bytes);
        srv->st_h[k].phase = kIdle;
        sl = SlotHost{};
        srv->active--;
        srv->completed++;
      }
      dirty = true;
    }
    srv->cv_out.notify_all();
  }
}

}  // namespace
}  // namespace srv
}  // namespace ainv

using ainv::srv::Request;

extern "C" {

int ainv_server_plan(int nslots, const int *rows, int grid, int *b0, int *nb) {
  if ((nslots > 0 && (!rows || !b0 || !nb)) || nslots > ainv::srv::kMaxSlots) {
    ainv::set_error("ainv_server_plan: invalid arguments");
    return AINV_ERR_ARG;
  }
  std::vector<int> ch((size_t)std::max(nslots, 0));
  for (int k = 0; k < nslots; k++) ch[(size_t)k] = ainv::srv::chunks_of(rows[k]);
  return ainv::srv::plan(nslots, ch.data(), grid, b0, nb);
}

size_t ainv_server_request_bytes(int n) { return n > 0 ? ainv::srv::request_bytes(n) : 0; }

int ainv_server_create(ainv_server **out, int max_slots, size_t hbm_bytes, int iters_per_launch) {
  using namespace ainv::srv;
  if (!out) {
    ainv::set_error("ainv_server_create: null pointer");
    return AINV_ERR_ARG;
  }
  *out = nullptr;
  if (max_slots < 1 || max_slots > kMaxSlots || iters_per_launch < 1 || iters_per_launch > 64) {
    ainv::set_error("ainv_server_create: max_slots must be 1..%d and iters_per_launch 1..64",
                    kMaxSlots);
    return AINV_ERR_ARG;
  }
  ainv_server *srv = new (std::nothrow) ainv_server;
  if (!srv) {
    ainv::set_error("ainv_server_create: host allocation failed");
    return AINV_ERR_ALLOC;
  }
  srv->max_slots = max_slots;
  srv->iters = iters_per_launch;
  srv->slots.resize((size_t)max_slots);
  srv->t0 = std::chrono::steady_clock::now();
  auto fail = [&](cudaError_t e, const char *what) {
    ainv::set_error("ainv_server_create: %s: %s", what, cudaGetErrorString(e));
    ainv_server_destroy(srv);
    return e == cudaErrorMemoryAllocation ? AINV_ERR_ALLOC : AINV_ERR_CUDA;
  };
  cudaError_t e = cudaGetDevice(&srv->device);
  int sms = 0;
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, srv->device);
  if (e != cudaSuccess) return fail(e, "device query");
  // 8 blocks of 256 threads per SM: a full wave for the light batched
  // kernels; the register-heavy SpMV / sweep kernels run it in a few waves.
  // (A grid of one wave of the heaviest kernel measured 35% fewer solves/s:
  // the light kernels, latency-bound, then had too few blocks.)
  srv->grid = std::min(kMaxGrid, std::max(max_slots, 8 * sms));
  // admission budget: the caller's bytes, or half of the free HBM
  size_t fr = 0, tot = 0;
  e = cudaMemGetInfo(&fr, &tot);
  if (e != cudaSuccess) return fail(e, "cudaMemGetInfo");
  size_t budget = hbm_bytes ? hbm_bytes : fr / 2;
  if (budget > fr) {
    ainv::set_error("ainv_server_create: %zu bytes requested, %zu free on the device", budget, fr);
    ainv_server_destroy(srv);
    return AINV_ERR_ALLOC;
  }
  budget = budget / 256 * 256;
  e = cudaMalloc(&srv->arena_d, budget);
  if (e != cudaSuccess) return fail(e, "arena");
  srv->arena.reset(budget);
  if ((e = cudaMalloc(&srv->tab_d, sizeof(Table))) != cudaSuccess) return fail(e, "table");
  if ((e = cudaMallocHost(&srv->tab_h, sizeof(Table))) != cudaSuccess) return fail(e, "table");
  if ((e = cudaMalloc(&srv->st_d, sizeof(SlotState) * (size_t)max_slots)) != cudaSuccess)
    return fail(e, "states");
  if ((e = cudaMallocHost(&srv->st_h, sizeof(SlotState) * (size_t)max_slots)) != cudaSuccess)
    return fail(e, "states");
  if ((e = cudaStreamCreateWithFlags(&srv->s, cudaStreamNonBlocking)) != cudaSuccess)
    return fail(e, "stream");
  std::memset(srv->tab_h, 0, sizeof(Table));
  std::fill(srv->tab_h->block_slot, srv->tab_h->block_slot + kMaxGrid, (short)-1);
  std::fill(srv->tab_h->block_group, srv->tab_h->block_group + kMaxGrid, (short)-1);
  std::memset(srv->st_h, 0, sizeof(SlotState) * (size_t)max_slots);
  e = cudaMemcpy(srv->tab_d, srv->tab_h, sizeof(Table), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(srv->st_d, srv->st_h, sizeof(SlotState) * (size_t)max_slots,
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(e, "initial table");
  if ((e = cudaMalloc(&srv->tab_empty_d, sizeof(Table))) != cudaSuccess) return fail(e, "table");
  e = cudaMemcpy(srv->tab_empty_d, srv->tab_h, sizeof(Table), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(e, "empty table");
  if ((e = capture_graph(srv, kFamStd)) != cudaSuccess) return fail(e, "graph capture");
  srv->running = true;
  srv->engine = std::thread(engine_loop, srv);
  *out = srv;
  return AINV_SUCCESS;
}

int ainv_server_add_operator(ainv_server *srv, const ainv_csr *a, const ainv_handle *h,
                             int *op) {
  if (!srv || !a || !h || !op) {
    ainv::set_error("ainv_server_add_operator: null argument");
    return AINV_ERR_ARG;
  }
  if (a->n != h->n || a->n < 1) {
    ainv::set_error("ainv_server_add_operator: operator size %d, factor size %d", a->n, h->n);
    return AINV_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(srv->mu);
  srv->fam |= ainv::srv::acc64_prec(h->prec) ? ainv::srv::kFamAcc64 : ainv::srv::kFamStd;
  srv->ops.push_back(ainv::srv::Operator{a, h});
  *op = (int)srv->ops.size() - 1;
  return AINV_SUCCESS;
}

int ainv_server_submit(ainv_server *srv, int op, const double *b, double *x, double eps,
                       int itmax, long long *id) {
  if (!srv || !b || !x || !id || !(eps > 0.0) || itmax < 0) {
    ainv::set_error("ainv_server_submit: invalid argument");
    return AINV_ERR_ARG;
  }
  Request *r = new (std::nothrow) Request;
  if (!r) {
    ainv::set_error("ainv_server_submit: host allocation failed");
    return AINV_ERR_ALLOC;
  }
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    if (op < 0 || op >= (int)srv->ops.size()) {
      delete r;
      ainv::set_error("ainv_server_submit: unknown operator %d", op);
      return AINV_ERR_ARG;
    }
    if (srv->error != AINV_SUCCESS || srv->stopping) {
      delete r;
      ainv::set_error("ainv_server_submit: server stopped (%s)", srv->error_msg.c_str());
      return srv->error != AINV_SUCCESS ? srv->error : AINV_ERR_INTERNAL;
    }
    r->id = srv->next_id++;
    r->op = op;
    r->opd = srv->ops[(size_t)op];
    r->n = r->opd.a->n;
    r->b = b;
    r->x = x;
    r->eps = eps;
    r->itmax = itmax;
    r->bytes = ainv::srv::request_bytes(r->n);
    if (r->bytes > srv->arena.size()) {
      const size_t need = r->bytes, have = srv->arena.size();
      delete r;
      ainv::set_error("ainv_server_submit: request needs %zu device bytes, the server holds %zu",
                      need, have);
      return AINV_ERR_ALLOC;
    }
    r->t_submit = srv->now();
    srv->reqs[r->id] = r;
    srv->queue.push_back(r);
    srv->submitted++;
    *id = r->id;
  }
  srv->cv_in.notify_one();
  return AINV_SUCCESS;
}

int ainv_server_wait(ainv_server *srv, long long id, double timeout_s, ainv_result *res) {
  if (!srv) {
    ainv::set_error("ainv_server_wait: null server");
    return AINV_ERR_ARG;
  }
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(id);
  if (it == srv->reqs.end()) {
    ainv::set_error("ainv_server_wait: unknown request %lld", id);
    return AINV_ERR_ARG;
  }
  Request *r = it->second;
  auto ready = [&] { return r->complete; };
  if (timeout_s < 0)
    srv->cv_out.wait(lk, ready);
  else if (!srv->cv_out.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
    ainv::set_error("ainv_server_wait: request %lld not complete after %.3f s", id, timeout_s);
    return AINV_ERR_TIMEOUT;
  }
  if (res) {
    res->id = r->id;
    res->op = r->op;
    res->status = r->status;
    res->iter = r->iter;
    res->err = r->err;
    res->t_submit = r->t_submit;
    res->t_admit = r->t_admit;
    res->t_done = r->t_done;
  }
  const int status = r->status;
  srv->reqs.erase(it);
  delete r;
  if (status != AINV_SUCCESS) {
    switch (status) {
      case AINV_ERR_NOCONV: ainv::set_error("request %lld: itmax reached", id); break;
      case AINV_ERR_BREAKDOWN: ainv::set_error("request %lld: Krylov breakdown", id); break;
      case AINV_ERR_NONFINITE: ainv::set_error("request %lld: non-finite residual", id); break;
      default: ainv::set_error("request %lld: %s", id, srv->error_msg.c_str()); break;
    }
  }
  return status;
}

int ainv_server_stats(ainv_server *srv, ainv_server_info *out) {
  if (!srv || !out) {
    ainv::set_error("ainv_server_stats: null argument");
    return AINV_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(srv->mu);
  out->submitted = srv->submitted;
  out->completed = srv->completed;
  out->graph_launches = srv->launches;
  out->kernel_launches = srv->launches *
      (1 + (long long)srv->iters *
               (ainv::srv::kLaunchesPerIteration + (srv->graph_fam == 3 ? 4 : 0)));
  out->active = srv->active;
  out->queued = (int)srv->queue.size();
  out->peak_active = srv->peak_active;
  out->max_slots = srv->max_slots;
  out->grid = srv->grid;
  out->iters_per_launch = srv->iters;
  out->arena_bytes = srv->arena.size();
  out->arena_used = srv->arena.used();
  out->arena_peak = srv->arena.peak();
  out->clock = srv->now();
  return srv->error;
}

int ainv_server_destroy(ainv_server *srv) {
  if (!srv) return AINV_SUCCESS;
  if (srv->running) {
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      srv->stopping = true;
    }
    srv->cv_in.notify_all();
    srv->engine.join();
  }
  if (srv->s) cudaStreamSynchronize(srv->s);
  for (auto &kv : srv->reqs) delete kv.second;
  if (srv->exec) cudaGraphExecDestroy(srv->exec);
  if (srv->arena_d) cudaFree(srv->arena_d);
  if (srv->tab_d) cudaFree(srv->tab_d);
  if (srv->tab_empty_d) cudaFree(srv->tab_empty_d);
  if (srv->tab_h) cudaFreeHost(srv->tab_h);
  if (srv->st_d) cudaFree(srv->st_d);
  if (srv->st_h) cudaFreeHost(srv->st_h);
  if (srv->s) cudaStreamDestroy(srv->s);
  delete srv;
  return AINV_SUCCESS;
}

}  // extern "C"
