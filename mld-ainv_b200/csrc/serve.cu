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
// Results do not depend on the mix, and they are the single-solve results:
// every dot is summed in the canonical order of the single-solve loop (the
// reducing kernels store one sum per 32-row slice, a fold kernel reduces
// them in fixed groups and ranges, the slot's last block doing the scalar
// step), and every kernel computes a member's rows with the single-solve
// arithmetic.  A request's iterates are thus bit-identical whether it runs
// alone, beside others, or through ainv_gpu_solve.
//
// Requests on the same operator share its reads.  Active slots are grouped
// by operator (up to kMaxMembers per group).  The kernels that read A or
// the factors (the two sweeps and the three A products) walk the
// operator's slices warp by warp, load each slice's values and columns
// once into registers and compute every member's rows from them, so the
// operator comes from HBM once per group and a member adds only its own
// gathers and epilogue.  A streamed form (the stream.cuh pipeline, each
// block working for one member, the members' blocks walking the same
// stages side by side) can be selected per kernel kind.
//
// The host side is an engine thread: requests queue on submit, are admitted
// first-come first-served while a slot is free and their vectors fit in the
// server's device arena (sized from free HBM at creation), are launched
// together, and are retired (x copied back, slot and memory released) as
// soon as their state reports completion.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "krylov_epi.cuh"

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
static_assert(kBlock == kFoldThreads, "the fold runs on the server's blocks");
// Resident blocks per SM of the streamed operator kernels (their register
// cap: 72 at 3 blocks) and the streamed grid's blocks per SM.  Their
// operator and member pointers come from the table, not from kernel
// parameters; at 4 blocks (56 registers) they spilled, and the served 200^3
// solve ran 17% slower.
#ifndef AINV_SRV_STREAM_BLOCKS
#define AINV_SRV_STREAM_BLOCKS 3
#endif
constexpr int kSrvStreamBlocks = AINV_SRV_STREAM_BLOCKS;
// Slice-shared operator kernels: resident blocks per SM (their register
// cap and grid) and members computed per step from one slice's registers.
// They are latency-bound: 5 blocks per SM (48 registers, a few spills)
// served the 200^3 batch 8% faster than 4 and 18% faster than 3; 6 was
// within 2%, and 7 or 8 (40, 32 registers) lost 19% to spills.
#ifndef AINV_SRV_SHARE_BLOCKS
#define AINV_SRV_SHARE_BLOCKS 5
#endif
#ifndef AINV_SRV_SHARE_UNROLL
#define AINV_SRV_SHARE_UNROLL 2
#endif
constexpr int kSrvShareBlocks = AINV_SRV_SHARE_BLOCKS;
constexpr int kShareUnroll = AINV_SRV_SHARE_UNROLL;

enum Vec { VX = 0, VB, VR, VRT, VP, VV, VF, VS, VZ, VT, VRTRUE, kNumVec };
enum Phase { kIdle = 0, kInitPhase = 1, kRun = 2 };
// Operator kernels that can run streamed: sweep 1 (W^T, D^-1 staged), sweep
// 2 (Z), the A products with one staged operand (sigma, omega) and the true
// residual (three staged operands).
enum StreamKind { kSkSweep1 = 0, kSkSweep2, kSkSpmv, kSkTrue, kNumSk };

struct Mat {
  int n, nslices, pack, prec;
  const int *sptr, *iptr, *idx;
  const void *val;
  const StageDesc *stages;
  int nstages;
};

struct SlotDesc {
  int b0, nb;    // launch blocks [b0, b0 + nb) of the vector kernels
  int fb0, fnb;  // fold blocks [fb0, fb0 + fnb), at most one per range
  int n, nchunks;
  Mat A, wt, z;
  const void *d;  // D^-1 in the factors' precision
  void *t;        // apply intermediate: double (FP64 factors) or float
  double *vec[kNumVec];
  // canonical-order reductions: slice sums of up to 3 dots (ld apart) and
  // range sums (ldr apart)
  double *sp, *rs;
  int ns, ng, nr, ld, ldr;
  // streamed operator kernels: layouts, and which kinds stream (bit k)
  StreamLayout L[kNumSk];
  unsigned smask;
};

// Slots on one operator, served together by the operator kernels.
struct GroupDesc {
  int b0, nb;    // slice-shared operator kernels: blocks [b0, b0 + nb)
  int bs0, nbs;  // streamed operator kernels: blocks [bs0, bs0 + nbs) (nbs >= nmem)
  int nchunks, nmem;
  short mem[kMaxMembers];
};

struct Table {
  SlotDesc slot[kMaxSlots];
  GroupDesc group[kMaxSlots];
  short block_slot[kMaxGrid];     // vector kernels: the block's slot, -1 idle
  short block_slot_f[kMaxGrid];   // folds: the block's slot, -1 idle
  short block_group[kMaxGrid];    // slice-shared operator kernels: the block's group
  short block_group_s[kMaxGrid];  // streamed operator kernels: the block's group
};

struct SlotState {
  KState k;
  int phase;
  int pad[3];
};

inline Mat mat_of(const DevSell &m) {
  return Mat{m.n, m.nslices, m.pack, m.prec, m.sptr, m.iptr, m.idx, m.val, m.stages, m.nstages};
}

// ---------------------------------------------------------------- device --
template <class V>
__device__ __forceinline__ SellView<V> sview(const Mat &m) {
  return SellView<V>{m.n, m.nslices, m.sptr, m.iptr, m.idx, (const V *)m.val};
}

// The members' vector pointers an operator kernel needs (up to 5 each),
// staged once per block in shared memory; the operator (A, W^T, Z, D^-1)
// is the same for every member and is read from member 0.
constexpr int kMemberVecs = 5;
struct MemberVecs {
  void *p[kMaxMembers][kMemberVecs];
};

// ---- slice-shared operator walk ------------------------------------------------
// The group's blocks walk the operator's slices warp by warp (lane = row;
// block lb takes slices 8 lb + warp, then every 8 nb-th).  A slice's
// values and columns are loaded once into registers and each active
// member's rows are computed from them, kShareUnroll members at a time (their
// gathers in flight together), so a member adds only its own gathers and
// epilogue.  Slots run in order with the
// products of zero slots adding zero, as group_slots forms them, so every
// member gets the single-solve row sums.  Slices wider than kShareSlots
// slots reload their values for each member, kShareSlots at a time.
// body(i, row, acc) runs for each member i (index into the group; its
// gathered vector is mv.p[i][0]) and row < n; end(i, s) then runs with the
// whole warp.  ml: the M active members (shared memory).
constexpr int kShareSlots = 8;

// Slots [k0, k0 + kShareSlots) of the lane's row of a slice into registers
// (zeros past w): values, and columns (offset mode: row + offset).
template <bool EF, int P, class V>
__device__ __forceinline__ void share_load(const SellView<V> &m, int w, int vb, int ib, bool om,
                                           int row, int k0,
                                           typename Acc<V>::type (&vv)[kShareSlots / P][P],
                                           int (&col)[kShareSlots / P][P]) {
  using A = typename Acc<V>::type;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < kShareSlots / P; j++) {
    const int k = k0 + j * P;
    const size_t pos = (size_t)(k / P) * (kSlice * P) + (size_t)lane * P;
    if (k < w) {
      Pack<V, P>::template load<EF>(m.val + vb + pos, vv[j]);
      if (om) {
        load_ints<P, false>(m.idx + ib + k, col[j]);
#pragma unroll
        for (int e = 0; e < P; e++) col[j][e] += row;
      } else {
        load_ints<P, EF>(m.idx + ib + pos, col[j]);
      }
    } else {
#pragma unroll
      for (int e = 0; e < P; e++) {
        vv[j][e] = A(0);
        col[j][e] = 0;
      }
    }
  }
}

// acc += the loaded slots dotted with x, in slot order (zero slots add 0).
template <int P, class A, class X>
__device__ __forceinline__ void share_dot(int n, const A (&vv)[kShareSlots / P][P],
                                          const int (&col)[kShareSlots / P][P],
                                          const X *__restrict__ x, A &acc) {
  A xv[kShareSlots / P][P];
#pragma unroll
  for (int j = 0; j < kShareSlots / P; j++)
#pragma unroll
    for (int e = 0; e < P; e++)
      xv[j][e] = (vv[j][e] != A(0) && (unsigned)col[j][e] < (unsigned)n) ? (A)__ldg(x + col[j][e])
                                                                         : A(0);
#pragma unroll
  for (int j = 0; j < kShareSlots / P; j++)
#pragma unroll
    for (int e = 0; e < P; e++) acc = madd(vv[j][e], xv[j][e], acc);
}

template <class V, int P, class X, class Body, class End>
__device__ __forceinline__ void shared_slices(const Mat &mm, int lb, int nb, const int *ml, int M,
                                              const MemberVecs &mv, Body &body, End &end) {
  using A = typename Acc<V>::type;
  constexpr int J = kShareSlots / P;
  const SellView<V> m = sview<V>(mm);
  const int lane = threadIdx.x & 31;
  for (int s = lb * kWarps + (int)(threadIdx.x >> 5); s < m.nslices; s += nb * kWarps) {
    int sp = 0, ip = 0;
    if (lane <= 1) {
      sp = __ldg(m.sptr + s + lane);
      ip = __ldg(m.iptr + s + lane);
    }
    const int vb = __shfl_sync(0xffffffffu, sp, 0), ve = __shfl_sync(0xffffffffu, sp, 1);
    const int ib = __shfl_sync(0xffffffffu, ip, 0), ie = __shfl_sync(0xffffffffu, ip, 1);
    const int w = (ve - vb) / kSlice;
    const bool om = (ie - ib) == w;
    const int row = s * kSlice + lane;
    if (w <= kShareSlots) {
      A vv[J][P];
      int col[J][P];
      share_load<true, P>(m, w, vb, ib, om, row, 0, vv, col);  // read once: evict-first
      for (int q = 0; q < M; q += kShareUnroll) {
        A a[kShareUnroll];
        int iu[kShareUnroll];
#pragma unroll
        for (int u = 0; u < kShareUnroll; u++) {
          iu[u] = q + u < M ? ml[q + u] : -1;
          a[u] = A(0);
          if (iu[u] >= 0) share_dot<P>(m.n, vv, col, (const X *)mv.p[iu[u]][0], a[u]);
        }
#pragma unroll
        for (int u = 0; u < kShareUnroll; u++)
          if (iu[u] >= 0) {
            if (row < m.n) body(iu[u], row, a[u]);
            end(iu[u], s);
          }
      }
    } else {
      for (int q = 0; q < M; q++) {
        const int i0 = ml[q];
        A a0 = A(0);
        for (int k0 = 0; k0 < w; k0 += kShareSlots) {
          A vv[J][P];
          int col[J][P];
          share_load<false, P>(m, w, vb, ib, om, row, k0, vv, col);  // every member: cached
          share_dot<P>(m.n, vv, col, (const X *)mv.p[i0][0], a0);
        }
        if (row < m.n) body(i0, row, a0);
        end(i0, s);
      }
    }
  }
}

// shared_slices for the operator's pack.
template <class V, class X, class Body, class End>
__device__ __forceinline__ void shared_slices_any(const Mat &m, int lb, int nb, const int *ml,
                                                  int M, const MemberVecs &mv, Body &body,
                                                  End &end) {
  if constexpr (pack_ok<V, 2>()) {
    if (m.pack == 2) return shared_slices<V, 2, X>(m, lb, nb, ml, M, mv, body, end);
  }
  if constexpr (pack_ok<V, 4>()) {
    if (m.pack == 4) return shared_slices<V, 4, X>(m, lb, nb, ml, M, mv, body, end);
  }
  if constexpr (pack_ok<V, 8>()) {
    if (m.pack == 8) return shared_slices<V, 8, X>(m, lb, nb, ml, M, mv, body, end);
  }
  shared_slices<V, 1, X>(m, lb, nb, ml, M, mv, body, end);
}

// The active members (bits of act) as a list of group indices in shared
// memory (thread 0 writes; the caller synchronises).
__device__ __forceinline__ void member_list(unsigned act, int nmem, int *ml) {
  if (threadIdx.x != 0) return;
  int M = 0;
  for (int i = 0; i < nmem; i++)
    if ((act >> i) & 1u) ml[M++] = i;
}

struct NoEnd {
  __device__ __forceinline__ void operator()(int, int) const {}
};

// Block prologue: the block's slot, or -1.  `need` decides from the slot's
// state whether this kernel acts on it; it is evaluated identically by
// every block of the slot (the state changes only in the last block of the
// slot's fold, after all blocks have passed this point).
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

// Prologue of the slice-shared operator kernels: the block's group (copied
// out of the table, so that the stores of the inner loops cannot force
// reloads), or return.
#define SRV_GROUP_PROLOGUE                                         \
  const int grp = tab->block_group[blockIdx.x];                   \
  if (grp < 0) return;                                            \
  const GroupDesc gd = tab->group[grp];                           \
  const int lb = blockIdx.x - gd.b0;

template <class F>
__device__ __forceinline__ void stage_members(const Table *tab, const GroupDesc &gd,
                                              MemberVecs &mv, F &&pick) {
  if ((int)threadIdx.x < gd.nmem) pick(tab->slot[gd.mem[threadIdx.x]], mv.p[threadIdx.x]);
  __syncthreads();
}

__device__ __forceinline__ bool slot_running(const SlotState *ss) {
  return ss->phase == kRun && !ss->k.done;
}

// The slot's slices, warp by warp over its blocks (lane = row): the walk of
// the vector kernels that reduce, so their slice sums see the lane order of
// the operator kernels.
#define SRV_SLICES(sl) \
  for (int sl = lb * kWarps + (int)(threadIdx.x >> 5); sl < sd.ns; sl += nb * kWarps)

// r = rt = b, x = p = v = 0; slice sums of b.b (the fold sets ||b|| and the
// first rho = r.r, x0 = 0).
__global__ void __launch_bounds__(kBlock) k_srv_init(const Table *tab, SlotState *sts) {
  SRV_PROLOGUE(ss->phase == kInitPhase)
  double *x = sd.vec[VX], *r = sd.vec[VR], *rt = sd.vec[VRT], *p = sd.vec[VP], *v = sd.vec[VV];
  const double *b = sd.vec[VB];
  SliceSums<1> sums{sd.sp, sd.ld, {0.0}};
  const int lane = threadIdx.x & 31;
  SRV_SLICES(sl) {
    const int i = sl * kSlice + lane;
    if (i < n) {
      const double bi = b[i];
      x[i] = 0.0;
      r[i] = bi;
      rt[i] = bi;
      p[i] = 0.0;
      v[i] = 0.0;
      sums.v[0] = bi * bi;
    }
    sums.end(sl);
  }
}

// p = r (first iteration) or p = r + beta (p - omega v).  When the last
// true-residual check asked for it, r := b - A x first (the single solve's
// replacement before its next p update; nothing reads r in between).
__global__ void __launch_bounds__(kBlock) k_srv_p(const Table *tab, SlotState *sts) {
  SRV_PROLOGUE(SRV_RUNNING)
  const double *rtrue = sd.vec[VRTRUE], *v = sd.vec[VV];
  double *r = sd.vec[VR], *p = sd.vec[VP];
  const bool first = st->iter == 0, repl = st->replace != 0;
  const double beta = st->beta, omega = st->omega;
  for (int i = lb * kBlock + threadIdx.x; i < n; i += nb * kBlock) {
    double ri;
    if (repl) {
      ri = rtrue[i];
      r[i] = ri;
    } else {
      ri = r[i];
    }
    p[i] = first ? ri : ri + beta * (p[i] - omega * v[i]);
  }
}

// s = r - alpha v.
__global__ void __launch_bounds__(kBlock) k_srv_s(const Table *tab, SlotState *sts) {
  SRV_PROLOGUE(SRV_RUNNING)
  const double *r = sd.vec[VR], *v = sd.vec[VV];
  double *s = sd.vec[VS];
  const double alpha = st->alpha;
  for (int i = lb * kBlock + threadIdx.x; i < n; i += nb * kBlock) s[i] = r[i] - alpha * v[i];
}

// x += alpha f + omega z, r = s - omega t; slice sums of r.r and rt.r.  Capped
// at 32 registers so that the grid's 8 blocks per SM are resident at once.
__global__ void __launch_bounds__(kBlock, 8) k_srv_xr(const Table *tab, SlotState *sts) {
  SRV_PROLOGUE(SRV_RUNNING)
  const double *f = sd.vec[VF], *z = sd.vec[VZ], *s = sd.vec[VS], *t = sd.vec[VT],
               *rt = sd.vec[VRT];
  double *x = sd.vec[VX], *r = sd.vec[VR];
  const double alpha = st->alpha, omega = st->omega;
  SliceSums<2> sums{sd.sp, sd.ld, {0.0, 0.0}};
  const int lane = threadIdx.x & 31;
  SRV_SLICES(sl) {
    const int i = sl * kSlice + lane;
    if (i < n) {
      x[i] = (x[i] + alpha * f[i]) + omega * z[i];
      const double ri = s[i] - omega * t[i];
      r[i] = ri;
      sums.v[0] = ri * ri;
      sums.v[1] = rt[i] * ri;
    }
    sums.end(sl);
  }
}

// ---- the fold ------------------------------------------------------------------
// The slot's fold blocks (their own small grid) fold its slice sums in the
// canonical order (the single-solve fold's steps): block lb takes ranges
// lb, lb + np, ... (np = the slot's fold blocks); the last block to finish (atomic
// ticket, no waiting) folds the range sums and runs fin.  fin.need(ss) is
// the producing kernel's test, so a reduction that did not run is not
// folded.
template <int NV, class Fin>
__global__ void __launch_bounds__(kBlock) k_srv_fold(const Table *tab, SlotState *sts, Fin fin) {
  const int slot = tab->block_slot_f[blockIdx.x];
  if (slot < 0) return;
  SlotState *ss = sts + slot;
  if (!fin.need(ss)) return;
  const SlotDesc &sd = tab->slot[slot];
  const int lb = blockIdx.x - sd.fb0, np = min(sd.fnb, sd.nr);
  if (lb >= np) return;
  __shared__ bool is_last;
  double v[NV];
  for (int r = lb; r < sd.nr; r += np) {
    fold_range<NV>(sd.sp, sd.ld, sd.ns, sd.ng, r, v);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < NV; k++) sd.rs[(size_t)k * sd.ldr + r] = v[k];
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();
    is_last = atomicAdd(&ss->k.ticket[3], 1u) == (unsigned)np - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  fold_total<NV>(sd.rs, sd.ldr, sd.nr, v);
  if (threadIdx.x == 0) {
    ss->k.ticket[3] = 0u;
    fin(ss, sd, v);
  }
}

struct FinInit {
  __device__ __forceinline__ bool need(const SlotState *ss) const { return ss->phase == kInitPhase; }
  __device__ __forceinline__ void operator()(SlotState *ss, const SlotDesc &,
                                             const double (&v)[1]) const {
    KState *st = &ss->k;
    const double bn = sqrt(v[0]);
    st->bn2 = (bn == 0.0) ? 1.0 : bn;
    const double pr[3] = {v[0], v[0], 0.0};
    finish_dots<kInit>(st, pr, false, nullptr);
    ss->phase = kRun;
  }
};

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
struct FinDotsSrv {
  __device__ __forceinline__ bool need(const SlotState *ss) const {
    bool v;
    return srv_spmv_active<MODE>(ss, &v);
  }
  __device__ __forceinline__ void operator()(SlotState *ss, const SlotDesc &sd,
                                             const double (&v)[dots_of(MODE)]) const {
    bool verify;
    srv_spmv_active<MODE>(ss, &verify);
    double pr[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < dots_of(MODE); k++) pr[k] = v[k];
    finish_dots<MODE>(&ss->k, pr, verify, sd.vec[VRT]);
  }
};

struct FinXr {
  __device__ __forceinline__ bool need(const SlotState *ss) const { return slot_running(ss); }
  __device__ __forceinline__ void operator()(SlotState *ss, const SlotDesc &,
                                             const double (&v)[2]) const {
    finish_iteration(&ss->k, v[0]);
    bicg_next_rho(&ss->k, v[1]);
  }
};

// ---- chunk-walking operator kernels ------------------------------------------
// For groups whose operator kind does not stream (smask bit clear): the
// group's blocks walk its 512-row chunks and compute each chunk for every
// active member in turn.
__host__ __device__ constexpr bool acc64_prec(int prec) {
  return prec == AINV_PREC_FP32_ACC64 || prec == AINV_PREC_BF16_ACC64;
}

// Members of the group (bit i: member i) that run the sweeps: running
// slots, when the group's operator belongs to family ACC and the sweep
// `kind` is chunk-walked (streamed == false) or streamed (true).
template <bool ACC>
__device__ __forceinline__ unsigned sweep_members(const SlotState *sts, const GroupDesc &gd,
                                                  int prec, unsigned smask, int kind,
                                                  bool streamed) {
  if (acc64_prec(prec) != ACC || (((smask >> kind) & 1u) != 0) != streamed) return 0u;
  unsigned act = 0u;
  for (int i = 0; i < gd.nmem; i++)
    if (slot_running(sts + gd.mem[i])) act |= 1u << i;
  return act;
}

// Sweep 1 of the apply: t = D^-1 .* (W^T src) for the members in ml.
template <class V, class T>
__device__ __forceinline__ void sweep1_group(const Mat &wt, const V *__restrict__ d,
                                             const GroupDesc &gd, const MemberVecs &mv,
                                             const int *ml, int M, int lb) {
  NoEnd end;
  auto body = [&](int i, int row, auto acc) { ((T *)mv.p[i][1])[row] = (T)(ldd(d + row) * acc); };
  shared_slices_any<V, double>(wt, lb, gd.nb, ml, M, mv, body, end);
}

// Slice-shared operator kernels, for groups whose kind does not stream:
// the members' vectors and the active-member list go to shared memory once
// per block.
#define SRV_SHARED_MEMBERS(act, pick)                 \
  __shared__ MemberVecs mv;                           \
  __shared__ int ml[kMaxMembers];                     \
  const int M = __popc(act);                          \
  member_list(act, gd.nmem, ml);                      \
  stage_members(tab, gd, mv, pick);

template <bool ACC>
__global__ void __launch_bounds__(kBlock, kSrvShareBlocks) k_srv_sweep1(const Table *tab, SlotState *sts,
                                                          int src) {
  SRV_GROUP_PROLOGUE
  const SlotDesc &s0 = tab->slot[gd.mem[0]];
  const Mat wt = s0.wt;
  const void *d = s0.d;
  const unsigned act = sweep_members<ACC>(sts, gd, wt.prec, s0.smask, kSkSweep1, false);
  if (!act) return;
  SRV_SHARED_MEMBERS(act, ([&](const SlotDesc &sd, void *(&p)[kMemberVecs]) {
                       p[0] = sd.vec[src];
                       p[1] = sd.t;
                     }))
  if constexpr (ACC) {
    if (wt.prec == AINV_PREC_FP32_ACC64)
      sweep1_group<f32w, double>(wt, (const f32w *)d, gd, mv, ml, M, lb);
    else
      sweep1_group<b16w, double>(wt, (const b16w *)d, gd, mv, ml, M, lb);
  } else {
    switch (wt.prec) {
      case AINV_PREC_FP64: sweep1_group<double, double>(wt, (const double *)d, gd, mv, ml, M, lb); break;
      case AINV_PREC_FP32: sweep1_group<float, float>(wt, (const float *)d, gd, mv, ml, M, lb); break;
      default:
        sweep1_group<__nv_bfloat16, float>(wt, (const __nv_bfloat16 *)d, gd, mv, ml, M, lb);
        break;
    }
  }
}

// Sweep 2 of the apply: dst = Z t (alpha = 1, beta = 0).
template <class V, class T>
__device__ __forceinline__ void sweep2_group(const Mat &z, const GroupDesc &gd,
                                             const MemberVecs &mv, const int *ml, int M, int lb) {
  NoEnd end;
  auto body = [&](int i, int row, auto acc) {
    ((double *)mv.p[i][1])[row] = axpby_row(1.0, (double)acc, 0.0, 0.0);
  };
  shared_slices_any<V, T>(z, lb, gd.nb, ml, M, mv, body, end);
}

template <bool ACC>
__global__ void __launch_bounds__(kBlock, kSrvShareBlocks) k_srv_sweep2(const Table *tab, SlotState *sts,
                                                          int dst) {
  SRV_GROUP_PROLOGUE
  const SlotDesc &s0 = tab->slot[gd.mem[0]];
  const Mat z = s0.z;
  const unsigned act = sweep_members<ACC>(sts, gd, z.prec, s0.smask, kSkSweep2, false);
  if (!act) return;
  SRV_SHARED_MEMBERS(act, ([&](const SlotDesc &sd, void *(&p)[kMemberVecs]) {
                       p[0] = sd.t;
                       p[1] = sd.vec[dst];
                     }))
  if constexpr (ACC) {
    if (z.prec == AINV_PREC_FP32_ACC64)
      sweep2_group<f32w, double>(z, gd, mv, ml, M, lb);
    else
      sweep2_group<b16w, double>(z, gd, mv, ml, M, lb);
  } else {
    switch (z.prec) {
      case AINV_PREC_FP64: sweep2_group<double, double>(z, gd, mv, ml, M, lb); break;
      case AINV_PREC_FP32: sweep2_group<float, float>(z, gd, mv, ml, M, lb); break;
      default: sweep2_group<__nv_bfloat16, float>(z, gd, mv, ml, M, lb); break;
    }
  }
}

// The vectors of an A product of MODE for one member: x, y, w1, w2, w3 of
// dots_row.
template <int MODE>
__device__ __forceinline__ void spmv_vectors(const SlotDesc &sd, void *(&p)[kMemberVecs]) {
  if (MODE == kBicgSigma) {
    p[0] = sd.vec[VF];
    p[1] = sd.vec[VV];
    p[2] = sd.vec[VRT];
    p[3] = nullptr;
    p[4] = nullptr;
  } else if (MODE == kBicgOmega) {
    p[0] = sd.vec[VZ];
    p[1] = sd.vec[VT];
    p[2] = sd.vec[VS];
    p[3] = nullptr;
    p[4] = nullptr;
  } else {
    p[0] = sd.vec[VX];
    p[1] = sd.vec[VRTRUE];
    p[2] = sd.vec[VB];
    p[3] = sd.vec[VRT];
    p[4] = sd.vec[VR];
  }
}

constexpr int spmv_kind(int mode) { return mode == kTrueRes ? kSkTrue : kSkSpmv; }

// Members that run the A product of MODE (streamed or chunk-walked).
template <int MODE>
__device__ __forceinline__ unsigned spmv_members(const SlotState *sts, const GroupDesc &gd,
                                                 unsigned smask, bool streamed) {
  if ((((smask >> spmv_kind(MODE)) & 1u) != 0) != streamed) return 0u;
  unsigned act = 0u;
  for (int i = 0; i < gd.nmem; i++) {
    bool v;
    if (srv_spmv_active<MODE>(sts + gd.mem[i], &v)) act |= 1u << i;
  }
  return act;
}

template <int MODE>
__global__ void __launch_bounds__(kBlock, kSrvShareBlocks) k_srv_spmv(const Table *tab, SlotState *sts) {
  SRV_GROUP_PROLOGUE
  const SlotDesc &s0 = tab->slot[gd.mem[0]];
  const unsigned act = spmv_members<MODE>(sts, gd, s0.smask, false);
  if (!act) return;
  const Mat A = s0.A;
  __shared__ double *msp[kMaxMembers];
  __shared__ int mld[kMaxMembers];
  SRV_SHARED_MEMBERS(act, ([&](const SlotDesc &sd, void *(&p)[kMemberVecs]) {
                       spmv_vectors<MODE>(sd, p);
                       msp[threadIdx.x] = sd.sp;
                       mld[threadIdx.x] = sd.ld;
                     }))
  SliceSums<dots_of(MODE)> cur{nullptr, 0, {}};
  auto body = [&](int i, int row, double acc) {
    dots_row<MODE>(row, acc, (const double *)mv.p[i][0], (double *)mv.p[i][1],
                   (const double *)mv.p[i][2], (double *)mv.p[i][3], (const double *)mv.p[i][4],
                   cur);
  };
  auto end = [&](int i, int s) {
    cur.sp = msp[i];
    cur.ld = mld[i];
    cur.end(s);
  };
  shared_slices_any<double, double>(A, lb, gd.nb, ml, M, mv, body, end);
}

// ---- streamed operator kernels -----------------------------------------------
// The stream.cuh pipeline applied to a group: each of the group's blocks
// works for one active member (block lb: member lb % M of the M active
// ones, stages lb / M, lb / M + nbs / M, ...), so the members' blocks walk
// the same stages side by side and a stage's values come from HBM once and
// from L2 for the other members.  The member's vectors are its own; the
// arithmetic is that of the single-solve streaming kernels.
struct MemberWalk {
  int slot, j0, jstride;
};
__device__ __forceinline__ bool member_walk(const GroupDesc &gd, unsigned act, int lb,
                                            SlotState *sts, MemberWalk &w) {
  const int M = __popc(act);
  if (M == 0) return false;
  const int per = gd.nbs / M;
  if (per == 0) {  // the plan gives every group at least nmem blocks
    if (lb == 0 && threadIdx.x == 0) atomicExch(&sts[gd.mem[0]].k.timeout, 1);
    return false;
  }
  if (lb >= per * M) return false;
  const int k = lb % M;  // k-th active member
  int i = 0, seen = 0;
  for (; i < gd.nmem; i++)
    if ((act >> i) & 1u) {
      if (seen == k) break;
      seen++;
    }
  w.slot = gd.mem[i];
  w.j0 = lb / M;
  w.jstride = per;
  return true;
}

#define SRV_STREAM_PROLOGUE                                        \
  const int grp = tab->block_group_s[blockIdx.x];                 \
  if (grp < 0) return;                                            \
  const GroupDesc &gd = tab->group[grp];                          \
  const SlotDesc &s0 = tab->slot[gd.mem[0]];                      \
  const int lb = blockIdx.x - gd.bs0;

template <class V>
constexpr int prec_of() {
  return std::is_same<V, double>::value   ? AINV_PREC_FP64
         : std::is_same<V, float>::value  ? AINV_PREC_FP32
         : std::is_same<V, f32w>::value   ? AINV_PREC_FP32_ACC64
         : std::is_same<V, b16w>::value   ? AINV_PREC_BF16_ACC64
                                          : AINV_PREC_BF16;
}

// Epilogues whose pointers live in shared memory (staged once per block):
// each call rebuilds the epilogue from the shared copy, so the pointers are
// loaded where they are used and hold no registers across the stage loop
// (the single-solve kernels take them as kernel parameters instead).
template <class E>
struct SharedEpi {
  const E *sh;
  __device__ __forceinline__ RowVecs row_vecs() const { return sh->row_vecs(); }
  template <class A>
  __device__ __forceinline__ void post(int row, A acc, const StagedRows &r) const {
    E e = *sh;
    e.post(row, acc, r);
  }
};
template <int MODE>
struct SharedEpiDots {
  static constexpr int NV = dots_of(MODE);
  const EpiDots<MODE> *sh;
  double v[NV];  // the lane's row products of the current slice
  __device__ __forceinline__ RowVecs row_vecs() const { return sh->row_vecs(); }
  __device__ __forceinline__ void post(int i, double acc, const StagedRows &r) {
    EpiDots<MODE> e = *sh;
#pragma unroll
    for (int k = 0; k < NV; k++) e.ss.v[k] = v[k];
    e.post(i, acc, r);
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = e.ss.v[k];
  }
  __device__ __forceinline__ void end_slice(int s) {
    SliceSums<NV> ss{sh->ss.sp, sh->ss.ld, {}};
#pragma unroll
    for (int k = 0; k < NV; k++) ss.v[k] = v[k];
    ss.end(s);
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = 0.0;
  }
};

// stream_rows over the member's walk, with the operator's view and layout
// staged in shared memory.
template <int P, int RMAX, class V, class X, class Epi>
__device__ __forceinline__ void srv_stream(const Mat &mat, const StreamLayout &Lg,
                                           const X *__restrict__ x, Epi &epi, int *status,
                                           const MemberWalk &w) {
  __shared__ SellView<V> m;
  __shared__ StreamLayout L;
  __shared__ const StageDesc *stages;
  __shared__ int nstages;
  if (threadIdx.x == 0) {
    m = sview<V>(mat);
    L = Lg;
    stages = mat.stages;
    nstages = mat.nstages;
  }
  __syncthreads();
  stream_rows<P, RMAX>(m, stages, nstages, x, L, epi, status, w.j0, w.jstride);
}

template <class V, class T, int P>
__global__ void __launch_bounds__(kStreamThreads, kSrvStreamBlocks)
    k_srv_stream_sweep1(const Table *tab, SlotState *sts, int src) {
  SRV_STREAM_PROLOGUE
  const Mat &wt = s0.wt;
  if (wt.prec != prec_of<V>() || wt.pack != P) return;
  const unsigned act =
      sweep_members<acc64_prec(prec_of<V>())>(sts, gd, wt.prec, s0.smask, kSkSweep1, true);
  MemberWalk w;
  if (!member_walk(gd, act, lb, sts, w)) return;
  const SlotDesc &sd = tab->slot[w.slot];
  __shared__ EpiDscale<V, T> sh;
  if (threadIdx.x == 0) sh = EpiDscale<V, T>{(const V *)s0.d, (T *)sd.t};
  SharedEpi<EpiDscale<V, T>> epi{&sh};
  srv_stream<P, stream_rmax<V>(), V>(wt, s0.L[kSkSweep1], (const double *)sd.vec[src], epi,
                                     &sts[w.slot].k.timeout, w);
}

template <class V, class T, int P>
__global__ void __launch_bounds__(kStreamThreads, kSrvStreamBlocks)
    k_srv_stream_sweep2(const Table *tab, SlotState *sts, int dst) {
  SRV_STREAM_PROLOGUE
  const Mat &z = s0.z;
  if (z.prec != prec_of<V>() || z.pack != P) return;
  const unsigned act =
      sweep_members<acc64_prec(prec_of<V>())>(sts, gd, z.prec, s0.smask, kSkSweep2, true);
  MemberWalk w;
  if (!member_walk(gd, act, lb, sts, w)) return;
  const SlotDesc &sd = tab->slot[w.slot];
  __shared__ EpiAxpby sh;
  if (threadIdx.x == 0) sh = EpiAxpby{1.0, 0.0, sd.vec[dst]};
  SharedEpi<EpiAxpby> epi{&sh};
  srv_stream<P, stream_rmax<V>(), V>(z, s0.L[kSkSweep2], (const T *)sd.t, epi,
                                     &sts[w.slot].k.timeout, w);
}

template <int MODE, int P>
__global__ void __launch_bounds__(kStreamThreads, kSrvStreamBlocks)
    k_srv_stream_spmv(const Table *tab, SlotState *sts) {
  SRV_STREAM_PROLOGUE
  const Mat &A = s0.A;
  if (A.pack != P) return;
  const unsigned act = spmv_members<MODE>(sts, gd, s0.smask, true);
  MemberWalk w;
  if (!member_walk(gd, act, lb, sts, w)) return;
  const SlotDesc &sd = tab->slot[w.slot];
  __shared__ EpiDots<MODE> sh;
  if (threadIdx.x == 0) {
    void *p[kMemberVecs];
    spmv_vectors<MODE>(sd, p);
    sh = EpiDots<MODE>{(double *)p[1], (const double *)p[0], (const double *)p[2], (double *)p[3],
                       (const double *)p[4], {sd.sp, sd.ld, {}}};
  }
  SharedEpiDots<MODE> epi{&sh, {}};
  void *p[kMemberVecs];
  spmv_vectors<MODE>(sd, p);
  srv_stream<P, 1, double>(A, s0.L[spmv_kind(MODE)], (const double *)p[0], epi,
                           &sts[w.slot].k.timeout, w);
}

// ---- launch plan -----------------------------------------------------------------
enum Family { kFamStd = 1, kFamAcc64 = 2 };

// What one batched iteration launches, from the registered operators: the
// streamed kernel variants (precision and pack of W^T / Z, pack of A) with
// their shared memory, and the chunk-walking kernels still needed.
struct LaunchPlan {
  std::vector<std::pair<int, int>> sw1, sw2;  // (prec, pack)
  std::vector<int> spmv, strue;               // packs of A
  size_t smem[kNumSk] = {0, 0, 0, 0};
  int fb_sweep1 = 0, fb_sweep2 = 0;  // families of chunk-walked sweeps
  bool fb_spmv = false, fb_true = false;
  bool operator==(const LaunchPlan &o) const {
    return sw1 == o.sw1 && sw2 == o.sw2 && spmv == o.spmv && strue == o.strue &&
           std::equal(smem, smem + kNumSk, o.smem) && fb_sweep1 == o.fb_sweep1 &&
           fb_sweep2 == o.fb_sweep2 && fb_spmv == o.fb_spmv && fb_true == o.fb_true;
  }
};

// The streamed sweep kernel (WHICH = 1 or 2) of one value type and pack.
template <int WHICH, class V, class T, int P>
void *sweep_kernel_vp() {
  return WHICH == 1 ? (void *)k_srv_stream_sweep1<V, T, P> : (void *)k_srv_stream_sweep2<V, T, P>;
}
template <int WHICH, class V, class T>
void *sweep_kernel_p(int pack) {
  switch (pack) {
    case 1: return sweep_kernel_vp<WHICH, V, T, 1>();
    case 2: if constexpr (pack_ok<V, 2>()) return sweep_kernel_vp<WHICH, V, T, 2>(); break;
    case 4: if constexpr (pack_ok<V, 4>()) return sweep_kernel_vp<WHICH, V, T, 4>(); break;
    case 8: if constexpr (pack_ok<V, 8>()) return sweep_kernel_vp<WHICH, V, T, 8>(); break;
  }
  return nullptr;
}
template <int WHICH>
void *sweep_kernel(int prec, int pack) {
  switch (prec) {
    case AINV_PREC_FP64: return sweep_kernel_p<WHICH, double, double>(pack);
    case AINV_PREC_FP32: return sweep_kernel_p<WHICH, float, float>(pack);
    case AINV_PREC_BF16: return sweep_kernel_p<WHICH, __nv_bfloat16, float>(pack);
    case AINV_PREC_FP32_ACC64: return sweep_kernel_p<WHICH, f32w, double>(pack);
    case AINV_PREC_BF16_ACC64: return sweep_kernel_p<WHICH, b16w, double>(pack);
  }
  return nullptr;
}
template <int MODE>
void *spmv_kernel(int pack) {
  switch (pack) {
    case 1: return (void *)k_srv_stream_spmv<MODE, 1>;
    case 2: return (void *)k_srv_stream_spmv<MODE, 2>;
  }
  return nullptr;
}

// Grids of the streamed and slice-shared operator kernels (one resident
// wave each) and of the folds (2 blocks per SM: a fold has one block per
// 256-group range, 123 for a 200^3 slot).
int stream_grid() { return std::min(kMaxGrid, kSrvStreamBlocks * sm_count()); }
int share_grid() { return std::min(kMaxGrid, kSrvShareBlocks * sm_count()); }
int fold_grid() { return std::min(kMaxGrid, std::max(kMaxSlots, 2 * sm_count())); }

cudaError_t launch_raw(void *k, int grid, int threads, size_t smem, cudaStream_t s, void **args) {
  return cudaLaunchKernel(k, dim3(grid), dim3(threads), args, smem, s);
}

void sweeps(const Table *tab, SlotState *sts, int grid, cudaStream_t s, const LaunchPlan &lp,
            int src, int dst, int *count) {
  const int gs = stream_grid();
  for (const auto &v : lp.sw1) {
    void *args[] = {(void *)&tab, (void *)&sts, (void *)&src};
    launch_raw(sweep_kernel<1>(v.first, v.second), gs, kStreamThreads, lp.smem[kSkSweep1], s, args);
    ++*count;
  }
  const int gh = share_grid();
  if (lp.fb_sweep1 & kFamStd) k_srv_sweep1<false><<<gh, kBlock, 0, s>>>(tab, sts, src), ++*count;
  if (lp.fb_sweep1 & kFamAcc64) k_srv_sweep1<true><<<gh, kBlock, 0, s>>>(tab, sts, src), ++*count;
  for (const auto &v : lp.sw2) {
    void *args[] = {(void *)&tab, (void *)&sts, (void *)&dst};
    launch_raw(sweep_kernel<2>(v.first, v.second), gs, kStreamThreads, lp.smem[kSkSweep2], s, args);
    ++*count;
  }
  if (lp.fb_sweep2 & kFamStd) k_srv_sweep2<false><<<gh, kBlock, 0, s>>>(tab, sts, dst), ++*count;
  if (lp.fb_sweep2 & kFamAcc64) k_srv_sweep2<true><<<gh, kBlock, 0, s>>>(tab, sts, dst), ++*count;
}

template <int MODE>
void spmv(const Table *tab, SlotState *sts, int grid, cudaStream_t s, const LaunchPlan &lp,
          int *count) {
  const std::vector<int> &packs = MODE == kTrueRes ? lp.strue : lp.spmv;
  for (int pk : packs) {
    void *args[] = {(void *)&tab, (void *)&sts};
    launch_raw(spmv_kernel<MODE>(pk), stream_grid(), kStreamThreads, lp.smem[spmv_kind(MODE)], s,
               args);
    ++*count;
  }
  if (MODE == kTrueRes ? lp.fb_true : lp.fb_spmv) {
    k_srv_spmv<MODE><<<share_grid(), kBlock, 0, s>>>(tab, sts);
    ++*count;
  }
  k_srv_fold<dots_of(MODE), FinDotsSrv<MODE>><<<fold_grid(), kBlock, 0, s>>>(tab, sts, FinDotsSrv<MODE>{});
  ++*count;
}

// Start of a graph launch: new slots' vectors and first scalars.
void enqueue_init(const Table *tab, SlotState *sts, int grid, cudaStream_t s, int *count) {
  k_srv_init<<<grid, kBlock, 0, s>>>(tab, sts);
  k_srv_fold<1, FinInit><<<fold_grid(), kBlock, 0, s>>>(tab, sts, FinInit{});
  *count += 2;
}

// One batched iteration on stream s, the single-solve BiCGSTAB sequence.
cudaError_t enqueue_iteration(const Table *tab, SlotState *sts, int grid, cudaStream_t s,
                              const LaunchPlan &lp, int *count) {
  k_srv_p<<<grid, kBlock, 0, s>>>(tab, sts);
  sweeps(tab, sts, grid, s, lp, VP, VF, count);
  spmv<kBicgSigma>(tab, sts, grid, s, lp, count);
  k_srv_s<<<grid, kBlock, 0, s>>>(tab, sts);
  sweeps(tab, sts, grid, s, lp, VS, VZ, count);
  spmv<kBicgOmega>(tab, sts, grid, s, lp, count);
  k_srv_xr<<<grid, kBlock, 0, s>>>(tab, sts);
  k_srv_fold<2, FinXr><<<fold_grid(), kBlock, 0, s>>>(tab, sts, FinXr{});
  spmv<kTrueRes>(tab, sts, grid, s, lp, count);
  *count += 4;
  return cudaGetLastError();
}

// ------------------------------------------------------------------ host --
size_t round256(size_t b) { return (b + 255) / 256 * 256; }
size_t vec_stride(int n) { return ((size_t)n + 31) / 32 * 32; }  // doubles
int chunks_of(int n) { return (n + kChunkRows - 1) / kChunkRows; }

// Sizes of a slot's canonical-order reduction buffers.
struct FoldSizes {
  int ns, ng, nr, ld, ldr;
};
FoldSizes fold_sizes(int n) {
  FoldSizes z;
  z.ns = (n + kSlice - 1) / kSlice;
  z.ng = (z.ns + kGroupSlices - 1) / kGroupSlices;
  z.nr = (z.ng + kFoldRange - 1) / kFoldRange;
  z.ld = (z.ns + 31) / 32 * 32;
  z.ldr = (z.nr + 31) / 32 * 32;
  return z;
}

// Device bytes of one request's vectors: 11 FP64 vectors, the apply
// intermediate (<= 8 B per row), and the slice and range sums of 3 dots.
size_t request_bytes(int n) {
  const size_t st = vec_stride(n) * sizeof(double);
  const FoldSizes z = fold_sizes(n);
  return round256((kNumVec + 1) * st + 3 * sizeof(double) * ((size_t)z.ld + (size_t)z.ldr));
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
  // streamed operator kernels: layout and shared memory per kind, and
  // which kinds stream (bit k)
  StreamLayout L[kNumSk] = {};
  size_t smem[kNumSk] = {0, 0, 0, 0};
  unsigned smask = 0;
};

// The operator's streamed kinds.  By default every kind runs slice-shared:
// at 5 blocks per SM it served the 200^3 batch 1.26x faster than the
// streamed kernels (whose shared memory holds them to 3 blocks per SM).
// AINV_SERVER_STREAM=<mask> streams the kinds of the mask (bit k:
// StreamKind k) whose matrix the streaming layout takes and whose kernel
// variant exists.
void plan_operator(Operator &op) {
  static const unsigned allow = [] {
    const char *e = std::getenv("AINV_SERVER_STREAM");
    return e ? (unsigned)std::strtoul(e, nullptr, 0) : 0u;
  }();
  const ainv_handle *h = op.h;
  const int tsz = (h->prec == AINV_PREC_FP32 || h->prec == AINV_PREC_BF16) ? 4 : 8;
  const struct {
    const DevSell *m;
    int xs, nrv;
  } k[kNumSk] = {{&h->wt, 8, 1}, {&h->z, tsz, 0}, {&op.a->a, 8, 1}, {&op.a->a, 8, 3}};
  op.smask = 0;
  for (int q = 0; q < kNumSk; q++) {
    if (!((allow >> q) & 1u)) continue;
    StreamLayout L;
    size_t smem = 0;
    if (stream_plan(*k[q].m, k[q].xs, k[q].nrv, L, smem) <= 0) continue;
    const int prec = k[q].m->prec, pack = k[q].m->pack;
    void *kern = q == kSkSweep1   ? sweep_kernel<1>(prec, pack)
                 : q == kSkSweep2 ? sweep_kernel<2>(prec, pack)
                 : q == kSkSpmv   ? spmv_kernel<kBicgSigma>(pack)
                                  : spmv_kernel<kTrueRes>(pack);
    if (!kern || (q >= kSkSpmv && prec != AINV_PREC_FP64)) continue;
    op.L[q] = L;
    op.smem[q] = smem;
    op.smask |= 1u << q;
  }
}

// Union of the registered operators' launch needs.
LaunchPlan make_plan(const std::vector<Operator> &ops) {
  LaunchPlan lp;
  auto add = [](auto &v, auto x) {
    if (std::find(v.begin(), v.end(), x) == v.end()) v.push_back(x);
  };
  for (const Operator &op : ops) {
    const int fam = acc64_prec(op.h->prec) ? kFamAcc64 : kFamStd;
    for (int q = 0; q < kNumSk; q++) {
      const bool st = (op.smask >> q) & 1u;
      if (st) lp.smem[q] = std::max(lp.smem[q], op.smem[q]);
      switch (q) {
        case kSkSweep1:
          if (st) add(lp.sw1, std::make_pair(op.h->wt.prec, op.h->wt.pack));
          else lp.fb_sweep1 |= fam;
          break;
        case kSkSweep2:
          if (st) add(lp.sw2, std::make_pair(op.h->z.prec, op.h->z.pack));
          else lp.fb_sweep2 |= fam;
          break;
        case kSkSpmv:
          if (st) add(lp.spmv, op.a->a.pack);
          else lp.fb_spmv = true;
          break;
        default:
          if (st) add(lp.strue, op.a->a.pack);
          else lp.fb_true = true;
          break;
      }
    }
  }
  return lp;
}

// Allow every streamed kernel of the plan its shared memory.
bool plan_smem(const LaunchPlan &lp) {
  bool ok = true;
  for (const auto &v : lp.sw1) ok = ok && set_smem_attr(sweep_kernel<1>(v.first, v.second), lp.smem[kSkSweep1]);
  for (const auto &v : lp.sw2) ok = ok && set_smem_attr(sweep_kernel<2>(v.first, v.second), lp.smem[kSkSweep2]);
  for (int pk : lp.spmv) {
    ok = ok && set_smem_attr(spmv_kernel<kBicgSigma>(pk), lp.smem[kSkSpmv]);
    ok = ok && set_smem_attr(spmv_kernel<kBicgOmega>(pk), lp.smem[kSkSpmv]);
  }
  for (int pk : lp.strue) ok = ok && set_smem_attr(spmv_kernel<kTrueRes>(pk), lp.smem[kSkTrue]);
  return ok;
}

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
  ainv::srv::LaunchPlan plan, graph_plan;   // launches the operators need / in the graph
  int graph_kernels = 0;                    // kernel launches per graph launch
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

// Capture (or re-capture) the step graph for the launch plan `lp`: the
// init kernels and `iters` batched iterations.  Every kernel of the graph is
// first launched once on an all-idle table, so nothing loads during capture
// and no admitted request is advanced.
cudaError_t capture_graph(ainv_server *srv, const LaunchPlan &lp) {
  if (!plan_smem(lp)) return cudaErrorInvalidConfiguration;
  int count = 0;
  enqueue_init(srv->tab_empty_d, srv->st_d, srv->grid, srv->s, &count);
  cudaError_t e = enqueue_iteration(srv->tab_empty_d, srv->st_d, srv->grid, srv->s, lp, &count);
  if (e == cudaSuccess) e = cudaStreamSynchronize(srv->s);
  if (e != cudaSuccess) return e;
  e = cudaStreamBeginCapture(srv->s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  count = 0;
  enqueue_init(srv->tab_d, srv->st_d, srv->grid, srv->s, &count);
  cudaError_t ce = cudaGetLastError();
  for (int k = 0; k < srv->iters && ce == cudaSuccess; k++)
    ce = enqueue_iteration(srv->tab_d, srv->st_d, srv->grid, srv->s, lp, &count);
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
  srv->graph_plan = lp;
  srv->graph_kernels = count;
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

// Streamed operator kernels: group k gets minb[k] blocks (its members) plus a
// share of the rest in proportion to weight[k]; contiguous ranges.
int plan_stream(int ng, const long long *weight, const int *minb, int grid, int *b0, int *nb) {
  long long total = 0;
  int fixed = 0;
  for (int k = 0; k < ng; k++) {
    total += std::max(1LL, weight[k]);
    fixed += minb[k];
  }
  if (fixed > grid) {
    set_error("server stream plan: %d members for a grid of %d blocks", fixed, grid);
    return AINV_ERR_ARG;
  }
  int at = 0;
  for (int k = 0; k < ng; k++) {
    nb[k] = minb[k] + (int)((long long)(grid - fixed) * std::max(1LL, weight[k]) / std::max(1LL, total));
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
  for (int q = 0; q < kNumSk; q++) d.L[q] = op.L[q];
  d.smask = op.smask;
  const size_t st = vec_stride(r->n);
  double *base = reinterpret_cast<double *>(srv->arena_d + off);
  for (int v = 0; v < kNumVec; v++) d.vec[v] = base + (size_t)v * st;
  d.t = base + (size_t)kNumVec * st;
  const FoldSizes z = fold_sizes(r->n);
  d.ns = z.ns;
  d.ng = z.ng;
  d.nr = z.nr;
  d.ld = z.ld;
  d.ldr = z.ldr;
  d.sp = base + (size_t)(kNumVec + 1) * st;
  d.rs = d.sp + 3 * (size_t)z.ld;
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
      // fold blocks: shares of the fold grid in proportion to the ranges
      {
        std::vector<long long> fw(order.size());
        std::vector<int> fcap(order.size()), fb0(order.size()), fnb(order.size());
        for (size_t q = 0; q < order.size(); q++) {
          fw[q] = fcap[q] = srv->tab_h->slot[order[q]].nr;
        }
        if (plan_weighted((int)order.size(), fw.data(), fcap.data(), fold_grid(), fb0.data(),
                          fnb.data()) != AINV_SUCCESS) {
          fail_all(srv, AINV_ERR_INTERNAL, "server fold plan failed");
          return;
        }
        std::fill(srv->tab_h->block_slot_f, srv->tab_h->block_slot_f + kMaxGrid, (short)-1);
        for (size_t q = 0; q < order.size(); q++) {
          SlotDesc &d = srv->tab_h->slot[order[q]];
          d.fb0 = fb0[q];
          d.fnb = fnb[q];
          for (int b = d.fb0; b < d.fb0 + d.fnb; b++) srv->tab_h->block_slot_f[b] = (short)order[q];
        }
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
      if (plan_weighted(ng, gw.data(), gcap.data(), share_grid(), gb0.data(), gnb.data()) !=
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
      // the streamed grid: at least one block per member
      for (int g = 0; g < ng; g++) gcap[(size_t)g] = srv->tab_h->group[g].nmem;
      if (plan_stream(ng, gw.data(), gcap.data(), stream_grid(), gb0.data(), gnb.data()) !=
          AINV_SUCCESS) {
        fail_all(srv, AINV_ERR_INTERNAL, "server stream plan failed");
        return;
      }
      std::fill(srv->tab_h->block_group_s, srv->tab_h->block_group_s + kMaxGrid, (short)-1);
      for (int g = 0; g < ng; g++) {
        GroupDesc &gd = srv->tab_h->group[g];
        gd.bs0 = gb0[(size_t)g];
        gd.nbs = gnb[(size_t)g];
        for (int b = gd.bs0; b < gd.bs0 + gd.nbs; b++) srv->tab_h->block_group_s[b] = (short)g;
      }
      ENG_TRY(cudaMemcpyAsync(srv->tab_d, srv->tab_h, sizeof(Table), cudaMemcpyHostToDevice,
                              srv->s));
      dirty = false;
    }
    LaunchPlan lp;
    {
      std::lock_guard<std::mutex> lk(srv->mu);
      lp = srv->plan;
    }
    if (!(lp == srv->graph_plan)) ENG_TRY(capture_graph(srv, lp));  // new operator kinds
    ENG_TRY(cudaGraphLaunch(srv->exec, srv->s));
    ENG_TRY(cudaMemcpyAsync(srv->st_h, srv->st_d, sizeof(SlotState) * (size_t)S,
                            cudaMemcpyDeviceToHost, srv->s));
    ENG_TRY(cudaStreamSynchronize(srv->s));
    srv->launches++;
    std::vector<int> done;
    for (int k = 0; k < S; k++) {
      const SlotHost &sl = srv->slots[(size_t)k];
      // finished, or a streamed kernel gave up a bounded wait for it
      if (sl.req && ((srv->st_h[k].phase == kRun && srv->st_h[k].k.done) || srv->st_h[k].k.timeout)) {
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
        r->status = f.timeout ? AINV_ERR_TIMEOUT : f.status;
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
  std::fill(srv->tab_h->block_slot_f, srv->tab_h->block_slot_f + kMaxGrid, (short)-1);
  std::fill(srv->tab_h->block_group, srv->tab_h->block_group + kMaxGrid, (short)-1);
  std::fill(srv->tab_h->block_group_s, srv->tab_h->block_group_s + kMaxGrid, (short)-1);
  std::memset(srv->st_h, 0, sizeof(SlotState) * (size_t)max_slots);
  e = cudaMemcpy(srv->tab_d, srv->tab_h, sizeof(Table), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(srv->st_d, srv->st_h, sizeof(SlotState) * (size_t)max_slots,
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(e, "initial table");
  if ((e = cudaMalloc(&srv->tab_empty_d, sizeof(Table))) != cudaSuccess) return fail(e, "table");
  e = cudaMemcpy(srv->tab_empty_d, srv->tab_h, sizeof(Table), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(e, "empty table");
  if ((e = capture_graph(srv, LaunchPlan{})) != cudaSuccess) return fail(e, "graph capture");
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
  ainv::srv::Operator o;
  o.a = a;
  o.h = h;
  ainv::srv::plan_operator(o);
  std::lock_guard<std::mutex> lk(srv->mu);
  srv->ops.push_back(o);
  srv->plan = ainv::srv::make_plan(srv->ops);
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
  out->kernel_launches = srv->launches * (long long)srv->graph_kernels;
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
