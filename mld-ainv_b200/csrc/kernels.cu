// sm_100a kernels for the factor sweeps of the AINV apply and the A SpMV.
//
// Layout: 32-row slices (see internal.h).  One warp owns one slice, one lane
// one row; slot k of a slice is a 32-wide contiguous run of values, so each
// value load of the warp is one coalesced 256 B (FP64) request.  Slices of
// stencil-derived factors store one shared list of column offsets instead of
// per-entry indices, so the streamed bytes are essentially the values alone
// and the gathers of a warp are contiguous.  Factor values are read exactly
// once per apply and use the streaming (evict-first) hint, so the gathered
// vectors (x and t: 64 MB at n = 8M, inside the 126 MB L2) stay resident
// between the two sweeps.
//
// Epilogues are fused: sweep 1 writes t = D^-1 .* (W^T x), sweep 2 writes
// y = alpha*Z t + beta*y, so the reference's three passes
// (src/impl/mld_d_base_ainv_solver_apply_vect.f90:114-119) become two.
// `stop` (optional) is a device flag set by the Krylov loop once it has
// converged; kernels launched after that return immediately.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <map>
#include <tuple>
#include <utility>

#include "stream.cuh"

namespace ainv {
namespace {

using namespace dev;

template <class V, class T, int S, int P>
__global__ void __launch_bounds__(kBlock)
    k_sweep_dscale(SellView<V> m, const double *__restrict__ x, const V *__restrict__ d,
                   T *__restrict__ t, const int *__restrict__ stop) {
  if (stop && *stop) return;
  for_each_row<S, P>(m, x, [&](int row, auto acc) { t[row] = (T)(ldd(d + row) * acc); });
}

// Every sweep-2 epilogue (register, slice-range, streaming and the host-array
// pipeline kernels) uses axpby_row, so all forms give the same bits.
template <class V, class T, int S, int P>
__global__ void __launch_bounds__(kBlock)
    k_sweep_axpby(SellView<V> m, const T *__restrict__ t, double alpha, double beta,
                  double *__restrict__ y, const int *__restrict__ stop) {
  if (stop && *stop) return;
  for_each_row<S, P>(m, t, [&](int row, auto acc) {
    y[row] = axpby_row(alpha, (double)acc, beta, beta == 0.0 ? 0.0 : y[row]);
  });
}

// Slice-range forms: groups [g0, g1) of S slices (the host-array pipeline).
template <class V, class T, int S, int P>
__global__ void __launch_bounds__(kBlock)
    k_sweep_dscale_range(SellView<V> m, const double *__restrict__ x, const V *__restrict__ d,
                         T *__restrict__ t, int g0, int g1) {
  for_each_row<S, P>(
      m, x, [&](int row, auto acc) { t[row] = (T)(ldd(d + row) * acc); }, g0, g1);
}

template <class V, class T, int S, int P>
__global__ void __launch_bounds__(kBlock)
    k_sweep_axpby_range(SellView<V> m, const T *__restrict__ t, double alpha, double beta,
                        double *__restrict__ y, int g0, int g1) {
  for_each_row<S, P>(
      m, t,
      [&](int row, auto acc) {
        y[row] = axpby_row(alpha, (double)acc, beta, beta == 0.0 ? 0.0 : y[row]);
      },
      g0, g1);
}

// ---- streaming variants (stream.cuh) ----------------------------------------
template <class V, class X, int P, class Epi>
__global__ void __launch_bounds__(kStreamThreads, kStreamMinBlocks)
    k_stream(SellView<V> m, const StageDesc *__restrict__ stages, int nstages,
             const X *__restrict__ x, StreamLayout L, Epi epi, int *status,
             const int *__restrict__ stop) {
  if (stop && *stop) return;
  stream_rows<P, stream_rmax<V>()>(m, stages, nstages, x, L, epi, status);
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

namespace dev {
int group_size(int prec) {
  static const int forced = [] {
    const char *e = std::getenv("AINV_SLICES_PER_WARP");
    const int v = e ? std::atoi(e) : 0;
    return (v == 1 || v == 2 || v == 4) ? v : 0;
  }();
  if (forced) return forced;
  return 2;
}

// Streaming (stream.cuh) is the default where it measured faster on B200 --
// FP32 and BF16 factors, and sweep 1 (the D^-1 epilogue) of FP64 factors
// (0.095 vs 0.102 ms at 200^3); FP64 sweep 2 (0.102 vs 0.086 ms) and the FP64
// operator A use the register kernels.  Both families sum the same products
// in the same slot order.  AINV_STREAM=0 / 1 forces one choice for every
// matrix.
namespace {
int stream_forced() {
  static const int forced = [] {
    const char *e = std::getenv("AINV_STREAM");
    return e ? (std::atoi(e) != 0 ? 1 : 0) : -1;
  }();
  return forced;
}
}  // namespace
bool stream_enabled(int prec) {
  if (stream_forced() >= 0) return stream_forced() == 1;
  return prec != AINV_PREC_FP64;
}
bool stream_enabled_sweep1(int prec) {
  if (stream_forced() >= 0) return stream_forced() == 1;
  (void)prec;
  return true;
}

int sm_count() {
  static int sms[64] = {};
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) d = 0;
  if (sms[d] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d) != cudaSuccess || v <= 0)
      v = 148;
    sms[d] = v;
  }
  return sms[d];
}

int occupancy_grid(const void *kernel, int threads, size_t smem, int grid) {
  // blocks of this kernel that fit on an SM at once (registers and shared
  // memory), cached per kernel, shared memory size and device
  static std::mutex mu;
  static std::map<std::tuple<const void *, size_t, int>, int> cache;
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) d = 0;
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find({kernel, smem, d});
    if (it != cache.end()) per_sm = it->second;
  }
  if (per_sm == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) !=
            cudaSuccess ||
        per_sm < 1) {
      cudaGetLastError();
      per_sm = 1;
    }
    std::lock_guard<std::mutex> lock(mu);
    cache[{kernel, smem, d}] = per_sm;
  }
  return std::max(1, std::min(grid, per_sm * sm_count()));
}

bool set_smem_attr(const void *kernel, size_t bytes) {
  // opt in to the dynamic shared memory this launch needs (kept per kernel
  // and device); a refusal leaves no error pending and reports false
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, size_t> granted;
  int d = 0;
  cudaGetDevice(&d);
  std::lock_guard<std::mutex> lock(mu);
  size_t &g = granted[{kernel, d}];
  if (bytes <= g || bytes <= 48 * 1024) return true;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
      cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  g = bytes;
  return true;
}

int stream_plan(const DevSell &m, int xs, int nrv, StreamLayout &L, size_t &smem_bytes) {
  if (m.nstages <= 0 || !m.stages || m.stage_slices <= 0) return 0;
  if (m.stage_slices % kConsumerWarps != 0 || m.stage_slices > kMaxStageSlices) return 0;
  auto r128 = [](long long b) { return (int)((b + 127) / 128 * 128); };
  L.R = m.stage_slices / kConsumerWarps;
  L.vb = r128(m.stage_vmax);
  L.ib = r128(m.stage_imax);
  // a window: the stage's rows, its offset cluster's span and granule slack
  L.xw = (int)(((long long)(m.stage_slices * kSlice + kWindowSpan) * xs + 32 + 15) / 16 * 16);
  L.nwin = m.stage_nwin_max;
  L.nrv = std::max(0, std::min(kMaxRowVecs, nrv));
  L.rw = (int)(((long long)m.stage_slices * kSlice * 8 + 15) / 16 * 16);
  L.stage = r128((long long)kHeaderBytes + L.vb + L.ib + (long long)L.nwin * L.xw +
                 (long long)L.nrv * L.rw);
  if (L.stage > kStreamStageMax) return 0;
  // shared memory per block (tunable: AINV_STREAM_SMEM_KB); a smaller budget
  // means fewer buffers per block but more blocks (producers) per SM
  static const int budget = [] {
    const char *e = std::getenv("AINV_STREAM_SMEM_KB");
    const int v = e ? std::atoi(e) : 0;
    return v >= 16 && v <= 220 ? v * 1024 : kStreamBlockBudget;
  }();
  L.D = std::max(2, std::min(8, budget / L.stage));
  smem_bytes = 128 + (size_t)L.D * L.stage;
  if (smem_bytes > (size_t)kStreamSmemMax) return 0;
  const int per_sm = std::max(1, std::min(4, (int)(kStreamSmemSM / (smem_bytes + 1024))));
  return std::min(m.nstages, per_sm * sm_count());
}

int wave_grid(const void *kernel, long long rows) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, int> cache;
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) d = 0;
  int wave;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find({d, kernel});
    if (it != cache.end()) {
      wave = it->second;
    } else {
      int per_sm = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0) !=
              cudaSuccess ||
          per_sm <= 0) {
        cudaGetLastError();
        per_sm = 1;
      }
      wave = per_sm * sm_count();
      cache[{d, kernel}] = wave;
    }
  }
  const long long units = (rows + kBlock - 1) / kBlock;
  return (int)std::max(1LL, std::min(units, (long long)wave));
}

int reduction_grid(long long rows) {
  static int sms[64] = {};
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) d = 0;
  if (sms[d] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d) != cudaSuccess || v <= 0)
      v = 148;
    sms[d] = v;
  }
  const long long units = (rows + kBlock - 1) / kBlock;
  const long long wave = 8LL * sms[d];
  return (int)std::max(1LL, std::min(units, wave));
}
}  // namespace dev

namespace {

template <class V, class T>
struct DscaleLaunch {
  const DevSell &m;
  const void *d;
  const double *x;
  void *t;
  cudaStream_t s;
  const int *stop;
  template <int S, int P>
  void run() const {
    launch(k_sweep_dscale<V, T, S, P>, grid_for_groups(m.nslices, S), kBlock, 0, s, view<V>(m),
           x, (const V *)d, (T *)t, stop);
  }
};

template <class V, class T>
struct AxpbyLaunch {
  const DevSell &m;
  const void *t;
  double alpha, beta;
  double *y;
  cudaStream_t s;
  const int *stop;
  template <int S, int P>
  void run() const {
    launch(k_sweep_axpby<V, T, S, P>, grid_for_groups(m.nslices, S), kBlock, 0, s, view<V>(m),
           (const T *)t, alpha, beta, y, stop);
  }
};

template <class V, class T>
struct DscaleRangeLaunch {
  const DevSell &m;
  const void *d;
  const double *x;
  void *t;
  int s0, s1;
  cudaStream_t s;
  template <int S, int P>
  void run() const {
    const int g0 = s0 / S, g1 = (s1 + S - 1) / S;
    k_sweep_dscale_range<V, T, S, P><<<grid_for(g1 - g0), kBlock, 0, s>>>(
        view<V>(m), x, (const V *)d, (T *)t, g0, g1);
  }
};

template <class V, class T>
struct AxpbyRangeLaunch {
  const DevSell &m;
  const void *t;
  double alpha, beta;
  double *y;
  int s0, s1;
  cudaStream_t s;
  template <int S, int P>
  void run() const {
    const int g0 = s0 / S, g1 = (s1 + S - 1) / S;
    k_sweep_axpby_range<V, T, S, P><<<grid_for(g1 - g0), kBlock, 0, s>>>(
        view<V>(m), (const T *)t, alpha, beta, y, g0, g1);
  }
};

// The epilogue's row vectors as seen from the host (same rule as row_vecs()).
template <class V, class T>
RowVecs host_row_vecs(const EpiDscale<V, T> &e) {
  return RowVecs{{e.d, nullptr, nullptr}, {(int)sizeof(V), 0, 0}};
}
inline RowVecs host_row_vecs(const EpiAxpby &e) {
  return RowVecs{{e.beta == 0.0 ? nullptr : e.y, nullptr, nullptr}, {8, 0, 0}};
}

template <class V, class X, class Epi>
struct StreamLaunch {
  const DevSell &m;
  const X *x;
  Epi epi;
  int *status;
  cudaStream_t s;
  const int *stop;
  int grid;
  StreamLayout L;
  size_t smem;
  bool *launched;
  template <int S, int P>
  void run() const {
    auto kern = k_stream<V, X, P, Epi>;
    if (!set_smem_attr((const void *)kern, smem)) return;
    const int g = occupancy_grid((const void *)kern, kStreamThreads, smem, grid);
    launch(kern, g, kStreamThreads, smem, s, view<V>(m), (const StageDesc *)m.stages, m.nstages,
           x, L, epi, status, stop);
    *launched = true;
  }
};

// Streaming launch when the layout allows it (returns false otherwise).
template <class V, class X, class Epi>
bool try_stream(const DevSell &m, const X *x, const Epi &epi, int *status, cudaStream_t s,
                const int *stop, bool sweep1 = false) {
  if (!status || !(sweep1 ? stream_enabled_sweep1(m.prec) : stream_enabled(m.prec)))
    return false;
  if ((reinterpret_cast<uintptr_t>(x) & 15u) != 0) return false;  // bulk copies need 16 B
  const RowVecs rv = host_row_vecs(epi);
  for (int i = 0; i < kMaxRowVecs; i++)
    if (rv.p[i] && (reinterpret_cast<uintptr_t>(rv.p[i]) & 15u) != 0) return false;
  StreamLayout L;
  size_t smem = 0;
  const int grid = stream_plan(m, (int)sizeof(X), Epi::kRowVecs, L, smem);
  if (grid <= 0) return false;
  bool launched = false;
  with_pack<V, 1>(m.pack, StreamLaunch<V, X, Epi>{m, x, epi, status, s, stop, grid, L, smem,
                                                   &launched});
  return launched;
}

template <class V, class T>
void sweep_dscale(const DevSell &m, const void *d, const double *x, void *t, cudaStream_t s,
                  const int *stop, int *status) {
  if (try_stream<V>(m, x, EpiDscale<V, T>{(const V *)d, (T *)t}, status, s, stop, true)) return;
  with_group_pack<V>(group_size(m.prec), m.pack, DscaleLaunch<V, T>{m, d, x, t, s, stop});
}

template <class V, class T>
void sweep_axpby(const DevSell &m, const void *t, double alpha, double beta, double *y,
                 cudaStream_t s, const int *stop, int *status) {
  if (try_stream<V>(m, (const T *)t, EpiAxpby{alpha, beta, y}, status, s, stop)) return;
  with_group_pack<V>(group_size(m.prec), m.pack,
                     AxpbyLaunch<V, T>{m, t, alpha, beta, y, s, stop});
}

}  // namespace

int launch_sweep_dscale(const DevSell &m, const void *d, const double *x, void *t,
                        cudaStream_t s, const int *stop, int *status) {
  if (m.nslices == 0) return AINV_SUCCESS;
  switch (m.prec) {
    case AINV_PREC_FP64: sweep_dscale<double, double>(m, d, x, t, s, stop, status); break;
    case AINV_PREC_FP32: sweep_dscale<float, float>(m, d, x, t, s, stop, status); break;
    case AINV_PREC_BF16: sweep_dscale<__nv_bfloat16, float>(m, d, x, t, s, stop, status); break;
    case AINV_PREC_FP32_ACC64: sweep_dscale<f32w, double>(m, d, x, t, s, stop, status); break;
    case AINV_PREC_BF16_ACC64: sweep_dscale<b16w, double>(m, d, x, t, s, stop, status); break;
    default:
      set_error("unknown precision %d", m.prec);
      return AINV_ERR_ARG;
  }
  return check_launch("sweep_dscale");
}

int launch_sweep_axpby(const DevSell &m, const void *t, double alpha, double beta,
                       double *y, cudaStream_t s, const int *stop, int *status) {
  if (m.nslices == 0) return AINV_SUCCESS;
  switch (m.prec) {
    case AINV_PREC_FP64: sweep_axpby<double, double>(m, t, alpha, beta, y, s, stop, status); break;
    case AINV_PREC_FP32: sweep_axpby<float, float>(m, t, alpha, beta, y, s, stop, status); break;
    case AINV_PREC_BF16: sweep_axpby<__nv_bfloat16, float>(m, t, alpha, beta, y, s, stop, status); break;
    case AINV_PREC_FP32_ACC64: sweep_axpby<f32w, double>(m, t, alpha, beta, y, s, stop, status); break;
    case AINV_PREC_BF16_ACC64: sweep_axpby<b16w, double>(m, t, alpha, beta, y, s, stop, status); break;
    default:
      set_error("unknown precision %d", m.prec);
      return AINV_ERR_ARG;
  }
  return check_launch("sweep_axpby");
}

namespace {
// Storage type V and intermediate type T of a precision, as a tag.
template <class V_, class T_>
struct Types {
  using V = V_;
  using T = T_;
};
template <class F>
int by_prec(int prec, F &&f) {
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

int check_range(const DevSell &m, int s0, int s1) {
  if (s0 < 0 || s1 > m.nslices || s0 > s1 || (s0 & 3) != 0) {
    set_error("slice range [%d, %d) invalid for %d slices", s0, s1, m.nslices);
    return AINV_ERR_ARG;
  }
  return AINV_SUCCESS;
}
}  // namespace

int launch_sweep_dscale_slices(const DevSell &m, const void *d, const double *x, void *t,
                               int s0, int s1, cudaStream_t s) {
  AINV_TRY(check_range(m, s0, s1));
  if (s0 == s1) return AINV_SUCCESS;
  AINV_TRY(by_prec(m.prec, [&](auto ty) {
    using V = typename decltype(ty)::V;
    using T = typename decltype(ty)::T;
    with_group_pack<V>(group_size(m.prec), m.pack, DscaleRangeLaunch<V, T>{m, d, x, t, s0, s1, s});
  }));
  return check_launch("sweep_dscale (slices)");
}

int launch_sweep_axpby_slices(const DevSell &m, const void *t, double alpha, double beta,
                              double *y, int s0, int s1, cudaStream_t s) {
  AINV_TRY(check_range(m, s0, s1));
  if (s0 == s1) return AINV_SUCCESS;
  AINV_TRY(by_prec(m.prec, [&](auto ty) {
    using V = typename decltype(ty)::V;
    using T = typename decltype(ty)::T;
    with_group_pack<V>(group_size(m.prec), m.pack,
                       AxpbyRangeLaunch<V, T>{m, t, alpha, beta, y, s0, s1, s});
  }));
  return check_launch("sweep_axpby (slices)");
}

int launch_spmv(const DevSell &a, double alpha, const double *x, double beta, double *y,
                cudaStream_t s, int *status) {
  if (a.prec != AINV_PREC_FP64) {
    set_error("operator A must be stored in FP64");
    return AINV_ERR_ARG;
  }
  if (a.nslices == 0) return AINV_SUCCESS;
  sweep_axpby<double, double>(a, x, alpha, beta, y, s, nullptr, status);
  return check_launch("spmv");
}

int ainv_apply_async(const ainv_handle *h, char trans, double alpha, const double *x,
                     double beta, double *y, cudaStream_t s, const int *stop, int *status) {
  int *st = status ? status : h->status;
  switch (trans) {
    case 'N': case 'n':
      AINV_TRY(launch_sweep_dscale(h->wt, h->d, x, h->t, s, stop, st));
      return launch_sweep_axpby(h->z, h->t, alpha, beta, y, s, stop, st);
    case 'T': case 't': case 'C': case 'c':
      AINV_TRY(launch_sweep_dscale(h->zt, h->d, x, h->t, s, stop, st));
      return launch_sweep_axpby(h->w, h->t, alpha, beta, y, s, stop, st);
    default:
      // psb_err_iarg_invalid_i_ (src/impl/mld_d_base_ainv_solver_apply_vect.f90:64-71)
      set_error("invalid trans '%c'", trans);
      return AINV_ERR_ARG;
  }
}

}  // namespace ainv
