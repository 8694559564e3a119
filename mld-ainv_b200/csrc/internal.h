// Internal declarations shared by the ainv_b200 translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "ainv_b200.h"

namespace ainv {

// ------------------------------------------------------------ errors --
void set_error(const char *fmt, ...);

#define AINV_CUDA_TRY(expr)                                                   \
  do {                                                                        \
    cudaError_t e_ = (expr);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      ::ainv::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                  \
      return AINV_ERR_CUDA;                                                   \
    }                                                                         \
  } while (0)

#define AINV_TRY(expr)           \
  do {                           \
    int rc_ = (expr);            \
    if (rc_ != AINV_SUCCESS) return rc_; \
  } while (0)

// ------------------------------------------------------ host sparse --
// 0-based CSR with sorted column indices inside each row.
struct HostCsr {
  int n = 0;
  std::vector<int> irp;  // n+1
  std::vector<int> ja;   // nnz
  std::vector<double> val;
  long long nnz() const { return irp.empty() ? 0 : irp.back(); }
};

// Validate and copy a caller CSR (optionally 1-based) into a HostCsr.
int import_csr(int n, const int *irp, const int *ja, const double *val,
               int one_based, HostCsr &out, const char *what);
// Transpose (CSR of A^T); indices come out sorted.
HostCsr transpose(const HostCsr &a);

// ------------------------------------------------------ device layout --
// Sliced layout, 32 rows per slice, slots stored column-major: slot k of
// lane l of slice s is value val[sptr[s] + 32*k + l].  Each slice picks the
// cheaper of two index encodings:
//   offset mode: the slice's rows share one sorted list of column offsets
//     (col - row); the slice stores that list once (iptr[s+1]-iptr[s] == w
//     entries) and slot k of every lane holds the value at offset idx[k], or
//     0 where that row has no entry.  Stencil-derived factors are all in
//     this mode, so almost no index bytes are streamed and the gathers of
//     the 32 lanes are contiguous.
//   column mode (SELL): one int32 column per slot (32*w entries); padding
//     slots carry value 0 and the row's own index.
// w is the slice width (slots per lane), a multiple of the pack P: the P
// slots kP..kP+P-1 of one lane are adjacent in memory, so a lane reads them
// with one vector load (slot k of lane l at sptr[s] + (k/P)*32P + l*P + k%P;
// per-slot columns use the same arrangement).  P is chosen per matrix (up to
// 16 bytes per load) as long as padding to a multiple of P costs <= 6%.
constexpr int kSlice = 32;
constexpr int kMaxOffsets = 64;  // offset mode only for slices with <= 64 offsets

// A stage is stage_slices consecutive slices (kConsumerSlices per consumer
// warp times a per-precision factor) streamed into shared memory by bulk
// asynchronous copies: its descriptor, its slice pointers, values, index
// words and, for uniform stages, the windows of the gathered vector.  A
// stage is "uniform" when all its slices use offset mode with one identical
// offset list of at most kStageMaxOffsets entries; its gathers then read
// contiguous windows x[r0+o, r1+o) that are copied too.  Offsets (sorted)
// within kWindowSpan elements of their cluster's first offset share one
// window, x[r0+o_first, r1+o_last): a new cluster starts at the first offset
// more than kWindowSpan past the current cluster's first offset.  Built on
// the host at upload; consumed by the streaming kernels.
constexpr int kConsumerSlices = 8;   // consumer warps per streaming block
constexpr int kStageMaxOffsets = 8;
constexpr int kWindowSpan = 16;
constexpr int kMaxStageSlices = 32;
struct alignas(16) StageDesc {
  int s0, s1;          // slice range [s0, s1)
  int vstart;          // first value (element index, = sptr[s0])
  int vbytes;          // value bytes (multiple of 16)
  long long ibyte0;    // first index byte copied (16-aligned)
  int ibytes;          // index bytes copied (multiple of 16)
  int noff;            // uniform: number of offsets (bits 0-7, else 0) and the
                       // offsets that start a window cluster (bit 8 + k)
  int off[kStageMaxOffsets];
};
static_assert(sizeof(StageDesc) == 64, "stage descriptor is one 64-byte copy");

struct DevSell {
  int n = 0;
  int nslices = 0;
  long long nnz = 0;    // real entries
  long long slots = 0;  // stored values incl. padding
  long long nidx = 0;   // stored index words
  int offset_slices = 0;
  int pack = 1;  // P
  int prec = AINV_PREC_FP64;
  int *sptr = nullptr;  // nslices+1 value offsets (+16 bytes of tail padding)
  int *iptr = nullptr;  // nslices+1 index offsets (+16 bytes of tail padding)
  int *idx = nullptr;   // nidx offsets / columns (+16 bytes of tail padding)
  void *val = nullptr;  // slots, element type from prec
  // streaming stages (see StageDesc); nstages = 0 when not streamable
  int nstages = 0;
  int stage_slices = 0;
  int stage_vmax = 0, stage_imax = 0, stage_noff_max = 0;
  int stage_nwin_max = 0;  // windows (offset clusters) of a uniform stage
  StageDesc *stages = nullptr;
  // host copy: the largest column each slice reads (-1 for an empty slice);
  // a sweep over rows of a slice range needs its input only up to there
  std::vector<int> slice_maxcol;
  size_t bytes() const;
};

size_t prec_size(int prec);
int upload_sell(const HostCsr &a, int prec, DevSell &out);
void free_sell(DevSell &m);

// Convert n doubles on the host to device storage of type prec.
int upload_values(const double *h, size_t n, int prec, void **dptr);

}  // namespace ainv

namespace ainv {
struct KrylovWs;
void destroy_ws(KrylovWs *w);
struct MrhsWs;
void destroy_mws(MrhsWs *w);
// Process-unique id for handles (keys cached CUDA graphs; never reused).
unsigned long long next_serial();
}  // namespace ainv

namespace ainv {
// Schedule of the host-array apply pipeline for one trans.  Chunk c of the
// vectors is slices [bound[c], bound[c+1]); sweep 1 of chunk c reads input
// chunks up to need1[c].  Sweep 2 and the copy out run in units: unit u is
// slices [u0[u], u1[u]) and reads t up to chunk need2[u].
struct HostPipe;
struct HostPlan {
  int cs = 0;  // nominal slices per chunk the plan was made for
  std::vector<int> bound, need1, u0, u1, need2;
};
}  // namespace ainv

// ------------------------------------------------------------- handles --
struct ainv_handle {
  unsigned long long serial = 0;
  int n = 0;
  int prec = AINV_PREC_FP64;
  ainv::DevSell wt;  // 'N' sweep 1: W^T
  ainv::DevSell z;   // 'N' sweep 2: Z
  ainv::DevSell zt;  // 'T' sweep 1: Z^T
  ainv::DevSell w;   // 'T' sweep 2: W
  void *d = nullptr;      // D^-1 in prec
  void *t = nullptr;      // intermediate D^-1 W^T x (double for FP64, float otherwise)
  double *xs = nullptr;   // device staging for the host-array apply
  double *ys = nullptr;
  int *status = nullptr;  // device word: nonzero after a streaming wait timed out
  // host-array apply pipeline: copy-in, sweep and copy-out streams, events,
  // and the schedule for 'N' and 'T'
  cudaStream_t hs[3] = {nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> hev;
  ainv::HostPlan hplan[2];
  ainv::HostPipe *pipe = nullptr;  // the persistent-kernel form of the pipeline
};

namespace ainv {
// The host-array apply as copies of x plus one persistent kernel
// (hostpipe.cu).  usable: the two sweeps share a pack width and y is
// device-mapped page-locked memory.  apply enqueues on si (copies) and sc
// (the kernel), ordered after whatever precedes them there; status reports
// a timed-out wait of the last call, after the streams are synchronised.
bool host_pipe_usable(const ainv_handle *h, bool tr, const double *y);
int host_pipe_apply(ainv_handle *h, bool tr, const HostPlan &p, double alpha, const double *x,
                    double beta, double *y, cudaStream_t si, cudaStream_t sc);
int host_pipe_status(const ainv_handle *h);
void destroy_host_pipe(HostPipe *hp);
}  // namespace ainv

struct ainv_csr {
  int n = 0;
  int *status = nullptr;  // device word: nonzero after a streaming wait timed out
  ainv::DevSell a;
  ainv::KrylovWs *ws = nullptr;  // Krylov vectors, state and captured graph
  ainv::MrhsWs *mws = nullptr;   // the same for multi-right-hand-side solves
};

// ------------------------------------------------------------- kernels --
namespace ainv {
// t = d .* (M x) with M, d in prec; t is double (FP64) or float (mixed).
// stop: optional device flag; when nonzero the kernel returns at once.
int launch_sweep_dscale(const DevSell &m, const void *d, const double *x, void *t,
                        cudaStream_t s, const int *stop = nullptr, int *status = nullptr);
// y = alpha * M t + beta * y; t as produced by launch_sweep_dscale.
int launch_sweep_axpby(const DevSell &m, const void *t, double alpha, double beta,
                       double *y, cudaStream_t s, const int *stop = nullptr,
                       int *status = nullptr);
// The same two sweeps over the rows of slices [s0, s1) only (register path;
// s0 a multiple of 4).  Rows outside the range are neither read nor written.
int launch_sweep_dscale_slices(const DevSell &m, const void *d, const double *x, void *t,
                               int s0, int s1, cudaStream_t s);
int launch_sweep_axpby_slices(const DevSell &m, const void *t, double alpha, double beta,
                              double *y, int s0, int s1, cudaStream_t s);
// y = alpha * A x + beta * y with an FP64 operator.
int launch_spmv(const DevSell &a, double alpha, const double *x, double beta,
                double *y, cudaStream_t s, int *status = nullptr);
// Both sweeps of the apply for trans 'N' or 'T'/'C'.
// status: device word for wait timeouts (the handle's own when null).
// update_a (src/impl/mld_d_base_ainv_update_a.f90:53-79) on stream s:
// d <- 1/(1/d_old + diag(W^T diag(x) Z)), d_old read from d64_in when given
// (FP64) else from the handle's device d; the new d is stored in the
// handle (its precision) and, when d64 is given, in FP64.  d64 may alias
// d64_in.
int update_a_async(ainv_handle *h, const double *x, const double *d64_in, double *d64,
                   cudaStream_t s);
int ainv_apply_async(const ainv_handle *h, char trans, double alpha, const double *x,
                     double beta, double *y, cudaStream_t s, const int *stop = nullptr,
                     int *status = nullptr);
}  // namespace ainv
