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
// SELL-32: rows are taken 32 at a time ("slices"); a slice of width w holds
// 32*w slots stored column-major, slot (k, lane) at sptr[s] + 32*k + lane.
// Padding slots carry value 0 and the row's own index as column, so every
// gather stays in bounds and lands next to data the warp already touches.
constexpr int kSlice = 32;

struct DevSell {
  int n = 0;
  int nslices = 0;
  long long nnz = 0;    // real entries
  long long slots = 0;  // stored entries incl. padding
  int prec = AINV_PREC_FP64;
  int *sptr = nullptr;  // nslices+1 slot offsets
  int *col = nullptr;   // slots
  void *val = nullptr;  // slots, element type from prec
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
// Process-unique id for handles (keys cached CUDA graphs; never reused).
unsigned long long next_serial();
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
};

struct ainv_csr {
  int n = 0;
  ainv::DevSell a;
  ainv::KrylovWs *ws = nullptr;  // Krylov vectors, state and captured graph
};

// ------------------------------------------------------------- kernels --
namespace ainv {
// t = d .* (M x) with M, d in prec; t is double (FP64) or float (mixed).
// stop: optional device flag; when nonzero the kernel returns at once.
int launch_sweep_dscale(const DevSell &m, const void *d, const double *x, void *t,
                        cudaStream_t s, const int *stop = nullptr);
// y = alpha * M t + beta * y; t as produced by launch_sweep_dscale.
int launch_sweep_axpby(const DevSell &m, const void *t, double alpha, double beta,
                       double *y, cudaStream_t s, const int *stop = nullptr);
// y = alpha * A x + beta * y with an FP64 operator.
int launch_spmv(const DevSell &a, double alpha, const double *x, double beta,
                double *y, cudaStream_t s);
// Both sweeps of the apply for trans 'N' or 'T'/'C'.
int ainv_apply_async(const ainv_handle *h, char trans, double alpha, const double *x,
                     double beta, double *y, cudaStream_t s, const int *stop = nullptr);
}  // namespace ainv
