// Apply entry point that allocates no memory.
//
// Some callers cannot allocate device memory at the moment they apply the
// preconditioner: an embedding framework that hands out all device memory
// from its own pool and forbids cudaMalloc outside it, or a host thread in
// a latency-critical section where a cudaMalloc/cudaFree (which may
// synchronise the device) is not acceptable.  Such a caller keeps W^T, Z
// and D^-1 in CSR arrays it allocated itself and calls
// ainv_gpu_apply_csr_noalloc, which reads those arrays directly.
//
// The only memory the apply needs besides its inputs and outputs is the
// intermediate t = D^-1 * W^T * x (n doubles).  Here it lives in a
// file-scope device array of fixed size (kNoallocMaxRows doubles, 8 MiB),
// which the CUDA runtime reserves when this file's module is loaded on a
// device and keeps until the process exits.  Host code cannot use the
// array's name as a device address; the first call on each device looks the
// address up with cudaGetSymbolAddress (which may load the module) and
// caches it, so that first call should happen before any stream capture.
//
// All calls share the one array and it keeps whatever the last call left
// there.  Nothing in it has to start at zero: sweep 1 writes t[i] for every
// row i < n before sweep 2 reads t[0..n).  Calls whose work overlaps on the
// GPU (different streams, or threads using the same device) race on the
// array and give wrong results; serialise them.
#include <cuda_runtime.h>

#include <mutex>

#include "internal.h"

namespace {

constexpr int kNoallocMaxRows = 1 << 20;  // 1,048,576 rows -> 8 MiB of doubles
constexpr int kMaxDevices = 64;
constexpr int kBlockRows = 256;

static __device__ __align__(256) double g_noalloc_t[kNoallocMaxRows];

std::mutex g_setup_mutex;
double *g_scratch[kMaxDevices] = {};

// Per-device set-up: the device address of g_noalloc_t on the current device.
int scratch_for_current_device(double **out) {
  int dev = -1;
  AINV_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    ainv::set_error("ainv_gpu_apply_csr_noalloc: device ordinal %d not supported", dev);
    return AINV_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_t);
    if (e != cudaSuccess || !p) {
      ainv::set_error("ainv_gpu_apply_csr_noalloc: cudaGetSymbolAddress failed: %s",
                      cudaGetErrorString(e));
      return AINV_ERR_CUDA;
    }
    g_scratch[dev] = static_cast<double *>(p);
  }
  *out = g_scratch[dev];
  return AINV_SUCCESS;
}

// Row range of a caller-owned CSR row, clamped to [0, nnz) so a damaged
// row pointer cannot send the loads outside the arrays.
__device__ __forceinline__ void row_range(const int *__restrict__ irp, int row, long long nnz,
                                          int &b, int &e) {
  long long lo = __ldg(irp + row), hi = __ldg(irp + row + 1);
  lo = lo < 0 ? 0 : (lo > nnz ? nnz : lo);
  hi = hi < lo ? lo : (hi > nnz ? nnz : hi);
  b = (int)lo;
  e = (int)hi;
}

// t[row] = dinv[row] * (W^T x)[row]; columns outside [0, n) are skipped.
__global__ void __launch_bounds__(kBlockRows)
    k_noalloc_sweep1(int n, const int *__restrict__ irp, const int *__restrict__ ja,
                     const double *__restrict__ val, long long nnz,
                     const double *__restrict__ dinv, const double *__restrict__ x,
                     double *__restrict__ t) {
  const int row = blockIdx.x * kBlockRows + threadIdx.x;
  if (row >= n) return;
  int b, e;
  row_range(irp, row, nnz, b, e);
  double acc = 0.0;
  for (int k = b; k < e; k++) {
    const int c = __ldg(ja + k);
    if ((unsigned)c < (unsigned)n) acc = fma(__ldg(val + k), __ldg(x + c), acc);
  }
  t[row] = __ldg(dinv + row) * acc;
}

// y[row] = alpha * (Z t)[row] + beta * y[row]  (y not read when beta == 0).
__global__ void __launch_bounds__(kBlockRows)
    k_noalloc_sweep2(int n, const int *__restrict__ irp, const int *__restrict__ ja,
                     const double *__restrict__ val, long long nnz,
                     const double *__restrict__ t, double alpha, double beta,
                     double *__restrict__ y) {
  const int row = blockIdx.x * kBlockRows + threadIdx.x;
  if (row >= n) return;
  int b, e;
  row_range(irp, row, nnz, b, e);
  double acc = 0.0;
  for (int k = b; k < e; k++) {
    const int c = __ldg(ja + k);
    if ((unsigned)c < (unsigned)n) acc = fma(__ldg(val + k), t[c], acc);
  }
  const double r = alpha * acc;
  y[row] = (beta == 0.0) ? r : r + beta * y[row];
}

}  // namespace

extern "C" int ainv_gpu_apply_csr_noalloc(int n, const int *wt_irp, const int *wt_ja,
                                          const double *wt_val, long long nnz_wt,
                                          const int *z_irp, const int *z_ja,
                                          const double *z_val, long long nnz_z,
                                          const double *dinv, double alpha,
                                          const double *x_dev, double beta, double *y_dev,
                                          void *stream) {
  if (n <= 0 || n > kNoallocMaxRows) {
    ainv::set_error("ainv_gpu_apply_csr_noalloc: n = %d is outside 1..%d, the size of the "
                    "built-in scratch; use ainv_gpu_create / ainv_gpu_apply instead",
                    n, kNoallocMaxRows);
    return AINV_ERR_ARG;
  }
  if (!wt_irp || !z_irp || !dinv || !x_dev || !y_dev || nnz_wt < 0 || nnz_z < 0 ||
      (nnz_wt > 0 && (!wt_ja || !wt_val)) || (nnz_z > 0 && (!z_ja || !z_val))) {
    ainv::set_error("ainv_gpu_apply_csr_noalloc: null or inconsistent argument");
    return AINV_ERR_ARG;
  }
  double *t = nullptr;
  AINV_TRY(scratch_for_current_device(&t));
  cudaStream_t s = (cudaStream_t)stream;
  const int grid = (n + kBlockRows - 1) / kBlockRows;
  k_noalloc_sweep1<<<grid, kBlockRows, 0, s>>>(n, wt_irp, wt_ja, wt_val, nnz_wt, dinv, x_dev, t);
  k_noalloc_sweep2<<<grid, kBlockRows, 0, s>>>(n, z_irp, z_ja, z_val, nnz_z, t, alpha, beta,
                                               y_dev);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    ainv::set_error("ainv_gpu_apply_csr_noalloc: launch failed: %s", cudaGetErrorString(e));
    return AINV_ERR_CUDA;
  }
  return AINV_SUCCESS;
}
