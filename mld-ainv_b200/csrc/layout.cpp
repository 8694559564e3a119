// Host-side CSR handling and the upload into the SELL-32 device layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "internal.h"

namespace ainv {

namespace {
thread_local std::string g_last_error;
}

void set_error(const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

const char *last_error() { return g_last_error.c_str(); }

size_t prec_size(int prec) {
  switch (prec) {
    case AINV_PREC_FP64: return 8;
    case AINV_PREC_FP32: return 4;
    case AINV_PREC_BF16: return 2;
    default: return 0;
  }
}

int import_csr(int n, const int *irp, const int *ja, const double *val,
               int one_based, HostCsr &out, const char *what) {
  if (n <= 0 || !irp) {
    set_error("%s: invalid size n=%d or null row pointer", what, n);
    return AINV_ERR_ARG;
  }
  const int base = one_based ? 1 : 0;
  if (irp[0] != base) {
    set_error("%s: row pointer must start at %d", what, base);
    return AINV_ERR_ARG;
  }
  long long nnz = (long long)irp[n] - base;
  if (nnz < 0 || nnz > INT_MAX || (nnz > 0 && (!ja || !val))) {
    set_error("%s: invalid nnz %lld", what, nnz);
    return AINV_ERR_ARG;
  }
  out.n = n;
  out.irp.resize((size_t)n + 1);
  out.ja.resize((size_t)nnz);
  out.val.assign(val, val + nnz);
  for (int i = 0; i <= n; i++) {
    int p = irp[i] - base;
    if (p < 0 || p > nnz || (i > 0 && p < out.irp[i - 1])) {
      set_error("%s: row pointer not monotone at row %d", what, i);
      return AINV_ERR_ARG;
    }
    out.irp[i] = p;
  }
  for (long long k = 0; k < nnz; k++) {
    int c = ja[k] - base;
    if (c < 0 || c >= n) {
      set_error("%s: column index %d out of range at entry %lld", what, ja[k], k);
      return AINV_ERR_ARG;
    }
    out.ja[k] = c;
  }
  // Sorted columns inside each row are part of the layout contract.
  for (int i = 0; i < n; i++)
    for (int k = out.irp[i] + 1; k < out.irp[i + 1]; k++)
      if (out.ja[k] <= out.ja[k - 1]) {
        set_error("%s: columns of row %d are not strictly increasing", what, i);
        return AINV_ERR_ARG;
      }
  return AINV_SUCCESS;
}

HostCsr transpose(const HostCsr &a) {
  HostCsr t;
  t.n = a.n;
  t.irp.assign((size_t)a.n + 1, 0);
  t.ja.resize(a.ja.size());
  t.val.resize(a.val.size());
  for (int c : a.ja) t.irp[c + 1]++;
  for (int i = 0; i < a.n; i++) t.irp[i + 1] += t.irp[i];
  std::vector<int> next(t.irp.begin(), t.irp.end() - 1);
  for (int r = 0; r < a.n; r++)
    for (int k = a.irp[r]; k < a.irp[r + 1]; k++) {
      int at = next[a.ja[k]]++;
      t.ja[at] = r;
      t.val[at] = a.val[k];
    }
  return t;
}

size_t DevSell::bytes() const {
  return (size_t)(nslices + 1) * sizeof(int) + (size_t)slots * (sizeof(int) + prec_size(prec));
}

namespace {

// bfloat16 storage is produced on the host as raw bits: the double is first
// rounded to float, then to the upper 16 bits with round-to-nearest-even.
uint16_t bf16_bits(double v) {
  float f = (float)v;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)((u >> 16) | ((u & 0xffff) ? 0x40 : 0));
  u += 0x7fffu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}

template <class V>
V cast_value(double v);
template <>
double cast_value<double>(double v) { return v; }
template <>
float cast_value<float>(double v) { return (float)v; }
template <>
uint16_t cast_value<uint16_t>(double v) { return bf16_bits(v); }

template <class V>
int upload_sell_t(const HostCsr &a, int prec, DevSell &out) {
  const int n = a.n;
  const int ns = (n + kSlice - 1) / kSlice;
  std::vector<int> sptr((size_t)ns + 1, 0);
  long long slots = 0;
  for (int s = 0; s < ns; s++) {
    int w = 0;
    for (int r = s * kSlice; r < std::min(n, (s + 1) * kSlice); r++)
      w = std::max(w, a.irp[r + 1] - a.irp[r]);
    slots += (long long)w * kSlice;
    if (slots > INT_MAX) {
      set_error("sliced layout exceeds 2^31 slots");
      return AINV_ERR_UNSUPPORTED;
    }
    sptr[s + 1] = (int)slots;
  }
  std::vector<int> col((size_t)slots);
  std::vector<V> val((size_t)slots);
  for (int s = 0; s < ns; s++) {
    const int w = (sptr[s + 1] - sptr[s]) / kSlice;
    for (int lane = 0; lane < kSlice; lane++) {
      const int r = s * kSlice + lane;
      const int rr = std::min(r, n - 1);
      const int beg = r < n ? a.irp[r] : 0, len = r < n ? a.irp[r + 1] - beg : 0;
      for (int k = 0; k < w; k++) {
        const size_t at = (size_t)sptr[s] + (size_t)k * kSlice + lane;
        if (k < len) {
          col[at] = a.ja[beg + k];
          val[at] = cast_value<V>(a.val[beg + k]);
        } else {
          col[at] = rr;
          val[at] = cast_value<V>(0.0);
        }
      }
    }
  }
  DevSell m;
  m.n = n;
  m.nslices = ns;
  m.nnz = a.nnz();
  m.slots = slots;
  m.prec = prec;
  cudaError_t e = cudaMalloc(&m.sptr, sizeof(int) * ((size_t)ns + 1));
  if (e == cudaSuccess && slots > 0) e = cudaMalloc(&m.col, sizeof(int) * (size_t)slots);
  if (e == cudaSuccess && slots > 0) e = cudaMalloc(&m.val, sizeof(V) * (size_t)slots);
  if (e == cudaSuccess)
    e = cudaMemcpy(m.sptr, sptr.data(), sizeof(int) * ((size_t)ns + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && slots > 0)
    e = cudaMemcpy(m.col, col.data(), sizeof(int) * (size_t)slots, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && slots > 0)
    e = cudaMemcpy(m.val, val.data(), sizeof(V) * (size_t)slots, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    free_sell(m);
    set_error("device upload of sliced matrix failed: %s", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? AINV_ERR_ALLOC : AINV_ERR_CUDA;
  }
  out = m;
  return AINV_SUCCESS;
}

}  // namespace

int upload_sell(const HostCsr &a, int prec, DevSell &out) {
  switch (prec) {
    case AINV_PREC_FP64: return upload_sell_t<double>(a, prec, out);
    case AINV_PREC_FP32: return upload_sell_t<float>(a, prec, out);
    case AINV_PREC_BF16: return upload_sell_t<uint16_t>(a, prec, out);
    default:
      set_error("unknown precision %d", prec);
      return AINV_ERR_ARG;
  }
}

void free_sell(DevSell &m) {
  if (m.sptr) cudaFree(m.sptr);
  if (m.col) cudaFree(m.col);
  if (m.val) cudaFree(m.val);
  m = DevSell{};
}

int upload_values(const double *h, size_t n, int prec, void **dptr) {
  *dptr = nullptr;
  size_t es = prec_size(prec);
  if (!es) {
    set_error("unknown precision %d", prec);
    return AINV_ERR_ARG;
  }
  std::vector<unsigned char> buf(n * es);
  for (size_t i = 0; i < n; i++) {
    if (prec == AINV_PREC_FP64) {
      std::memcpy(&buf[i * es], &h[i], 8);
    } else if (prec == AINV_PREC_FP32) {
      float f = (float)h[i];
      std::memcpy(&buf[i * es], &f, 4);
    } else {
      uint16_t b = bf16_bits(h[i]);
      std::memcpy(&buf[i * es], &b, 2);
    }
  }
  cudaError_t e = cudaMalloc(dptr, n * es);
  if (e == cudaSuccess) e = cudaMemcpy(*dptr, buf.data(), n * es, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    if (*dptr) cudaFree(*dptr);
    *dptr = nullptr;
    set_error("device upload of a vector failed: %s", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? AINV_ERR_ALLOC : AINV_ERR_CUDA;
  }
  return AINV_SUCCESS;
}

}  // namespace ainv
