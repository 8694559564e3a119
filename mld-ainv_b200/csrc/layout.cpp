// Host-side CSR handling and the upload into the SELL-32 device layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cstdlib>

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
    case AINV_PREC_FP32_ACC64: return 4;
    case AINV_PREC_BF16_ACC64: return 2;
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
  return (size_t)(nslices + 1) * 2 * sizeof(int) + (size_t)nidx * sizeof(int) +
         (size_t)slots * prec_size(prec);
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
  // pass 1: per-slice encoding, width and offset list
  std::vector<char> om((size_t)ns);
  std::vector<int> width((size_t)ns);
  std::vector<int> offs_ptr((size_t)ns + 1, 0);
  std::vector<int> offs_all;
  std::vector<int> offs;
  std::vector<int> maxcol((size_t)ns, -1);
  long long base_slots = 0;
  for (int s = 0; s < ns; s++) {
    const int r0 = s * kSlice, r1 = std::min(n, r0 + kSlice);
    int w = 0;
    offs.clear();
    for (int r = r0; r < r1; r++) {
      w = std::max(w, a.irp[r + 1] - a.irp[r]);
      for (int k = a.irp[r]; k < a.irp[r + 1]; k++) {
        offs.push_back(a.ja[k] - r);
        maxcol[(size_t)s] = std::max(maxcol[(size_t)s], a.ja[k]);
      }
    }
    std::sort(offs.begin(), offs.end());
    offs.erase(std::unique(offs.begin(), offs.end()), offs.end());
    const long long u = (long long)offs.size();
    const long long cost_off = u * kSlice * (long long)sizeof(V) + u * 4;
    const long long cost_col = (long long)w * kSlice * (long long)(sizeof(V) + 4);
    om[s] = u <= kMaxOffsets && cost_off <= cost_col;
    width[s] = om[s] ? (int)u : w;
    if (om[s]) offs_all.insert(offs_all.end(), offs.begin(), offs.end());
    offs_ptr[s + 1] = (int)offs_all.size();
    base_slots += (long long)width[s] * kSlice;
  }
  // pack P: largest power of two with P*sizeof(V) <= 16 and <= 6% padding
  int P = 1;
  for (int p = (int)(16 / sizeof(V)); p > 1; p /= 2) {
    long long padded = 0;
    for (int s = 0; s < ns; s++) padded += (long long)((width[s] + p - 1) / p * p) * kSlice;
    if (padded * 100 <= base_slots * 106) {
      P = p;
      break;
    }
  }
  // pass 2: fill
  std::vector<int> sptr((size_t)ns + 1, 0), iptr((size_t)ns + 1, 0);
  std::vector<int> idx;
  std::vector<V> val;
  idx.reserve((size_t)offs_all.size() + 64);
  val.reserve((size_t)(base_slots + base_slots / 8 + 64));
  int offset_slices = 0;
  auto at = [P](int k, int lane) { return (size_t)(k / P) * kSlice * P + (size_t)lane * P + k % P; };
  for (int s = 0; s < ns; s++) {
    const int r0 = s * kSlice, r1 = std::min(n, r0 + kSlice);
    const int wp = (width[s] + P - 1) / P * P;
    const size_t vbase = val.size();
    if (vbase + (size_t)wp * kSlice > (size_t)INT_MAX) {
      set_error("sliced layout exceeds 2^31 slots");
      return AINV_ERR_UNSUPPORTED;
    }
    val.resize(vbase + (size_t)wp * kSlice, cast_value<V>(0.0));
    if (om[s]) {
      offset_slices++;
      const int *o = offs_all.data() + offs_ptr[s];
      const int u = offs_ptr[s + 1] - offs_ptr[s];
      idx.insert(idx.end(), o, o + u);
      idx.resize(idx.size() + (size_t)(wp - u), 0);  // padding offsets hold value 0
      for (int r = r0; r < r1; r++) {
        const int lane = r - r0;
        for (int k = a.irp[r]; k < a.irp[r + 1]; k++) {
          const int pos = (int)(std::lower_bound(o, o + u, a.ja[k] - r) - o);
          val[vbase + at(pos, lane)] = cast_value<V>(a.val[k]);
        }
      }
    } else {
      const size_t ibase = idx.size();
      idx.resize(ibase + (size_t)wp * kSlice);
      for (int lane = 0; lane < kSlice; lane++) {
        const int r = r0 + lane;
        const int rr = std::min(r, n - 1);
        const int beg = r < n ? a.irp[r] : 0, len = r < n ? a.irp[r + 1] - beg : 0;
        for (int k = 0; k < wp; k++) {
          const size_t p = at(k, lane);
          if (k < len) {
            idx[ibase + p] = a.ja[beg + k];
            val[vbase + p] = cast_value<V>(a.val[beg + k]);
          } else {
            idx[ibase + p] = rr;
          }
        }
      }
    }
    if (idx.size() > (size_t)INT_MAX) {
      set_error("sliced layout exceeds 2^31 index words");
      return AINV_ERR_UNSUPPORTED;
    }
    sptr[s + 1] = (int)val.size();
    iptr[s + 1] = (int)idx.size();
  }
  DevSell m;
  m.n = n;
  m.nslices = ns;
  m.nnz = a.nnz();
  m.slots = (long long)val.size();
  m.nidx = (long long)idx.size();
  m.offset_slices = offset_slices;
  m.pack = P;
  m.prec = prec;
  m.slice_maxcol = std::move(maxcol);
  // streaming stages: kConsumerSlices warps, each with 8/sizeof(V) slices,
  // so a warp's share of a stage is about 1 KB of values at every precision
  // (AINV_STAGE_R = 1 or 2 caps the slices per warp, for tuning)
  std::vector<StageDesc> stages;
  static const int rcap = [] {
    const char *e = std::getenv("AINV_STAGE_R");
    const int v = e ? std::atoi(e) : 0;
    return (v == 1 || v == 2) ? v : 8;
  }();
  const int stage_slices =
      kConsumerSlices * std::min(rcap, (int)std::max<size_t>(1, 8 / sizeof(V)));
  {
    const int nst = (ns + stage_slices - 1) / stage_slices;
    stages.resize((size_t)nst);
    for (int st = 0; st < nst; st++) {
      StageDesc &d = stages[(size_t)st];
      std::memset(&d, 0, sizeof d);
      d.s0 = st * stage_slices;
      d.s1 = std::min(ns, d.s0 + stage_slices);
      d.vstart = sptr[d.s0];
      d.vbytes = (int)((sptr[d.s1] - sptr[d.s0]) * sizeof(V));
      const long long ib0 = (long long)iptr[d.s0] * 4, ib1 = (long long)iptr[d.s1] * 4;
      d.ibyte0 = ib0 / 16 * 16;
      d.ibytes = (int)((ib1 + 15) / 16 * 16 - d.ibyte0);
      // uniform: every slice in offset mode with the same offset list
      // (AINV_STREAM_NO_WINDOWS=1 disables staging of the gathered windows)
      static const bool no_windows = std::getenv("AINV_STREAM_NO_WINDOWS") != nullptr;
      bool uni = !no_windows && om[d.s0] && width[d.s0] > 0 && width[d.s0] <= kStageMaxOffsets;
      const int *o0 = offs_all.data() + offs_ptr[d.s0];
      const int u0 = offs_ptr[d.s0 + 1] - offs_ptr[d.s0];
      for (int s = d.s0 + 1; uni && s < d.s1; s++) {
        const int u = offs_ptr[s + 1] - offs_ptr[s];
        uni = om[s] && u == u0 && std::equal(o0, o0 + u0, offs_all.data() + offs_ptr[s]);
      }
      // a window must not need bytes past the end of the gathered vector
      const long long r0 = (long long)d.s0 * kSlice, r1 = std::min<long long>(n, (long long)d.s1 * kSlice);
      for (int k = 0; uni && k < u0; k++) {
        const long long hi = std::min<long long>(n, r1 + o0[k]);
        // each window copy rounds its end up to 16 bytes: it must not pass the
        // end of a vector of n doubles or of n floats
        for (long long xs : {4LL, 8LL})
          if ((hi * xs + 15) / 16 * 16 > (long long)n * xs) uni = false;
        if (r0 + o0[k] >= n || r1 + o0[k] <= 0) uni = false;
      }
      if (uni) {
        d.noff = u0;
        for (int k = 0; k < u0; k++) d.off[k] = o0[k];
        // windows: clusters of offsets within kWindowSpan of their first
        int nwin = 0, first = 0;
        for (int k = 0; k < u0; k++)
          if (k == 0 || o0[k] - first > kWindowSpan) {
            nwin++;
            first = o0[k];
            d.noff |= 1 << (8 + k);
          }
        m.stage_nwin_max = std::max(m.stage_nwin_max, nwin);
      }
      m.stage_vmax = std::max(m.stage_vmax, d.vbytes);
      m.stage_imax = std::max(m.stage_imax, d.ibytes);
      m.stage_noff_max = std::max(m.stage_noff_max, d.noff & 0xff);
    }
    m.nstages = nst;
    m.stage_slices = stage_slices;
  }
  idx.resize(idx.size() + 4, 0);  // tail padding: index copies round up to 16 bytes
  sptr.resize(sptr.size() + 4, sptr.back());  // and so do the slice-pointer copies
  iptr.resize(iptr.size() + 4, iptr.back());
  cudaError_t e = cudaMalloc(&m.sptr, sizeof(int) * sptr.size());
  if (e == cudaSuccess) e = cudaMalloc(&m.iptr, sizeof(int) * iptr.size());
  if (e == cudaSuccess && !idx.empty()) e = cudaMalloc(&m.idx, sizeof(int) * idx.size());
  if (e == cudaSuccess && !stages.empty())
    e = cudaMalloc(&m.stages, sizeof(StageDesc) * stages.size());
  if (e == cudaSuccess && !stages.empty())
    e = cudaMemcpy(m.stages, stages.data(), sizeof(StageDesc) * stages.size(),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !val.empty()) e = cudaMalloc(&m.val, sizeof(V) * val.size());
  if (e == cudaSuccess)
    e = cudaMemcpy(m.sptr, sptr.data(), sizeof(int) * sptr.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(m.iptr, iptr.data(), sizeof(int) * iptr.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !idx.empty())
    e = cudaMemcpy(m.idx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !val.empty())
    e = cudaMemcpy(m.val, val.data(), sizeof(V) * val.size(), cudaMemcpyHostToDevice);
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
    case AINV_PREC_FP32_ACC64: return upload_sell_t<float>(a, prec, out);
    case AINV_PREC_BF16_ACC64: return upload_sell_t<uint16_t>(a, prec, out);
    default:
      set_error("unknown precision %d", prec);
      return AINV_ERR_ARG;
  }
}

void free_sell(DevSell &m) {
  if (m.stages) cudaFree(m.stages);
  if (m.sptr) cudaFree(m.sptr);
  if (m.iptr) cudaFree(m.iptr);
  if (m.idx) cudaFree(m.idx);
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
    } else if (prec == AINV_PREC_FP32 || prec == AINV_PREC_FP32_ACC64) {
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
