// update_a on the device: the diagonal refresh that reuses the factors of A
// for the shifted system A + diag(x),
//   d <- 1 / (1/d + diag(W^T diag(x) Z))
// (mld_d_base_ainv_update_a, src/impl/mld_d_base_ainv_update_a.f90:53-79).
//
// Row i of the handle's W^T layout is the sparse row the reference takes
// from sv%w, and row i of its Z^T layout (uploaded for the 'T' apply) is
// column i of Z, so each row's term is one sorted sparse dot
// (psb_spdot_srtd): the entries of W^T's row are visited in ascending
// column order (the slot order of both encodings), each matched against
// Z^T's row, and the products x_k * z_ki * w_ik are summed from zero in that
// order.  Products and sums are explicitly rounded (no fused multiply-add)
// so an FP64 handle reproduces the host arithmetic exactly.
#include "sell_device.cuh"

namespace ainv {
namespace {

using namespace dev;

// Column and value of slot k of row `lane` in slice s; value 0 for padding.
template <class V>
__device__ __forceinline__ void slot_of(const SellView<V> &m, int pack, int s, int lane, int k,
                                        int vb, int ib, bool om, int &col, double &val) {
  const int pos = (k / pack) * (kSlice * pack) + lane * pack + (k % pack);
  val = (double)ldd(m.val + vb + pos);
  col = om ? s * kSlice + lane + __ldg(m.idx + ib + k) : __ldg(m.idx + ib + pos);
}

// d64_in (optional): the old d in FP64, read instead of the device copy d
// (which is rounded for FP32/BF16 handles); may alias d64 (each thread
// reads its row before writing it).
template <class V>
__global__ void __launch_bounds__(kBlock)
    k_update_a(SellView<V> wt, int wpack, SellView<V> zt, int zpack, const double *__restrict__ x,
               V *__restrict__ d, const double *d64_in, double *d64) {
  const int row = blockIdx.x * kBlock + threadIdx.x;
  if (row >= wt.n) return;
  const int s = row / kSlice, lane = row % kSlice;
  const int wvb = __ldg(wt.sptr + s), wib = __ldg(wt.iptr + s);
  const int ww = (__ldg(wt.sptr + s + 1) - wvb) / kSlice;
  const bool wom = (__ldg(wt.iptr + s + 1) - wib) == ww;
  const int zvb = __ldg(zt.sptr + s), zib = __ldg(zt.iptr + s);
  const int zw = (__ldg(zt.sptr + s + 1) - zvb) / kSlice;
  const bool zom = (__ldg(zt.iptr + s + 1) - zib) == zw;
  double e = 0.0;
  int kz = 0;  // merge cursor over Z^T's row (both rows ascend in column)
  for (int kw = 0; kw < ww; kw++) {
    int cw;
    double vw;
    slot_of(wt, wpack, s, lane, kw, wvb, wib, wom, cw, vw);
    if (vw == 0.0) continue;
    for (; kz < zw; kz++) {
      int cz;
      double vz;
      slot_of(zt, zpack, s, lane, kz, zvb, zib, zom, cz, vz);
      if (vz == 0.0) continue;
      if (cz > cw) break;
      if (cz == cw) {
        // (diag(x) Z)(k, i) = x_k * z_ki, then w_ik times it
        e = __dadd_rn(e, __dmul_rn(vw, __dmul_rn(x[cw], vz)));
        kz++;
        break;
      }
    }
  }
  const double dold = d64_in ? d64_in[row] : (double)ldd(d + row);
  const double dd = __ddiv_rn(1.0, __dadd_rn(__ddiv_rn(1.0, dold), e));
  d[row] = (V)dd;
  if (d64) d64[row] = dd;
}

}  // namespace

int update_a_async(ainv_handle *h, const double *x, const double *d64_in, double *d64,
                   cudaStream_t s) {
  const int G = (h->n + kBlock - 1) / kBlock;
  switch (h->prec) {
    case AINV_PREC_FP64:
      k_update_a<double><<<G, kBlock, 0, s>>>(view<double>(h->wt), h->wt.pack,
                                               view<double>(h->zt), h->zt.pack, x, (double *)h->d,
                                               d64_in, d64);
      break;
    case AINV_PREC_FP32:
      k_update_a<float><<<G, kBlock, 0, s>>>(view<float>(h->wt), h->wt.pack, view<float>(h->zt),
                                              h->zt.pack, x, (float *)h->d, d64_in, d64);
      break;
    case AINV_PREC_FP32_ACC64:
      k_update_a<f32w><<<G, kBlock, 0, s>>>(view<f32w>(h->wt), h->wt.pack, view<f32w>(h->zt),
                                             h->zt.pack, x, (f32w *)h->d, d64_in, d64);
      break;
    case AINV_PREC_BF16_ACC64:
      k_update_a<b16w><<<G, kBlock, 0, s>>>(view<b16w>(h->wt), h->wt.pack, view<b16w>(h->zt),
                                             h->zt.pack, x, (b16w *)h->d, d64_in, d64);
      break;
    default:
      k_update_a<__nv_bfloat16><<<G, kBlock, 0, s>>>(view<__nv_bfloat16>(h->wt), h->wt.pack,
                                                      view<__nv_bfloat16>(h->zt), h->zt.pack, x,
                                                      (__nv_bfloat16 *)h->d, d64_in, d64);
      break;
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("update_a launch failed: %s", cudaGetErrorString(e));
    return AINV_ERR_CUDA;
  }
  return AINV_SUCCESS;
}

}  // namespace ainv

extern "C" int ainv_gpu_update_a(ainv_handle *h, const double *x_dev, double *d_dev_out,
                                 void *stream) {
  if (!h || !x_dev) {
    ainv::set_error("ainv_gpu_update_a: null argument");
    return AINV_ERR_ARG;
  }
  return ainv::update_a_async(h, x_dev, nullptr, d_dev_out, (cudaStream_t)stream);
}
