// Row epilogues of the A products inside the Krylov loops (shared by the
// single-solve loop and the solve server, so both compute the same bits):
// the product y = A x, the vector the recurrence needs from it, and the
// row terms of the dots that follow, which go to per-slice sums
// (SliceSums) in the canonical order of sell_device.cuh.
#pragma once

#include "kstate.cuh"
#include "stream.cuh"

namespace ainv {
namespace dev {

using kstate::kBicgOmega;
using kstate::kBicgSigma;
using kstate::kCgSigma;
using kstate::kInit;
using kstate::kTrueRes;

// Dots of each MODE (see dots_row).
constexpr int dots_of(int mode) {
  return mode == kTrueRes ? 3 : (mode == kInit || mode == kBicgOmega) ? 2 : 1;
}

// y = A x with the reductions each caller needs (see MODE):
//   kCgSigma:   sigma = x.y, alpha = rho/sigma               (q = A p)
//   kBicgSigma: sigma = w1.y, alpha = rho/sigma              (v = A f, w1 = rt)
//   kBicgOmega: omega = (y.w1)/(y.y)                         (t = A z, w1 = s)
//   kInit:      y = w1 - A x, optional copy into w2 (rt), initial norm/rho
//   kTrueRes:   y = w1 - A x (true residual, w1 = b) compared with the
//               recurrence residual w3 = r; runs every check_every
//               iterations and once when the recurrence claims convergence.
//               Decides whether r is replaced and whether the convergence
//               stands; w2 = rt for BiCGSTAB's rho.
// The row products of the dots go to ss; the fold does the scalar step.
template <int MODE, class SS>
__device__ __forceinline__ void dots_row(int i, double acc, const double *__restrict__ x,
                                         double *__restrict__ y, const double *w1, double *w2,
                                         const double *w3, SS &ss) {
  if constexpr (MODE == kTrueRes || MODE == kInit) {
    const double ri = w1[i] - acc;
    y[i] = ri;
    ss.v[0] = ri * ri;
    if constexpr (MODE == kInit) {
      if (w2) {
        w2[i] = ri;
        ss.v[1] = ri * ri;
      }
    } else {
      const double g = ri - w3[i];
      ss.v[1] = g * g;
      if (w2) ss.v[2] = w2[i] * ri;
    }
  } else {
    y[i] = acc;
    if constexpr (MODE == kCgSigma) ss.v[0] = x[i] * acc;
    if constexpr (MODE == kBicgSigma) ss.v[0] = w1[i] * acc;
    if constexpr (MODE == kBicgOmega) {
      ss.v[0] = acc * acc;
      ss.v[1] = acc * w1[i];
    }
  }
}

// Streaming form of dots_row (stream.cuh): the per-row operands are staged
// with the stage's copies, the row products go to the slice sums.
template <int MODE>
struct EpiDots {
  double *__restrict__ y;
  const double *__restrict__ x;
  const double *__restrict__ w1;
  double *__restrict__ w2;
  const double *__restrict__ w3;
  SliceSums<dots_of(MODE)> ss;
  static constexpr int kRowVecs = (MODE == kTrueRes) ? 3 : 1;
  // row operands: b (init / true residual, with r and rt), p (CG sigma),
  // rt (BiCGSTAB sigma), s (BiCGSTAB omega)
  __device__ __host__ __forceinline__ RowVecs row_vecs() const {
    if (MODE == kTrueRes) return RowVecs{{w1, w3, w2}, {8, 8, w2 ? 8 : 0}};
    if (MODE == kCgSigma) return RowVecs{{x, nullptr, nullptr}, {8, 0, 0}};
    return RowVecs{{w1, nullptr, nullptr}, {8, 0, 0}};
  }
  __device__ __forceinline__ void post(int i, double acc, const StagedRows &r) {
    if constexpr (MODE == kTrueRes || MODE == kInit) {
      const double ri = r.get<double>(0, i) - acc;
      y[i] = ri;
      ss.v[0] = ri * ri;
      if constexpr (MODE == kInit) {
        if (w2) {
          w2[i] = ri;
          ss.v[1] = ri * ri;
        }
      } else {
        const double g = ri - r.get<double>(1, i);
        ss.v[1] = g * g;
        if (w2) ss.v[2] = r.get<double>(2, i) * ri;
      }
    } else {
      y[i] = acc;
      const double a = r.get<double>(0, i);
      if constexpr (MODE == kCgSigma || MODE == kBicgSigma) ss.v[0] = a * acc;
      if constexpr (MODE == kBicgOmega) {
        ss.v[0] = acc * acc;
        ss.v[1] = acc * a;
      }
    }
  }
  __device__ __forceinline__ void end_slice(int s) { ss.end(s); }
};

}  // namespace dev
}  // namespace ainv
