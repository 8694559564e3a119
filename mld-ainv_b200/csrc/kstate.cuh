// Scalar state of the preconditioned Krylov recurrences (PSBLAS psb_dcg /
// psb_dbicgstab with istop=2, driven at tests/pdegen/ppde3d.f90:280-281) and
// the bookkeeping that the last block of each reduction kernel applies to
// it.  Shared by the single-solve loop and the batched solve server, so both
// follow one recurrence.
#pragma once

#include <cmath>

#include "internal.h"

namespace ainv {

struct KState {
  double rho, rho_old, alpha, beta, omega, rn2, bn2, eps;
  int iter, itmax, done, status, check_every, method;
  int verified;  // convergence confirmed on the true residual b - A x
  int replace;   // r := b - A x pending (cleared by the next reduction kernel)
  int fails;     // convergence claims the true residual did not confirm
  int replacements;
  int timeout;  // a streaming kernel gave up a bounded wait
  unsigned ticket[4];
  double *hist;  // ||r_k||/||b|| of iteration k at hist[k-1] (k <= hist_cap), or null
  int hist_cap;
};

namespace kstate {

enum { kCgSigma = 0, kBicgSigma = 1, kBicgOmega = 2, kTrueRes = 3, kInit = 4 };
constexpr double kDrift = 1e-6;   // replace r when ||(b - A x) - r|| > kDrift ||b - A x||
constexpr int kMaxVerifyFails = 3;

__device__ __forceinline__ void finish_iteration(KState *st, double rn2) {
  st->rn2 = rn2;
  st->iter += 1;
  const double err = sqrt(rn2) / st->bn2;
  if (st->hist && st->iter <= st->hist_cap) st->hist[st->iter - 1] = err;
  if (!isfinite(rn2)) {
    st->status = AINV_ERR_NONFINITE;
    st->done = 1;
  } else if (err <= st->eps) {
    st->status = AINV_SUCCESS;
    st->done = 1;
  } else if (st->iter >= st->itmax) {
    st->status = AINV_ERR_NOCONV;
    st->done = 1;
  }
}

// CG: rho = r.z from the preconditioner sweep, then beta = rho / rho_old.
__device__ __forceinline__ void cg_take_rho(KState *st, double rho) {
  st->replace = 0;
  st->rho_old = st->rho;
  st->rho = rho;
  if (st->iter > 0) {
    if (st->rho_old == 0.0) {
      st->status = AINV_ERR_BREAKDOWN;
      st->done = 1;
    } else {
      st->beta = st->rho / st->rho_old;
    }
  }
}

// BiCGSTAB: start the next iteration's scalars from rho = rt.r.
__device__ __forceinline__ void bicg_next_rho(KState *st, double rr) {
  if (st->done) return;
  st->rho_old = st->rho;
  st->rho = rr;
  if (rr == 0.0) {
    st->status = AINV_ERR_BREAKDOWN;
    st->done = 1;
  } else {
    st->beta = (st->rho / st->rho_old) * (st->alpha / st->omega);
  }
}

// Scalar bookkeeping done by the last block of an SpMV-with-dots kernel
// (thread 0), from the grid totals pr.
template <int MODE>
__device__ __forceinline__ void finish_dots(KState *st, const double (&pr)[3], bool verify,
                                            const double *w2) {
  if (MODE == kCgSigma || MODE == kBicgSigma) {
    if (MODE == kBicgSigma) st->replace = 0;
    if (pr[0] == 0.0) {
      st->status = AINV_ERR_BREAKDOWN;
      st->done = 1;
    } else {
      st->alpha = st->rho / pr[0];
    }
  } else if (MODE == kBicgOmega) {
    const double om = (pr[0] == 0.0) ? 0.0 : pr[1] / pr[0];
    if (pr[0] == 0.0 || om == 0.0) {
      st->status = AINV_ERR_BREAKDOWN;
      st->done = 1;
    } else {
      st->omega = om;
    }
  } else if (MODE == kInit) {
    st->rn2 = pr[0];
    const double err = sqrt(pr[0]) / st->bn2;
    if (!isfinite(pr[0])) {
      st->status = AINV_ERR_NONFINITE;
      st->done = 1;
    } else if (err <= st->eps) {
      st->status = AINV_SUCCESS;
      st->done = 1;
      st->verified = 1;  // computed from b - A x already
    } else if (st->itmax <= 0) {
      st->status = AINV_ERR_NOCONV;
      st->done = 1;
    }
    st->rho = pr[1];
  } else {  // kTrueRes
    const double tn = sqrt(pr[0]), gap = sqrt(pr[1]);
    bool replace;
    if (verify) {
      if (tn / st->bn2 <= st->eps || !isfinite(pr[0])) {
        st->verified = 1;
        st->rn2 = pr[0];
        if (!isfinite(pr[0])) st->status = AINV_ERR_NONFINITE;
        replace = false;
      } else if (st->fails >= kMaxVerifyFails || st->iter >= st->itmax) {
        st->verified = 1;
        st->rn2 = pr[0];
        st->status = AINV_ERR_NOCONV;
        replace = false;
      } else {
        // the recurrence drifted: continue from the true residual
        st->fails += 1;
        st->done = 0;
        st->status = AINV_SUCCESS;
        replace = true;
        if (w2) st->rho_old = st->rho;  // k_bicg_xr skipped its rho step
      }
    } else {
      replace = gap > kDrift * tn;
    }
    if (replace) {
      st->replace = 1;
      st->replacements += 1;
      st->rn2 = pr[0];
      if (w2) {  // BiCGSTAB: rho and beta follow the replaced residual
        st->rho = pr[2];
        if (pr[2] == 0.0) {
          st->status = AINV_ERR_BREAKDOWN;
          st->done = 1;
        } else {
          st->beta = (st->rho / st->rho_old) * (st->alpha / st->omega);
        }
      }
    }
  }
}

}  // namespace kstate
}  // namespace ainv
