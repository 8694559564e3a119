// The host solver object behind the mld_d_solver_* C-ABI (shared by the
// translation units that fill it: solver.cpp and io.cpp).
#pragma once

#include <string>
#include <vector>

#include "host_build.h"

namespace ainv {
enum SolverKind { kAinv = 0, kInvk = 1, kInvt = 2 };
}  // namespace ainv

struct mld_d_solver {
  int kind = ainv::kAinv;
  // AINV: alg, fill_in, thresh.  INVK: fill_in, inv_fill.  INVT: all four.
  int alg = ainv::kAlgLLK;
  int fill_in = 0;
  double thresh = 0.0;
  int inv_fill = 0;
  double inv_thresh = 0.0;
  bool built = false;
  ainv::HostCsr wt, z;  // wt holds W^T (sv%w), z holds Z (sv%z)
  std::vector<double> d;
  int dev_prec = -1;  // device storage requested by cnv (-1: none yet)
  ainv_handle *h = nullptr;
};

namespace ainv {
// Replace sv's factors by (wt, z, d), mark it built and upload them when a
// device precision was requested.
int install_factors(mld_d_solver *sv, HostCsr wt, HostCsr z, std::vector<double> d);
int load_matrix_market(mld_d_solver *sv, const std::string &prefix);
int save_cache(const mld_d_solver *sv, const std::string &path);
int load_cache(mld_d_solver *sv, const std::string &path);
}  // namespace ainv
