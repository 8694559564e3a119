// Host factor builders (the reference's host biconjugation / sparse inverse
// tools, restated in C++).  Outputs are 0-based sorted CSR.
#pragma once

#include <vector>

#include "internal.h"

namespace ainv {

// Algorithm ids, in the order of src/mld_base_ainv_mod.F90:50-55.
constexpr int kAlgLLK = 0;      // 'LLK'
constexpr int kAlgSymLLK = 1;   // 'SYM-LLK'
constexpr int kAlgStabLLK = 2;  // 'STAB-LLK'
constexpr int kAlgLLKNoth = 3;  // left-looking without the alpha test
constexpr int kAlgMLK = 4;      // 'MLK'

// AINV: W^T (CSR), Z (CSR), d = D^-1.
int ainv_biconjg_build(const HostCsr &a, int alg, int fill_in, double thresh, HostCsr &wt,
                       HostCsr &z, std::vector<double> &d);

// INVK: ILU(fill1) then level-fill2 sparse inverses of U and L.
int invk_build(const HostCsr &a, int fill1, int fill2, HostCsr &wt, HostCsr &z,
               std::vector<double> &d);

// INVT: ILUT(fill, thresh) with maxval scaling, then sparse inverses of U
// and L with (invfill, invthresh).
int invt_build(const HostCsr &a, int fill, double thresh, int invfill, double invthresh,
               HostCsr &wt, HostCsr &z, std::vector<double> &d);

}  // namespace ainv
