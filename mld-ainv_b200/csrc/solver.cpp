// Host mirror of the plugin's solver types: mld_d_ainv_solver_type
// (src/mld_d_ainv_solver.F90:46-67), mld_d_invk_solver_type
// (src/mld_d_invk_solver.f90:47-57) and mld_d_invt_solver_type
// (src/mld_d_invt_solver.f90:46-58), with the type-bound procedures of the
// common base (src/mld_d_base_ainv_mod.F90:45-68).  The factors are built
// on the host; `cnv` plays the mold conversion that moves them to the
// device layout (src/impl/mld_d_base_ainv_solver_cnv.f90:56-60), after
// which `apply` runs on the GPU.  There is no host apply.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include <cuda_runtime.h>

#include "solver_impl.h"

namespace {

using ainv::kAinv;
using ainv::kInvk;
using ainv::kInvt;

std::string upper(const char *s) {
  std::string u = s ? s : "";
  while (!u.empty() && std::isspace((unsigned char)u.back())) u.pop_back();
  size_t b = 0;
  while (b < u.size() && std::isspace((unsigned char)u[b])) b++;
  u = u.substr(b);
  for (char &c : u) c = (char)std::toupper((unsigned char)c);
  return u;
}

}  // namespace


namespace {

void drop_device(mld_d_solver *sv) {
  if (sv->h) ainv_gpu_destroy(sv->h);
  sv->h = nullptr;
}

void clear_data(mld_d_solver *sv) {
  drop_device(sv);
  sv->wt = ainv::HostCsr{};
  sv->z = ainv::HostCsr{};
  sv->d.clear();
  sv->d.shrink_to_fit();
  sv->built = false;
}

int upload(mld_d_solver *sv) {
  drop_device(sv);
  const ainv::HostCsr &wt = sv->wt, &z = sv->z;
  return ainv_gpu_create(&sv->h, wt.n, wt.irp.data(), wt.ja.data(), wt.val.data(),
                         z.irp.data(), z.ja.data(), z.val.data(), sv->d.data(),
                         sv->dev_prec, 0);
}

}  // namespace

int ainv::install_factors(mld_d_solver *sv, HostCsr wt, HostCsr z, std::vector<double> d) {
  clear_data(sv);
  sv->wt = std::move(wt);
  sv->z = std::move(z);
  sv->d = std::move(d);
  sv->built = true;
  if (sv->dev_prec >= 0) return upload(sv);
  return AINV_SUCCESS;
}

namespace {

// d_ainv_stringval (src/mld_d_ainv_solver.F90:232-258); unknown names map
// to an invalid algorithm, which build rejects as "Invalid alg".
int alg_from_string(const std::string &s) {
  if (s == "LLK") return ainv::kAlgLLK;
  if (s == "STAB-LLK") return ainv::kAlgStabLLK;
  if (s == "SYM-LLK") return ainv::kAlgSymLLK;
  if (s == "MLK") return ainv::kAlgMLK;
  return -1;
}

const char *alg_name(int alg) {
  // d_ainv_algname (src/mld_d_ainv_solver.F90:261-298)
  switch (alg) {
    case ainv::kAlgMLK: return "Left-looking, list merge";
    case ainv::kAlgLLK: return "Left-looking";
    case ainv::kAlgSymLLK: return "Symmetric Left-looking";
    case ainv::kAlgStabLLK: return "Stabilized Left-looking";
    case ainv::kAlgLLKNoth: return "Left-looking, no alpha test";
    default: return "Unknown alg variant";
  }
}

}  // namespace

extern "C" {

int mld_d_solver_create(mld_d_solver **out, const char *type) {
  if (!out) {
    ainv::set_error("mld_d_solver_create: null pointer");
    return AINV_ERR_ARG;
  }
  *out = nullptr;
  const std::string t = upper(type);
  int kind;
  if (t == "AINV")
    kind = kAinv;
  else if (t == "INVK")
    kind = kInvk;
  else if (t == "INVT")
    kind = kInvt;
  else {
    ainv::set_error("mld_d_solver_create: unknown solver type '%s'", type ? type : "");
    return AINV_ERR_ARG;
  }
  mld_d_solver *sv = new (std::nothrow) mld_d_solver;
  if (!sv) {
    ainv::set_error("mld_d_solver_create: host allocation failed");
    return AINV_ERR_ALLOC;
  }
  sv->kind = kind;
  mld_d_solver_default(sv);
  *out = sv;
  return AINV_SUCCESS;
}

int mld_d_solver_destroy(mld_d_solver *sv) {
  if (sv) {
    clear_data(sv);
    delete sv;
  }
  return AINV_SUCCESS;
}

int mld_d_solver_default(mld_d_solver *sv) {
  if (!sv) return AINV_ERR_ARG;
  // d_ainv_solver_default (src/mld_d_ainv_solver.F90:206-220),
  // d_invk_solver_default (src/mld_d_invk_solver.f90:243-256),
  // d_invt_solver_default (src/mld_d_invt_solver.f90:256-271)
  sv->alg = ainv::kAlgLLK;
  sv->fill_in = 0;
  sv->thresh = 0.0;
  sv->inv_fill = 0;
  sv->inv_thresh = 0.0;
  return AINV_SUCCESS;
}

int mld_d_solver_cseti(mld_d_solver *sv, const char *what, int val) {
  if (!sv) return AINV_ERR_ARG;
  const std::string w = upper(what);
  // src/impl/mld_d_ainv_solver_cseti.f90:55-62, mld_d_invk_solver_cseti.f90:55-62,
  // mld_d_invt_solver_cseti.f90
  if (w == "SUB_FILLIN") {
    sv->fill_in = val;
  } else if (w == "AINV_ALG" && sv->kind == kAinv) {
    sv->alg = val;
  } else if (w == "INV_FILLIN" && sv->kind != kAinv) {
    sv->inv_fill = val;
  }
  return AINV_SUCCESS;  // other keys belong to the base solver: ignored
}

int mld_d_solver_csetr(mld_d_solver *sv, const char *what, double val) {
  if (!sv) return AINV_ERR_ARG;
  const std::string w = upper(what);
  // src/impl/mld_d_ainv_solver_csetr.f90:55-60, mld_d_invt_solver_csetr.f90:55-62
  if (w == "SUB_ILUTHRS" && sv->kind != kInvk) {
    sv->thresh = val;
  } else if (w == "INV_THRESH" && sv->kind == kInvt) {
    sv->inv_thresh = val;
  }
  return AINV_SUCCESS;
}

int mld_d_solver_csetc(mld_d_solver *sv, const char *what, const char *val) {
  if (!sv) return AINV_ERR_ARG;
  const std::string w = upper(what);
  // src/impl/mld_d_ainv_solver_csetc.f90:56-61
  if (w == "AINV_ALG" && sv->kind == kAinv) sv->alg = alg_from_string(upper(val));
  return AINV_SUCCESS;
}

int mld_d_solver_check(mld_d_solver *sv) {
  if (!sv) return AINV_ERR_ARG;
  // mld_check_def: illegal values fall back to the default with a warning
  // (src/impl/mld_d_ainv_solver_check.f90:53-56, mld_d_invk_solver_check.f90:52-55,
  // mld_d_invt_solver_check.f90:53-60)
  auto fix_i = [](int &v, int lo, int def, const char *name) {
    if (v < lo) {
      std::fprintf(stderr, " Illegal value for %s : %d. defaulting to %d\n", name, v, def);
      v = def;
    }
  };
  auto fix_r = [](double &v, const char *name) {
    if (!(v >= 0.0)) {
      std::fprintf(stderr, " Illegal value for %s : %g. defaulting to 0\n", name, v);
      v = 0.0;
    }
  };
  if (sv->kind == kAinv) {
    fix_i(sv->fill_in, 1, 1, "Nzmin");
    fix_r(sv->thresh, "Eps");
  } else {
    fix_i(sv->fill_in, 0, 0, "Level");
    fix_i(sv->inv_fill, 0, 0, "Level");
    if (sv->kind == kInvt) {
      fix_r(sv->thresh, "Eps");
      fix_r(sv->inv_thresh, "Eps");
    }
  }
  return AINV_SUCCESS;
}

int mld_d_solver_build(mld_d_solver *sv, int n, const int *irp, const int *ja,
                       const double *val, int one_based) {
  if (!sv) return AINV_ERR_ARG;
  ainv::HostCsr a;
  AINV_TRY(ainv::import_csr(n, irp, ja, val, one_based, a, "A"));
  clear_data(sv);
  int rc;
  if (sv->kind == kAinv) {
    rc = ainv::ainv_biconjg_build(a, sv->alg, sv->fill_in, sv->thresh, sv->wt, sv->z, sv->d);
  } else if (sv->kind == kInvk) {
    // src/impl/mld_d_invk_solver_bld.f90:68-69: (fill_in, inv_fill) -> (w, d, z)
    rc = ainv::invk_build(a, sv->fill_in, sv->inv_fill, sv->wt, sv->z, sv->d);
  } else {
    // src/impl/mld_d_invt_solver_bld.f90:68-70
    rc = ainv::invt_build(a, sv->fill_in, sv->thresh, sv->inv_fill, sv->inv_thresh, sv->wt,
                          sv->z, sv->d);
  }
  if (rc != AINV_SUCCESS) return rc;
  sv->built = true;
  // src/impl/mld_d_ainv_solver_bld.f90:71-82: convert when a mold is present
  if (sv->dev_prec >= 0) return upload(sv);
  return AINV_SUCCESS;
}

int mld_d_solver_load(mld_d_solver *sv, const char *prefix) {
  if (!sv || !prefix) return AINV_ERR_ARG;
  return ainv::load_matrix_market(sv, prefix);
}

int mld_d_solver_save(const mld_d_solver *sv, const char *path) {
  if (!sv || !path) return AINV_ERR_ARG;
  return ainv::save_cache(sv, path);
}

int mld_d_solver_restore(mld_d_solver *sv, const char *path) {
  if (!sv || !path) return AINV_ERR_ARG;
  return ainv::load_cache(sv, path);
}

int mld_d_solver_cnv(mld_d_solver *sv, int prec) {
  if (!sv) return AINV_ERR_ARG;
  if (ainv::prec_size(prec) == 0) {
    ainv::set_error("cnv: unknown precision %d", prec);
    return AINV_ERR_ARG;
  }
  sv->dev_prec = prec;
  if (!sv->built) return AINV_SUCCESS;  // applied at the end of the next build
  return upload(sv);
}

int mld_d_solver_apply(mld_d_solver *sv, double alpha, const double *x_dev, double beta,
                       double *y_dev, char trans, void *stream) {
  if (!sv) return AINV_ERR_ARG;
  if (!sv->h) {
    ainv::set_error("apply: factors are not on the device (build, then cnv)");
    return AINV_ERR_NOT_BUILT;
  }
  return ainv_gpu_apply(sv->h, trans, alpha, x_dev, beta, y_dev, stream);
}

int mld_d_solver_apply_host(mld_d_solver *sv, double alpha, const double *x, double beta,
                            double *y, char trans) {
  if (!sv) return AINV_ERR_ARG;
  if (!sv->h) {
    ainv::set_error("apply: factors are not on the device (build, then cnv)");
    return AINV_ERR_NOT_BUILT;
  }
  return ainv_gpu_apply_host(sv->h, trans, alpha, x, beta, y);
}

int mld_d_solver_update_a(mld_d_solver *sv, const double *x, int nx) {
  if (!sv || !x) return AINV_ERR_ARG;
  // src/impl/mld_d_base_ainv_update_a.f90:53-79 on the device; sv%d and the
  // device copy are both replaced.  Wrong size: info = -1 there (:54-58).
  if (sv->built && nx < (int)sv->d.size()) {
    ainv::set_error("update_a: x has %d entries, the factors %d", nx, (int)sv->d.size());
    return AINV_ERR_ARG;
  }
  if (!sv->h) {
    ainv::set_error("update_a: factors are not on the device (build, then cnv)");
    return AINV_ERR_NOT_BUILT;
  }
  // The old d enters in FP64 from sv%d (the device copy may be rounded to
  // FP32/BF16), so the host d keeps the reference's FP64 recurrence across
  // repeated updates; the kernel overwrites dd with the new FP64 d.
  const size_t bytes = sizeof(double) * sv->d.size();
  double *xd = nullptr, *dd = nullptr;
  cudaError_t e = cudaMalloc(&xd, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&dd, bytes);
  if (e == cudaSuccess) e = cudaMemcpy(xd, x, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dd, sv->d.data(), bytes, cudaMemcpyHostToDevice);
  int rc = AINV_SUCCESS;
  if (e == cudaSuccess) {
    rc = ainv::update_a_async(sv->h, xd, dd, dd, nullptr);
    if (rc == AINV_SUCCESS) e = cudaStreamSynchronize(nullptr);
  }
  if (e == cudaSuccess && rc == AINV_SUCCESS)
    e = cudaMemcpy(sv->d.data(), dd, bytes, cudaMemcpyDeviceToHost);
  if (xd) cudaFree(xd);
  if (dd) cudaFree(dd);
  if (e != cudaSuccess) {
    ainv::set_error("update_a: %s", cudaGetErrorString(e));
    return AINV_ERR_CUDA;
  }
  return rc;
}

ainv_handle *mld_d_solver_handle(mld_d_solver *sv) { return sv ? sv->h : nullptr; }

int mld_d_solver_get_factors(const mld_d_solver *sv, int *n, long long *nnz_wt,
                             long long *nnz_z, int *wt_irp, int *wt_ja, double *wt_val,
                             int *z_irp, int *z_ja, double *z_val, double *d) {
  if (!sv) return AINV_ERR_ARG;
  if (!sv->built) {
    ainv::set_error("get_factors: solver not built");
    return AINV_ERR_NOT_BUILT;
  }
  if (n) *n = sv->wt.n;
  if (nnz_wt) *nnz_wt = sv->wt.nnz();
  if (nnz_z) *nnz_z = sv->z.nnz();
  auto cp = [](auto *dst, const auto &src) {
    if (dst && !src.empty()) std::memcpy(dst, src.data(), sizeof(src[0]) * src.size());
  };
  cp(wt_irp, sv->wt.irp);
  cp(wt_ja, sv->wt.ja);
  cp(wt_val, sv->wt.val);
  cp(z_irp, sv->z.irp);
  cp(z_ja, sv->z.ja);
  cp(z_val, sv->z.val);
  cp(d, sv->d);
  return AINV_SUCCESS;
}

int mld_d_solver_clone_settings(const mld_d_solver *sv, mld_d_solver *out) {
  if (!sv || !out) return AINV_ERR_ARG;
  if (sv->kind != out->kind) {
    // clone_settings requires the same dynamic type (select type, class default)
    ainv::set_error("clone_settings: solver types differ");
    return AINV_ERR_INTERNAL;
  }
  out->alg = sv->alg;
  out->fill_in = sv->fill_in;
  out->thresh = sv->thresh;
  out->inv_fill = sv->inv_fill;
  out->inv_thresh = sv->inv_thresh;
  return AINV_SUCCESS;
}

int mld_d_solver_clone(const mld_d_solver *sv, mld_d_solver **out) {
  if (!sv || !out) return AINV_ERR_ARG;
  // src/impl/mld_d_ainv_solver_clone.f90:57-78: settings, d, dv, w, z
  mld_d_solver *c = new (std::nothrow) mld_d_solver;
  if (!c) {
    ainv::set_error("clone: host allocation failed");
    return AINV_ERR_ALLOC;
  }
  c->kind = sv->kind;
  mld_d_solver_clone_settings(sv, c);
  c->built = sv->built;
  c->wt = sv->wt;
  c->z = sv->z;
  c->d = sv->d;
  c->dev_prec = sv->dev_prec;
  if (sv->h) {
    int rc = upload(c);
    if (rc != AINV_SUCCESS) {
      mld_d_solver_destroy(c);
      return rc;
    }
  }
  *out = c;
  return AINV_SUCCESS;
}

int mld_d_solver_free(mld_d_solver *sv) {
  if (!sv) return AINV_ERR_ARG;
  clear_data(sv);
  return AINV_SUCCESS;
}

size_t mld_d_solver_sizeof(const mld_d_solver *sv) {
  if (!sv) return 0;
  // base fields + dv + w + z (d_base_ainv_solver_sizeof, src/mld_d_base_ainv_mod.F90:194-207)
  auto csr_bytes = [](const ainv::HostCsr &m) {
    return m.irp.size() * sizeof(int) + m.ja.size() * sizeof(int) + m.val.size() * sizeof(double);
  };
  size_t b = 2 * sizeof(int) + sizeof(double);
  b += sv->d.size() * sizeof(double) + csr_bytes(sv->wt) + csr_bytes(sv->z);
  b += ainv_gpu_sizeof(sv->h);
  return b;
}

long long mld_d_solver_get_nzeros(const mld_d_solver *sv) {
  if (!sv || !sv->built) return 0;
  return (long long)sv->d.size() + sv->wt.nnz() + sv->z.nnz();
}

int mld_d_solver_get_wrksz(void) { return 2; }

int mld_d_solver_descr(const mld_d_solver *sv, char *buf, size_t len) {
  if (!sv || !buf || len == 0) return AINV_ERR_ARG;
  // src/impl/mld_d_ainv_solver_descr.f90:63-66, mld_d_invk_solver_descr.f90,
  // mld_d_invt_solver_descr.f90
  if (sv->kind == kAinv)
    std::snprintf(buf, len,
                  "  AINV: Approximate Inverse with sparse biconjugation \n"
                  "  Algorithm variant      : %s\n"
                  "  Fill level             : %d\n"
                  "  Fill threshold         : %g\n",
                  alg_name(sv->alg), sv->fill_in, sv->thresh);
  else if (sv->kind == kInvk)
    std::snprintf(buf, len,
                  "  INVK Approximate Inverse with ILU(N) \n"
                  "  Fill level             :%d\n"
                  "  Inverse fill level     :%d\n",
                  sv->fill_in, sv->inv_fill);
  else
    std::snprintf(buf, len,
                  "  INVT Approximate Inverse with ILU(T,P) \n"
                  "  Fill level             :%d\n"
                  "  Fill threshold         :%g\n"
                  "  Inverse fill level     :%d\n"
                  "  Inverse fill threshold :%g\n",
                  sv->fill_in, sv->thresh, sv->inv_fill, sv->inv_thresh);
  return AINV_SUCCESS;
}

int mld_d_solver_dump(const mld_d_solver *sv, const char *prefix) {
  if (!sv || !prefix) return AINV_ERR_ARG;
  if (!sv->built) {
    ainv::set_error("dump: solver not built");
    return AINV_ERR_NOT_BUILT;
  }
  // src/impl/mld_d_base_ainv_solver_dmp.f90:82-108: wmat, diag, zmat
  auto write_csr = [](const std::string &fn, const ainv::HostCsr &m) {
    FILE *f = std::fopen(fn.c_str(), "w");
    if (!f) return false;
    std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n");
    std::fprintf(f, "%d %d %lld\n", m.n, m.n, m.nnz());
    for (int i = 0; i < m.n; i++)
      for (int k = m.irp[i]; k < m.irp[i + 1]; k++)
        std::fprintf(f, "%d %d %.17g\n", i + 1, m.ja[k] + 1, m.val[k]);
    return std::fclose(f) == 0;
  };
  const std::string p = prefix;
  bool ok = write_csr(p + "_wmat.mtx", sv->wt) && write_csr(p + "_zmat.mtx", sv->z);
  if (ok) {
    FILE *f = std::fopen((p + "_diag.mtx").c_str(), "w");
    ok = f != nullptr;
    if (ok) {
      std::fprintf(f, "%%%%MatrixMarket matrix array real general\n%zu 1\n", sv->d.size());
      for (double v : sv->d) std::fprintf(f, "%.17g\n", v);
      ok = std::fclose(f) == 0;
    }
  }
  if (!ok) {
    ainv::set_error("dump: cannot write files with prefix '%s'", prefix);
    return AINV_ERR_INTERNAL;
  }
  return AINV_SUCCESS;
}

}  // extern "C"
