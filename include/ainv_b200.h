/*
 * ainv_b200 -- B200 (sm_100a) application phase of the MLD2P4 AINV plugin.
 *
 * C-ABI boundary.  Plain pointers and sizes only; no exceptions cross it.
 * Every entry point returns 0 (AINV_SUCCESS, the reference's psb_success_)
 * or a nonzero status; ainv_last_error() gives a message for the calling
 * thread.  Device pointers are CUDA global-memory addresses on the current
 * device; `stream` is a cudaStream_t passed as void* (NULL = legacy
 * default stream).  Host arrays passed to *_create are copied and not
 * retained.  A handle is not thread-safe; one stream per call.
 *
 * Reference interfaces replaced (paths inside sfilippone/mld-ainv):
 *   ainv_gpu_create      mold conversion of the factors:
 *                        src/impl/mld_d_ainv_solver_bld.f90:71-82 and
 *                        src/impl/mld_d_base_ainv_solver_cnv.f90:56-60
 *   ainv_gpu_apply       mld_d_base_ainv_solver_apply_vect
 *                        src/impl/mld_d_base_ainv_solver_apply_vect.f90:35-166
 *   ainv_gpu_apply_host  mld_d_base_ainv_solver_apply (array form)
 *                        src/impl/mld_d_base_ainv_solver_apply.f90:35-152
 *   ainv_gpu_destroy     mld_d_base_ainv_solver_free / clear_data
 *                        src/impl/mld_d_base_ainv_solver_free.f90:35-60,
 *                        src/impl/mld_d_base_ainv_solver_clear_data.f90:35-70
 *   ainv_gpu_sizeof      d_base_ainv_solver_sizeof src/mld_d_base_ainv_mod.F90:194-207
 *   ainv_gpu_get_nzeros  d_base_ainv_get_nzeros    src/mld_d_base_ainv_mod.F90:179-192
 *   ainv_csr_* / ainv_gpu_solve
 *                        psb_spmm(A) and psb_krylov('CG'|'BICGSTAB', ..., istop=2)
 *                        as called at tests/pdegen/ppde3d.f90:280-281 (PSBLAS)
 *   mld_d_solver_*       the solver types mld_d_ainv_solver_type
 *                        (src/mld_d_ainv_solver.F90:46-67), mld_d_invk_solver_type
 *                        (src/mld_d_invk_solver.f90:47-57), mld_d_invt_solver_type
 *                        (src/mld_d_invt_solver.f90:46-58) with their
 *                        build / cseti / csetr / csetc / check / default / descr /
 *                        clone / clone_settings / free / sizeof / get_nzeros /
 *                        get_wrksz / dump procedures.
 */
#ifndef AINV_B200_H
#define AINV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define AINV_SUCCESS          0    /* psb_success_                        */
#define AINV_ERR_ARG          30   /* invalid argument (bad trans, sizes)  */
#define AINV_ERR_ALLOC        4025 /* allocation request refused            */
#define AINV_ERR_INTERNAL     4000 /* internal error / inconsistent state   */
#define AINV_ERR_CUDA         4100 /* a CUDA runtime call failed            */
#define AINV_ERR_NOT_BUILT    4101 /* solver has no factors yet             */
#define AINV_ERR_BREAKDOWN    4102 /* Krylov breakdown (rho, sigma or omega = 0) */
#define AINV_ERR_NONFINITE    4103 /* non-finite residual in the Krylov loop */
#define AINV_ERR_NOCONV       4104 /* itmax reached before the tolerance    */
#define AINV_ERR_UNSUPPORTED  4105 /* option not built into this library   */
#define AINV_ERR_TIMEOUT      4106 /* a device-side wait ran past its limit  */

/* ---- factor storage precision (values of W^T, Z and D^-1) ------------- */
#define AINV_PREC_FP64 0
#define AINV_PREC_FP32 1
#define AINV_PREC_BF16 2
/* FP32 / BF16 storage with FP64 accumulation and an FP64 intermediate: the
 * same factor bytes as FP32 / BF16, arithmetic as the FP64 apply. */
#define AINV_PREC_FP32_ACC64 3
#define AINV_PREC_BF16_ACC64 4

/* ---- Krylov methods --------------------------------------------------- */
#define AINV_KRYLOV_CG       0
#define AINV_KRYLOV_BICGSTAB 1

/* ---- AINV_ALG values (cseti), in the order of src/mld_base_ainv_mod.F90:50-55;
 * csetc accepts 'LLK', 'SYM-LLK', 'STAB-LLK', 'MLK'. ------------------------ */
#define MLD_AINV_LLK       0
#define MLD_AINV_S_LLK     1
#define MLD_AINV_S_FT_LLK  2
#define MLD_AINV_LLK_NOTH  3
#define MLD_AINV_MLK       4

typedef struct ainv_handle ainv_handle; /* device factors W^T, Z, D^-1    */
typedef struct ainv_csr ainv_csr;       /* device sparse operator A        */
typedef struct mld_d_solver mld_d_solver; /* host solver type (AINV/INVK/INVT) */

const char *ainv_last_error(void);
/* Library version string. */
const char *ainv_version(void);

/* ---- device factors: upload / apply / release ------------------------ */
/* Upload W^T (CSR, lower, row i = column w_i), Z (CSR, upper) and
 * dinv = D^-1 into the device layout, stored in precision `prec`.
 * one_based != 0 accepts Fortran 1-based irp/ja. */
int ainv_gpu_create(ainv_handle **h, int n,
                    const int *wt_irp, const int *wt_ja, const double *wt_val,
                    const int *z_irp, const int *z_ja, const double *z_val,
                    const double *dinv, int prec, int one_based);
/* y = alpha * Z * D^-1 * W^T * x + beta * y   (trans 'N')
 * y = alpha * W * D^-1 * Z^T * x + beta * y   (trans 'T' or 'C')
 * x_dev, y_dev: n doubles on the device.  beta == 0 ignores y's contents. */
int ainv_gpu_apply(ainv_handle *h, char trans, double alpha, const double *x_dev,
                   double beta, double *y_dev, void *stream);
/* One sweep of the apply, for overlapping the two sweeps with other work
 * or timing them apart: stage 1 computes the handle's intermediate
 * t = D^-1 * (W^T x) ('N') or D^-1 * (Z^T x) ('T'); stage 2 computes
 * y = alpha * Z t + beta * y ('N') or alpha * W t + beta * y ('T') from the
 * t left by the last stage 1 on this handle (x is ignored in stage 2). */
int ainv_gpu_apply_stage(ainv_handle *h, char trans, int stage, double alpha,
                         const double *x_dev, double beta, double *y_dev, void *stream);
/* Same on host arrays: copies x (and y when beta != 0) in, y out, and
 * returns when y is written.  Device staging is owned by h.  With page-locked
 * x and y (cudaHostAlloc / cudaHostRegister) the copies run chunk by chunk on
 * streams of h and overlap the sweeps; pageable arrays, and x and y that
 * overlap (x == y included), are copied whole.  y is written by the device:
 * do not register it with cudaHostRegisterReadOnly. */
int ainv_gpu_apply_host(ainv_handle *h, char trans, double alpha, const double *x,
                        double beta, double *y);
int ainv_gpu_destroy(ainv_handle *h);
/* Synchronise and report whether any kernel working on h gave up a wait
 * (the streaming kernels bound every wait to about 2 s); clears the flag.
 * AINV_SUCCESS or AINV_ERR_TIMEOUT. */
int ainv_gpu_check(const ainv_handle *h);
size_t ainv_gpu_sizeof(const ainv_handle *h);
long long ainv_gpu_get_nzeros(const ainv_handle *h);
int ainv_gpu_get_n(const ainv_handle *h);
int ainv_gpu_get_prec(const ainv_handle *h);
/* Device layout of one operand: which = 0 W^T, 1 Z (the 'N' sweeps),
 * 2 Z^T, 3 W (the 'T' sweeps).  nnz: entries; slots: stored values incl.
 * padding; nidx: stored index words; nslices: 32-row slices;
 * offset_slices: slices that share one column-offset list. */
int ainv_gpu_layout_info(const ainv_handle *h, int which, long long *nnz, long long *slots,
                         long long *nidx, int *nslices, int *offset_slices);

/* No counterpart in the reference.  The 'N' apply for callers that may not
 * allocate device memory when they apply (a framework that owns all device
 * memory through its own pool, or a latency-critical section where
 * cudaMalloc/cudaFree and the synchronisation they can cause are not
 * allowed).  Every argument is caller-owned device memory: W^T and Z as
 * 0-based CSR (irp n+1, ja/val nnz), dinv, x and y (n doubles); columns
 * outside [0, n) are skipped.  Computes y = alpha * Z * D^-1 * W^T * x +
 * beta * y without allocating: the intermediate vector lives in a built-in
 * device array of 2^20 doubles (8 MiB, held on each device where the
 * library's module is loaded until the process exits), so n must be at most
 * 1,048,576 (larger n returns AINV_ERR_ARG).  The first call on each device
 * looks up that array's address (cudaGetSymbolAddress); make it before any
 * stream capture.  All calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller. */
int ainv_gpu_apply_csr_noalloc(int n, const int *wt_irp, const int *wt_ja,
                               const double *wt_val, long long nnz_wt,
                               const int *z_irp, const int *z_ja, const double *z_val,
                               long long nnz_z, const double *dinv, double alpha,
                               const double *x_dev, double beta, double *y_dev,
                               void *stream);

/* ---- operator A and the Krylov loop ---------------------------------- */
int ainv_csr_create(ainv_csr **a, int n, const int *irp, const int *ja,
                    const double *val, int one_based);
/* y = alpha * A * x + beta * y on device vectors. */
int ainv_csr_spmv(const ainv_csr *a, double alpha, const double *x_dev, double beta,
                  double *y_dev, void *stream);
int ainv_csr_destroy(ainv_csr *a);
/* As ainv_gpu_check, for kernels working on the operator A. */
int ainv_csr_check(const ainv_csr *a);
/* Preconditioned CG / BiCGSTAB with istop=2 (||r||_2 <= eps*||b||_2).
 * x_dev holds x0 on entry and the solution on exit; h may be NULL (no
 * preconditioner).  Returns AINV_SUCCESS on convergence, AINV_ERR_NOCONV
 * at itmax, AINV_ERR_BREAKDOWN / AINV_ERR_NONFINITE on breakdown; *iter and
 * *err (relative residual) are set in every case. */
int ainv_gpu_solve(ainv_handle *h, const ainv_csr *a, const double *b_dev,
                   double *x_dev, int method, double eps, int itmax, int *iter,
                   double *err, void *stream);
/* Statistics of the last ainv_gpu_solve on a: how often the recurrence
 * claimed convergence the true residual did not confirm, and how often the
 * recurrence residual was replaced by b - A x. */
int ainv_csr_solve_info(const ainv_csr *a, int *verify_fails, int *replacements);
/* Relative residual ||r_k||/||b|| after each iteration k of the last
 * ainv_gpu_solve on this operator (the first 8192 iterations), written to
 * rel_res[0 .. min(cap, count)); *count receives the number recorded.  The
 * reference prints the same quantity per iteration when its itrace > 0
 * (psb_krylov's trace; tests/pdegen/ppde3d.f90:280-281 passes itrace). */
int ainv_csr_solve_history(const ainv_csr *a, double *rel_res, int cap, int *count);

/* update_a (src/impl/mld_d_base_ainv_update_a.f90:53-79): reuse the factors
 * for the shifted system A + diag(x) by refreshing the diagonal,
 *   d <- 1 / (1/d + diag(W^T diag(x) Z)),
 * on the device.  x_dev: n doubles on the device.  d_dev_out (may be NULL):
 * n doubles on the device receiving the new d in FP64 (the handle keeps it
 * in its own precision).  Asynchronous on `stream`. */
int ainv_gpu_update_a(ainv_handle *h, const double *x_dev, double *d_dev_out, void *stream);

/* Preconditioned CG on m (1..32) right-hand sides at once: column l solves
 * A x_l = b_l with its own CG recurrence (psb_dcg, istop=2, as
 * ainv_gpu_solve) while every product with A and with the factors is one
 * SpMM over all columns.  B and X are device arrays of n rows by m columns,
 * row-interleaved (entry (i, l) at B[i*ldb + l]); X holds x0 on entry and
 * the solutions on exit.  iters / errs / status (each m entries, may be
 * NULL) receive per column the iterations, the relative residual and the
 * status; the return value is AINV_SUCCESS when every column converged, else
 * the first failing column's status.  h may be NULL (no preconditioner). */
int ainv_gpu_block_solve(ainv_handle *h, const ainv_csr *a, int m, const double *B, int ldb,
                         double *X, int ldx, double eps, int itmax, int *iters, double *errs,
                         int *status, void *stream);

/* ---- host solver types (mirror of the Fortran plugin types) ----------- */
/* type: "AINV", "INVK" or "INVT".  default() is applied on creation. */
int mld_d_solver_create(mld_d_solver **sv, const char *type);
int mld_d_solver_destroy(mld_d_solver *sv);
int mld_d_solver_default(mld_d_solver *sv);
/* String-keyed setters; keys as in the reference: SUB_FILLIN, AINV_ALG,
 * SUB_ILUTHRS, INV_FILLIN, INV_THRESH.  Unknown keys are ignored with
 * success, as the base-solver fallthrough does. */
int mld_d_solver_cseti(mld_d_solver *sv, const char *what, int val);
int mld_d_solver_csetr(mld_d_solver *sv, const char *what, double val);
int mld_d_solver_csetc(mld_d_solver *sv, const char *what, const char *val);
/* Validate the parameters like mld_check_def: an illegal value is reset to
 * its default with a warning on stderr (fill_in >= 1 for AINV, levels >= 0
 * for INVK/INVT, thresholds >= 0); returns AINV_SUCCESS. */
int mld_d_solver_check(mld_d_solver *sv);
/* Host factor construction from A (n x n CSR; entries outside the local
 * n x n block are clipped).  When a device precision has been set with
 * mld_d_solver_cnv, the factors are uploaded at the end of build, as the
 * reference converts them when amold/vmold are present. */
int mld_d_solver_build(mld_d_solver *sv, int n, const int *irp, const int *ja,
                       const double *val, int one_based);
/* Convert (upload) the built factors to the device in precision prec. */
int mld_d_solver_cnv(mld_d_solver *sv, int prec);
int mld_d_solver_apply(mld_d_solver *sv, double alpha, const double *x_dev,
                       double beta, double *y_dev, char trans, void *stream);
/* Host-array form of the apply (apply_a). */
int mld_d_solver_apply_host(mld_d_solver *sv, double alpha, const double *x,
                            double beta, double *y, char trans);
/* Device handle owned by sv (NULL before cnv). */
ainv_handle *mld_d_solver_handle(mld_d_solver *sv);
/* Copy the host factors out.  Call with NULL arrays to get the sizes. */
int mld_d_solver_get_factors(const mld_d_solver *sv, int *n, long long *nnz_wt,
                             long long *nnz_z, int *wt_irp, int *wt_ja,
                             double *wt_val, int *z_irp, int *z_ja, double *z_val,
                             double *d);
int mld_d_solver_clone(const mld_d_solver *sv, mld_d_solver **out);
int mld_d_solver_clone_settings(const mld_d_solver *sv, mld_d_solver *out);
int mld_d_solver_free(mld_d_solver *sv);       /* drop host and device data */
size_t mld_d_solver_sizeof(const mld_d_solver *sv);
long long mld_d_solver_get_nzeros(const mld_d_solver *sv);
int mld_d_solver_get_wrksz(void);              /* 2, like get_wrksz */
/* Human-readable description into buf (always NUL-terminated). */
int mld_d_solver_descr(const mld_d_solver *sv, char *buf, size_t len);
/* Load factors from the MatrixMarket files of a dump: <prefix>_wmat.mtx
 * (W^T), <prefix>_diag.mtx (d) and <prefix>_zmat.mtx (Z), as this library's
 * dump and the reference's (src/impl/mld_d_base_ainv_solver_dmp.f90:82-108,
 * full prefix such as "dump_ainv_d_p000_l001") write them.  The solver is
 * then built (and uploaded if cnv was called), whatever its type. */
int mld_d_solver_load(mld_d_solver *sv, const char *prefix);
/* Binary factor cache (host factors + settings, checksummed): save writes
 * it, restore reads it into a solver of the same type.  No counterpart in
 * the reference; it skips the host build when factors are reused. */
int mld_d_solver_save(const mld_d_solver *sv, const char *path);
int mld_d_solver_restore(mld_d_solver *sv, const char *path);
/* update(x) of the plugin type (src/impl/mld_d_base_ainv_update_a.f90:35-79):
 * the device update_a on the uploaded factors, x being nx host doubles.
 * As in the reference (:54-58, info = -1 when size(x) < size(d)), nx < n is
 * an argument error and nothing is read.  The new d is formed in FP64 from
 * the host's FP64 d whatever the device precision, stored in the host
 * factors and uploaded rounded to the device precision. */
int mld_d_solver_update_a(mld_d_solver *sv, const double *x, int nx);
/* MatrixMarket dump of W^T, D^-1 and Z as <prefix>_wmat.mtx,
 * <prefix>_diag.mtx, <prefix>_zmat.mtx. */
int mld_d_solver_dump(const mld_d_solver *sv, const char *prefix);

/* ---- solve server: continuous batching of many solves ----------------- */
/* The reference solves one system at a time (psb_krylov at
 * tests/pdegen/ppde3d.f90:280-281).  The server keeps preconditioned
 * BiCGSTAB solves (istop=2, the loop of ainv_gpu_solve) against resident
 * operators in flight together: every graph launch advances all admitted
 * requests, whatever their operator and size, by a fixed number of
 * iterations, and requests are admitted first-come first-served as slots
 * and device memory free up.  A request's result does not depend on what
 * else runs beside it (bit-identical iterates alone or in a mix).
 * x0 = 0 for every request. */
typedef struct ainv_server ainv_server;

typedef struct {
  long long id;
  int op;          /* operator index from ainv_server_add_operator */
  int status;      /* AINV_SUCCESS, AINV_ERR_NOCONV, ... as ainv_gpu_solve */
  int iter;        /* BiCGSTAB iterations */
  double err;      /* final relative residual (confirmed on b - A x) */
  double t_submit; /* server clock (seconds since creation) */
  double t_admit;
  double t_done;   /* x written back to the caller's buffer */
} ainv_result;

typedef struct {
  long long submitted, completed, graph_launches, kernel_launches;
  int active, queued, peak_active, max_slots, grid, iters_per_launch;
  size_t arena_bytes, arena_used, arena_peak;
  double clock;
} ainv_server_info;

/* max_slots (1..64): requests in flight together.  hbm_bytes: device bytes
 * for the requests' vectors (0: half of the free HBM); a request is admitted
 * only while its vectors fit (ainv_server_request_bytes).  iters_per_launch
 * (1..64): iterations per graph launch, i.e. how often completion is
 * checked.  Starts the server's engine thread on the current device. */
int ainv_server_create(ainv_server **srv, int max_slots, size_t hbm_bytes,
                       int iters_per_launch);
/* Register a resident operator A with its factors h (AINV, INVK or INVT,
 * any precision; FP32/BF16 factors get true-residual replacement every 50
 * iterations).  Both must outlive the server. */
int ainv_server_add_operator(ainv_server *srv, const ainv_csr *a, const ainv_handle *h,
                             int *op);
/* Queue a solve of A_op x = b.  b (host, n doubles) is read at admission and
 * x (host, n doubles) written at completion: both must stay valid until
 * ainv_server_wait returns for *id.  Thread-safe. */
int ainv_server_submit(ainv_server *srv, int op, const double *b, double *x, double eps,
                       int itmax, long long *id);
/* Wait for request id (timeout_s < 0: no limit); fills *res (may be NULL)
 * and returns the request's status, or AINV_ERR_TIMEOUT if it is still
 * running.  Each id is waited for once. */
int ainv_server_wait(ainv_server *srv, long long id, double timeout_s, ainv_result *res);
int ainv_server_stats(ainv_server *srv, ainv_server_info *out);
/* Finishes every queued request, stops the engine, frees the server. */
int ainv_server_destroy(ainv_server *srv);
/* Device bytes one request of n rows holds while admitted. */
size_t ainv_server_request_bytes(int n);
/* The block plan of a launch: grid blocks shared among nslots requests of
 * rows[k] rows in proportion to their 512-row chunks (at least one each,
 * never more than their chunks).  Host-only; b0/nb receive nslots entries. */
int ainv_server_plan(int nslots, const int *rows, int grid, int *b0, int *nb);

#ifdef __cplusplus
}
#endif
#endif /* AINV_B200_H */
