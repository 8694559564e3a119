/*
 * CPU oracle for the AINV preconditioner application phase.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links, loads or calls
 * this code; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only as the checker / the timed CPU reference.
 *
 * PARITY UNPINNED: the reference (Fortran 2003 on PSBLAS >= 3.4 and
 * MLD2P4 >= 2.1.1) cannot be compiled here -- there is no Fortran compiler,
 * no MPI, no PSBLAS and no MLD2P4 -- and the reference ships no golden
 * vectors.  This file is a plain-C restatement of the reference's algorithm,
 * each function citing the reference file:line it follows, checked against
 * mathematical known-answer tests and an independent pure-Python
 * restatement (tests/golden/).
 *
 * Conventions: all index arrays are 0-based; CSR/CSC arrays are
 * (ptr[n+1], idx[nnz], val[nnz]) with sorted indices inside each row/column.
 */
#ifndef AINV_ORACLE_H
#define AINV_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Biconjugation variants (src/mld_base_ainv_mod.F90:50-56). */
enum { ORC_ALG_LLK = 0, ORC_ALG_S_LLK = 1, ORC_ALG_LLK_NOTH = 2, ORC_ALG_S_FT_LLK = 3, ORC_ALG_MLK = 4 };

/* PSBLAS d_epstol (unit roundoff guard used by the pivot checks). */
#define ORC_EPSTOL 1.1e-16

/* ---- synthetic inputs ---------------------------------------------------*/
/* 7-point 3-D operator on an idim^3 grid, x fastest.  kind 0: Poisson with
 * diagonal 6 and off-diagonals -1 (unscaled).  kind 1: -Lap(u) + b.grad(u)
 * with h = 1/(idim+1), central diffusion, first-order upwind convection.
 * Returns nnz; arrays must hold 7*idim^3 entries. */
long orc_gen_pde3d(int idim, int kind, double bx, double by, double bz,
                   int *irp, int *ja, double *val);
/* Counter-based splitmix64 streams: U[0,1) -> lo + (hi-lo)*u, and N(0,1). */
void orc_rand_uniform(uint64_t seed, long n, double lo, double hi, double *out);
void orc_rand_normal(uint64_t seed, long n, double *out);

/* ---- factor construction (host; fixes the Z/W patterns) ----------------*/
/* mld_d_ainv_bld (src/impl/mld_d_ainv_bld.F90:35-194) with iscale=maxval
 * (src/impl/mld_d_ainv_solver_bld.f90:68-69).  Outputs:
 *   Wt in CSR (row i = column w_i, the reference's sv%w),
 *   Z  in CSR (the reference's sv%z), d = D^-1 (sv%d).
 * Output capacity must be n*fill_in for both factors.
 * Returns 0 on success; *nnz_wt / *nnz_z receive the counts. */
int orc_ainv_build(int alg, int n, const int *irp, const int *ja,
                   const double *val, int fill_in, double thresh,
                   int *wt_irp, int *wt_ja, double *wt_val, long *nnz_wt,
                   int *z_irp, int *z_ja, double *z_val, long *nnz_z,
                   double *d);

/* mld_d_invk_bld (src/impl/mld_d_invk_bld.f90:104-125): ILU(fill1), then
 * the level-fill2 sparse inverses of U and L (via L^T).  mld_d_invt_bld
 * (src/impl/mld_d_invt_bld.f90:108-136): ILUT(fillin, thresh) with maxval
 * scaling, then the (invfill, invthresh) sparse inverses.  Both produce
 * W^T ~ L^-1 (CSR), Z ~ U^-1 (CSR) and d = D^-1 (n entries, caller-owned).
 * The factor arrays are allocated here; release each with orc_free.
 * Returns 0, or a negative value (-(row+1) for a too-small pivot). */
int orc_invk_build(int n, const int *irp, const int *ja, const double *val,
                   int fill1, int fill2,
                   int **wt_irp, int **wt_ja, double **wt_val, long *nnz_wt,
                   int **z_irp, int **z_ja, double **z_val, long *nnz_z, double *d);
int orc_invt_build(int n, const int *irp, const int *ja, const double *val,
                   int fillin, double thresh, int invfill, double invthresh,
                   int **wt_irp, int **wt_ja, double **wt_val, long *nnz_wt,
                   int **z_irp, int **z_ja, double **z_val, long *nnz_z, double *d);
void orc_free(void *p);

/* mld_d_base_ainv_update_a (src/impl/mld_d_base_ainv_update_a.f90:53-79):
 * d_out = 1 / (1/d + diag(W^T diag(x) Z)), Wt and Z in CSR. */
int orc_update_a(int n, const int *wt_irp, const int *wt_ja, const double *wt_val,
                 const int *z_irp, const int *z_ja, const double *z_val,
                 const double *d, const double *x, double *d_out);

/* ---- application phase --------------------------------------------------*/
/* y = alpha*A*x + beta*y (PSBLAS CSR csmv, trans='N'); OpenMP over rows. */
void orc_csr_spmv(int n, const int *irp, const int *ja, const double *val,
                  double alpha, const double *x, double beta, double *y);
/* y = alpha*A^T*x + beta*y (scatter form, serial). */
void orc_csr_spmv_t(int n, const int *irp, const int *ja, const double *val,
                    double alpha, const double *x, double beta, double *y);
/* mld_d_base_ainv_solver_apply_vect
 * (src/impl/mld_d_base_ainv_solver_apply_vect.f90:112-127):
 *   'N': y = alpha*Z*(d.*(Wt*x)) + beta*y
 *   'T'/'C': y = alpha*W*(d.*(Z^T*x)) + beta*y
 * work must hold n doubles.  Returns 0, or -1 for an invalid trans. */
int orc_ainv_apply(int n, const int *wt_irp, const int *wt_ja,
                   const double *wt_val, const int *z_irp, const int *z_ja,
                   const double *z_val, const double *d, char trans,
                   double alpha, const double *x, double beta, double *y,
                   double *work);

/* ---- Krylov loop --------------------------------------------------------*/
/* Preconditioned CG / BiCGSTAB in the PSBLAS psb_dcg / psb_dbicgstab form
 * (called at tests/pdegen/ppde3d.f90:280-281) with istop=2:
 * stop when ||r||_2 <= eps*||b||_2.  x holds x0 on entry.  The
 * preconditioner is the AINV apply above ('N', alpha=1, beta=0).
 * Returns 0 on convergence, 1 if itmax was reached, <0 on breakdown. */
int orc_cg(int n, const int *irp, const int *ja, const double *val,
           const int *wt_irp, const int *wt_ja, const double *wt_val,
           const int *z_irp, const int *z_ja, const double *z_val,
           const double *d, const double *b, double *x, double eps,
           int itmax, int *iter, double *err);
int orc_bicgstab(int n, const int *irp, const int *ja, const double *val,
                 const int *wt_irp, const int *wt_ja, const double *wt_val,
                 const int *z_irp, const int *z_ja, const double *z_val,
                 const double *d, const double *b, double *x, double eps,
                 int itmax, int *iter, double *err);

/* Summation order of the Krylov dots (see ainv_oracle.c): the device
 * library's canonical order (default; iterates equal the device's bit for
 * bit) or a sequential sum (the reference BLAS ddot). */
enum { ORC_DOT_DEVICE = 0, ORC_DOT_SEQUENTIAL = 1 };
void orc_set_dot_order(int order);
double orc_dot_device_order(int n, const double *a, const double *b);
/* Record ||r_k||/||b|| of iteration k at rel_res[k-1] (k <= cap) during the
 * following solves; NULL stops recording. */
void orc_set_history(double *rel_res, int cap);

/* OpenMP thread control for the timed CPU baseline. */
void orc_set_threads(int nthreads);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
