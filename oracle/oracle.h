/*
 * oracle.h -- CPU restatement (FP64) of LFRic Core's Krylov-solve hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the correctness oracle and the
 * timed CPU baseline. Only tests/, __graft_entry__.smoke() and the CPU legs of
 * bench.py load it, and only as the checker; the product path
 * (lfric_core_b200) never links or calls it.
 *
 * Reference files restated (paths inside the reference project):
 *   matrix_vector_code      components/science/source/kernel/algebra/matrix_vector_kernel_mod.F90:107-140
 *   transpose_matrix_vector components/science/source/kernel/algebra/transpose_matrix_vector_kernel_mod.F90:107-146
 *   dg_matrix_vector        components/science/source/kernel/algebra/dg_matrix_vector_kernel_mod.F90:113-156
 *   mm_diagonal             components/science/source/kernel/algebra/sci_mm_diagonal_kernel_mod.F90:99-125
 *   mass_matrix_operator    components/science/source/algorithm/solver/sci_mass_matrix_operator_alg_mod.x90:72-119
 *   diagonal_preconditioner components/science/source/algorithm/solver/sci_diagonal_preconditioner_alg_mod.x90:71-106
 *   field_vector ops        components/science/source/algorithm/solver/sci_field_vector_mod.x90:132-466
 *   CMA asm/app/appinv      components/science/source/kernel/columnwise_operators/sci_columnwise_op_{asm,app,appinv}_kernel_mod.F90
 *   tri_solve               components/science/source/kernel/solver/sci_tri_solve_kernel_mod.f90:72-156
 *   cg/bicgstab/gmres       components/science/source/solver/sci_iterative_solver_mod.f90:495-592, 645-779, 830-1003
 *   operator_x_plus_ay      components/science/source/kernel/algebra/sci_operator_algebra_kernel_mod.F90:92-119
 *
 * Arithmetic conventions (shared with the device path so FP64 results can be
 * compared bit for bit): every "a = a + b*c" of the reference is one fused
 * multiply-add, fma(b, c, a); nothing else is contracted (-ffp-contract=off).
 * Global sums use the fixed blocked order described at or_dot().
 */
#ifndef LFX_ORACLE_H
#define LFX_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* reduction order: 0 = blocked order shared with the device (default),
 *                  1 = plain sequential sum (the reference loop read literally) */
void or_set_reduction_order(int mode);
void or_set_threads(int nthreads);

/* ---- PSyclone builtins / field_vector ops on one field of length n ---- */
double or_dot(const double* x, const double* y, int64_t n);
double or_sumsq(const double* x, int64_t n);
void or_setval_c(double* x, double c, int64_t n);
void or_setval_x(double* y, const double* x, int64_t n);
void or_inc_x_plus_by(double* x, double b, const double* y, int64_t n);   /* x += b*y  (axpy) */
void or_inc_ax_plus_y(double a, double* x, const double* y, int64_t n);   /* x = a*x + y (aypx) */
void or_ax_plus_by(double* z, double a, const double* x, double b, const double* y, int64_t n);
void or_inc_a_times_x(double a, double* x, int64_t n);                    /* x = a*x */
void or_x_divideby_y(double* z, const double* x, const double* y, int64_t n);

/* ---- kernels, one cell column (cell is 1-based; maps are 1-based) ---- */
void or_matrix_vector_code(int32_t cell, int32_t nlayers, double* lhs, const double* x,
                           int64_t ncell_3d, const double* matrix, int32_t ndf1,
                           const int32_t* map1, int32_t ndf2, const int32_t* map2);
void or_transpose_matrix_vector_code(int32_t cell, int32_t nlayers, double* lhs,
                                     const double* x, int64_t ncell_3d, const double* matrix,
                                     int32_t ndf1, const int32_t* map1, int32_t ndf2,
                                     const int32_t* map2);
void or_dg_matrix_vector_code(int32_t cell, int32_t nlayers, double* lhs, const double* x,
                              int64_t ncell_3d, const double* matrix, int32_t ndf1,
                              const int32_t* map1, int32_t ndf2, const int32_t* map2);
/* operator_x_plus_ay_kernel_code for one cell column: x_plus_ay(ik,:,:) =
 * x(ik,:,:) + a*y(ik,:,:), ik = k + 1 + (cell-1)*nlayers, k = 0..nlayers-1,
 * on (ncell_3d, ndf1, ndf2) operators */
void or_operator_x_plus_ay_code(int32_t cell, int32_t nlayers, int64_t ncell_3d, double* x_plus_ay,
                                const double* x, double a, const double* y, int32_t ndf1,
                                int32_t ndf2);
void or_tri_solve_code(int32_t nlayers, double* y, const double* x, const double* tri_0,
                       const double* tri_plus, const double* tri_minus, const int32_t* map);
void or_columnwise_op_asm_code(int32_t cell, int32_t nlayers, int32_t ncell_2d,
                               int64_t ncell_3d, const double* local_stencil,
                               double* columnwise_matrix, int32_t nrow, int32_t ncol,
                               int32_t bandwidth, int32_t alpha, int32_t beta,
                               int32_t gamma_m, int32_t gamma_p, int32_t ndf_to,
                               const int32_t* column_banded_dofmap_to, int32_t ndf_from,
                               const int32_t* column_banded_dofmap_from);
void or_columnwise_op_app_code(int32_t cell, double* lhs, const double* x,
                               const double* columnwise_matrix, int32_t nrow, int32_t ncol,
                               int32_t bandwidth, int32_t alpha, int32_t beta,
                               int32_t gamma_m, int32_t gamma_p, const int32_t* map1,
                               const int32_t* indirection_to, const int32_t* map2,
                               const int32_t* indirection_from);
void or_columnwise_op_appinv_code(int32_t cell, double* lhs, const double* x,
                                  const double* columnwise_matrix, int32_t nrow,
                                  int32_t bandwidth, const int32_t* map,
                                  const int32_t* indirection);

/* ---- operators and preconditioners (objects keep the caller's pointers) ---- */
typedef struct or_op or_op;
typedef struct or_prec or_prec;

/* CMA set-up kernels, one column (cell, 1-based) of Fortran band arrays
 * (bw, nrow, ncell_2d) and local stencils (ncell_3d, ndf_to, ndf_from):
 *   mul        sci_columnwise_op_mul_kernel_mod.F90 (C += A B)
 *   scaledadd  sci_columnwise_op_scaledadd_kernel_mod.F90 (C = alpha A + beta B)
 *   m2v_lumped_inv  sci_columnwise_op_asm_m2v_lumped_inv_krnl_mod.F90:74-132
 *   diag_hmht  sci_columnwise_op_asm_diag_hmht_kernel_mod.F90:78-151 */
void or_columnwise_op_mul_code(int32_t cell, int32_t ncell_2d, const double* A, int32_t nrow_A,
                               int32_t ncol_A, int32_t bw_A, int32_t alpha_A, int32_t beta_A,
                               int32_t gm_A, int32_t gp_A, const double* B, int32_t nrow_B,
                               int32_t ncol_B, int32_t bw_B, int32_t alpha_B, int32_t beta_B,
                               int32_t gm_B, int32_t gp_B, double* C, int32_t nrow_C,
                               int32_t ncol_C, int32_t bw_C, int32_t alpha_C, int32_t beta_C,
                               int32_t gm_C, int32_t gp_C);
void or_columnwise_op_scaledadd_code(int32_t cell, int32_t ncell_2d, const double* A,
                                     int32_t nrow_A, int32_t ncol_A, int32_t bw_A, int32_t alpha_A,
                                     int32_t beta_A, int32_t gm_A, int32_t gp_A, const double* B,
                                     int32_t nrow_B, int32_t ncol_B, int32_t bw_B, int32_t alpha_B,
                                     int32_t beta_B, int32_t gm_B, int32_t gp_B, double* C,
                                     int32_t nrow_C, int32_t ncol_C, int32_t bw_C, int32_t alpha_C,
                                     int32_t beta_C, int32_t gm_C, int32_t gp_C, double alpha,
                                     double beta);
void or_columnwise_op_asm_m2v_lumped_inv_code(int32_t cell, int32_t nlayers, int32_t ncell_2d,
                                              int32_t ncell_3d, const double* local_stencil,
                                              double* C, int32_t nrow, int32_t bw, int32_t ndf,
                                              const int32_t* column_banded_dofmap);
void or_columnwise_op_asm_diag_hmht_code(int32_t cell, int32_t nlayers, int32_t ncell_2d,
                                         int32_t ncell_3d, const double* Dh, const double* M2h,
                                         double* C, int32_t nrow, int32_t bw, int32_t alpha,
                                         int32_t beta, int32_t gamma_m, int32_t gamma_p,
                                         int32_t ndf_w3, const int32_t* column_banded_dofmap,
                                         int32_t ndf_w2h);

/* W2 split / combine for the lowest-order spaces (ndf_w2 6, ndf_w2h 4,
 * ndf_w2v 2), one cell (maps of that cell, 1-based):
 *   face_selector  sci_face_selector_kernel_mod.F90 (face_counter on W2h)
 *   split          split_w2_field_kernel_mod.F90 (uvw -> uv, w)
 *   combine        combine_w2_field_kernel_mod.F90 (uv, w -> uvw)
 * Arrays are 0-based host arrays indexed by the 1-based map values minus 1. */
void or_face_selector_code(int32_t* face_selector_ew, int32_t* face_selector_ns,
                           int32_t* face_counter, const int32_t* map_w3, const int32_t* map_w2h);
void or_split_w2_field_code(int32_t nlayers, double* uv, double* w, const double* uvw,
                            const int32_t* face_selector_ew, const int32_t* face_selector_ns,
                            const int32_t* map_w2h, const int32_t* map_w2v, const int32_t* map_w2,
                            const int32_t* map_w3_2d);
void or_combine_w2_field_code(int32_t nlayers, double* uvw, const double* uv, const double* w,
                              const int32_t* face_selector_ew, const int32_t* face_selector_ns,
                              const int32_t* map_w2, const int32_t* map_w2h,
                              const int32_t* map_w2v, const int32_t* map_w3_2d);

/* LMA operator: y = A x, coloured loop over cell columns. maps [ncell_2d][ndf],
 * cells_in_colour Fortran (ncolours, maxc), 1-based. mode 0 = matrix_vector
 * (GH_INC after setval_c(y,0)), 1 = transpose_matrix_vector. */
or_op* or_lma_create(int32_t ncell_2d, int32_t nlayers, int32_t ndf_to, int32_t ndf_from,
                     const int32_t* map_to, const int32_t* map_from, int64_t undf_to,
                     int64_t undf_from, const double* stencil, int32_t ncolours,
                     const int32_t* ncells_per_colour, const int32_t* cells_in_colour,
                     int32_t maxc, int32_t mode);
void or_op_apply(or_op* op, const double* x, double* y);
void or_op_destroy(or_op* op);
/* diag(A) assembled by mm_diagonal over the same colouring (to-space == from-space) */
void or_lma_diagonal(const or_op* op, double* diag);

or_prec* or_null_prec_create(int64_t n);
or_prec* or_diag_prec_create(const double* diag, int64_t n);
/* CMA Thomas inverse on the rows of every column given by
 * first_dof[c] + indirection[i] - 1 (1-based), and y = x/diag on all other rows
 * (diag may be NULL when the CMA covers every row). */
or_prec* or_cma_prec_create(int32_t ncell_2d, int32_t nrow, int32_t bandwidth,
                            const int32_t* first_dof, const int32_t* indirection,
                            const double* columnwise_matrix, const double* diag, int64_t n);
void or_prec_apply(or_prec* p, const double* x, double* y);
void or_prec_destroy(or_prec* p);

typedef struct {
  int32_t iterations; /* CG/BiCGStab: iterations; GMRES: restart cycles */
  int32_t converged;
  double initial_norm; /* ||b - A x0|| */
  double final_norm;   /* last monitored residual norm */
  double final_rel;    /* last monitored relative residual */
  int32_t applies;     /* operator applications */
} or_info;

int or_cg(or_op* A, or_prec* P, double* x, const double* b, int64_t n, double r_tol,
          double a_tol, int32_t max_iter, or_info* info);
int or_bicgstab(or_op* A, or_prec* P, double* x, const double* b, int64_t n, double r_tol,
                double a_tol, int32_t max_iter, or_info* info);
int or_gmres(or_op* A, or_prec* P, double* x, const double* b, int64_t n, int32_t gcrk,
             double r_tol, double a_tol, int32_t max_iter, or_info* info);
/* fgmres_solve (sci_iterative_solver_mod.f90:1055-1237): flexible GMRES with
 * the preconditioned basis Pv kept; the residual starts from b (the reference
 * assumes a zero initial guess) and x += dx at the end. iterations = cycles. */
int or_fgmres(or_op* A, or_prec* P, double* x, const double* b, int64_t n, int32_t gcrk,
              double r_tol, double a_tol, int32_t max_iter, or_info* info);
/* gcr_solve (sci_iterative_solver_mod.f90:1288-1408): right-preconditioned
 * GCR(gcrk) with dx0 = P b, relative to ||b||. iterations = outer restarts;
 * *iv_final = the inner step at the last check. */
int or_gcr(or_op* A, or_prec* P, double* x, const double* b, int64_t n, int32_t gcrk,
           double r_tol, double a_tol, int32_t max_iter, or_info* info, int32_t* iv_final);
/* precondition_only_solve (:1664-1694): x = P b, then (monitoring) the
 * residual ||b - A x|| against ||b||. */
int or_precondition_only(or_op* A, or_prec* P, double* x, const double* b, int64_t n,
                         or_info* info);
/* jacobi_solve (:1745-1815): x += -rho P (A x - b) until ||r||/||r_1|| <= r_tol
 * or ||r|| <= a_tol (checked before each update); iterations = checks made. */
int or_jacobi(or_op* A, or_prec* P, double* x, const double* b, int64_t n, double r_tol,
              double a_tol, int32_t max_iter, double rho_relax, or_info* info);
/* chebyshev_solve (:1868-1940): max_iter steps from x = 0 with eigenvalue
 * bounds lmin, lmax; final ||A x - b|| / max(1, ||b||). */
int or_chebyshev(or_op* A, or_prec* P, double* x, const double* b, int64_t n, int32_t max_iter,
                 double lmin, double lmax, or_info* info);

#ifdef __cplusplus
}
#endif
#endif
