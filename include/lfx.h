/*
 * lfx.h -- C ABI of the B200-native Krylov-solve path for LFRic-style
 * extruded-mesh finite-element operators (single GPU, sm_100a).
 *
 * Drop-in surface: the three abstract types a Krylov solver of the reference
 * talks to, plus an optional whole-solve object.
 *   abstract_vector_type          infrastructure/source/field/vector_mod.F90:17-189
 *   abstract_linear_operator_type components/science/source/solver/sci_linear_operator_mod.f90:18-36
 *   abstract_preconditioner_type  components/science/source/solver/sci_preconditioner_mod.f90:19-38
 *   abstract_iterative_solver_type components/science/source/solver/sci_iterative_solver_mod.f90:38-57
 * A Fortran shim (lfric_core_b200/fortran/lfx_device_mod.f90) extends each
 * abstract type with one bind(C) call per type-bound procedure.
 *
 * Conventions
 *  - Every function returns an lfx_status; 0 is success. No function aborts;
 *    lfx_last_error() gives the message of the last failure on a context.
 *  - Array arguments are the reference's native arrays: dof ids and cell ids
 *    are 1-based, multi-dimensional arrays are in Fortran (column-major)
 *    order. Scalars are double at the ABI (the reference's r_def).
 *  - Data passed at create time is copied to the device; the caller may free
 *    its arrays afterwards.
 *  - Objects belong to one context; a context owns one CUDA stream and is
 *    used from one host thread at a time. Operations are stream-ordered;
 *    functions that return a scalar (dot, norm) synchronise the stream.
 */
#ifndef LFX_H
#define LFX_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  LFX_OK = 0,
  LFX_NOT_CONVERGED = 1,
  LFX_NAN_DETECTED = 2,
  LFX_OUT_OF_MEMORY = 3,
  LFX_INVALID_ARGUMENT = 4,
  LFX_TYPE_MISMATCH = 5,
  LFX_TIMEOUT = 6,
  LFX_CUDA_ERROR = 7,
  LFX_NOT_SUPPORTED = 8
} lfx_status;

/* storage precision of a vector or operator: r_def (FP64) or r_solver (FP32) */
enum { LFX_R64 = 64, LFX_R32 = 32 };

typedef struct lfx_ctx lfx_ctx;
typedef struct lfx_vec lfx_vec;
typedef struct lfx_op lfx_op;
typedef struct lfx_prec lfx_prec;
typedef struct lfx_cma lfx_cma;
typedef struct lfx_solver lfx_solver;

/* ------------------------------------------------------------------ context */
int lfx_ctx_create(int device, lfx_ctx** out);
int lfx_ctx_destroy(lfx_ctx* ctx);
const char* lfx_last_error(const lfx_ctx* ctx);
int lfx_ctx_synchronize(lfx_ctx* ctx);
/* the context's cudaStream_t, for callers that time or order work around it */
void* lfx_ctx_stream(lfx_ctx* ctx);
/* device bytes currently held by objects of this context */
int64_t lfx_ctx_device_bytes(const lfx_ctx* ctx);

/* ------------------------------------------------------------------ vectors
 * field_vector_type (sci_field_vector_mod.x90:24-468) and, for precision 32,
 * r_solver_field_vector_type (sci_r_solver_field_vector_mod.x90:26-479):
 * nfields fields of undf[i] values each. Inner products always accumulate
 * in FP64 (sci_psykal_light_mod.f90:72-214). */
int lfx_vec_create(lfx_ctx* ctx, int32_t nfields, const int64_t* undf, int32_t precision,
                   lfx_vec** out);
/* duplicate: same shape and precision, contents undefined (vector_mod duplicate) */
int lfx_vec_duplicate(const lfx_vec* src, lfx_vec** out);
int lfx_vec_destroy(lfx_vec* v);
int lfx_vec_set_scalar(lfx_vec* v, double scalar);                      /* setval_c      */
int lfx_vec_axpy(lfx_vec* y, double alpha, const lfx_vec* x);           /* y = y + a x   */
int lfx_vec_aypx(lfx_vec* y, double alpha, const lfx_vec* x);           /* y = a y + x   */
int lfx_vec_axpby(lfx_vec* z, double a, const lfx_vec* x, double b, const lfx_vec* y);
int lfx_vec_norm(const lfx_vec* v, double* out);                        /* sqrt(sum v^2) */
int lfx_vec_field_norm(const lfx_vec* v, int32_t position, double* out);/* 1-based field */
int lfx_vec_dot(const lfx_vec* v, const lfx_vec* x, double* out);
int lfx_vec_scale(lfx_vec* v, double scalar);
int lfx_vec_copy(lfx_vec* dst, const lfx_vec* src);                     /* dst = src     */
int lfx_vec_size(const lfx_vec* v, int32_t* nfields);
/* import_field / export_field (sci_field_vector_mod.x90:294-334): host FP64
 * data of field `position` (1-based); converts to/from FP32 storage. */
int lfx_vec_import_field(lfx_vec* v, int32_t position, const double* host, int64_t n);
int lfx_vec_export_field(const lfx_vec* v, int32_t position, double* host, int64_t n);
/* the same transfers for an FP64 field, queued on `stream` (a cudaStream_t;
 * NULL = the context's stream) without waiting: with pinned host memory they
 * overlap work on other streams (e.g. the next request's right-hand side
 * arriving while a solve runs). The caller orders `stream` against the
 * context's stream (lfx_ctx_stream, events) and keeps `host` alive until the
 * copy is done. No counterpart in the reference (its fields live on the host). */
int lfx_vec_import_field_async(lfx_vec* v, int32_t position, const double* host, int64_t n,
                               void* stream);
int lfx_vec_export_field_async(const lfx_vec* v, int32_t position, double* host, int64_t n,
                               void* stream);
/* raw device pointer of a field (for zero-copy callers); precision tells the type */
int lfx_vec_field_device_ptr(const lfx_vec* v, int32_t position, void** out);

/* ------------------------------------------------------------------ operators
 * LMA operator (operator_type, operator_mod.t90:31-122) applied as the
 * reference's matrix_vector_kernel over a cell colouring
 * (sci_mass_matrix_operator_alg_mod.x90:98, matrix_vector_kernel_mod.F90:107-140):
 * y is overwritten with A x. Colour order fixes the summation order, which the
 * device reproduces bit for bit in FP64.
 *   map_to / map_from   Fortran (ndf, ncell_2d): dof id of layer 0 of each local dof
 *   local_stencil       Fortran (ncell_2d*nlayers, ndf_to, ndf_from)
 *   cells_in_colour     Fortran (ncolours, max_cells_per_colour), 1-based cell ids
 *   precision           device storage: LFX_R64, or LFX_R32 (rounded copy)
 * local_stencil may be host or device memory. */
int lfx_lma_create(lfx_ctx* ctx, int32_t ncell_2d, int32_t nlayers, int32_t ndf_to,
                   int32_t ndf_from, const int32_t* map_to, const int32_t* map_from,
                   int64_t undf_to, int64_t undf_from, const double* local_stencil,
                   int32_t ncolours, const int32_t* ncells_per_colour,
                   const int32_t* cells_in_colour, int32_t max_cells_per_colour,
                   int32_t precision, lfx_op** out);
/* A second operator sharing the dofmaps and colouring of `src` but holding
 * its own local matrices (e.g. the FP32 copy of an FP64 operator). */
int lfx_lma_create_like(const lfx_op* src, const double* local_stencil, int32_t precision,
                        lfx_op** out);
int lfx_op_apply(lfx_op* op, const lfx_vec* x, lfx_vec* y);
int lfx_op_destroy(lfx_op* op);
/* operator_x_plus_ay (components/science/source/kernel/algebra/
 * sci_operator_algebra_kernel_mod.F90:92-119): a new operator x + a y, entry
 * by entry (each entry one fma, as the oracle computes it), for two operators
 * of one precision sharing one layout (made from one another by
 * lfx_lma_create_like, e.g. the mass matrix and tau D^T D); the result shares
 * that layout. An FP32 pair sums in FP32. */
int lfx_lma_sum(const lfx_op* x, double a, const lfx_op* y, lfx_op** out);
/* Apply autotuner (no counterpart in the reference, whose loop shape is fixed
 * by PSyclone): times each launch configuration of the apply on this
 * operator -- the register gather, the register gather with prefetched
 * column descriptors (at two register caps, stages 0 and 1; columns reading
 * at most two blocks from at most two cells, e.g. W2 and W3), the bulk-copy
 * pipeline with 2..8 stages and 1..8 warps per block, and the copy-staged
 * pipeline with 2..6 stages and 2..8 warps, those that fit the shared memory,
 * and the cell scatter (square operators on one dofmap; one launch per
 * colour, reading a symmetric operator's packed upper triangle; or, ndf 6
 * or 8 with at most 31 levels, one persistent launch whose colours meet at
 * bounded grid barriers, 4 or 6 ring stages of 4 or 8 warps) -- over
 * `reps` launches and keeps the fastest for later applies. Outputs
 * (nullable) name the choice: kernel 0 pipeline / 1 register gather / 2
 * generic / 3 register gather with prefetched descriptors / 4 copy-staged
 * pipeline (matrix blocks and x values both staged in shared memory) / 5 cell
 * scatter / 6 persistent cell scatter, and its time per apply. */
int lfx_op_autotune(lfx_op* op, int32_t reps, int32_t* kernel, int32_t* stages, int32_t* warps,
                    float* us);
/* time one configuration (as above) without keeping it. Both time on
 * scratch vectors allocated for the call: consecutive applies take different
 * x and y (pairs enough to hold twice the L2), so the vectors travel to and
 * from HBM on every apply, as the local matrices do. */
int lfx_op_time_apply(lfx_op* op, int32_t kernel, int32_t stages, int32_t warps, int32_t reps,
                      float* us);
/* keep one configuration (as above) for later applies, as the autotuner
 * would; LFX_NOT_SUPPORTED if it does not fit the operator. Kernel 5 takes
 * stages 0 (one cell per warp) or 2, 3 (cells staged ahead in shared memory);
 * kernel 6 stages 4 or 6 (ring stages per warp) and warps 4 or 8 per block. */
int lfx_op_set_apply(lfx_op* op, int32_t kernel, int32_t stages, int32_t warps);
/* bytes of the stored local matrices: the full copy every kernel can read
 * and the packed upper triangle of a bitwise symmetric operator on one
 * dofmap (0 when there is none), which the cell scatter reads instead */
int lfx_op_storage(const lfx_op* op, int64_t* full_bytes, int64_t* packed_bytes);
/* diag(A) by mm_diagonal_kernel (sci_mm_diagonal_kernel_mod.F90:99-125) */
int lfx_lma_diagonal(lfx_op* op, lfx_vec* diag);
/* transpose apply y = A^T x for a matrix stored as (ncell_3d, ndf_to, ndf_from)
 * (transpose_matrix_vector_kernel_mod.F90); y is overwritten */
int lfx_op_apply_transpose(lfx_op* op, const lfx_vec* x, lfx_vec* y);

/* ------------------------------------------------------------------ FEM set-up
 * Device assembly of the local matrices by 3x3x3 Gauss quadrature on the
 * trilinear hexahedra of an extruded mesh (the role of the reference's
 * compute_mass_matrix_kernel_w_scalar / _w2 and compute_div_operator_kernel,
 * components/science/source/kernel/fem/), followed by lfx_lma_create. Either
 * output may be NULL; both share one layout.
 *   verts_on_cell  [ncell_2d][4] 1-based (SW, SE, NE, NW)
 *   xyz3d          [nvert_2d][nlayers+1][3] vertex positions
 *   cell_next      [ncell_2d][4] 1-based (W, S, E, N): orients the RT0 faces
 * W0: A = M + nu K (Q1 mass + diffusion). W2: A = M2 + tau D^T D (RT0 mass
 * plus the W3 divergence penalty). */
int lfx_fem_w0_operator(lfx_ctx* ctx, int32_t ncell_2d, int32_t nlayers,
                        const int32_t* verts_on_cell, int64_t nvert_2d, const double* xyz3d,
                        double nu, const int32_t* map, int64_t undf, int32_t ncolours,
                        const int32_t* ncells_per_colour, const int32_t* cells_in_colour,
                        int32_t max_cells_per_colour, lfx_op** op64, lfx_op** op32);
int lfx_fem_w2_operator(lfx_ctx* ctx, int32_t ncell_2d, int32_t nlayers, const int32_t* cell_next,
                        const int32_t* verts_on_cell, int64_t nvert_2d, const double* xyz3d,
                        double tau, const int32_t* map, int64_t undf, int32_t ncolours,
                        const int32_t* ncells_per_colour, const int32_t* cells_in_colour,
                        int32_t max_cells_per_colour, lfx_op** op64, lfx_op** op32);

/* ------------------------------------------------------------------ CMA
 * columnwise_operator_type (columnwise_operator_mod.f90:42-469): one banded
 * matrix columnwise_matrix(bandwidth, nrow, ncell_2d) per column.
 *   first_dof[c]   dof id (1-based) of the column's first dof (map(1) of the
 *                  CMA space, which may point into a larger vector)
 *   indirection    (nrow) indirection_dofmap, 1-based offsets within a column */
int lfx_cma_create(lfx_ctx* ctx, int32_t ncell_2d, int32_t nrow, int32_t ncol,
                   int32_t bandwidth, int32_t alpha, int32_t beta, int32_t gamma_m,
                   int32_t gamma_p, const int32_t* first_dof, const int32_t* indirection,
                   const double* columnwise_matrix, lfx_cma** out);
/* columnwise_op_asm (sci_columnwise_op_asm_kernel_mod.F90:72-128) on the
 * device: assembles the band from the sub-block of an FP64 LMA operator
 * formed by its local dofs `dfs` (1-based, nsub of them), which must map to
 * the column's rows through column_banded_dofmap (Fortran (nsub, nlayers)). */
int lfx_cma_assemble_from_lma(const lfx_op* lma, int32_t nsub, const int32_t* dfs,
                              const int32_t* column_banded_dofmap, int32_t alpha,
                              int32_t beta, int32_t gamma_m, int32_t gamma_p,
                              int32_t bandwidth, int32_t nrow, const int32_t* first_dof,
                              const int32_t* indirection, lfx_cma** out);
/* CMA set-up algebra (the Helmholtz column operators of the reference's
 * pressure preconditioner are built this way). Operators made here have no
 * dofmap (lfx_cma_set_dofmap attaches one to a square operator before
 * lfx_cma_apply / lfx_cma_prec_create) and may be rectangular (nrow != ncol).
 * Band parameters must satisfy bandwidth >= 1 + ceiling((g_m + g_p)/beta). */
int lfx_cma_create_banded(lfx_ctx* ctx, int32_t ncell_2d, int32_t nrow, int32_t ncol,
                          int32_t bandwidth, int32_t alpha, int32_t beta, int32_t gamma_m,
                          int32_t gamma_p, const double* columnwise_matrix, lfx_cma** out);
int lfx_cma_set_dofmap(lfx_cma* cma, const int32_t* first_dof, const int32_t* indirection);
/* C += A B: columnwise_op_mul_kernel (sci_columnwise_op_mul_kernel_mod.F90) */
int lfx_cma_mul(const lfx_cma* A, const lfx_cma* B, lfx_cma* C);
/* new C = A B: columnwise_operator_product (columnwise_operator_mod.f90) + mul;
 * alpha/beta/gamma from the product rule, divided by gcd(alpha, beta) */
int lfx_cma_product(const lfx_cma* A, const lfx_cma* B, lfx_cma** C);
/* C = alpha A + beta B: columnwise_op_scaledadd_kernel
 * (sci_columnwise_op_scaledadd_kernel_mod.F90); C's band must hold A's and B's */
int lfx_cma_scaledadd(const lfx_cma* A, const lfx_cma* B, lfx_cma* C, double alpha, double beta);
/* new C = alpha A + beta B: columnwise_operator_sum + scaledadd */
int lfx_cma_sum(const lfx_cma* A, const lfx_cma* B, double alpha, double beta, lfx_cma** C);
/* columnwise_op_asm_m2v_lumped_inv_krnl (..._krnl_mod.F90:74-132): inverse of
 * the lumped (diagonal) square FP64 LMA, in band entry 1 of each row;
 * column_banded_dofmap Fortran (ndf, nlayers) */
int lfx_cma_assemble_m2v_lumped_inv(const lfx_op* lma, const int32_t* column_banded_dofmap,
                                    int32_t alpha, int32_t beta, int32_t gamma_m, int32_t gamma_p,
                                    int32_t bandwidth, int32_t nrow, lfx_cma** out);
/* columnwise_op_asm_diag_hmht_kernel (..._kernel_mod.F90:78-151): sum over the
 * W2h dofs of Dh Dh^T / diag(M2h), Dh the FP64 W2h -> W3 LMA and M2h the FP64
 * W2h mass LMA; column_banded_dofmap Fortran (ndf_w3, nlayers) */
int lfx_cma_assemble_diag_hmht(const lfx_op* Dh, const lfx_op* M2h,
                               const int32_t* column_banded_dofmap, int32_t alpha, int32_t beta,
                               int32_t gamma_m, int32_t gamma_p, int32_t bandwidth, int32_t nrow,
                               lfx_cma** out);
/* copy of the band back to the host, Fortran (bandwidth, nrow, ncell_2d) */
int lfx_cma_get_band(const lfx_cma* cma, double* band);
/* y += A x (columnwise_op_app_kernel_mod.F90:73-124) */
int lfx_cma_apply(lfx_cma* cma, const lfx_vec* x, lfx_vec* y);
int lfx_cma_destroy(lfx_cma* cma);

/* ------------------------------------------------------------------ W2 split / combine
 * split_w2_field_kernel_mod.F90 / combine_w2_field_kernel_mod.F90 for the
 * lowest-order spaces: W2 (6 dofs per cell, faces W S E N B T) to and from its
 * horizontal part W2h (4) and vertical part W2v (2, one column of nlayers + 1
 * dofs). Maps are Fortran (ndf, ncell_2d), 1-based; the face selectors
 * (get_face_selector_ew / _ns: 1 or 2 per W3-2D dof) choose which cells copy
 * their E and N faces, as in the reference. */
typedef struct lfx_w2_split lfx_w2_split;
int lfx_w2_split_create(lfx_ctx* ctx, int32_t ncell_2d, int32_t nlayers, const int32_t* map_w2,
                        const int32_t* map_w2h, const int32_t* map_w2v, const int32_t* map_w3_2d,
                        int64_t undf_w3_2d, const int32_t* face_selector_ew,
                        const int32_t* face_selector_ns, lfx_w2_split** out);
/* uv, w from uvw (split_w2_field) */
int lfx_w2_split_field(lfx_w2_split* s, const lfx_vec* uvw, lfx_vec* uv, lfx_vec* w);
/* uvw from uv, w (combine_w2_field) */
int lfx_w2_combine_field(lfx_w2_split* s, const lfx_vec* uv, const lfx_vec* w, lfx_vec* uvw);
int lfx_w2_split_destroy(lfx_w2_split* s);

/* ------------------------------------------------------------------ preconditioners
 * apply writes y = P^{-1} x (sci_preconditioner_mod.f90:19-38). */
int lfx_null_prec_create(lfx_ctx* ctx, lfx_prec** out);                 /* y = x        */
int lfx_diag_prec_create(lfx_ctx* ctx, const lfx_vec* diag, lfx_prec** out); /* y = x/diag */
/* Column-tridiagonal (Thomas, columnwise_op_appinv_kernel_mod.F90:77-145) on
 * the rows the CMA covers, y = x / diag on every other row (diag may be NULL
 * if the CMA covers all rows). The factorisation is done once, in FP64.
 * precision selects the vectors it will be applied to. */
int lfx_cma_prec_create(lfx_ctx* ctx, const lfx_cma* cma, const lfx_vec* diag,
                        int32_t precision, lfx_prec** out);
int lfx_prec_apply(lfx_prec* p, const lfx_vec* x, lfx_vec* y);
int lfx_prec_destroy(lfx_prec* p);

/* ------------------------------------------------------------------ solvers
 * Device-resident Krylov solves (sci_iterative_solver_mod.f90): every
 * scalar recurrence stays on the device; the host only launches work and
 * polls a convergence flag. */
enum {
  LFX_SOLVER_CG = 1,        /* cg_solve       :495-592  */
  LFX_SOLVER_BICGSTAB = 2,  /* bicgstab_solve :645-779  */
  LFX_SOLVER_GMRES = 3,     /* gmres_solve    :830-1003 */
  /* Flexible GMRES and GCR run their vector operations, applies and
   * preconditioners on the device in the reference's order, with the short
   * scalar recurrences on the host (each inner product returns to the host,
   * as in the reference). As in the reference, FGMRES starts its residual
   * from b (it assumes a zero initial guess) and adds the correction to x;
   * GCR starts from dx = P b, measures against ||b||, and reports
   * non-convergence (with monitoring on) as LFX_NOT_CONVERGED whatever
   * fail_on_non_converged says, as the reference logs it as an error in both
   * branches. iterations = restart cycles; GCR's inner_iterations = the inner
   * step of the last check. */
  LFX_SOLVER_FGMRES = 4,    /* fgmres_solve   :1055-1237 */
  LFX_SOLVER_GCR = 5,       /* gcr_solve      :1288-1408 */
  /* made by their own constructors below */
  LFX_SOLVER_PRECONDITION_ONLY = 6, /* precondition_only_solve :1664-1694 */
  LFX_SOLVER_JACOBI = 7,            /* jacobi_solve            :1745-1815 */
  LFX_SOLVER_CHEBYSHEV = 8          /* chebyshev_solve         :1868-1940 */
};

typedef struct {
  double r_tol;                  /* relative tolerance                       */
  double a_tol;                  /* absolute tolerance                       */
  int32_t max_iter;              /* iterations (CG/BiCGStab) or cycles (GMRES) */
  int32_t gcrk;                  /* GMRES / FGMRES / GCR restart length      */
  int32_t monitor_convergence;   /* 0: run exactly max_iter, as the reference */
  int32_t fail_on_non_converged; /* 1: return LFX_NOT_CONVERGED              */
} lfx_solver_cfg;

typedef struct {
  int32_t iterations;   /* iterations (CG/BiCGStab) or restart cycles (GMRES) */
  int32_t converged;
  double initial_norm;  /* ||b - A x0||                                       */
  double final_norm;    /* last monitored residual norm                       */
  double final_rel;     /* last monitored relative residual                   */
  int32_t applies;      /* operator applications                              */
  int32_t status;       /* lfx_status of the solve                            */
  int32_t outer_iterations; /* refinement steps (refined solver only)         */
  int32_t inner_iterations; /* total inner iterations (refined solver only)   */
} lfx_solve_info;

int lfx_solver_create(lfx_ctx* ctx, int32_t kind, lfx_op* op, lfx_prec* prec,
                      const lfx_solver_cfg* cfg, lfx_solver** out);
/* x: initial guess on entry, solution on exit; b unchanged */
int lfx_solver_apply(lfx_solver* s, lfx_vec* x, const lfx_vec* b, lfx_solve_info* info);
int lfx_solver_destroy(lfx_solver* s);
/* precondition_only_constructor (:1642-1657): x = P b; with monitoring the
 * info reports ||b - A x|| against ||b||. */
int lfx_precondition_only_solver_create(lfx_ctx* ctx, lfx_op* op, lfx_prec* prec,
                                        int32_t monitor_convergence, lfx_solver** out);
/* jacobi_constructor (:1715-1739): x += -rho_relax P (A x - b), converged when
 * ||r||/||r_1|| <= r_tol or ||r|| <= a_tol (checked before each update);
 * iterations = residual checks made. */
int lfx_jacobi_solver_create(lfx_ctx* ctx, lfx_op* op, lfx_prec* prec, double r_tol, double a_tol,
                             int32_t max_iter, int32_t monitor_convergence,
                             int32_t fail_on_non_converged, double rho_relax, lfx_solver** out);
/* chebyshev_constructor (:1836-1862): exactly max_iter steps from x = 0 (the
 * initial guess is ignored, as in the reference) for eigenvalue bounds
 * [lmin, lmax] of P A; with monitoring the info reports ||A x - b|| /
 * max(1, ||b||). As in the reference, fail_on_non_converged with monitoring
 * makes every solve return LFX_NOT_CONVERGED (it logs its result as an
 * error). */
int lfx_chebyshev_solver_create(lfx_ctx* ctx, lfx_op* op, lfx_prec* prec, double r_tol,
                                double a_tol, int32_t max_iter, int32_t monitor_convergence,
                                int32_t fail_on_non_converged, double lmin, double lmax,
                                lfx_solver** out);
/* change r_tol / a_tol for the next solves (keeps the solver's CUDA graphs) */
int lfx_solver_set_tolerance(lfx_solver* s, double r_tol, double a_tol);

/* Mixed-precision solve with FP64 iterative refinement: the residual
 * b - A x and the solution update stay FP64 (op64, FP64 vectors); each
 * correction comes from `inner` (typically an FP32 GMRES on an FP32 copy of
 * the operator) solved to inner_rtol. Converged when ||b - A x||/||b - A x0||
 * <= cfg->r_tol, with at most cfg->max_iter refinement steps. When `inner`
 * is an FP32 GMRES, each refinement step runs one of its restart cycles
 * (stopping early once the cycle's own estimate reaches inner_rtol), queued
 * with the step's FP64 residual so that a step costs one host round trip;
 * the cycle forms no FP32 residual of its own. Other inner solvers run their
 * full solve per step. */
int lfx_refined_solver_create(lfx_ctx* ctx, lfx_op* op64, lfx_solver* inner,
                              double inner_rtol, const lfx_solver_cfg* cfg,
                              lfx_solver** out);

/* Per-kernel device timing of the operator apply: when enabled, CUDA events
 * bracket every LMA apply launched on this context; lfx_ctx_apply_timing
 * returns the count and total milliseconds of the applies of the given
 * storage precision (0 = all) accumulated since the last reset. */
int lfx_ctx_enable_apply_timing(lfx_ctx* ctx, int32_t enable);
int lfx_ctx_apply_timing(lfx_ctx* ctx, int32_t precision, int64_t* launches, double* total_ms,
                         int32_t reset);
/* number of kernels this context has launched so far */
int64_t lfx_ctx_launch_count(const lfx_ctx* ctx);
/* LMA apply kernel for every operator of the context: -1 = each operator's
 * autotuned choice, else the register gather with prefetched descriptors
 * where it fits, else the register gather (default); 0 = force the
 * bulk-copy pipeline; 1 = force the register gather; 3 = force the register
 * gather with prefetched descriptors (the register gather where the operator
 * does not fit it); 4 = force the copy-staged pipeline; 5 = force the cell
 * scatter where the operator fits it; 6 = force the cell scatter as one
 * persistent (cooperative) launch over the colours where the operator fits
 * it (ndf 6 or 8, at most 31 levels and 16 colours). All give bit-identical
 * results. */
int lfx_ctx_set_apply_kernel(lfx_ctx* ctx, int32_t which);
/* LFX_TIMEOUT if a kernel's bounded device-side wait ran out since the last
 * check (the kernel then skipped its work); synchronises the stream */
int lfx_ctx_check_device_error(lfx_ctx* ctx);

/* ------------------------------------------------------------------ batched solves
 * Continuous batching of many independent SPD solves (no counterpart in the
 * reference, which solves one system per call: each slot replaces one
 * cg_solve of sci_iterative_solver_mod.f90:495-592). Each slot runs
 * preconditioned CG in FP32 with the solution accumulated in FP64 and
 * reliable updates: the true residual b - A x is recomputed with the FP64
 * operator whenever the FP32 residual has dropped by 1e-3 since the last one,
 * and a slot converges only when ||b - A x|| / ||b - A x0|| <= tol.
 * One CUDA graph replay is ONE persistent (cooperative) kernel launch that
 * runs `iters_per_launch` super-iterations of every admitted slot, phase by
 * phase with grid-wide barriers; the operator apply is the reference's
 * coloured cell loop over each slot's packed FP32 local matrices (the FP64
 * ones for the true residuals). A slot's result does not depend on the other
 * slots or on the launch shape. Admission allocates the slot's Krylov state
 * (28 bytes per dof) from the device's stream-ordered memory pool and is
 * refused (LFX_OUT_OF_MEMORY) while it would leave less than reserve_bytes of
 * device memory free, or when all max_slots slots are taken. Every slot of a
 * batch has ndf 8 (W0) or 6 (W2) dofs per cell. A bounded wait that runs out
 * returns LFX_TIMEOUT from lfx_batch_step; the batch must then be destroyed. */
typedef struct lfx_batch lfx_batch;
int lfx_batch_create(lfx_ctx* ctx, int32_t ndf, int32_t max_slots, int64_t reserve_bytes,
                     int32_t iters_per_launch, lfx_batch** out);
int lfx_batch_destroy(lfx_batch* b);
/* op64/op32: FP64 and FP32 copies of one symmetric operator on one dofmap
 * (lfx_lma_create_like), which therefore carry the packed cell-scatter
 * copies; prec32: its FP32 Jacobi or column preconditioner; b, x: FP64
 * vectors kept alive, with the operators, until the slot is retired (x:
 * initial guess in, solution out). */
int lfx_batch_admit(lfx_batch* b, lfx_op* op64, lfx_op* op32, lfx_prec* prec32, const lfx_vec* rhs,
                    lfx_vec* x, double tol, int32_t max_iter, int64_t tag, int32_t* slot);
/* one graph replay (one kernel launch) for every slot; *ndone = slots done
 * and not yet retired */
int lfx_batch_step(lfx_batch* b, int32_t* ndone);
/* phase: 0 empty, 1 starting, 2 iterating, 3 done; info as lfx_solve_info
 * (iterations = CG iterations, outer_iterations = true residuals taken) */
int lfx_batch_slot_info(const lfx_batch* b, int32_t slot, int32_t* phase, int64_t* tag,
                        lfx_solve_info* info);
int lfx_batch_retire(lfx_batch* b, int32_t slot);
/* launch shape of the persistent kernel: cell columns per apply work item
 * (the colour block one warp takes), blocks per SM, and the bytes of vectors of one L2 group
 * of slots (slots of a group run their colour phases together, so their
 * vectors stay in L2 across the colours) */
typedef struct {
  int32_t cells_per_item;
  int32_t blocks_per_sm;
  int32_t grid;
  int32_t cooperative;      /* 1: cooperative launch inside the graph      */
  int64_t group_bytes;
  int64_t replays;          /* graph replays (kernel launches) so far       */
  float us_per_iteration;   /* the tuner's best time per super-iteration   */
} lfx_batch_tuning;
/* Batch autotuner: times one replay of `iters` super-iterations per candidate
 * shape on the admitted slots (these replays advance the solves, which do not
 * depend on the shape) -- blocks per SM, then 1/2/4/8 columns per item,
 * then L2 groups of a quarter, half, all of L2 or one group -- and keeps the
 * fastest. A trial with no running slot measures nothing and is not chosen
 * (step the batch once after admitting, so the slots are running). */
int lfx_batch_autotune(lfx_batch* b, int32_t iters, lfx_batch_tuning* out);
int lfx_batch_get_tuning(const lfx_batch* b, lfx_batch_tuning* out);
/* pin a launch shape (cells_per_item 1 to 8) */
int lfx_batch_set_tuning(lfx_batch* b, int32_t cells_per_item, int32_t blocks_per_sm,
                         int64_t group_bytes);
/* upper bound in seconds of one grid-barrier wait (default 2) */
int lfx_batch_set_wait_limit(lfx_batch* b, double seconds);

/* ------------------------------------------------------------------ many right-hand sides
 * One operator applied to, and solved for, nrhs right-hand sides at once (no
 * counterpart in the reference, whose solvers take one field_vector_type).
 * The per-cell product becomes an (nrhs x 8) by (8 x 8) small GEMM on the
 * tensor cores, in TF32 or BF16 with FP32 accumulation. Operators with the
 * lowest-order nodal (W0) dofmap only: ndf = 8, map_to == map_from, dofs 4..7
 * one level above dofs 0..3. */
typedef struct lfx_mrhs lfx_mrhs;
enum { LFX_MRHS_TF32 = 1, LFX_MRHS_BF16 = 2 };
/* From an FP64 (or FP32) LMA operator: its matrices rounded to `kind`, the
 * cell columns split into patches of about cells_per_patch (0: 16). nrhs is
 * 16, 32 or 64. */
int lfx_mrhs_create(const lfx_op* op, int32_t kind, int32_t nrhs, int32_t cells_per_patch,
                    lfx_mrhs** out);
int lfx_mrhs_destroy(lfx_mrhs* m);
/* patches, cell levels computed per apply (halo cells of two patches count
 * twice), most vertex columns one patch owns, most colours in one patch, and
 * the bytes of the rounded matrices */
int lfx_mrhs_info(const lfx_mrhs* m, int32_t* npatch, int64_t* cell_levels, int32_t* max_owned,
                  int32_t* max_colours, int64_t* matrix_bytes);
/* y = A x for device arrays x, y of undf x nrhs FP32 values, dof-major
 * (element (dof, rhs) at dof * nrhs + rhs); x and y must differ */
int lfx_mrhs_apply(lfx_mrhs* m, const float* x, float* y);
/* mean time of one apply over reps applies (after one untimed), microseconds */
int lfx_mrhs_time_apply(lfx_mrhs* m, const float* x, float* y, int32_t reps, float* us);
/* apply autotuner: times 2, 4 and 8 levels per shared-memory block (those
 * that fit) over reps applies and keeps the fastest; outputs (nullable) the
 * choice and its time per apply in microseconds */
int lfx_mrhs_autotune(lfx_mrhs* m, int32_t reps, int32_t* levels_per_block, float* us);
enum { LFX_MRHS_PER_RHS_CG = 0, LFX_MRHS_BLOCK_CG = 1 };
typedef struct {
  double r_tol;      /* per right-hand side: ||b - A x|| <= r_tol ||b - A x0|| */
  double inner_tol;  /* each inner FP32 solve reduces its residual by this */
  int32_t max_outer; /* refinement steps, at most */
  int32_t max_inner; /* iterations of one inner solve, at most */
  /* inner solver: LFX_MRHS_PER_RHS_CG, CG on every right-hand side with its
   * own step lengths; LFX_MRHS_BLOCK_CG, breakdown-free block CG over the
   * 64 right-hand sides together (64 only): one search space for all of
   * them, directions that become dependent dropped by a pivoted Cholesky
   * orthonormalisation (the block Krylov idea of block_gcr_solve,
   * sci_iterative_solver_mod.f90:1461-1628, in CG form) */
  int32_t method;
} lfx_mrhs_cfg;
/* FP64 iterative refinement around an FP32 Jacobi-preconditioned CG run on
 * all right-hand sides together (cfg->method: each with its own step
 * lengths, or one block CG), with the tensor-core apply. op64: the FP64 operator (residuals); diag: its FP64
 * diagonal (lfx_lma_diagonal). b, x: device arrays of nrhs FP64 vectors,
 * right-hand side r at b + r * ld (x: initial guess in, solution out). info:
 * nrhs entries; iterations = inner iterations of that right-hand side,
 * outer_iterations = refinement steps it took part in. */
int lfx_mrhs_solve(lfx_mrhs* m, lfx_op* op64, const lfx_vec* diag, const double* b, double* x,
                   int64_t ld, const lfx_mrhs_cfg* cfg, lfx_solve_info* info);
/* Where the block CG's Gram products U^T V (n x 64 blocks) run: tensor = 1
 * on the tcgen05 tensor cores, each FP32 value split into two TF32 parts
 * (three MMAs per step, about FP32 accuracy, FP32 accumulation in tensor
 * memory per block, FP64 across blocks); 0 (default) on the FP32 cores. */
int lfx_mrhs_set_gram(lfx_mrhs* m, int32_t tensor);
/* One Gram product with either path: out (device, nv x 64 x 64 FP64,
 * [v][i][j]) = sum over rows of U[row][i] V_v[row][j], for device arrays U,
 * V0, V1 of undf x 64 FP32 values, dof-major. LFX_TIMEOUT if a bounded
 * tensor-core wait ran out. */
int lfx_mrhs_gram(lfx_mrhs* m, const float* U, const float* V0, const float* V1, int32_t nv,
                  int32_t tensor, double* out);

/* ------------------------------------------------------------------ no allocation
 * Allocation-free inner product (no counterpart in the reference): for
 * callers that cannot allocate device memory where they need a dot product --
 * device memory owned by another runtime's pool, or a loop that must not take
 * cudaMalloc's implicit synchronisation. x, y (n FP64 values) and result (one FP64 value) are device
 * pointers owned by the caller; the work is queued on `stream` (a
 * cudaStream_t, NULL for the default stream) and *result is valid once it
 * completes. The reduction scratch is a fixed array built into the library
 * (about 64 KiB on every GPU that loads it, held until exit), so n is limited
 * to lfx_dot_noalloc_max_n() (16 Mi) values; larger n is rejected with
 * LFX_INVALID_ARGUMENT and a message from lfx_noalloc_last_error(). The first
 * call on each device looks up the array's device address; make that first
 * call before any stream capture. A device reset (cudaDeviceReset) may move
 * the array; do not call this again in a process after one. n = 0 gives 0.0.
 * All calls share the array: calls that
 * overlap on the GPU (different streams, or concurrent host threads) race and
 * must be serialised by the caller. The result equals lfx_vec_dot's bit for
 * bit. */
int lfx_dot_noalloc(const double* x, const double* y, int64_t n, double* result, void* stream);
int64_t lfx_dot_noalloc_max_n(void);
const char* lfx_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
