/*
 * oracle.c -- CPU restatement (FP64) of the Krylov-solve hot path.
 * TEST INFRASTRUCTURE ONLY: the checker and the timed CPU baseline, never the
 * product. See oracle.h for the reference file:line each function follows.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_order = 0;
void or_set_reduction_order(int mode) { g_order = mode; }
void or_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* constants_mod.F90:167, EPS = epsilon(1.0_r_def) */
#define EPS_RDEF DBL_EPSILON

/* ------------------------------------------------------------------------ */
/* Global sums. The reference sums per OpenMP thread and then across ranks
 * (sci_psykal_light_mod.f90:72-214, scalar_mod.t90:82-93), so its order
 * depends on the thread count. The oracle fixes one order, the one the
 * device reduction uses:
 *   chunk j = elements [2048 j, 2048 j + 2048); lane t = 0..255 of the chunk
 *   accumulates, in this order, elements 256 m + t (m = 0..7) with
 *   acc = fma(x, y, acc); the 32 lanes of each warp are combined by a xor
 *   butterfly (offsets 16, 8, 4, 2, 1); the 8 warp sums are added left to
 *   right. The chunk partials are then reduced the same way, lane t adding
 *   partials t, t+256, t+512, ... in order.                                 */
/* ------------------------------------------------------------------------ */
#define RCHUNK 2048
#define RTHREADS 256

static double block_combine(double* lane /* [256], destroyed */) {
  double total = 0.0;
  for (int w = 0; w < RTHREADS / 32; ++w) {
    double* v = lane + 32 * w;
    for (int off = 16; off >= 1; off >>= 1) {
      double t[32];
      for (int l = 0; l < 32; ++l) t[l] = v[l] + v[l ^ off];
      memcpy(v, t, sizeof t);
    }
    total = (w == 0) ? v[0] : total + v[0];
  }
  return total;
}

static double chunk_dot(const double* x, const double* y, int64_t n, int64_t j) {
  double lane[RTHREADS];
  for (int t = 0; t < RTHREADS; ++t) {
    double acc = 0.0;
    for (int m = 0; m < 8; ++m) {
      int64_t i = j * RCHUNK + 256 * m + t;
      if (i < n) acc = fma(x[i], y[i], acc);
    }
    lane[t] = acc;
  }
  return block_combine(lane);
}

static double reduce_partials(const double* p, int64_t np) {
  double lane[RTHREADS];
  for (int t = 0; t < RTHREADS; ++t) {
    double acc = 0.0;
    for (int64_t i = t; i < np; i += RTHREADS) acc = acc + p[i];
    lane[t] = acc;
  }
  return block_combine(lane);
}

double or_dot(const double* x, const double* y, int64_t n) {
  if (g_order == 1) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s = fma(x[i], y[i], s);
    return s;
  }
  int64_t nc = (n + RCHUNK - 1) / RCHUNK;
  if (nc == 0) return 0.0;
  double* part = (double*)malloc(sizeof(double) * nc);
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < nc; ++j) part[j] = chunk_dot(x, y, n, j);
  double s = reduce_partials(part, nc);
  free(part);
  return s;
}

double or_sumsq(const double* x, int64_t n) { return or_dot(x, x, n); }

/* ------------------------------------------------------------------------ */
/* PSyclone builtins (semantics; their source is generated by PSyclone)     */
/* ------------------------------------------------------------------------ */
void or_setval_c(double* x, double c, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) x[i] = c;
}
void or_setval_x(double* y, const double* x, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) y[i] = x[i];
}
void or_inc_x_plus_by(double* x, double b, const double* y, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) x[i] = fma(b, y[i], x[i]);
}
void or_inc_ax_plus_y(double a, double* x, const double* y, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) x[i] = fma(a, x[i], y[i]);
}
void or_ax_plus_by(double* z, double a, const double* x, double b, const double* y,
                   int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) z[i] = fma(a, x[i], b * y[i]);
}
void or_inc_a_times_x(double a, double* x, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) x[i] = a * x[i];
}
void or_x_divideby_y(double* z, const double* x, const double* y, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) z[i] = x[i] / y[i];
}

/* ------------------------------------------------------------------------ */
/* kernels                                                                  */
/* ------------------------------------------------------------------------ */
#define MAT(m, ik, i, j, ndf1, nc3) \
  (m)[(int64_t)(ik) + (int64_t)(nc3) * ((int64_t)(i) + (int64_t)(ndf1) * (j))]

/* matrix_vector_kernel_mod.F90:130-138: for df2, df: lhs(i1:i1+nl) += M*x */
void or_matrix_vector_code(int32_t cell, int32_t nlayers, double* lhs, const double* x,
                           int64_t ncell_3d, const double* matrix, int32_t ndf1,
                           const int32_t* map1, int32_t ndf2, const int32_t* map2) {
  int64_t ik = (int64_t)(cell - 1) * nlayers;
  for (int32_t df2 = 0; df2 < ndf2; ++df2) {
    int64_t i2 = map2[df2] - 1;
    for (int32_t df = 0; df < ndf1; ++df) {
      int64_t i1 = map1[df] - 1;
      for (int32_t k = 0; k < nlayers; ++k)
        lhs[i1 + k] = fma(MAT(matrix, ik + k, df, df2, ndf1, ncell_3d), x[i2 + k], lhs[i1 + k]);
    }
  }
}

/* transpose_matrix_vector_kernel_mod.F90:128-144: per layer, lhs_e = M^T x_e,
 * then lhs += lhs_e; matrix is (ncell_3d, ndf2, ndf1). matmul sums over df2. */
void or_transpose_matrix_vector_code(int32_t cell, int32_t nlayers, double* lhs,
                                     const double* x, int64_t ncell_3d, const double* matrix,
                                     int32_t ndf1, const int32_t* map1, int32_t ndf2,
                                     const int32_t* map2) {
  for (int32_t k = 0; k < nlayers; ++k) {
    int64_t ik = (int64_t)(cell - 1) * nlayers + k;
    for (int32_t df = 0; df < ndf1; ++df) {
      double s = 0.0;
      for (int32_t j = 0; j < ndf2; ++j)
        s = fma(MAT(matrix, ik, j, df, ndf2, ncell_3d), x[map2[j] - 1 + k], s);
      lhs[map1[df] - 1 + k] = lhs[map1[df] - 1 + k] + s;
    }
  }
}

/* dg_matrix_vector_kernel_mod.F90:135-154: zero the cell's lhs, then as
 * matrix_vector_code (df2 outer, df1 inner). */
void or_dg_matrix_vector_code(int32_t cell, int32_t nlayers, double* lhs, const double* x,
                              int64_t ncell_3d, const double* matrix, int32_t ndf1,
                              const int32_t* map1, int32_t ndf2, const int32_t* map2) {
  for (int32_t df = 0; df < ndf1; ++df)
    for (int32_t k = 0; k < nlayers; ++k) lhs[map1[df] - 1 + k] = 0.0;
  or_matrix_vector_code(cell, nlayers, lhs, x, ncell_3d, matrix, ndf1, map1, ndf2, map2);
}

/* sci_operator_algebra_kernel_mod.F90:92-119 (operator_x_plus_ay_kernel_code):
 *   do k = 0, nlayers - 1
 *     ik = k + 1 + (cell-1)*nlayers
 *     x_plus_ay(ik,:,:) = x(ik,:,:) + a*y(ik,:,:)
 * the a*y + x of each entry is one fma, as everywhere in this restatement */
void or_operator_x_plus_ay_code(int32_t cell, int32_t nlayers, int64_t ncell_3d, double* x_plus_ay,
                                const double* x, double a, const double* y, int32_t ndf1,
                                int32_t ndf2) {
  for (int32_t k = 0; k < nlayers; ++k) {
    const int64_t ik = k + (int64_t)(cell - 1) * nlayers; /* 0-based */
    for (int32_t j = 0; j < ndf2; ++j)
      for (int32_t i = 0; i < ndf1; ++i) {
        const int64_t e = ik + ncell_3d * (i + (int64_t)ndf1 * j);
        x_plus_ay[e] = fma(a, y[e], x[e]);
      }
  }
}

/* sci_tri_solve_kernel_mod.f90:125-154 */
void or_tri_solve_code(int32_t nlayers, double* y, const double* x, const double* tri_0,
                       const double* tri_plus, const double* tri_minus, const int32_t* map) {
  double* xn = (double*)malloc(sizeof(double) * nlayers);
  double* tp = (double*)malloc(sizeof(double) * nlayers);
  int64_t ij = map[0] - 1;
  double denom = 1.0 / tri_0[ij];
  tp[0] = tri_plus[ij] * denom;
  xn[0] = x[ij] * denom;
  for (int32_t k = 1; k < nlayers; ++k) {
    denom = 1.0 / fma(-tri_minus[ij + k], tp[k - 1], tri_0[ij + k]);
    tp[k] = tri_plus[ij + k] * denom;
    xn[k] = fma(-tri_minus[ij + k], xn[k - 1], x[ij + k]) * denom;
  }
  y[ij + nlayers - 1] = xn[nlayers - 1];
  for (int32_t k = nlayers - 2; k >= 0; --k) y[ij + k] = fma(-tp[k], y[ij + k + 1], xn[k]);
  free(xn);
  free(tp);
}

static int32_t ceil_div_r(int32_t a, int32_t b) { return (int32_t)ceil((double)a / (double)b); }
static int32_t floor_div_r(int32_t a, int32_t b) { return (int32_t)floor((double)a / (double)b); }

/* sci_columnwise_op_asm_kernel_mod.F90:107-126 */
void or_columnwise_op_asm_code(int32_t cell, int32_t nlayers, int32_t ncell_2d,
                               int64_t ncell_3d, const double* local_stencil,
                               double* cm, int32_t nrow, int32_t ncol, int32_t bw,
                               int32_t alpha, int32_t beta, int32_t gamma_m, int32_t gamma_p,
                               int32_t ndf_to, const int32_t* cbd_to, int32_t ndf_from,
                               const int32_t* cbd_from) {
  (void)ncell_2d;
  (void)ncol;
  (void)gamma_m;
  double* col = cm + (int64_t)(cell - 1) * bw * nrow;
  memset(col, 0, sizeof(double) * bw * nrow);
  for (int32_t k = 1; k <= nlayers; ++k) {
    int64_t ik = (int64_t)(cell - 1) * nlayers + k - 1;
    for (int32_t df1 = 1; df1 <= ndf_to; ++df1) {
      int32_t i = cbd_to[(df1 - 1) + ndf_to * (k - 1)];
      int32_t jm = ceil_div_r(alpha * i - gamma_p, beta);
      for (int32_t df2 = 1; df2 <= ndf_from; ++df2) {
        int32_t j = cbd_from[(df2 - 1) + ndf_from * (k - 1)];
        double* e = &col[(j - jm) + (int64_t)bw * (i - 1)];
        *e = *e + MAT(local_stencil, ik, df1 - 1, df2 - 1, ndf_to, ncell_3d);
      }
    }
  }
}

/* sci_columnwise_op_app_kernel_mod.F90:109-122 */
void or_columnwise_op_app_code(int32_t cell, double* lhs, const double* x, const double* cm,
                               int32_t nrow, int32_t ncol, int32_t bw, int32_t alpha,
                               int32_t beta, int32_t gamma_m, int32_t gamma_p,
                               const int32_t* map1, const int32_t* ind_to,
                               const int32_t* map2, const int32_t* ind_from) {
  const double* col = cm + (int64_t)(cell - 1) * bw * nrow;
  for (int32_t i = 1; i <= nrow; ++i) {
    int64_t mu_i = map1[0] + ind_to[i - 1] - 1 - 1;
    int32_t jm = ceil_div_r(alpha * i - gamma_p, beta);
    int32_t jp = floor_div_r(alpha * i + gamma_m, beta);
    for (int32_t j = (jm > 1 ? jm : 1); j <= (jp < ncol ? jp : ncol); ++j) {
      int64_t mu_j = map2[0] + ind_from[j - 1] - 1 - 1;
      lhs[mu_i] = fma(col[(j - jm) + (int64_t)bw * (i - 1)], x[mu_j], lhs[mu_i]);
    }
  }
}

/* sci_columnwise_op_appinv_kernel_mod.F90:116-143 (writes, not increments) */
void or_columnwise_op_appinv_code(int32_t cell, double* lhs, const double* x,
                                  const double* cm, int32_t nrow, int32_t bw,
                                  const int32_t* map, const int32_t* ind) {
  const double* col = cm + (int64_t)(cell - 1) * bw * nrow;
#define B(r, i) col[(r) - 1 + (int64_t)bw * ((i) - 1)]
  double cp[512], dp[512];
  double* c_prime = nrow <= 512 ? cp : (double*)malloc(sizeof(double) * nrow);
  double* d_prime = nrow <= 512 ? dp : (double*)malloc(sizeof(double) * nrow);
  for (int32_t i = 1; i <= nrow; ++i) {
    int64_t mu = map[0] + ind[i - 1] - 1 - 1;
    double inv_denom;
    if (i == 1) {
      inv_denom = 1.0 / B(2, i);
      c_prime[0] = inv_denom * B(3, i);
      d_prime[0] = inv_denom * x[mu];
    } else {
      inv_denom = 1.0 / fma(-B(1, i), c_prime[i - 2], B(2, i));
      if (i < nrow) c_prime[i - 1] = inv_denom * B(3, i);
      d_prime[i - 1] = inv_denom * fma(-B(1, i), d_prime[i - 2], x[mu]);
    }
  }
  for (int32_t i = nrow; i >= 1; --i) {
    int64_t mu = map[0] + ind[i - 1] - 1 - 1;
    if (i < nrow) d_prime[i - 1] = fma(-c_prime[i - 1], d_prime[i], d_prime[i - 1]);
    lhs[mu] = d_prime[i - 1];
  }
#undef B
  if (c_prime != cp) free(c_prime);
  if (d_prime != dp) free(d_prime);
}

/* ------------------------------------------------------------------------ */
/* operator / preconditioner objects                                        */
/* ------------------------------------------------------------------------ */
struct or_op {
  int32_t ncell_2d, nlayers, ndf_to, ndf_from, ncolours, maxc, mode;
  const int32_t *map_to, *map_from, *ncells_per_colour, *cells_in_colour;
  int64_t undf_to, undf_from;
  const double* stencil;
};

/* columnwise_op_mul_kernel_code, sci_columnwise_op_mul_kernel_mod.F90 */
#define BAND(M, b, i, bw, nrow, cell) (M)[((b) - 1) + (int64_t)(bw) * ((i) - 1) + (int64_t)(bw) * (nrow) * ((cell) - 1)]
void or_columnwise_op_mul_code(int32_t cell, int32_t ncell_2d, const double* A, int32_t nrow_A,
                               int32_t ncol_A, int32_t bw_A, int32_t alpha_A, int32_t beta_A,
                               int32_t gm_A, int32_t gp_A, const double* B, int32_t nrow_B,
                               int32_t ncol_B, int32_t bw_B, int32_t alpha_B, int32_t beta_B,
                               int32_t gm_B, int32_t gp_B, double* C, int32_t nrow_C,
                               int32_t ncol_C, int32_t bw_C, int32_t alpha_C, int32_t beta_C,
                               int32_t gm_C, int32_t gp_C) {
  (void)ncell_2d;
  (void)ncol_B;
  (void)gm_C;
  for (int32_t i = 1; i <= nrow_C; ++i) {
    const int32_t jmA = ceil_div_r(alpha_A * i - gp_A, beta_A);
    const int32_t jpA = floor_div_r(alpha_A * i + gm_A, beta_A);
    const int32_t jmC = ceil_div_r(alpha_C * i - gp_C, beta_C);
    const int32_t jpC = floor_div_r(alpha_C * i + gm_C, beta_C);
    for (int32_t j = (jmC > 1 ? jmC : 1); j <= (ncol_C < jpC ? ncol_C : jpC); ++j) {
      double e = 0.0;
      for (int32_t l = (jmA > 1 ? jmA : 1); l <= (ncol_A < jpA ? ncol_A : jpA); ++l) {
        const int32_t jmB = ceil_div_r(alpha_B * l - gp_B, beta_B);
        const int32_t jpB = floor_div_r(alpha_B * l + gm_B, beta_B);
        if (jmB <= j && j <= jpB)
          e = fma(BAND(A, l - jmA + 1, i, bw_A, nrow_A, cell),
                  BAND(B, j - jmB + 1, l, bw_B, nrow_B, cell), e);
      }
      BAND(C, j - jmC + 1, i, bw_C, nrow_C, cell) = BAND(C, j - jmC + 1, i, bw_C, nrow_C, cell) + e;
    }
  }
}

/* columnwise_op_scaledadd_kernel_code, sci_columnwise_op_scaledadd_kernel_mod.F90 */
void or_columnwise_op_scaledadd_code(int32_t cell, int32_t ncell_2d, const double* A,
                                     int32_t nrow_A, int32_t ncol_A, int32_t bw_A, int32_t alpha_A,
                                     int32_t beta_A, int32_t gm_A, int32_t gp_A, const double* B,
                                     int32_t nrow_B, int32_t ncol_B, int32_t bw_B, int32_t alpha_B,
                                     int32_t beta_B, int32_t gm_B, int32_t gp_B, double* C,
                                     int32_t nrow_C, int32_t ncol_C, int32_t bw_C, int32_t alpha_C,
                                     int32_t beta_C, int32_t gm_C, int32_t gp_C, double alpha,
                                     double beta) {
  (void)ncell_2d;
  (void)ncol_B;
  (void)ncol_C;
  (void)gm_C;
  for (int64_t q = 0; q < (int64_t)bw_C * nrow_C; ++q) C[q + (int64_t)bw_C * nrow_C * (cell - 1)] = 0.0;
  for (int32_t i = 1; i <= nrow_A; ++i) {
    const int32_t jmA = ceil_div_r(alpha_A * i - gp_A, beta_A);
    const int32_t jpA = floor_div_r(alpha_A * i + gm_A, beta_A);
    const int32_t jmB = ceil_div_r(alpha_B * i - gp_B, beta_B);
    const int32_t jpB = floor_div_r(alpha_B * i + gm_B, beta_B);
    const int32_t jmC = ceil_div_r(alpha_C * i - gp_C, beta_C);
    for (int32_t j = (jmA > 1 ? jmA : 1); j <= (ncol_A < jpA ? ncol_A : jpA); ++j) {
      double* e = &BAND(C, j - jmC + 1, i, bw_C, nrow_C, cell);
      *e = fma(alpha, BAND(A, j - jmA + 1, i, bw_A, nrow_A, cell), *e);
    }
    for (int32_t j = (jmB > 1 ? jmB : 1); j <= (ncol_A < jpB ? ncol_A : jpB); ++j) {
      double* e = &BAND(C, j - jmC + 1, i, bw_C, nrow_C, cell);
      *e = fma(beta, BAND(B, j - jmB + 1, i, bw_B, nrow_B, cell), *e);
    }
  }
}

/* columnwise_op_asm_m2v_lumped_inv_krnl_code, ..._asm_m2v_lumped_inv_krnl_mod.F90:74-132 */
void or_columnwise_op_asm_m2v_lumped_inv_code(int32_t cell, int32_t nlayers, int32_t ncell_2d,
                                              int32_t ncell_3d, const double* local_stencil,
                                              double* C, int32_t nrow, int32_t bw, int32_t ndf,
                                              const int32_t* column_banded_dofmap) {
  (void)ncell_2d;
  double* col = C + (int64_t)bw * nrow * (cell - 1);
  for (int64_t q = 0; q < (int64_t)bw * nrow; ++q) col[q] = 0.0;
  for (int32_t k = 1; k <= nlayers; ++k) {
    const int64_t ik = (int64_t)(cell - 1) * nlayers + k;
    for (int32_t df1 = 1; df1 <= ndf; ++df1) {
      const int32_t i = column_banded_dofmap[(df1 - 1) + (int64_t)ndf * (k - 1)];
      col[(int64_t)bw * (i - 1)] = col[(int64_t)bw * (i - 1)] +
          local_stencil[(ik - 1) + (int64_t)ncell_3d * ((df1 - 1) + (int64_t)ndf * (df1 - 1))];
    }
  }
  for (int64_t q = 0; q < (int64_t)bw * nrow; ++q)
    if (col[q] != 0.0) col[q] = 1.0 / col[q];
}

/* columnwise_op_asm_diag_hmht_kernel_code, ..._asm_diag_hmht_kernel_mod.F90:78-151 */
void or_columnwise_op_asm_diag_hmht_code(int32_t cell, int32_t nlayers, int32_t ncell_2d,
                                         int32_t ncell_3d, const double* Dh, const double* M2h,
                                         double* C, int32_t nrow, int32_t bw, int32_t alpha,
                                         int32_t beta, int32_t gamma_m, int32_t gamma_p,
                                         int32_t ndf_w3, const int32_t* column_banded_dofmap,
                                         int32_t ndf_w2h) {
  (void)ncell_2d;
  (void)gamma_m;
  double* col = C + (int64_t)bw * nrow * (cell - 1);
  for (int64_t q = 0; q < (int64_t)bw * nrow; ++q) col[q] = 0.0;
#define DH(ik, a, b) Dh[((ik) - 1) + (int64_t)ncell_3d * (((a) - 1) + (int64_t)ndf_w3 * ((b) - 1))]
#define MH(ik, a, b) M2h[((ik) - 1) + (int64_t)ncell_3d * (((a) - 1) + (int64_t)ndf_w2h * ((b) - 1))]
  for (int32_t k = 1; k <= nlayers; ++k) {
    const int64_t ik = (int64_t)(cell - 1) * nlayers + k;
    for (int32_t df1 = 1; df1 <= ndf_w3; ++df1) {
      const int32_t i = column_banded_dofmap[(df1 - 1) + (int64_t)ndf_w3 * (k - 1)];
      const int32_t jm = ceil_div_r(alpha * i - gamma_p, beta);
      for (int32_t df2 = 1; df2 <= ndf_w3; ++df2) {
        double tmp = 0.0;
        for (int32_t df3 = 1; df3 <= ndf_w2h; ++df3)
          tmp = tmp + DH(ik, df1, df3) * DH(ik, df2, df3) / MH(ik, df3, df3);
        const int32_t j = column_banded_dofmap[(df2 - 1) + (int64_t)ndf_w3 * (k - 1)];
        col[(j - jm) + (int64_t)bw * (i - 1)] = col[(j - jm) + (int64_t)bw * (i - 1)] + tmp;
      }
    }
  }
#undef DH
#undef MH
}
#undef BAND

/* face_selector_code, sci_face_selector_kernel_mod.F90: the first cell (in
 * loop order) whose E (N) face a W2h face is marks it and selects 2 */
void or_face_selector_code(int32_t* face_selector_ew, int32_t* face_selector_ns,
                           int32_t* face_counter, const int32_t* map_w3, const int32_t* map_w2h) {
  const int32_t e = map_w2h[2] - 1, nn = map_w2h[3] - 1, c3 = map_w3[0] - 1;
  if (face_counter[e] == 0) {
    face_selector_ew[c3] = 2;
    face_counter[e] = 1;
  }
  if (face_counter[nn] == 0) {
    face_selector_ns[c3] = 2;
    face_counter[nn] = 1;
  }
}

/* the horizontal faces a cell copies: W, S, then E or N (or both), as
 * split_w2_field_code / combine_w2_field_code select them */
static int32_t hori_faces(const int32_t* ew, const int32_t* ns, const int32_t* map_w3_2d,
                          int32_t* dof3) {
  const int32_t c = map_w3_2d[0] - 1;
  *dof3 = (ns[c] == 2 && ew[c] == 1) ? 4 : 3; /* N = 4, E = 3 */
  return ew[c] + ns[c];
}

/* split_w2_field_code_r_double, split_w2_field_kernel_mod.F90 (lowest order) */
void or_split_w2_field_code(int32_t nlayers, double* uv, double* w, const double* uvw,
                            const int32_t* face_selector_ew, const int32_t* face_selector_ns,
                            const int32_t* map_w2h, const int32_t* map_w2v, const int32_t* map_w2,
                            const int32_t* map_w3_2d) {
  int32_t dof3;
  const int32_t todo = hori_faces(face_selector_ew, face_selector_ns, map_w3_2d, &dof3);
  for (int32_t j = 1; j <= todo; ++j) {
    const int32_t df = (j == 3) ? dof3 : j;
    for (int32_t k = 0; k <= nlayers - 1; ++k) uv[map_w2h[df - 1] - 1 + k] = uvw[map_w2[df - 1] - 1 + k];
  }
  for (int32_t k = 0; k <= nlayers; ++k) w[map_w2v[0] - 1 + k] = uvw[map_w2[4] - 1 + k];
}

/* combine_w2_field_code_r_double, combine_w2_field_kernel_mod.F90 (lowest order) */
void or_combine_w2_field_code(int32_t nlayers, double* uvw, const double* uv, const double* w,
                              const int32_t* face_selector_ew, const int32_t* face_selector_ns,
                              const int32_t* map_w2, const int32_t* map_w2h,
                              const int32_t* map_w2v, const int32_t* map_w3_2d) {
  int32_t dof3;
  const int32_t todo = hori_faces(face_selector_ew, face_selector_ns, map_w3_2d, &dof3);
  for (int32_t j = 1; j <= todo; ++j) {
    const int32_t df = (j == 3) ? dof3 : j;
    for (int32_t k = 0; k <= nlayers - 1; ++k) uvw[map_w2[df - 1] - 1 + k] = uv[map_w2h[df - 1] - 1 + k];
  }
  for (int32_t k = 0; k <= nlayers; ++k) uvw[map_w2[4] - 1 + k] = w[map_w2v[0] - 1 + k];
}

or_op* or_lma_create(int32_t ncell_2d, int32_t nlayers, int32_t ndf_to, int32_t ndf_from,
                     const int32_t* map_to, const int32_t* map_from, int64_t undf_to,
                     int64_t undf_from, const double* stencil, int32_t ncolours,
                     const int32_t* ncells_per_colour, const int32_t* cells_in_colour,
                     int32_t maxc, int32_t mode) {
  or_op* op = (or_op*)calloc(1, sizeof(or_op));
  op->ncell_2d = ncell_2d;
  op->nlayers = nlayers;
  op->ndf_to = ndf_to;
  op->ndf_from = ndf_from;
  op->map_to = map_to;
  op->map_from = map_from;
  op->undf_to = undf_to;
  op->undf_from = undf_from;
  op->stencil = stencil;
  op->ncolours = ncolours;
  op->ncells_per_colour = ncells_per_colour;
  op->cells_in_colour = cells_in_colour;
  op->maxc = maxc;
  op->mode = mode;
  return op;
}
void or_op_destroy(or_op* op) { free(op); }

/* sci_mass_matrix_operator_alg_mod.x90:98: invoke(setval_c(y, 0), matrix_vector_kernel)
 * with the PSy layer's colour loop (cells of one colour share no dof, so the
 * cells within a colour run in parallel). */
void or_op_apply(or_op* op, const double* x, double* y) {
  or_setval_c(y, 0.0, op->mode == 1 ? op->undf_from : op->undf_to);
  int64_t nc3 = (int64_t)op->ncell_2d * op->nlayers;
  for (int32_t colour = 0; colour < op->ncolours; ++colour) {
    int32_t nc = op->ncells_per_colour[colour];
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < nc; ++i) {
      int32_t cell = op->cells_in_colour[colour + (int64_t)op->ncolours * i];
      const int32_t* m1 = op->map_to + (int64_t)(cell - 1) * op->ndf_to;
      const int32_t* m2 = op->map_from + (int64_t)(cell - 1) * op->ndf_from;
      if (op->mode == 1) /* lhs on the from-space, matrix (nc3, ndf_to, ndf_from) */
        or_transpose_matrix_vector_code(cell, op->nlayers, y, x, nc3, op->stencil,
                                        op->ndf_from, m2, op->ndf_to, m1);
      else
        or_matrix_vector_code(cell, op->nlayers, y, x, nc3, op->stencil, op->ndf_to, m1,
                              op->ndf_from, m2);
    }
  }
}

/* sci_mm_diagonal_kernel_mod.F90:117-122 over the colour loop */
void or_lma_diagonal(const or_op* op, double* diag) {
  or_setval_c(diag, 0.0, op->undf_to);
  int64_t nc3 = (int64_t)op->ncell_2d * op->nlayers;
  for (int32_t colour = 0; colour < op->ncolours; ++colour) {
    int32_t nc = op->ncells_per_colour[colour];
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < nc; ++i) {
      int32_t cell = op->cells_in_colour[colour + (int64_t)op->ncolours * i];
      const int32_t* m = op->map_to + (int64_t)(cell - 1) * op->ndf_to;
      for (int32_t k = 0; k < op->nlayers; ++k) {
        int64_t ik = (int64_t)(cell - 1) * op->nlayers + k;
        for (int32_t df = 0; df < op->ndf_to; ++df)
          diag[m[df] - 1 + k] = diag[m[df] - 1 + k] + MAT(op->stencil, ik, df, df, op->ndf_to, nc3);
      }
    }
  }
}

enum { P_NULL = 0, P_DIAG = 1, P_CMA = 2 };
struct or_prec {
  int kind;
  int64_t n;
  const double* diag;
  int32_t ncell_2d, nrow, bw;
  const int32_t *first_dof, *indirection;
  const double* cm;
  char* covered; /* rows owned by the CMA */
};

or_prec* or_null_prec_create(int64_t n) {
  or_prec* p = (or_prec*)calloc(1, sizeof(or_prec));
  p->kind = P_NULL;
  p->n = n;
  return p;
}
or_prec* or_diag_prec_create(const double* diag, int64_t n) {
  or_prec* p = or_null_prec_create(n);
  p->kind = P_DIAG;
  p->diag = diag;
  return p;
}
or_prec* or_cma_prec_create(int32_t ncell_2d, int32_t nrow, int32_t bw,
                            const int32_t* first_dof, const int32_t* indirection,
                            const double* cm, const double* diag, int64_t n) {
  or_prec* p = or_null_prec_create(n);
  p->kind = P_CMA;
  p->ncell_2d = ncell_2d;
  p->nrow = nrow;
  p->bw = bw;
  p->first_dof = first_dof;
  p->indirection = indirection;
  p->cm = cm;
  p->diag = diag;
  p->covered = (char*)calloc((size_t)n, 1);
  for (int32_t c = 0; c < ncell_2d; ++c)
    for (int32_t i = 0; i < nrow; ++i) p->covered[first_dof[c] + indirection[i] - 2] = 1;
  return p;
}
void or_prec_destroy(or_prec* p) {
  if (!p) return;
  free(p->covered);
  free(p);
}

void or_prec_apply(or_prec* p, const double* x, double* y) {
  if (p->kind == P_NULL) {
    or_setval_x(y, x, p->n);
  } else if (p->kind == P_DIAG) {
    or_x_divideby_y(y, x, p->diag, p->n);
  } else {
    if (p->diag) {
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < p->n; ++i)
        if (!p->covered[i]) y[i] = x[i] / p->diag[i];
    }
#pragma omp parallel for schedule(static)
    for (int32_t c = 1; c <= p->ncell_2d; ++c)
      or_columnwise_op_appinv_code(c, y, x, p->cm, p->nrow, p->bw, &p->first_dof[c - 1],
                                   p->indirection);
  }
}

/* ------------------------------------------------------------------------ */
/* Krylov solvers, sci_iterative_solver_mod.f90 with monitor_convergence on */
/* ------------------------------------------------------------------------ */
static double* vnew(int64_t n) { return (double*)calloc((size_t)n, sizeof(double)); }
static double vnorm(const double* x, int64_t n) { return sqrt(or_sumsq(x, n)); }

/* cg_solve, :495-592 */
int or_cg(or_op* A, or_prec* P, double* x, const double* b, int64_t n, double r_tol,
          double a_tol, int32_t max_iter, or_info* info) {
  double *r = vnew(n), *p = vnew(n), *z = vnew(n);
  double alpha, beta, r_nrm = 0.0, r_nrm_0, rz, rz_new;
  int32_t iter, converged = 0;
  memset(info, 0, sizeof *info);
  or_op_apply(A, x, r);
  info->applies++;
  or_inc_a_times_x(-1.0, r, n);
  or_inc_x_plus_by(r, 1.0, b, n);
  r_nrm_0 = vnorm(r, n);
  info->initial_norm = r_nrm_0;
  if (r_nrm_0 < EPS_RDEF) {
    info->converged = 1;
    info->final_norm = r_nrm_0;
    goto done;
  }
  or_prec_apply(P, r, z);
  rz = or_dot(r, z, n);
  or_setval_x(p, z, n);
  for (iter = 1; iter <= max_iter; ++iter) {
    or_op_apply(A, p, z);
    info->applies++;
    alpha = rz / or_dot(p, z, n);
    or_inc_x_plus_by(x, alpha, p, n);
    or_inc_x_plus_by(r, -alpha, z, n);
    r_nrm = vnorm(r, n);
    info->iterations = iter;
    info->final_norm = r_nrm;
    info->final_rel = r_nrm / r_nrm_0;
    if (r_nrm / r_nrm_0 <= r_tol || r_nrm <= a_tol) {
      converged = 1;
      break;
    }
    or_prec_apply(P, r, z);
    rz_new = or_dot(r, z, n);
    beta = rz_new / rz;
    or_inc_ax_plus_y(beta, p, z, n);
    rz = rz_new;
  }
  info->converged = converged;
done:
  free(r);
  free(p);
  free(z);
  return 0;
}

/* bicgstab_solve, :645-779 */
int or_bicgstab(or_op* A, or_prec* P, double* x, const double* b, int64_t n, double r_tol,
                double a_tol, int32_t max_iter, or_info* info) {
  double *r = vnew(n), *r0 = vnew(n), *p = vnew(n), *v = vnew(n), *t = vnew(n);
  double *s = vnew(n), *y = vnew(n), *z = vnew(n);
  double alpha, beta, rho, omega, rho_old, err, sc_err, tt, ts;
  int32_t iter;
  memset(info, 0, sizeof *info);
  or_setval_x(r, b, n);
  or_op_apply(A, x, v);
  info->applies++;
  or_inc_x_plus_by(r, -1.0, v, n);
  or_setval_x(r0, r, n);
  sc_err = vnorm(r, n);
  info->initial_norm = sc_err;
  if (sc_err < EPS_RDEF) {
    info->converged = 1;
    info->final_norm = sc_err;
    goto done;
  }
  sc_err = fmax(sc_err, a_tol);
  alpha = 1.0;
  omega = 1.0;
  rho_old = 1.0;
  or_setval_c(v, 0.0, n);
  or_setval_c(p, 0.0, n);
  for (iter = 1; iter <= max_iter; ++iter) {
    rho = or_dot(r, r0, n);
    beta = (rho / rho_old) * (alpha / omega);
    or_setval_x(t, r, n);
    or_inc_x_plus_by(t, -beta * omega, v, n);
    or_prec_apply(P, t, y);
    or_inc_ax_plus_y(beta, p, y, n);
    or_op_apply(A, p, v);
    alpha = rho / or_dot(r0, v, n);
    or_setval_x(s, r, n);
    or_inc_x_plus_by(s, -alpha, v, n);
    or_prec_apply(P, s, z);
    or_op_apply(A, z, t);
    info->applies += 2;
    tt = or_dot(t, t, n);
    ts = or_dot(t, s, n);
    omega = ts / tt;
    or_inc_x_plus_by(x, omega, z, n);
    or_inc_x_plus_by(x, alpha, p, n);
    or_setval_x(r, s, n);
    or_inc_x_plus_by(r, -omega, t, n);
    rho_old = rho;
    err = vnorm(r, n) / sc_err;
    info->iterations = iter;
    info->final_rel = err;
    info->final_norm = err * sc_err;
    if (err < r_tol) {
      info->converged = 1;
      break;
    }
  }
done:
  free(r);
  free(r0);
  free(p);
  free(v);
  free(t);
  free(s);
  free(y);
  free(z);
  return 0;
}

/* gmres_solve, :830-1003 (left preconditioned, restart gcrk, no early exit
 * inside a cycle; the true residual is tested once per cycle) */
int or_gmres(or_op* A, or_prec* P, double* x, const double* b, int64_t n, int32_t gcrk,
             double r_tol, double a_tol, int32_t max_iter, or_info* info) {
  double *s = vnew(n), *w = vnew(n), *Ax = vnew(n), *res = vnew(n);
  double** v = (double**)calloc((size_t)gcrk, sizeof(double*));
  double* h = (double*)calloc((size_t)(gcrk + 1) * gcrk, sizeof(double));
  double* g = (double*)calloc((size_t)gcrk + 1, sizeof(double));
  double* u = (double*)calloc((size_t)gcrk, sizeof(double));
#define H(i, j) h[((i) - 1) + (int64_t)(gcrk + 1) * ((j) - 1)]
  double beta, si, ci, nrm, h1, h2, pp, q, res_norm, err = 0.0, sc_err;
  int32_t iv, ivj, iter;
  memset(info, 0, sizeof *info);
  for (iv = 0; iv < gcrk; ++iv) v[iv] = vnew(n);
  or_op_apply(A, x, Ax);
  info->applies++;
  or_setval_x(res, b, n);
  or_inc_x_plus_by(res, -1.0, Ax, n);
  sc_err = vnorm(res, n);
  info->initial_norm = sc_err;
  if (sc_err < EPS_RDEF) {
    info->converged = 1;
    info->final_norm = sc_err;
    goto done;
  }
  sc_err = fmax(sc_err, a_tol);
  for (iter = 1; iter <= max_iter; ++iter) {
    or_prec_apply(P, res, s);
    beta = vnorm(s, n);
    or_setval_x(v[0], s, n);
    or_inc_a_times_x(1.0 / beta, v[0], n);
    for (iv = 0; iv <= gcrk; ++iv) g[iv] = 0.0;
    g[0] = beta;
    for (iv = 1; iv <= gcrk; ++iv) {
      or_setval_x(w, v[iv - 1], n);
      or_op_apply(A, w, s);
      info->applies++;
      or_prec_apply(P, s, w);
      for (ivj = 1; ivj <= iv; ++ivj) {
        H(ivj, iv) = or_dot(v[ivj - 1], w, n);
        or_inc_x_plus_by(w, -H(ivj, iv), v[ivj - 1], n);
      }
      H(iv + 1, iv) = vnorm(w, n);
      if (iv < gcrk) {
        or_setval_x(v[iv], w, n);
        or_inc_a_times_x(1.0 / H(iv + 1, iv), v[iv], n);
      }
    }
    for (iv = 1; iv <= gcrk; ++iv) {
      nrm = sqrt(fma(H(iv, iv), H(iv, iv), H(iv + 1, iv) * H(iv + 1, iv)));
      si = H(iv + 1, iv) / nrm;
      ci = H(iv, iv) / nrm;
      pp = fma(ci, g[iv - 1], si * g[iv]);
      q = fma(-si, g[iv - 1], ci * g[iv]);
      g[iv - 1] = pp;
      g[iv] = q;
      for (ivj = iv; ivj <= gcrk; ++ivj) {
        h1 = fma(ci, H(iv, ivj), si * H(iv + 1, ivj));
        h2 = fma(-si, H(iv, ivj), ci * H(iv + 1, ivj));
        H(iv, ivj) = h1;
        H(iv + 1, ivj) = h2;
      }
    }
    u[gcrk - 1] = g[gcrk - 1] / H(gcrk, gcrk);
    for (iv = gcrk - 1; iv >= 1; --iv) {
      u[iv - 1] = g[iv - 1];
      for (ivj = iv + 1; ivj <= gcrk; ++ivj) u[iv - 1] = fma(-H(iv, ivj), u[ivj - 1], u[iv - 1]);
      u[iv - 1] = u[iv - 1] / H(iv, iv);
    }
    for (iv = 1; iv <= gcrk; ++iv) or_inc_x_plus_by(x, u[iv - 1], v[iv - 1], n);
    or_op_apply(A, x, Ax);
    info->applies++;
    or_setval_x(res, Ax, n);
    or_inc_ax_plus_y(-1.0, res, b, n);
    res_norm = vnorm(res, n);
    err = res_norm / sc_err;
    info->iterations = iter;
    info->final_norm = res_norm;
    info->final_rel = err;
    if (err < r_tol) {
      info->converged = 1;
      break;
    }
  }
done:
#undef H
  for (iv = 0; iv < gcrk; ++iv) free(v[iv]);
  free(v);
  free(h);
  free(g);
  free(u);
  free(s);
  free(w);
  free(Ax);
  free(res);
  return 0;
}

/* Givens reduction of the (gcrk+1) x gcrk Hessenberg matrix and back
 * substitution, shared by or_fgmres: sci_iterative_solver_mod.f90:1153-1182
 * (the same steps as gmres_solve :931-960). */
static void hessenberg_solve(double* h, double* g, double* u, int32_t gcrk) {
#define H(i, j) h[((i) - 1) + (int64_t)(gcrk + 1) * ((j) - 1)]
  for (int32_t iv = 1; iv <= gcrk; ++iv) {
    const double nrm = sqrt(fma(H(iv, iv), H(iv, iv), H(iv + 1, iv) * H(iv + 1, iv)));
    const double si = H(iv + 1, iv) / nrm;
    const double ci = H(iv, iv) / nrm;
    const double p = fma(ci, g[iv - 1], si * g[iv]);
    const double q = fma(-si, g[iv - 1], ci * g[iv]);
    g[iv - 1] = p;
    g[iv] = q;
    for (int32_t ivj = iv; ivj <= gcrk; ++ivj) {
      const double h1 = fma(ci, H(iv, ivj), si * H(iv + 1, ivj));
      const double h2 = fma(-si, H(iv, ivj), ci * H(iv + 1, ivj));
      H(iv, ivj) = h1;
      H(iv + 1, ivj) = h2;
    }
  }
  u[gcrk - 1] = g[gcrk - 1] / H(gcrk, gcrk);
  for (int32_t iv = gcrk - 1; iv >= 1; --iv) {
    u[iv - 1] = g[iv - 1];
    for (int32_t ivj = iv + 1; ivj <= gcrk; ++ivj) u[iv - 1] = fma(-H(iv, ivj), u[ivj - 1], u[iv - 1]);
    u[iv - 1] = u[iv - 1] / H(iv, iv);
  }
#undef H
}

/* fgmres_solve, sci_iterative_solver_mod.f90:1055-1237, monitor_convergence on */
int or_fgmres(or_op* A, or_prec* P, double* x, const double* b, int64_t n, int32_t gcrk,
              double r_tol, double a_tol, int32_t max_iter, or_info* info) {
  double *s = vnew(n), *w = vnew(n), *dx = vnew(n), *Ax = vnew(n), *res = vnew(n);
  double** v = (double**)calloc((size_t)gcrk, sizeof(double*));
  double** Pv = (double**)calloc((size_t)gcrk, sizeof(double*));
  double* h = (double*)calloc((size_t)(gcrk + 1) * gcrk, sizeof(double));
  double* g = (double*)calloc((size_t)gcrk + 1, sizeof(double));
  double* u = (double*)calloc((size_t)gcrk, sizeof(double));
#define H(i, j) h[((i) - 1) + (int64_t)(gcrk + 1) * ((j) - 1)]
  double beta, err = 0.0, sc_err;
  int32_t iv, ivj, iter;
  memset(info, 0, sizeof *info);
  for (iv = 0; iv < gcrk; ++iv) {
    v[iv] = vnew(n);
    Pv[iv] = vnew(n);
  }
  /* :1079-1087 dx = 0, Ax = 0, res = b */
  or_setval_x(res, b, n);
  sc_err = vnorm(res, n);
  info->initial_norm = sc_err;
  if (sc_err < EPS_RDEF) { /* :1092-1097, returns before x += dx */
    info->converged = 1;
    info->final_norm = sc_err;
    goto done;
  }
  sc_err = fmax(sc_err, a_tol);
  or_setval_x(s, res, n);
  beta = vnorm(s, n);
  or_setval_x(v[0], s, n);
  or_inc_a_times_x(1.0 / beta, v[0], n);
  for (iv = 0; iv <= gcrk; ++iv) g[iv] = 0.0;
  g[0] = beta;
  for (iter = 1; iter <= max_iter; ++iter) {
    for (iv = 1; iv <= gcrk; ++iv) { /* :1134-1151 */
      or_prec_apply(P, v[iv - 1], Pv[iv - 1]);
      or_op_apply(A, Pv[iv - 1], s);
      info->applies++;
      or_setval_x(w, s, n);
      for (ivj = 1; ivj <= iv; ++ivj) {
        H(ivj, iv) = or_dot(v[ivj - 1], w, n);
        or_inc_x_plus_by(w, -H(ivj, iv), v[ivj - 1], n);
      }
      H(iv + 1, iv) = vnorm(w, n);
      if (iv < gcrk) {
        or_setval_x(v[iv], w, n);
        or_inc_a_times_x(1.0 / H(iv + 1, iv), v[iv], n);
      }
    }
    hessenberg_solve(h, g, u, gcrk);
    for (iv = 1; iv <= gcrk; ++iv) or_inc_x_plus_by(dx, u[iv - 1], Pv[iv - 1], n); /* :1185-1188 */
    or_op_apply(A, dx, Ax); /* :1191-1193 */
    info->applies++;
    or_setval_x(res, Ax, n);
    or_inc_ax_plus_y(-1.0, res, b, n);
    beta = vnorm(res, n);
    err = beta / sc_err;
    info->iterations = iter;
    info->final_norm = beta;
    info->final_rel = err;
    if (err < r_tol) {
      info->converged = 1;
      break;
    }
    or_setval_x(s, res, n); /* :1208-1213 */
    or_setval_c(v[0], 0.0, n);
    or_inc_x_plus_by(v[0], 1.0 / beta, s, n);
    for (iv = 0; iv <= gcrk; ++iv) g[iv] = 0.0;
    g[0] = beta;
  }
  or_inc_x_plus_by(x, 1.0, dx, n); /* :1228 */
done:
#undef H
  for (iv = 0; iv < gcrk; ++iv) {
    free(v[iv]);
    free(Pv[iv]);
  }
  free(v);
  free(Pv);
  free(h);
  free(g);
  free(u);
  free(s);
  free(w);
  free(dx);
  free(Ax);
  free(res);
  return 0;
}

/* gcr_solve, sci_iterative_solver_mod.f90:1288-1408, monitor_convergence on */
int or_gcr(or_op* A, or_prec* P, double* x, const double* b, int64_t n, int32_t gcrk,
           double r_tol, double a_tol, int32_t max_iter, or_info* info, int32_t* iv_final) {
  double *dx = vnew(n), *res = vnew(n), *Ax = vnew(n);
  double** v = (double**)calloc((size_t)gcrk, sizeof(double*));
  double** Pv = (double**)calloc((size_t)gcrk, sizeof(double*));
  double alpha, beta, err = 0.0, sc_err, rn = 0.0;
  int32_t iv, ivj, iter, ivf = 0;
  memset(info, 0, sizeof *info);
  for (iv = 0; iv < gcrk; ++iv) {
    v[iv] = vnew(n);
    Pv[iv] = vnew(n);
  }
  /* :1321-1327 dx = P b, res = b - A dx */
  or_prec_apply(P, b, dx);
  or_op_apply(A, dx, Ax);
  info->applies++;
  or_setval_x(res, b, n);
  or_inc_x_plus_by(res, -1.0, Ax, n);
  sc_err = vnorm(b, n); /* :1330 */
  info->initial_norm = sc_err;
  if (sc_err < EPS_RDEF) {
    info->converged = 1;
    info->final_norm = sc_err;
    goto done;
  }
  sc_err = fmax(sc_err, a_tol);
  for (iter = 1; iter <= max_iter; ++iter) {
    for (iv = 1; iv <= gcrk; ++iv) { /* :1356-1380 */
      or_prec_apply(P, res, Pv[iv - 1]);
      or_op_apply(A, Pv[iv - 1], v[iv - 1]);
      info->applies++;
      for (ivj = 1; ivj <= iv - 1; ++ivj) {
        alpha = or_dot(v[iv - 1], v[ivj - 1], n);
        or_inc_x_plus_by(v[iv - 1], -alpha, v[ivj - 1], n);
        or_inc_x_plus_by(Pv[iv - 1], -alpha, Pv[ivj - 1], n);
      }
      alpha = vnorm(v[iv - 1], n);
      beta = 1.0 / alpha;
      or_inc_a_times_x(beta, v[iv - 1], n);
      or_inc_a_times_x(beta, Pv[iv - 1], n);
      alpha = or_dot(res, v[iv - 1], n);
      or_inc_x_plus_by(dx, alpha, Pv[iv - 1], n);
      or_inc_x_plus_by(res, -alpha, v[iv - 1], n);
      rn = vnorm(res, n);
      err = rn / sc_err;
      ivf = iv;
      if (err < r_tol) break;
    }
    info->iterations = iter;
    info->final_norm = rn;
    info->final_rel = err;
    if (err < r_tol) {
      info->converged = 1;
      break;
    }
  }
  or_inc_x_plus_by(x, 1.0, dx, n); /* :1400 */
done:
  if (iv_final) *iv_final = ivf;
  for (iv = 0; iv < gcrk; ++iv) {
    free(v[iv]);
    free(Pv[iv]);
  }
  free(v);
  free(Pv);
  free(dx);
  free(res);
  free(Ax);
  return 0;
}

/* precondition_only_solve, sci_iterative_solver_mod.f90:1664-1694 (monitoring on) */
int or_precondition_only(or_op* A, or_prec* P, double* x, const double* b, int64_t n,
                         or_info* info) {
  double *res = vnew(n), *Ax = vnew(n);
  memset(info, 0, sizeof *info);
  or_prec_apply(P, b, x);
  or_setval_x(res, b, n);
  const double e0 = vnorm(res, n);
  or_op_apply(A, x, Ax);
  info->applies = 1;
  or_inc_x_plus_by(res, -1.0, Ax, n);
  const double e = vnorm(res, n);
  info->iterations = 1;
  info->converged = 1;
  info->initial_norm = e0;
  info->final_norm = e;
  info->final_rel = e / e0;
  free(res);
  free(Ax);
  return 0;
}

/* jacobi_solve, sci_iterative_solver_mod.f90:1745-1815 (monitoring on) */
int or_jacobi(or_op* A, or_prec* P, double* x, const double* b, int64_t n, double r_tol,
              double a_tol, int32_t max_iter, double rho_relax, or_info* info) {
  double *r = vnew(n), *z = vnew(n);
  double r_nrm = 0.0, r_nrm_0 = 0.0;
  const double cst = -rho_relax;
  memset(info, 0, sizeof *info);
  for (int32_t iter = 1; iter <= max_iter; ++iter) {
    or_op_apply(A, x, r);
    info->applies++;
    or_inc_x_plus_by(r, -1.0, b, n);
    r_nrm = vnorm(r, n);
    if (iter == 1) r_nrm_0 = r_nrm;
    info->iterations = iter;
    info->final_norm = r_nrm;
    info->final_rel = r_nrm / r_nrm_0;
    if (r_nrm / r_nrm_0 <= r_tol || r_nrm <= a_tol) {
      info->converged = 1;
      break;
    }
    or_prec_apply(P, r, z);
    or_inc_x_plus_by(x, cst, z, n);
  }
  info->initial_norm = r_nrm_0;
  free(r);
  free(z);
  return 0;
}

/* chebyshev_solve, sci_iterative_solver_mod.f90:1868-1940 (monitoring on) */
int or_chebyshev(or_op* A, or_prec* P, double* x, const double* b, int64_t n, int32_t max_iter,
                 double lmin, double lmax, or_info* info) {
  double *xp = vnew(n), *xo = vnew(n), *z = vnew(n), *r = vnew(n);
  memset(info, 0, sizeof *info);
  or_setval_c(x, 0.0, n);
  const double init_norm = fmax(1.0, vnorm(b, n));
  const double a1 = 2.0 / (lmax - lmin);
  const double a2 = (lmax + lmin) / (lmax - lmin);
  const double a_over_b = a1 / a2;
  double w = 1.0;
  for (int32_t iter = 1; iter <= max_iter; ++iter) {
    or_op_apply(A, xo, z);
    info->applies++;
    or_ax_plus_by(r, 1.0, b, -1.0, z, n);
    or_prec_apply(P, r, z);
    w = 1.0 / (1.0 - w / (4.0 * (a2 * a2)));
    const double wa_over_b = w * a_over_b;
    or_ax_plus_by(x, wa_over_b, z, w, xo, n);
    or_inc_x_plus_by(x, 1.0 - w, xp, n);
    if (iter < max_iter) {
      or_setval_x(xp, xo, n);
      or_setval_x(xo, x, n);
    }
  }
  or_op_apply(A, x, z);
  info->applies++;
  or_inc_x_plus_by(z, -1.0, b, n);
  const double fn = vnorm(z, n);
  info->iterations = max_iter;
  info->converged = 1;
  info->initial_norm = init_norm;
  info->final_norm = fn;
  info->final_rel = fn / init_norm;
  free(xp);
  free(xo);
  free(z);
  free(r);
  return 0;
}
