// Columnwise-assembled (CMA) operators and the preconditioners.
//
//  * lfx_cma: columnwise_operator_type (columnwise_operator_mod.f90:42-469),
//    banded storage columnwise_matrix(bandwidth, nrow, ncell_2d).
//  * assembly from an LMA sub-block: columnwise_op_asm_kernel_code
//    (sci_columnwise_op_asm_kernel_mod.F90:72-128), one thread per column.
//  * y += A x: columnwise_op_app_kernel_code (sci_columnwise_op_app_kernel_mod.F90:73-124).
//  * preconditioners: null (y = x), diagonal (X_divideby_Y,
//    sci_diagonal_preconditioner_alg_mod.x90:92) and column-tridiagonal
//    (columnwise_op_appinv_kernel_code, sci_columnwise_op_appinv_kernel_mod.F90:77-145)
//    with the Jacobi diagonal on the rows the columns do not cover.
//
// The Thomas recurrences of appinv split into an x-independent part (c' and
// the inverse denominators) and the sweeps. The device computes the first
// part once, in FP64, with the same operations as the reference (so every
// value is bit-identical to recomputing it per apply) and stores the factors
// row-major over columns ([row][column]) so that one thread per column reads
// them with coalesced loads.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "lfx_internal.cuh"

using namespace lfx;

namespace {

__host__ __device__ inline int ceil_div_i(int a, int b) {  // b > 0, as ceiling(real(a)/b)
  return a >= 0 ? (a + b - 1) / b : -((-a) / b);
}
__host__ __device__ inline int floor_div_i(int a, int b) {
  return a >= 0 ? a / b : -((-a + b - 1) / b);
}

// columnwise_op_asm on a sub-block (dfs) of an FP64 LMA stored [c][df] blocks
// of blk elements, [df2][k] inside
__global__ void cma_asm(int ncell, int nl, int ndf_full, int blk, const double* __restrict__ M,
                        int nsub, const int* __restrict__ dfs, const int* __restrict__ cbd,
                        int nrow, int bw, int alpha, int beta, int gamma_p,
                        double* __restrict__ band) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  double* col = band + (size_t)c * bw * nrow;
  for (int i = 0; i < bw * nrow; ++i) col[i] = 0.0;
  const double* Mc = M + (size_t)c * ndf_full * blk;
  for (int k = 1; k <= nl; ++k)
    for (int a = 0; a < nsub; ++a) {
      const int i = cbd[a + nsub * (k - 1)];
      const int jm = ceil_div_i(alpha * i - gamma_p, beta);
      for (int b = 0; b < nsub; ++b) {
        const int j = cbd[b + nsub * (k - 1)];
        if (j - jm < 0 || j - jm >= bw) continue;  // outside the band (host validates)
        double* e = &col[(j - jm) + (size_t)bw * (i - 1)];
        *e = *e + Mc[(size_t)dfs[a] * blk + (size_t)dfs[b] * nl + (k - 1)];
      }
    }
}

template <class T>
__global__ void cma_app(int ncell, int nrow, int ncol, int bw, int alpha, int beta, int gamma_m,
                        int gamma_p, const int* __restrict__ first, const int* __restrict__ ind,
                        const double* __restrict__ band, const T* __restrict__ x, T* __restrict__ y) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const double* col = band + (size_t)c * bw * nrow;
  for (int i = 1; i <= nrow; ++i) {
    const int mu_i = first[c] + ind[i - 1];
    const int jm = ceil_div_i(alpha * i - gamma_p, beta);
    const int jp = floor_div_i(alpha * i + gamma_m, beta);
    T acc = y[mu_i];
    for (int j = max(1, jm); j <= min(ncol, jp); ++j)
      acc = fmaT((T)col[(j - jm) + (size_t)bw * (i - 1)], x[first[c] + ind[j - 1]], acc);
    y[mu_i] = acc;
  }
}

// x-independent Thomas factors per column (FP64), stored [row][column] in T;
// flags a zero or non-finite pivot in *bad
template <class T>
__global__ void thomas_factor(int ncell, int nrow, const double* __restrict__ band, T* fa, T* finv,
                              T* fc, int* bad) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const double* col = band + (size_t)c * 3 * nrow;
  double cprev = 0.0;
  for (int i = 0; i < nrow; ++i) {
    const double a = col[3 * i + 0], b = col[3 * i + 1], u = col[3 * i + 2];
    const double inv = (i == 0) ? 1.0 / b : 1.0 / fma(-a, cprev, b);
    const double cp = (i < nrow - 1) ? inv * u : 0.0;
    if (!isfinite(inv)) atomicExch(bad, 1);
    fa[(size_t)i * ncell + c] = (T)a;
    finv[(size_t)i * ncell + c] = (T)inv;
    fc[(size_t)i * ncell + c] = (T)cp;
    cprev = cp;
  }
}

// Thomas sweeps (one thread per column) and y = x / diag on uncovered runs
// (one warp per run), in one launch.
template <class T>
__global__ void __launch_bounds__(128) cma_prec_apply(
    int ncell, int nrow, const int* __restrict__ first, const int* __restrict__ ind,
    const T* __restrict__ fa, const T* __restrict__ finv, const T* __restrict__ fc,
    const T* __restrict__ x, T* __restrict__ y, int thomas_blocks, int nruns,
    const int* __restrict__ run_start, const int* __restrict__ run_len, const T* __restrict__ diag,
    const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  if ((int)blockIdx.x < thomas_blocks) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    thomas_sweep<8>(first[c], ind, nrow, ncell, c, fa, finv, fc, x, y);
  } else {
    const int lane = threadIdx.x & 31;
    const int64_t w = ((int64_t)(blockIdx.x - thomas_blocks) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)(gridDim.x - thomas_blocks) * blockDim.x) >> 5;
    for (int64_t r = w; r < nruns; r += nw) {
      const int s = run_start[r], len = run_len[r];
      for (int l = lane; l < len; l += 32) y[s + l] = x[s + l] / diag[s + l];
    }
  }
}

template <class T>
int k_divide(lfx_ctx* ctx, T* y, const T* x, const T* d, int64_t n, const int* skip) {
  return launch_chunks<0>(
      ctx, n, [=] __device__(int64_t i) { return V2<T>{x[i], d[i]}; },
      [=] __device__(int64_t i, const V2<T>& v, double*) { y[i] = v.a / v.b; }, NoFin{}, skip);
}
template <class S, class D>
int k_cast(lfx_ctx* ctx, D* d, const S* s, int64_t n, const int* skip) {
  return launch_chunks<0>(
      ctx, n, [=] __device__(int64_t i) { return V1<S>{s[i]}; },
      [=] __device__(int64_t i, const V1<S>& v, double*) { d[i] = (D)v.a; }, NoFin{}, skip);
}

}  // namespace

namespace lfx {

int prec_apply_impl(lfx_prec* p, int32_t precision, const void* x, void* y, int64_t n,
                    const int* skip) {
  lfx_ctx* ctx = p->ctx;
  const bool r64 = precision == LFX_R64;
  switch (p->kind) {
    case PREC_NULL:
      return r64 ? k_cast(ctx, (double*)y, (const double*)x, n, skip)
                 : k_cast(ctx, (float*)y, (const float*)x, n, skip);
    case PREC_DIAG:
      return r64 ? k_divide(ctx, (double*)y, (const double*)x, (const double*)p->rdiag, n, skip)
                 : k_divide(ctx, (float*)y, (const float*)x, (const float*)p->rdiag, n, skip);
    case PREC_CMA: {
      ctx->launches++;
      const int tb = (p->ncell_2d + 127) / 128;
      int rb = (int)std::min<int64_t>(((int64_t)p->nruns + 3) / 4, (int64_t)ctx->num_sms * 8);
      if (p->nruns == 0) rb = 0;
      if (r64)
        cma_prec_apply<double><<<tb + rb, 128, 0, ctx->stream>>>(
            p->ncell_2d, p->nrow, p->first_dof, p->indirection, (const double*)p->fa,
            (const double*)p->finv, (const double*)p->fc, (const double*)x, (double*)y, tb,
            p->nruns, p->run_start, p->run_len, (const double*)p->rdiag, skip);
      else
        cma_prec_apply<float><<<tb + rb, 128, 0, ctx->stream>>>(
            p->ncell_2d, p->nrow, p->first_dof, p->indirection, (const float*)p->fa,
            (const float*)p->finv, (const float*)p->fc, (const float*)x, (float*)y, tb, p->nruns,
            p->run_start, p->run_len, (const float*)p->rdiag, skip);
      LFX_CK(ctx, cudaGetLastError());
      return LFX_OK;
    }
  }
  return LFX_INVALID_ARGUMENT;
}

}  // namespace lfx

static int copy_diag(lfx_ctx* ctx, const lfx_vec* diag, int32_t precision, void** out) {
  const int64_t n = diag->undf[0];
  const size_t esz = precision == LFX_R64 ? 8 : 4;
  int rc = dmalloc(ctx, out, n * esz);
  if (rc) return rc;
  if (diag->precision == precision) {
    LFX_CK(ctx, cudaMemcpyAsync(*out, diag->data[0], n * esz, cudaMemcpyDeviceToDevice, ctx->stream));
  } else if (precision == LFX_R32) {
    rc = k_cast(ctx, (float*)*out, (const double*)diag->data[0], n, nullptr);
  } else {
    rc = k_cast(ctx, (double*)*out, (const float*)diag->data[0], n, nullptr);
  }
  return rc;
}

extern "C" {

int lfx_cma_create(lfx_ctx* ctx, int32_t ncell_2d, int32_t nrow, int32_t ncol, int32_t bandwidth,
                   int32_t alpha, int32_t beta, int32_t gamma_m, int32_t gamma_p,
                   const int32_t* first_dof, const int32_t* indirection,
                   const double* columnwise_matrix, lfx_cma** out) {
  if (!ctx || !out || !first_dof || !indirection) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  if (ncell_2d < 1 || nrow < 1 || ncol != nrow || bandwidth < 1 || beta < 1)
    return fail(ctx, LFX_INVALID_ARGUMENT, "bad CMA dimensions (square operators only)");
  lfx_cma* m = new lfx_cma();
  m->ctx = ctx;
  m->ncell_2d = ncell_2d;
  m->nrow = nrow;
  m->ncol = ncol;
  m->bw = bandwidth;
  m->alpha = alpha;
  m->beta = beta;
  m->gamma_m = gamma_m;
  m->gamma_p = gamma_p;
  m->h_first.resize(ncell_2d);
  m->h_ind.resize(nrow);
  int32_t maxf = 0, maxi = 0;
  for (int c = 0; c < ncell_2d; ++c) {
    m->h_first[c] = first_dof[c] - 1;
    maxf = std::max(maxf, m->h_first[c]);
    if (m->h_first[c] < 0) {
      delete m;
      return fail(ctx, LFX_INVALID_ARGUMENT, "first_dof must be >= 1");
    }
  }
  for (int i = 0; i < nrow; ++i) {
    m->h_ind[i] = indirection[i] - 1;
    maxi = std::max(maxi, m->h_ind[i]);
    if (m->h_ind[i] < 0) {
      delete m;
      return fail(ctx, LFX_INVALID_ARGUMENT, "indirection entries must be >= 1");
    }
  }
  m->max_row = (int64_t)maxf + maxi;
  int rc = dmalloc(ctx, (void**)&m->first_dof, 4 * (size_t)ncell_2d);
  if (!rc) rc = dmalloc(ctx, (void**)&m->indirection, 4 * (size_t)nrow);
  if (!rc) rc = dmalloc(ctx, (void**)&m->band, 8 * (size_t)bandwidth * nrow * ncell_2d);
  if (rc) {
    lfx_cma_destroy(m);
    return rc;
  }
  cudaMemcpy(m->first_dof, m->h_first.data(), 4 * (size_t)ncell_2d, cudaMemcpyHostToDevice);
  cudaMemcpy(m->indirection, m->h_ind.data(), 4 * (size_t)nrow, cudaMemcpyHostToDevice);
  if (columnwise_matrix)
    cudaMemcpy(m->band, columnwise_matrix, 8 * (size_t)bandwidth * nrow * ncell_2d,
               cudaMemcpyHostToDevice);
  else
    cudaMemset(m->band, 0, 8 * (size_t)bandwidth * nrow * ncell_2d);
  LFX_CK(ctx, cudaGetLastError());
  *out = m;
  return LFX_OK;
}

int lfx_cma_assemble_from_lma(const lfx_op* lma, int32_t nsub, const int32_t* dfs,
                              const int32_t* column_banded_dofmap, int32_t alpha, int32_t beta,
                              int32_t gamma_m, int32_t gamma_p, int32_t bandwidth, int32_t nrow,
                              const int32_t* first_dof, const int32_t* indirection, lfx_cma** out) {
  if (!lma || !dfs || !column_banded_dofmap || !out) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = lma->ctx;
  const lfx_lma_layout* L = lma->lay;
  if (lma->precision != LFX_R64 || L->ndf_to != L->ndf_from)
    return fail(ctx, LFX_INVALID_ARGUMENT, "CMA assembly needs a square FP64 LMA");
  std::vector<int32_t> d0(nsub);
  for (int a = 0; a < nsub; ++a) {
    d0[a] = dfs[a] - 1;
    if (d0[a] < 0 || d0[a] >= L->ndf_to) return fail(ctx, LFX_INVALID_ARGUMENT, "bad local dof");
  }
  for (int64_t q = 0; q < (int64_t)nsub * L->nlayers; ++q)
    if (column_banded_dofmap[q] < 1 || column_banded_dofmap[q] > nrow)
      return fail(ctx, LFX_INVALID_ARGUMENT, "column_banded_dofmap out of range");
  if (beta < 1) return fail(ctx, LFX_INVALID_ARGUMENT, "beta must be positive");
  for (int k = 0; k < L->nlayers; ++k)
    for (int a = 0; a < nsub; ++a) {
      const int i = column_banded_dofmap[a + nsub * k];
      const int jm = ceil_div_i(alpha * i - gamma_p, beta);
      for (int b = 0; b < nsub; ++b) {
        const int j = column_banded_dofmap[b + nsub * k];
        if (j - jm < 0 || j - jm >= bandwidth)
          return fail(ctx, LFX_INVALID_ARGUMENT, "LMA entry falls outside the band");
      }
    }
  int rc = lfx_cma_create(ctx, L->ncell_2d, nrow, nrow, bandwidth, alpha, beta, gamma_m, gamma_p,
                          first_dof, indirection, nullptr, out);
  if (rc) return rc;
  int *d_dfs = nullptr, *d_cbd = nullptr;
  rc = dmalloc(ctx, (void**)&d_dfs, 4 * (size_t)nsub);
  if (!rc) rc = dmalloc(ctx, (void**)&d_cbd, 4 * (size_t)nsub * L->nlayers);
  if (!rc) {
    cudaMemcpy(d_dfs, d0.data(), 4 * (size_t)nsub, cudaMemcpyHostToDevice);
    cudaMemcpy(d_cbd, column_banded_dofmap, 4 * (size_t)nsub * L->nlayers, cudaMemcpyHostToDevice);
    cma_asm<<<(L->ncell_2d + 127) / 128, 128, 0, ctx->stream>>>(
        L->ncell_2d, L->nlayers, L->ndf_to, lma->blk, (const double*)lma->mat, nsub, d_dfs, d_cbd,
        nrow, bandwidth, alpha, beta, gamma_p, (*out)->band);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      rc = fail(ctx, LFX_CUDA_ERROR, "CMA assembly kernel failed");
  }
  dfree(ctx, d_dfs, 4 * (size_t)nsub);
  dfree(ctx, d_cbd, 4 * (size_t)nsub * L->nlayers);
  if (rc) {
    lfx_cma_destroy(*out);
    *out = nullptr;
  }
  return rc;
}

int lfx_cma_get_band(const lfx_cma* m, double* band) {
  if (!m || !band) return LFX_INVALID_ARGUMENT;
  LFX_CK(m->ctx, cudaStreamSynchronize(m->ctx->stream));
  LFX_CK(m->ctx, cudaMemcpy(band, m->band, 8 * (size_t)m->bw * m->nrow * m->ncell_2d,
                            cudaMemcpyDeviceToHost));
  return LFX_OK;
}

int lfx_cma_apply(lfx_cma* m, const lfx_vec* x, lfx_vec* y) {
  if (!m || !x || !y) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = m->ctx;
  if (x->precision != y->precision || x->undf != y->undf)
    return fail(ctx, LFX_TYPE_MISMATCH, "vectors differ in shape or precision");
  if (m->max_row >= x->undf[0])
    return fail(ctx, LFX_TYPE_MISMATCH, "CMA rows fall outside the vector");
  const int grid = (m->ncell_2d + 127) / 128;
  if (x->precision == LFX_R64)
    cma_app<double><<<grid, 128, 0, ctx->stream>>>(m->ncell_2d, m->nrow, m->ncol, m->bw, m->alpha,
                                                   m->beta, m->gamma_m, m->gamma_p, m->first_dof,
                                                   m->indirection, m->band,
                                                   (const double*)x->data[0], (double*)y->data[0]);
  else
    cma_app<float><<<grid, 128, 0, ctx->stream>>>(m->ncell_2d, m->nrow, m->ncol, m->bw, m->alpha,
                                                  m->beta, m->gamma_m, m->gamma_p, m->first_dof,
                                                  m->indirection, m->band,
                                                  (const float*)x->data[0], (float*)y->data[0]);
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

int lfx_cma_destroy(lfx_cma* m) {
  if (!m) return LFX_OK;
  dfree(m->ctx, m->first_dof, 4 * (size_t)m->ncell_2d);
  dfree(m->ctx, m->indirection, 4 * (size_t)m->nrow);
  dfree(m->ctx, m->band, 8 * (size_t)m->bw * m->nrow * m->ncell_2d);
  delete m;
  return LFX_OK;
}

int lfx_null_prec_create(lfx_ctx* ctx, lfx_prec** out) {
  if (!ctx || !out) return LFX_INVALID_ARGUMENT;
  lfx_prec* p = new lfx_prec();
  p->ctx = ctx;
  p->kind = PREC_NULL;
  p->precision = 0;  // any
  *out = p;
  return LFX_OK;
}

// The reference copies the diagonal into the preconditioner
// (sci_diagonal_preconditioner_alg_mod.x90:60), so does this.
int lfx_diag_prec_create(lfx_ctx* ctx, const lfx_vec* diag, lfx_prec** out) {
  if (!ctx || !diag || !out) return LFX_INVALID_ARGUMENT;
  if (diag->undf.size() != 1) return fail(ctx, LFX_NOT_SUPPORTED, "single-field diagonal only");
  lfx_prec* p = new lfx_prec();
  p->ctx = ctx;
  p->kind = PREC_DIAG;
  p->precision = diag->precision;
  p->rdiag_n = diag->undf[0];
  int rc = copy_diag(ctx, diag, p->precision, &p->rdiag);
  if (rc) {
    delete p;
    return rc;
  }
  p->bytes = p->rdiag_n * diag->elem();
  *out = p;
  return LFX_OK;
}

int lfx_cma_prec_create(lfx_ctx* ctx, const lfx_cma* m, const lfx_vec* diag, int32_t precision,
                        lfx_prec** out) {
  if (!ctx || !m || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  if (m->bw != 3) return fail(ctx, LFX_NOT_SUPPORTED, "column inverse needs a tridiagonal band");
  if (precision != LFX_R64 && precision != LFX_R32) return LFX_INVALID_ARGUMENT;
  const size_t esz = precision == LFX_R64 ? 8 : 4;
  lfx_prec* p = new lfx_prec();
  p->ctx = ctx;
  p->kind = PREC_CMA;
  p->precision = precision;
  p->ncell_2d = m->ncell_2d;
  p->nrow = m->nrow;
  p->max_row = m->max_row;
  const size_t nf = (size_t)m->nrow * m->ncell_2d;
  int rc = dmalloc(ctx, &p->fa, nf * esz);
  if (!rc) rc = dmalloc(ctx, &p->finv, nf * esz);
  if (!rc) rc = dmalloc(ctx, &p->fc, nf * esz);
  if (!rc) rc = dmalloc(ctx, (void**)&p->first_dof, 4 * (size_t)m->ncell_2d);
  if (!rc) rc = dmalloc(ctx, (void**)&p->indirection, 4 * (size_t)m->nrow);
  p->bytes = 3 * nf * esz;
  int* bad = nullptr;
  if (!rc) rc = dmalloc(ctx, (void**)&bad, 4);
  if (rc) {
    lfx_prec_destroy(p);
    return rc;
  }
  cudaMemcpy(p->first_dof, m->first_dof, 4 * (size_t)m->ncell_2d, cudaMemcpyDeviceToDevice);
  cudaMemcpy(p->indirection, m->indirection, 4 * (size_t)m->nrow, cudaMemcpyDeviceToDevice);
  cudaMemset(bad, 0, 4);
  const int grid = (m->ncell_2d + 127) / 128;
  if (precision == LFX_R64)
    thomas_factor<double><<<grid, 128, 0, ctx->stream>>>(m->ncell_2d, m->nrow, m->band,
                                                         (double*)p->fa, (double*)p->finv,
                                                         (double*)p->fc, bad);
  else
    thomas_factor<float><<<grid, 128, 0, ctx->stream>>>(m->ncell_2d, m->nrow, m->band,
                                                        (float*)p->fa, (float*)p->finv,
                                                        (float*)p->fc, bad);
  int hbad = 0;
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess ||
      cudaMemcpy(&hbad, bad, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = fail(ctx, LFX_CUDA_ERROR, "column factorisation failed");
  dfree(ctx, bad, 4);
  if (!rc && hbad) rc = fail(ctx, LFX_NAN_DETECTED, "zero or non-finite pivot in a column tridiagonal");
  if (!rc && diag) {
    // rows the columns do not cover, as runs of consecutive dofs
    const int64_t n = diag->undf[0];
    std::vector<char> cov((size_t)n, 0);
    for (int c = 0; c < m->ncell_2d && !rc; ++c)
      for (int i = 0; i < m->nrow; ++i) {
        const int64_t mu = (int64_t)m->h_first[c] + m->h_ind[i];
        if (mu < 0 || mu >= n) {
          rc = fail(ctx, LFX_INVALID_ARGUMENT, "CMA rows fall outside the vector");
          break;
        }
        cov[mu] = 1;
      }
    std::vector<int32_t> rs, rl;
    for (int64_t i = 0; i < n && !rc;) {
      if (cov[i]) {
        ++i;
        continue;
      }
      int64_t j = i;
      while (j < n && !cov[j] && j - i < 1024) ++j;
      rs.push_back((int32_t)i);
      rl.push_back((int32_t)(j - i));
      i = j;
    }
    p->nruns = (int32_t)rs.size();
    if (!rc) rc = dmalloc(ctx, (void**)&p->run_start, 4 * rs.size());
    if (!rc) rc = dmalloc(ctx, (void**)&p->run_len, 4 * rl.size());
    if (!rc && !rs.empty()) {
      cudaMemcpy(p->run_start, rs.data(), 4 * rs.size(), cudaMemcpyHostToDevice);
      cudaMemcpy(p->run_len, rl.data(), 4 * rl.size(), cudaMemcpyHostToDevice);
    }
    p->rdiag_n = n;
    if (!rc) rc = copy_diag(ctx, diag, precision, &p->rdiag);
  }
  if (rc) {
    lfx_prec_destroy(p);
    return rc;
  }
  *out = p;
  return LFX_OK;
}

int lfx_prec_apply(lfx_prec* p, const lfx_vec* x, lfx_vec* y) {
  if (!p || !x || !y) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = p->ctx;
  if (x->precision != y->precision || x->undf != y->undf)
    return fail(ctx, LFX_TYPE_MISMATCH, "vectors differ in shape or precision");
  if (p->kind != PREC_NULL && x->precision != p->precision)
    return fail(ctx, LFX_TYPE_MISMATCH, "preconditioner and vector precision differ");
  if ((p->kind == PREC_DIAG || (p->kind == PREC_CMA && p->rdiag)) && x->undf[0] != p->rdiag_n)
    return fail(ctx, LFX_TYPE_MISMATCH, "vector length does not match the diagonal");
  if (p->kind == PREC_CMA && p->max_row >= x->undf[0])
    return fail(ctx, LFX_TYPE_MISMATCH, "CMA rows fall outside the vector");
  if (x->data[0] == y->data[0]) return fail(ctx, LFX_INVALID_ARGUMENT, "x and y must differ");
  for (size_t f = 0; f < x->data.size(); ++f) {
    if (f > 0 && p->kind != PREC_NULL) return fail(ctx, LFX_NOT_SUPPORTED, "single-field only");
    int rc = prec_apply_impl(p, x->precision, x->data[f], y->data[f], x->undf[f], nullptr);
    if (rc) return rc;
  }
  return LFX_OK;
}

int lfx_prec_destroy(lfx_prec* p) {
  if (!p) return LFX_OK;
  lfx_ctx* ctx = p->ctx;
  const size_t esz = p->precision == LFX_R32 ? 4 : 8;
  if (p->kind == PREC_CMA) {
    const size_t nf = (size_t)p->nrow * p->ncell_2d;
    dfree(ctx, p->fa, nf * esz);
    dfree(ctx, p->finv, nf * esz);
    dfree(ctx, p->fc, nf * esz);
    dfree(ctx, p->first_dof, 4 * (size_t)p->ncell_2d);
    dfree(ctx, p->indirection, 4 * (size_t)p->nrow);
    dfree(ctx, p->run_start, 4 * (size_t)p->nruns);
    dfree(ctx, p->run_len, 4 * (size_t)p->nruns);
  }
  dfree(ctx, p->rdiag, (size_t)p->rdiag_n * esz);
  delete p;
  return LFX_OK;
}

}  // extern "C"
