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
#include <initializer_list>
#include <vector>

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

// Band of one columnwise operator as the set-up kernels see it.
struct BandArg {
  double* band;
  int nrow, ncol, bw, alpha, beta, gm, gp;
};

// columnwise_op_mul_kernel_code (sci_columnwise_op_mul_kernel_mod.F90): C += A B,
// one thread per column, the reference's loops and order (matrixentry as one fma chain)
__global__ void cma_mul(int ncell, BandArg A, BandArg B, BandArg C) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const double* a = A.band + (size_t)c * A.bw * A.nrow;
  const double* bb = B.band + (size_t)c * B.bw * B.nrow;
  double* cc = C.band + (size_t)c * C.bw * C.nrow;
  for (int i = 1; i <= C.nrow; ++i) {
    const int jmA = ceil_div_i(A.alpha * i - A.gp, A.beta);
    const int jpA = floor_div_i(A.alpha * i + A.gm, A.beta);
    const int jmC = ceil_div_i(C.alpha * i - C.gp, C.beta);
    const int jpC = floor_div_i(C.alpha * i + C.gm, C.beta);
    for (int j = max(1, jmC); j <= min(C.ncol, jpC); ++j) {
      double e = 0.0;
      for (int l = max(1, jmA); l <= min(A.ncol, jpA); ++l) {
        const int jmB = ceil_div_i(B.alpha * l - B.gp, B.beta);
        const int jpB = floor_div_i(B.alpha * l + B.gm, B.beta);
        if (jmB <= j && j <= jpB)
          e = fma(a[(l - jmA) + (size_t)A.bw * (i - 1)], bb[(j - jmB) + (size_t)B.bw * (l - 1)], e);
      }
      double* t = &cc[(j - jmC) + (size_t)C.bw * (i - 1)];
      *t = *t + e;
    }
  }
}

// columnwise_op_scaledadd_kernel_code (sci_columnwise_op_scaledadd_kernel_mod.F90):
// C = alpha A + beta B over the rows of A
__global__ void cma_scaledadd(int ncell, BandArg A, BandArg B, BandArg C, double alpha,
                              double beta) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const double* a = A.band + (size_t)c * A.bw * A.nrow;
  const double* bb = B.band + (size_t)c * B.bw * B.nrow;
  double* cc = C.band + (size_t)c * C.bw * C.nrow;
  for (int q = 0; q < C.bw * C.nrow; ++q) cc[q] = 0.0;
  for (int i = 1; i <= A.nrow; ++i) {
    const int jmA = ceil_div_i(A.alpha * i - A.gp, A.beta);
    const int jpA = floor_div_i(A.alpha * i + A.gm, A.beta);
    const int jmB = ceil_div_i(B.alpha * i - B.gp, B.beta);
    const int jpB = floor_div_i(B.alpha * i + B.gm, B.beta);
    const int jmC = ceil_div_i(C.alpha * i - C.gp, C.beta);
    for (int j = max(1, jmA); j <= min(A.ncol, jpA); ++j) {
      double* t = &cc[(j - jmC) + (size_t)C.bw * (i - 1)];
      *t = fma(alpha, a[(j - jmA) + (size_t)A.bw * (i - 1)], *t);
    }
    for (int j = max(1, jmB); j <= min(A.ncol, jpB); ++j) {
      double* t = &cc[(j - jmC) + (size_t)C.bw * (i - 1)];
      *t = fma(beta, bb[(j - jmB) + (size_t)B.bw * (i - 1)], *t);
    }
  }
}

// columnwise_op_asm_m2v_lumped_inv_krnl_code (..._krnl_mod.F90:74-132): the
// diagonal entries of the LMA summed into band entry 1 of each row, then
// every nonzero band entry inverted. M: [c][df] blocks of blk, [df2][k] inside.
__global__ void cma_m2v_lumped_inv(int ncell, int nl, int ndf, int blk, const double* __restrict__ M,
                                   const int* __restrict__ cbd, BandArg C) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  double* cc = C.band + (size_t)c * C.bw * C.nrow;
  for (int q = 0; q < C.bw * C.nrow; ++q) cc[q] = 0.0;
  const double* Mc = M + (size_t)c * ndf * blk;
  for (int k = 1; k <= nl; ++k)
    for (int df = 0; df < ndf; ++df) {
      const int i = cbd[df + ndf * (k - 1)];
      double* t = &cc[(size_t)C.bw * (i - 1)];
      *t = *t + Mc[(size_t)df * blk + (size_t)df * nl + (k - 1)];
    }
  for (int q = 0; q < C.bw * C.nrow; ++q)
    if (cc[q] != 0.0) cc[q] = 1.0 / cc[q];
}

// columnwise_op_asm_diag_hmht_kernel_code (..._kernel_mod.F90:78-151):
// sum_df3 Dh(df1, df3) Dh(df2, df3) / M2h(df3, df3) into the band.
__global__ void cma_diag_hmht(int ncell, int nl, int ndf3, int ndfh, int blkD, int blkM,
                              const double* __restrict__ Dh, const double* __restrict__ Mh,
                              const int* __restrict__ cbd, BandArg C) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  double* cc = C.band + (size_t)c * C.bw * C.nrow;
  for (int q = 0; q < C.bw * C.nrow; ++q) cc[q] = 0.0;
  const double* Dc = Dh + (size_t)c * ndf3 * blkD;
  const double* Mc = Mh + (size_t)c * ndfh * blkM;
  for (int k = 1; k <= nl; ++k)
    for (int d1 = 0; d1 < ndf3; ++d1) {
      const int i = cbd[d1 + ndf3 * (k - 1)];
      const int jm = ceil_div_i(C.alpha * i - C.gp, C.beta);
      for (int d2 = 0; d2 < ndf3; ++d2) {
        double tmp = 0.0;
        for (int d3 = 0; d3 < ndfh; ++d3)
          tmp = tmp + Dc[(size_t)d1 * blkD + (size_t)d3 * nl + (k - 1)] *
                          Dc[(size_t)d2 * blkD + (size_t)d3 * nl + (k - 1)] /
                          Mc[(size_t)d3 * blkM + (size_t)d3 * nl + (k - 1)];
        const int j = cbd[d2 + ndf3 * (k - 1)];
        double* t = &cc[(j - jm) + (size_t)C.bw * (i - 1)];
        *t = *t + tmp;
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

// The same Thomas sweeps with each block's kStageCols columns staged through
// shared memory. The block's x rows are copied in by one warp per column
// (a column's rows are contiguous dofs, so the copies coalesce) and, with SF,
// its factor rows too ([row][column] in memory: one coalesced run of
// kStageCols per row), all by asynchronous copies issued before any is waited
// for; each of the first kStageCols threads then runs its column's
// recurrences on the staged copy and the result is copied out the same way.
// Row i of column j sits at [i * (kStageCols + 1) + j], conflict-free for the
// row-wise copies and the column-wise sweeps. Same arithmetic as
// thomas_sweep, so the same bits. Factors, read once per application, carry
// an evict-first L2 policy so that x and y stay in L2.
//
// Rows the columns do not cover get y = x / diag: where the diagonal carries
// zeros on the column rows (zero_sentinel), elementwise in a launch of its
// own that runs beside the sweeps (jacobi_sentinel), else by runs of rows in
// the blocks after the Thomas blocks.
constexpr int kStageCols = 64;
constexpr int kStageThreads = 128;

// asynchronous global -> shared copy of one element (the thread holds no
// register for it while it is in flight); the factor copies carry an L2
// evict-first policy, as they are read once per application
__device__ __forceinline__ uint32_t stage_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
template <int B>
__device__ __forceinline__ void stage_copy(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(stage_addr(dst)), "l"(src), "n"(B)
               : "memory");
}
template <int B>
__device__ __forceinline__ void stage_copy_once(void* dst, const void* src, uint64_t pol) {
  asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], %2, %3;" ::"r"(stage_addr(dst)),
               "l"(src), "n"(B), "l"(pol)
               : "memory");
}

template <class T, bool SF>
__global__ void __launch_bounds__(kStageThreads) cma_prec_staged(
    int ncell, int nrow, const int* __restrict__ first, const int* __restrict__ ind,
    const T* __restrict__ fa, const T* __restrict__ finv, const T* __restrict__ fc,
    const T* __restrict__ x, T* __restrict__ y, int thomas_blocks, int nruns,
    const int* __restrict__ run_start, const int* __restrict__ run_len, const T* __restrict__ diag,
    const int* skip) {
  // a programmatic dependent launch after this one (the Jacobi rows) may
  // start at once and run beside the sweeps
  asm volatile("griddepcontrol.launch_dependents;");
  if (skip && *((volatile const int*)skip)) return;
  constexpr int LD = kStageCols + 1;
  constexpr int NW = kStageThreads / 32;
  extern __shared__ __align__(16) unsigned char stage_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if ((int)blockIdx.x < thomas_blocks) {
    T* xs = reinterpret_cast<T*>(stage_raw);
    T* as = xs + (size_t)nrow * LD;
    T* is = as + (size_t)nrow * LD;
    T* cs = is + (size_t)nrow * LD;
    __shared__ int fs[kStageCols];
    const int c0 = blockIdx.x * kStageCols;
    const int nc = min(kStageCols, ncell - c0);
    if (threadIdx.x < nc) fs[threadIdx.x] = __ldg(first + c0 + threadIdx.x);
    __syncthreads();
    // every staging copy of the block is in flight before any is waited for:
    // lane l copies row r0 + l of the warp's columns warp, warp + NW, ...
    // (one contiguous run of rows per column), and with SF thread t copies
    // column t % kStageCols of the factor rows t / kStageCols + RS m (one
    // contiguous run of kStageCols per row)
    constexpr int CPW = kStageCols / NW;
    for (int r0 = 0; r0 < nrow; r0 += 32) {
      const int i = r0 + lane;
      if (i < nrow) {
        const int il = __ldg(ind + i);
#pragma unroll
        for (int k = 0; k < CPW; ++k) {
          const int j = warp + NW * k;
          if (j < nc) stage_copy<sizeof(T)>(&xs[i * LD + j], x + fs[j] + il);
        }
      }
    }
    if (SF) {
      uint64_t pol;
      asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
      const int j = threadIdx.x % kStageCols, i0 = threadIdx.x / kStageCols;
      constexpr int RS = kStageThreads / kStageCols;
      if (j < nc)
        for (int i = i0; i < nrow; i += RS) {
          const size_t g = (size_t)i * ncell + c0 + j;
          stage_copy_once<sizeof(T)>(&as[i * LD + j], fa + g, pol);
          stage_copy_once<sizeof(T)>(&is[i * LD + j], finv + g, pol);
          stage_copy_once<sizeof(T)>(&cs[i * LD + j], fc + g, pol);
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();
    const int j = threadIdx.x;
    if (j < nc) {
      const int c = c0 + j;
      T* col = xs + j;
      double d = 0.0;
      if (SF) {
        for (int i = 0; i < nrow; ++i) {
          const double xv = (double)col[i * LD], iv = (double)is[i * LD + j];
          d = (i == 0) ? iv * xv : iv * fma(-(double)as[i * LD + j], d, xv);
          col[i * LD] = (T)d;
        }
        for (int i = nrow - 2; i >= 0; --i) {
          d = fma(-(double)cs[i * LD + j], d, (double)col[i * LD]);
          col[i * LD] = (T)d;
        }
      } else {
        constexpr int R = 8;
        for (int i0 = 0; i0 < nrow; i0 += R) {
          double iv[R], av[R];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int i = i0 + r;
            if (i < nrow) {
              iv[r] = (double)__ldcs(finv + (size_t)i * ncell + c);
              av[r] = (double)__ldcs(fa + (size_t)i * ncell + c);
            }
          }
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int i = i0 + r;
            if (i < nrow) {
              const double xv = (double)col[i * LD];
              d = (i == 0) ? iv[r] * xv : iv[r] * fma(-av[r], d, xv);
              col[i * LD] = (T)d;
            }
          }
        }
        for (int i0 = nrow - 2; i0 >= 0; i0 -= R) {
          double cv[R];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int i = i0 - r;
            if (i >= 0) cv[r] = (double)__ldcs(fc + (size_t)i * ncell + c);
          }
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int i = i0 - r;
            if (i >= 0) {
              d = fma(-cv[r], d, (double)col[i * LD]);
              col[i * LD] = (T)d;
            }
          }
        }
      }
    }
    __syncthreads();
    for (int r0 = 0; r0 < nrow; r0 += 32) {
      const int i = r0 + lane;
      if (i < nrow) {
        const int il = __ldg(ind + i);
#pragma unroll
        for (int k = 0; k < CPW; ++k) {
          const int j = warp + NW * k;
          if (j < nc) y[fs[j] + il] = xs[i * LD + j];
        }
      }
    }
  } else {
    const int64_t w = ((int64_t)(blockIdx.x - thomas_blocks) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)(gridDim.x - thomas_blocks) * blockDim.x) >> 5;
    for (int64_t r = w; r < nruns; r += nw) {
      const int s0 = run_start[r], len = run_len[r];
      for (int l = lane; l < len; l += 32) y[s0 + l] = x[s0 + l] / diag[s0 + l];
    }
  }
}

// y = x / diag on the rows whose diagonal is not zero (the diagonal carries
// zeros on the column rows): eight rows per thread per pass, loads first.
// Launched as a programmatic dependent of the column sweeps (it shares no
// row of y with them), it waits for them only before it completes.
template <class T>
__global__ void __launch_bounds__(256) jacobi_sentinel(int64_t n, const T* __restrict__ x,
                                                       T* __restrict__ y,
                                                       const T* __restrict__ diag,
                                                       const int* skip) {
  if (skip && *((volatile const int*)skip)) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    return;
  }
  constexpr int U = 8;
  for (int64_t b0 = (int64_t)blockIdx.x * U * 256; b0 < n; b0 += (int64_t)gridDim.x * U * 256) {
    T dv[U], xv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = b0 + u * 256 + threadIdx.x;
      dv[u] = i < n ? __ldcs(diag + i) : T(0);
      xv[u] = i < n ? x[i] : T(0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = b0 + u * 256 + threadIdx.x;
      if (dv[u] != T(0)) y[i] = xv[u] / dv[u];
    }
  }
  // launched beside the column sweeps: this grid completes only after them,
  // so work queued after it sees both
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// shared memory of the staged sweeps (0: the column does not fit)
constexpr size_t kStageSmemMax = 200 * 1024;
size_t staged_smem(int nrow, size_t esz, bool sf) {
  const size_t b = (size_t)nrow * (kStageCols + 1) * esz * (sf ? 4 : 1);
  return b <= kStageSmemMax ? b : 0;
}
// factors are staged while the block's shared memory stays at most this
constexpr size_t kStageFactorsMax = 100 * 1024;
// resident blocks per SM given to the elementwise Jacobi rows beside the
// column sweeps (each loops over its share of the rows)
constexpr int kJacobiBlocksPerSm = 4;

template <class T, bool SF>
void launch_staged(lfx_ctx* ctx, const lfx_prec* p, const T* x, T* y, size_t smem,
                   const int* skip) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(cma_prec_staged<T, SF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kStageSmemMax);
    attr = true;
  }
  const int tb = (p->ncell_2d + kStageCols - 1) / kStageCols;
  if (p->rdiag && p->zero_sentinel) {
    // the column sweeps, then the Jacobi rows as a programmatic dependent
    // launch: its blocks start as soon as every sweep block has started and
    // fill the SMs beside them (the two write disjoint rows of y)
    cma_prec_staged<T, SF><<<tb, kStageThreads, smem, ctx->stream>>>(
        p->ncell_2d, p->nrow, p->first_dof, p->indirection, (const T*)p->fa, (const T*)p->finv,
        (const T*)p->fc, x, y, tb, 0, nullptr, nullptr, nullptr, skip);
    const int g = (int)std::max<int64_t>(
        1, std::min<int64_t>((p->rdiag_n + 8 * 256 - 1) / (8 * 256),
                             (int64_t)ctx->num_sms * kJacobiBlocksPerSm));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.gridDim = dim3((unsigned)g);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = ctx->stream;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, jacobi_sentinel<T>, p->rdiag_n, x, y, (const T*)p->rdiag, skip);
    ctx->launches++;
    return;
  }
  const int jb =
      p->nruns ? (int)std::min<int64_t>(((int64_t)p->nruns + 3) / 4, (int64_t)ctx->num_sms * 8) : 0;
  cma_prec_staged<T, SF><<<tb + jb, kStageThreads, smem, ctx->stream>>>(
      p->ncell_2d, p->nrow, p->first_dof, p->indirection, (const T*)p->fa, (const T*)p->finv,
      (const T*)p->fc, x, y, tb, p->nruns, p->run_start, p->run_len, (const T*)p->rdiag, skip);
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
      {
        const size_t esz = r64 ? 8 : 4;
        size_t smem = staged_smem(p->nrow, esz, true);
        const bool sf = smem && smem <= kStageFactorsMax;
        if (!sf) smem = staged_smem(p->nrow, esz, false);
        if (smem) {
          if (r64) {
            if (sf)
              launch_staged<double, true>(ctx, p, (const double*)x, (double*)y, smem, skip);
            else
              launch_staged<double, false>(ctx, p, (const double*)x, (double*)y, smem, skip);
          } else {
            if (sf)
              launch_staged<float, true>(ctx, p, (const float*)x, (float*)y, smem, skip);
            else
              launch_staged<float, false>(ctx, p, (const float*)x, (float*)y, smem, skip);
          }
          LFX_CK(ctx, cudaGetLastError());
          return LFX_OK;
        }
      }
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

template <class T>
static int zero_rows_t(lfx_ctx* ctx, lfx_prec* p, const std::vector<char>& cov) {
  const int64_t n = p->rdiag_n;
  std::vector<T> d((size_t)n);
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  LFX_CK(ctx, cudaMemcpy(d.data(), p->rdiag, n * sizeof(T), cudaMemcpyDeviceToHost));
  bool ok = true;
  for (int64_t i = 0; i < n; ++i) {
    if (cov[i])
      d[i] = T(0);
    else if (d[i] == T(0))
      ok = false;
  }
  LFX_CK(ctx, cudaMemcpy(p->rdiag, d.data(), n * sizeof(T), cudaMemcpyHostToDevice));
  p->jacobi_zeroed = true;
  p->zero_sentinel = ok;
  return LFX_OK;
}

static int zero_column_rows(lfx_ctx* ctx, lfx_prec* p, const std::vector<char>& cov) {
  return p->precision == LFX_R64 ? zero_rows_t<double>(ctx, p, cov)
                                 : zero_rows_t<float>(ctx, p, cov);
}

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
  if (!m->first_dof || m->nrow != m->ncol)
    return fail(ctx, LFX_NOT_SUPPORTED, "apply needs a square CMA operator with a dofmap");
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

// ------------------------------------------------------------------ CMA set-up
namespace {

bool band_consistent(int bw, int beta, int gm, int gp) {
  return beta >= 1 && gm >= 0 && gp >= 0 && bw >= 1 + ceil_div_i(gm + gp, beta);
}

BandArg arg_of(const lfx_cma* m) {
  return BandArg{m->band, m->nrow, m->ncol, m->bw, m->alpha, m->beta, m->gamma_m, m->gamma_p};
}

int gcd_i(int a, int b) {
  while (b) {
    const int t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// a map-free operator with a zero band: the parameters divided by
// gcd(alpha, beta) and bandwidth 1 + ceiling((g_m + g_p)/beta), as
// columnwise_operator_initialiser_custom (columnwise_operator_mod.f90:216-247)
int cma_new(lfx_ctx* ctx, int ncell_2d, int nrow, int ncol, int alpha, int beta, int gm, int gp,
            lfx_cma** out) {
  const int g = gcd_i(alpha, beta);
  if (g > 1) {
    alpha /= g;
    beta /= g;
    gm /= g;
    gp /= g;
  }
  const int bw = 1 + ceil_div_i(gm + gp, beta);
  return lfx_cma_create_banded(ctx, ncell_2d, nrow, ncol, bw, alpha, beta, gm, gp, nullptr, out);
}

int run_sync(lfx_ctx* ctx, const char* what) {
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(ctx->stream) != cudaSuccess)
    return fail(ctx, LFX_CUDA_ERROR, what);
  return LFX_OK;
}

int upload_cbd(lfx_ctx* ctx, const int32_t* cbd, size_t n, int** d) {
  int rc = dmalloc(ctx, (void**)d, 4 * n);
  if (!rc && cudaMemcpy(*d, cbd, 4 * n, cudaMemcpyHostToDevice) != cudaSuccess)
    rc = fail(ctx, LFX_CUDA_ERROR, "upload of column_banded_dofmap failed");
  return rc;
}

}  // namespace

int lfx_cma_create_banded(lfx_ctx* ctx, int32_t ncell_2d, int32_t nrow, int32_t ncol,
                          int32_t bandwidth, int32_t alpha, int32_t beta, int32_t gamma_m,
                          int32_t gamma_p, const double* columnwise_matrix, lfx_cma** out) {
  if (!ctx || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  if (ncell_2d < 1 || nrow < 1 || ncol < 1 || !band_consistent(bandwidth, beta, gamma_m, gamma_p))
    return fail(ctx, LFX_INVALID_ARGUMENT, "bad CMA dimensions or band parameters");
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
  const size_t bytes = 8 * (size_t)bandwidth * nrow * ncell_2d;
  int rc = dmalloc(ctx, (void**)&m->band, bytes);
  if (!rc) {
    if (columnwise_matrix)
      rc = cudaMemcpy(m->band, columnwise_matrix, bytes, cudaMemcpyHostToDevice) == cudaSuccess
               ? LFX_OK
               : fail(ctx, LFX_CUDA_ERROR, "band upload failed");
    else
      rc = cudaMemset(m->band, 0, bytes) == cudaSuccess ? LFX_OK
                                                         : fail(ctx, LFX_CUDA_ERROR, "memset failed");
  }
  if (rc) {
    lfx_cma_destroy(m);
    return rc;
  }
  *out = m;
  return LFX_OK;
}

int lfx_cma_set_dofmap(lfx_cma* m, const int32_t* first_dof, const int32_t* indirection) {
  if (!m || !first_dof || !indirection) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = m->ctx;
  if (m->nrow != m->ncol) return fail(ctx, LFX_NOT_SUPPORTED, "dofmaps for square operators only");
  std::vector<int32_t> f(m->ncell_2d), ind(m->nrow);
  int32_t maxf = 0, maxi = 0;
  for (int c = 0; c < m->ncell_2d; ++c) {
    f[c] = first_dof[c] - 1;
    if (f[c] < 0) return fail(ctx, LFX_INVALID_ARGUMENT, "first_dof must be >= 1");
    maxf = std::max(maxf, f[c]);
  }
  for (int i = 0; i < m->nrow; ++i) {
    ind[i] = indirection[i] - 1;
    if (ind[i] < 0) return fail(ctx, LFX_INVALID_ARGUMENT, "indirection entries must be >= 1");
    maxi = std::max(maxi, ind[i]);
  }
  if (!m->first_dof) {
    int rc = dmalloc(ctx, (void**)&m->first_dof, 4 * (size_t)m->ncell_2d);
    if (!rc) rc = dmalloc(ctx, (void**)&m->indirection, 4 * (size_t)m->nrow);
    if (rc) return rc;
  }
  LFX_CK(ctx, cudaMemcpy(m->first_dof, f.data(), 4 * f.size(), cudaMemcpyHostToDevice));
  LFX_CK(ctx, cudaMemcpy(m->indirection, ind.data(), 4 * ind.size(), cudaMemcpyHostToDevice));
  m->h_first = f;
  m->h_ind = ind;
  m->max_row = (int64_t)maxf + maxi;
  return LFX_OK;
}

// C += A B (columnwise_op_mul_kernel_code)
int lfx_cma_mul(const lfx_cma* A, const lfx_cma* B, lfx_cma* C) {
  if (!A || !B || !C) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = C->ctx;
  if (A->ncell_2d != B->ncell_2d || A->ncell_2d != C->ncell_2d || A->ncol != B->nrow ||
      C->nrow != A->nrow || C->ncol != B->ncol)
    return fail(ctx, LFX_INVALID_ARGUMENT, "operator shapes do not chain");
  for (const lfx_cma* m : std::initializer_list<const lfx_cma*>{A, B, C})
    if (!band_consistent(m->bw, m->beta, m->gamma_m, m->gamma_p))
      return fail(ctx, LFX_INVALID_ARGUMENT, "inconsistent band parameters");
  cma_mul<<<(C->ncell_2d + 127) / 128, 128, 0, ctx->stream>>>(C->ncell_2d, arg_of(A), arg_of(B),
                                                               arg_of(C));
  ctx->launches++;
  return run_sync(ctx, "CMA product failed");
}

// columnwise_operator_product (columnwise_operator_mod.f90) followed by the
// mul kernel: a new C = A B
int lfx_cma_product(const lfx_cma* A, const lfx_cma* B, lfx_cma** out) {
  if (!A || !B || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  lfx_cma* C = nullptr;
  int rc = cma_new(A->ctx, A->ncell_2d, A->nrow, B->ncol, A->alpha * B->alpha, A->beta * B->beta,
                   B->alpha * A->gamma_m + A->beta * B->gamma_m,
                   B->alpha * A->gamma_p + A->beta * B->gamma_p, &C);
  if (!rc) rc = lfx_cma_mul(A, B, C);
  if (rc) {
    lfx_cma_destroy(C);
    return rc;
  }
  *out = C;
  return LFX_OK;
}

// C = alpha A + beta B (columnwise_op_scaledadd_kernel_code); C's band must
// hold the bands of A and B row by row
int lfx_cma_scaledadd(const lfx_cma* A, const lfx_cma* B, lfx_cma* C, double alpha, double beta) {
  if (!A || !B || !C) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = C->ctx;
  if (A->ncell_2d != B->ncell_2d || A->ncell_2d != C->ncell_2d || C->nrow < A->nrow ||
      B->nrow < A->nrow)
    return fail(ctx, LFX_INVALID_ARGUMENT, "operator shapes differ");
  for (const lfx_cma* m : std::initializer_list<const lfx_cma*>{A, B, C})
    if (!band_consistent(m->bw, m->beta, m->gamma_m, m->gamma_p))
      return fail(ctx, LFX_INVALID_ARGUMENT, "inconsistent band parameters");
  for (int i = 1; i <= A->nrow; ++i) {
    const int jmC = ceil_div_i(C->alpha * i - C->gamma_p, C->beta);
    for (const lfx_cma* m : std::initializer_list<const lfx_cma*>{A, B}) {
      const int lo = std::max(1, ceil_div_i(m->alpha * i - m->gamma_p, m->beta));
      const int hi = std::min(A->ncol, floor_div_i(m->alpha * i + m->gamma_m, m->beta));
      if (lo <= hi && (lo - jmC < 0 || hi - jmC >= C->bw))
        return fail(ctx, LFX_INVALID_ARGUMENT, "C's band does not cover A and B");
    }
  }
  cma_scaledadd<<<(C->ncell_2d + 127) / 128, 128, 0, ctx->stream>>>(
      C->ncell_2d, arg_of(A), arg_of(B), arg_of(C), alpha, beta);
  ctx->launches++;
  return run_sync(ctx, "CMA scaled add failed");
}

// columnwise_operator_sum followed by the scaledadd kernel: a new C = alpha A + beta B
int lfx_cma_sum(const lfx_cma* A, const lfx_cma* B, double alpha, double beta, lfx_cma** out) {
  if (!A || !B || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  lfx_ctx* ctx = A->ctx;
  if (A->alpha != B->alpha || A->beta != B->beta)
    return fail(ctx, LFX_INVALID_ARGUMENT, "parameters alpha / beta of the operators differ");
  if (A->nrow != B->nrow || A->ncol != B->ncol)
    return fail(ctx, LFX_INVALID_ARGUMENT, "operator shapes differ");
  lfx_cma* C = nullptr;
  int rc = cma_new(ctx, A->ncell_2d, A->nrow, A->ncol, A->alpha, A->beta,
                   std::max(A->gamma_m, B->gamma_m), std::max(A->gamma_p, B->gamma_p), &C);
  if (!rc) rc = lfx_cma_scaledadd(A, B, C, alpha, beta);
  if (rc) {
    lfx_cma_destroy(C);
    return rc;
  }
  *out = C;
  return LFX_OK;
}

int lfx_cma_assemble_m2v_lumped_inv(const lfx_op* lma, const int32_t* column_banded_dofmap,
                                    int32_t alpha, int32_t beta, int32_t gamma_m, int32_t gamma_p,
                                    int32_t bandwidth, int32_t nrow, lfx_cma** out) {
  if (!lma || !column_banded_dofmap || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  lfx_ctx* ctx = lma->ctx;
  const lfx_lma_layout* L = lma->lay;
  if (lma->precision != LFX_R64 || L->ndf_to != L->ndf_from)
    return fail(ctx, LFX_INVALID_ARGUMENT, "lumped inverse needs a square FP64 LMA");
  const size_t ncbd = (size_t)L->ndf_to * L->nlayers;
  for (size_t q = 0; q < ncbd; ++q)
    if (column_banded_dofmap[q] < 1 || column_banded_dofmap[q] > nrow)
      return fail(ctx, LFX_INVALID_ARGUMENT, "column_banded_dofmap out of range");
  int rc = lfx_cma_create_banded(ctx, L->ncell_2d, nrow, nrow, bandwidth, alpha, beta, gamma_m,
                                 gamma_p, nullptr, out);
  if (rc) return rc;
  int* d_cbd = nullptr;
  rc = upload_cbd(ctx, column_banded_dofmap, ncbd, &d_cbd);
  if (!rc) {
    cma_m2v_lumped_inv<<<(L->ncell_2d + 127) / 128, 128, 0, ctx->stream>>>(
        L->ncell_2d, L->nlayers, L->ndf_to, lma->blk, (const double*)lma->mat, d_cbd,
        arg_of(*out));
    ctx->launches++;
    rc = run_sync(ctx, "lumped inverse assembly failed");
  }
  dfree(ctx, d_cbd, 4 * ncbd);
  if (rc) {
    lfx_cma_destroy(*out);
    *out = nullptr;
  }
  return rc;
}

int lfx_cma_assemble_diag_hmht(const lfx_op* Dh, const lfx_op* M2h,
                               const int32_t* column_banded_dofmap, int32_t alpha, int32_t beta,
                               int32_t gamma_m, int32_t gamma_p, int32_t bandwidth, int32_t nrow,
                               lfx_cma** out) {
  if (!Dh || !M2h || !column_banded_dofmap || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  lfx_ctx* ctx = Dh->ctx;
  const lfx_lma_layout *LD = Dh->lay, *LM = M2h->lay;
  if (Dh->precision != LFX_R64 || M2h->precision != LFX_R64)
    return fail(ctx, LFX_INVALID_ARGUMENT, "diag_hmht needs FP64 LMAs");
  if (LM->ndf_to != LM->ndf_from || LD->ndf_from != LM->ndf_to || LD->ncell_2d != LM->ncell_2d ||
      LD->nlayers != LM->nlayers)
    return fail(ctx, LFX_INVALID_ARGUMENT, "Dh (W2h -> W3) and M2h (W2h) do not match");
  const int ndf3 = LD->ndf_to, nl = LD->nlayers;
  if (beta < 1) return fail(ctx, LFX_INVALID_ARGUMENT, "beta must be positive");
  for (int k = 0; k < nl; ++k)
    for (int a = 0; a < ndf3; ++a) {
      const int i = column_banded_dofmap[a + ndf3 * k];
      if (i < 1 || i > nrow) return fail(ctx, LFX_INVALID_ARGUMENT, "column_banded_dofmap out of range");
      const int jm = ceil_div_i(alpha * i - gamma_p, beta);
      for (int b = 0; b < ndf3; ++b) {
        const int j = column_banded_dofmap[b + ndf3 * k];
        if (j - jm < 0 || j - jm >= bandwidth)
          return fail(ctx, LFX_INVALID_ARGUMENT, "entry falls outside the band");
      }
    }
  int rc = lfx_cma_create_banded(ctx, LD->ncell_2d, nrow, nrow, bandwidth, alpha, beta, gamma_m,
                                 gamma_p, nullptr, out);
  if (rc) return rc;
  int* d_cbd = nullptr;
  const size_t ncbd = (size_t)ndf3 * nl;
  rc = upload_cbd(ctx, column_banded_dofmap, ncbd, &d_cbd);
  if (!rc) {
    cma_diag_hmht<<<(LD->ncell_2d + 127) / 128, 128, 0, ctx->stream>>>(
        LD->ncell_2d, nl, ndf3, LM->ndf_to, Dh->blk, M2h->blk, (const double*)Dh->mat,
        (const double*)M2h->mat, d_cbd, arg_of(*out));
    ctx->launches++;
    rc = run_sync(ctx, "diag_hmht assembly failed");
  }
  dfree(ctx, d_cbd, 4 * ncbd);
  if (rc) {
    lfx_cma_destroy(*out);
    *out = nullptr;
  }
  return rc;
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
  if (!m->first_dof || m->nrow != m->ncol)
    return fail(ctx, LFX_NOT_SUPPORTED, "column inverse needs a square CMA operator with a dofmap");
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
    // zeros on the column rows mark them for the elementwise Jacobi pass,
    // unless an uncovered row has a zero diagonal of its own
    if (!rc) rc = zero_column_rows(ctx, p, cov);
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
