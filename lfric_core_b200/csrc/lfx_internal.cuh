// Internal definitions shared by the liblfx translation units.
//
// Reduction order (shared with the CPU oracle so FP64 results match bit for
// bit): a vector of n values is cut into chunks of RCHUNK = 2048; in chunk j,
// lane t (0..255) accumulates elements 2048 j + 256 m + t for m = 0..7 with
// acc = fma(a, b, acc); each warp combines its 32 lanes with a xor butterfly
// (16, 8, 4, 2, 1); the 8 warp sums are added left to right. The per-chunk
// partials are reduced by the last block to finish (atomic ticket) in the same
// way, lane t adding partials t, t + 256, ... in order. The result does not
// depend on the grid size.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "lfx.h"

// a start/stop event pair around one timed operator apply
struct TimedPair {
  cudaEvent_t a, b;
  int prec;
};

struct lfx_ctx {
  int device = 0;
  int num_sms = 148;
  int l2_bytes = 126 << 20;  // the device's L2 size (queried at creation)
  cudaStream_t stream = nullptr;
  std::string err;
  // reduction scratch: partials of up to 4 simultaneous sums, one ticket
  double* d_partials = nullptr;
  int64_t partials_cap = 0;  // doubles
  unsigned* d_ticket = nullptr;
  // small device scratch for scalar results of the C-ABI reductions
  double* d_scalars = nullptr;
  double* h_scalars = nullptr;      // pinned, mapped into the device's address space
  double* h_scalars_dev = nullptr;  // its device address
  int64_t device_bytes = 0;
  // operator-apply timing: event pairs, the precision of each timed apply,
  // and running totals per precision (index 0: FP64, 1: FP32)
  bool time_applies = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<int> ev_prec;
  int ev_used = 0;
  int64_t timed_launches[2] = {0, 0};
  double timed_ms[2] = {0.0, 0.0};
  int64_t launches = 0;  // kernels launched on this context
  int lma_kernel = -1;   // -1: per-operator choice, 0: force pipeline, 1: force gather
  int* d_err = nullptr;  // [0] set by a kernel whose bounded wait ran out; [2..3] grid barrier words
  // while a solver captures a CUDA graph, timed applies record into fresh
  // event pairs owned by that graph
  std::vector<TimedPair>* capture_ev = nullptr;
};

namespace lfx {

constexpr int RT = 256;
constexpr int RCHUNK = 2048;
constexpr int RPER = RCHUNK / RT;  // 8 elements per lane per chunk

// ---------------------------------------------------------------- errors
int fail(lfx_ctx* ctx, int status, const std::string& msg);
int cuda_fail(lfx_ctx* ctx, cudaError_t e, const char* what);

#define LFX_CK(ctx, call)                                   \
  do {                                                      \
    cudaError_t _e = (call);                                \
    if (_e != cudaSuccess) return lfx::cuda_fail((ctx), _e, #call); \
  } while (0)

// ---------------------------------------------------------------- memory
int dmalloc(lfx_ctx* ctx, void** p, size_t bytes);
void dfree(lfx_ctx* ctx, void* p, size_t bytes);
int ensure_partials(lfx_ctx* ctx, int64_t n, int nsums);

inline int64_t nchunks(int64_t n) { return (n + RCHUNK - 1) / RCHUNK; }
inline int grid_for(const lfx_ctx* ctx, int64_t n) {
  int64_t nc = nchunks(n);
  int64_t cap = (int64_t)ctx->num_sms * 32;
  int64_t g = nc < cap ? nc : cap;
  return (int)(g < 1 ? 1 : g);
}

// ---------------------------------------------------------------- device math
__device__ __forceinline__ double fmaT(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float fmaT(float a, float b, float c) { return fmaf(a, b, c); }

__device__ __forceinline__ double warp_butterfly(double v) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// block sum in the fixed order; result valid in thread 0
__device__ __forceinline__ double block_sum(double acc, double* sm) {
  acc = warp_butterfly(acc);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sm[w] = acc;
  __syncthreads();
  double tot = 0.0;
  if (threadIdx.x == 0) {
    tot = sm[0];
#pragma unroll
    for (int i = 1; i < RT / 32; ++i) tot = tot + sm[i];
  }
  __syncthreads();
  return tot;
}

// small tuples returned by the load phase of a chunk kernel
template <class T> struct V1 { T a; };
template <class T> struct V2 { T a, b; };
template <class T> struct V3 { T a, b, c; };
template <class T> struct V4 { T a, b, c, d; };

// Chunked elementwise kernel with NR fixed-order reductions.
//   ld(i)           : load phase for element i, returns a small tuple
//   op(i, v, acc)   : compute/store phase for element i, adds into acc[0..NR)
//   fin(tot)        : run by one thread after every chunk is done, tot[NR]
// All RPER loads of a lane are issued before any store, so stores (which the
// compiler must assume may alias) do not serialise the loads.
// skip: optional device flag; when non-zero the kernel does nothing (used by
// device-resident solvers to idle after convergence).
template <int NR, class Ld, class Op, class Fin>
__global__ void __launch_bounds__(RT) chunk_kernel(int64_t n, Ld ld, Op op, Fin fin,
                                                   double* partials, unsigned* ticket,
                                                   const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  __shared__ double sm[RT / 32];
  __shared__ int am_last;
  using V = decltype(ld(int64_t(0)));
  const int64_t nch = (n + RCHUNK - 1) / RCHUNK;
  for (int64_t ch = blockIdx.x; ch < nch; ch += gridDim.x) {
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int r = 0; r < (NR > 0 ? NR : 1); ++r) acc[r] = 0.0;
    const int64_t base = ch * RCHUNK + threadIdx.x;
    V v[RPER];
#pragma unroll
    for (int m = 0; m < RPER; ++m) {
      const int64_t i = base + (int64_t)m * RT;
      if (i < n) v[m] = ld(i);
    }
#pragma unroll
    for (int m = 0; m < RPER; ++m) {
      const int64_t i = base + (int64_t)m * RT;
      if (i < n) op(i, v[m], acc);
    }
    if constexpr (NR > 0) {
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        double t = block_sum(acc[r], sm);
        if (threadIdx.x == 0) partials[(int64_t)r * nch + ch] = t;
      }
    }
  }
  if constexpr (NR > 0) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (am_last) {
      __threadfence();
      double tot[NR];
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        double a = 0.0;
        for (int64_t i = threadIdx.x; i < nch; i += RT) a = a + __ldcg(&partials[(int64_t)r * nch + i]);
        tot[r] = block_sum(a, sm);
      }
      if (threadIdx.x == 0) {
        fin(tot);
        *ticket = 0u;
      }
    }
  }
}

struct NoFin {
  __device__ void operator()(const double*) const {}
};

template <int NR, class Ld, class Op, class Fin>
int launch_chunks(lfx_ctx* ctx, int64_t n, Ld ld, Op op, Fin fin, const int* skip = nullptr) {
  if (NR > 0) {
    int rc = ensure_partials(ctx, n, NR);
    if (rc) return rc;
  }
  chunk_kernel<NR><<<grid_for(ctx, n), RT, 0, ctx->stream>>>(n, ld, op, fin, ctx->d_partials,
                                                              ctx->d_ticket, skip);
  ctx->launches++;
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

// ints of one group and of one column in the per-column descriptors of the
// prefetching gather (fdesc of lfx_lma_layout)
__host__ __device__ constexpr int fd_group_ints(int ndf2) { return (2 + ndf2 + 3) / 4 * 4; }
__host__ __device__ constexpr int fd_ints(int ndf2) { return 4 + 2 * fd_group_ints(ndf2); }

// Thomas sweeps of one column with x-independent factors stored [row][column]
// (nc columns): y = T^{-1} x on rows f + ind[i], i < nrow, in FP64 with the
// forward result rounded to TX between the sweeps. The loads of R rows are
// issued ahead of their dependent recurrence steps, so a column costs about
// 2 nrow / R memory latencies instead of 2 nrow. Every row is read before it
// is written, so x == y is allowed.
template <int R, class TF, class TX>
__device__ __forceinline__ void thomas_sweep(int f, const int* __restrict__ ind, int nrow, int nc,
                                             int c, const TF* __restrict__ fa,
                                             const TF* __restrict__ finv,
                                             const TF* __restrict__ fc, const TX* x, TX* y) {
  double d = 0.0;
  for (int i0 = 0; i0 < nrow; i0 += R) {
    int mu[R];
    double xv[R], iv[R], av[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int i = i0 + j;
      if (i < nrow) {
        mu[j] = f + __ldg(ind + i);
        xv[j] = (double)x[mu[j]];
        iv[j] = (double)__ldg(finv + (size_t)i * nc + c);
        av[j] = (double)__ldg(fa + (size_t)i * nc + c);
      }
    }
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int i = i0 + j;
      if (i < nrow) {
        d = (i == 0) ? iv[j] * xv[j] : iv[j] * fma(-av[j], d, xv[j]);
        y[mu[j]] = (TX)d;
      }
    }
  }
  // back substitution; d holds row nrow-1, already final
  for (int i0 = nrow - 2; i0 >= 0; i0 -= R) {
    int mu[R];
    double yv[R], cv[R];
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int i = i0 - j;
      if (i >= 0) {
        mu[j] = f + __ldg(ind + i);
        yv[j] = (double)y[mu[j]];
        cv[j] = (double)__ldg(fc + (size_t)i * nc + c);
      }
    }
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int i = i0 - j;
      if (i >= 0) {
        d = fma(-cv[j], d, yv[j]);
        y[mu[j]] = (TX)d;
      }
    }
  }
}

}  // namespace lfx

// ---------------------------------------------------------------- objects

struct lfx_vec {
  lfx_ctx* ctx = nullptr;
  int32_t precision = LFX_R64;
  std::vector<int64_t> undf;
  std::vector<void*> data;
  size_t elem() const { return precision == LFX_R64 ? 8 : 4; }
};

// Gather form of the coloured LMA apply: for every to-space "entity column"
// (a run of consecutive dof ids touched by the same (cell, local dof) pairs)
// the device keeps the contributing cells in colour order and, per cell, the
// local dofs (df, vertical offset off) that land on the column. The dof
// base+l then receives M(c; l-off, df, df2) * x(map_from(c, df2) + l - off) in
// the reference's order: colour, cell, df2, df.
struct lfx_lma_layout {
  int32_t ncell_2d = 0, nlayers = 0, ndf_to = 0, ndf_from = 0;
  int64_t undf_to = 0, undf_from = 0;
  int32_t nent = 0, ngrp = 0, max_h = 0, max_off = 0, max_nrec = 0;
  bool full_cover = true;
  // device arrays
  int32_t* ent_base = nullptr;   // [nent] 0-based first dof
  int32_t* ent_h = nullptr;      // [nent] height
  int32_t* ent_grp = nullptr;    // [nent+1] group range
  int32_t* grp_cell = nullptr;   // [ngrp] 0-based cell
  uint32_t* grp_rec = nullptr;   // [ngrp] packed records
  int32_t* map_from = nullptr;   // [ncell_2d*ndf_from] 0-based
  int32_t* map_to = nullptr;     // [ncell_2d*ndf_to] 0-based
  // packed copies read by the fast kernels: per entity {base, h, g0, g1};
  // per group {cell, record, map_from row...} padded to gp_stride ints
  int4* ent_pack = nullptr;
  int32_t* grp_pack = nullptr;
  int32_t gp_stride = 0;
  // per entity column one descriptor of 32 * desc_ipl ints: {base, h, groups,
  // blocks} then per group {cell, record, map_from row} (0 when not built)
  int32_t* desc = nullptr;
  int32_t desc_ipl = 0;
  // per entity column fd_ints ints for the prefetching gather: {base, h,
  // groups, 0} then per group {cell, record, map_from row} padded to 4 ints
  // (built when a column reads at most two blocks from at most two cells)
  int32_t* fdesc = nullptr;
  int32_t fd_ints = 0;
  int32_t max_groups = 0;  // groups of one entity column, at most
  int32_t max_blocks = 0;  // (cell, df) matrix blocks one entity column reads, at most
  int refcount = 1;
  std::vector<int32_t> rank;         // colour-loop position of every cell
  lfx_lma_layout* tlay = nullptr;    // from-space layout for the transpose apply
  // cell-scatter plan (square operators on one dofmap whose dof columns each
  // get the same records from every cell that touches them, at most two per
  // cell at consecutive offsets): cells in colour-loop order with the start of
  // each colour, and per cell {map row, flags, partners} padded to cs_ints
  // ints, stored in the same colour-loop order. flags bit df: this cell is the first (in colour order) on the
  // column of df; bit 8+df: df is the lower record of a pair; bit 16+df: the
  // upper one; bit 24+df: this cell is the last on the column of df.
  // partners: 4 bits per df, the upper record of df's pair.
  bool cs_ok = false;
  int32_t cs_ints = 0;
  // the cells' vertical-pair structure (descriptor flag bits 8-23: lower and
  // upper records; partners) when every cell has the same one
  bool cs_uniform = false;
  uint32_t cs_struct_flags = 0, cs_struct_part = 0;
  std::vector<int32_t> colour_start;
  int32_t* cs_cells = nullptr;
  int32_t* cs_desc = nullptr;
};

struct lfx_op {
  lfx_ctx* ctx = nullptr;
  lfx_lma_layout* lay = nullptr;  // shared with ops made by lfx_lma_create_like
  int32_t precision = LFX_R64;
  // local matrices [cell][df][df2][k]; each (cell, df) block of ndf2*nlayers
  // values starts at a multiple of blk elements (blk*elem a multiple of 16
  // bytes, so a block is one aligned bulk copy)
  void* mat = nullptr;
  size_t mat_bytes = 0;
  int32_t blk = 0;
  // apply launch configuration (set by lfx_op_autotune; kernel -1 = default):
  // kernel 0 bulk-copy pipelined with `stages` and `warps` per block,
  // kernel 1 register gather, kernel 2 generic gather
  int32_t tune_kernel = -1, tune_stages = 0, tune_warps = 0;
  float tune_us = 0.f;
  // the upper triangle [q][p][k] of bitwise symmetric local matrices
  // (p = packed (df, df2), df <= df2), blocks in the colour-loop order of
  // the cell scatter (block q: cell cs_cells[q]), stride sblk elements; null
  // when the operator is not square on one dofmap or not symmetric
  void* smat = nullptr;
  size_t smat_bytes = 0;
  int32_t sblk = 0;
  // FP32 only, made on first use by the batch engine: the same upper
  // triangles level-major, [q][k][p] with each level's entries padded to a
  // multiple of four (lnpv float4 per level), so a lane loads its level with
  // 16-byte loads and a warp's levels are one contiguous run
  void* lmat = nullptr;
  size_t lmat_bytes = 0;
  int32_t lnpv = 0;
};

struct lfx_cma {
  lfx_ctx* ctx = nullptr;
  int32_t ncell_2d = 0, nrow = 0, ncol = 0, bw = 0, alpha = 0, beta = 0, gamma_m = 0, gamma_p = 0;
  int32_t* first_dof = nullptr;    // [ncell_2d] 0-based
  int32_t* indirection = nullptr;  // [nrow] 0-based offsets
  int32_t* ind_from = nullptr;     // [ncol] 0-based offsets
  double* band = nullptr;          // Fortran (bw, nrow, ncell_2d)
  std::vector<int32_t> h_first, h_ind;
  int64_t max_row = 0;             // largest 0-based dof the columns touch
};

enum { PREC_NULL = 0, PREC_DIAG = 1, PREC_CMA = 2 };
struct lfx_prec {
  lfx_ctx* ctx = nullptr;
  int kind = PREC_NULL;
  int32_t precision = LFX_R64;  // for PREC_CMA: the vectors it applies to
  const lfx_vec* diag = nullptr;  // not owned (PREC_DIAG)
  // PREC_CMA: factors [row][column]
  int32_t ncell_2d = 0, nrow = 0;
  int32_t* first_dof = nullptr;
  int32_t* indirection = nullptr;
  void* fa = nullptr;     // sub-diagonal a_i
  void* finv = nullptr;   // 1 / (b_i - a_i c'_{i-1})
  void* fc = nullptr;     // c'_i
  void* rdiag = nullptr;  // diagonal on uncovered rows, by run
  int32_t nruns = 0;
  int32_t* run_start = nullptr;
  int32_t* run_len = nullptr;
  int32_t* run_off = nullptr;  // offset of each run in rdiag
  int64_t rdiag_n = 0;
  size_t bytes = 0;
  int64_t max_row = -1;  // PREC_CMA: largest 0-based dof the columns touch
  bool jacobi_zeroed = false;  // PREC_CMA: rdiag zeroed on the column rows
  bool zero_sentinel = false;  // ... and non-zero on every other row
};

namespace lfx {
// The vertical-pair structure of the reference elements, as cell
// descriptors encode it (flag bits 8-15: lower records, 16-23: upper
// records; each lower dof's partner in its nibble): W0 (8 dofs), bottom
// vertices 0-3 under top vertices 4-7; W2 (6 dofs), the bottom face 4 under
// the top face 5. Other dof counts have none (never used with CANON).
template <int NDF>
struct Canon {
  static constexpr uint32_t lower = 0u, upper = 0u, part = 0u;
};
template <>
struct Canon<8> {
  static constexpr uint32_t lower = 0x0Fu, upper = 0xF0u, part = 0x7654u;
};
template <>
struct Canon<6> {
  static constexpr uint32_t lower = 0x10u, upper = 0x20u, part = 0x50000u;
};
inline bool layout_canon(const lfx_lma_layout* L, int ndf) {
  if (!L->cs_uniform || (ndf != 6 && ndf != 8)) return false;
  const uint32_t fl = ndf == 8 ? ((Canon<8>::lower << 8) | (Canon<8>::upper << 16))
                               : ((Canon<6>::lower << 8) | (Canon<6>::upper << 16));
  const uint32_t pt = ndf == 8 ? Canon<8>::part : Canon<6>::part;
  return L->cs_struct_flags == fl && L->cs_struct_part == pt;
}
// a descriptor's pair tests, compile-time constants with CANON
template <int NDF, bool CANON>
__device__ __forceinline__ bool is_lower(uint32_t flags, int df) {
  return CANON ? ((Canon<NDF>::lower >> df) & 1u) : ((flags >> (8 + df)) & 1u);
}
template <int NDF, bool CANON>
__device__ __forceinline__ bool is_upper(uint32_t flags, int df) {
  return CANON ? ((Canon<NDF>::upper >> df) & 1u) : ((flags >> (16 + df)) & 1u);
}
template <int NDF, bool CANON>
__device__ __forceinline__ int partner(uint32_t prt, int df) {
  return CANON ? (int)((Canon<NDF>::part >> (4 * df)) & 15u) : (int)((prt >> (4 * df)) & 15u);
}
}  // namespace lfx

namespace lfx {
int op_apply_impl(lfx_op* op, const void* x, void* y, const void* b, const int* skip);
// bytes of the level-major copy an FP32 operator with a packed copy would
// take, and its creation (a no-op when it exists); both LFX_NOT_SUPPORTED
// without an FP32 packed copy
size_t op_level_major_bytes(const lfx_op* op);
int op_level_major(lfx_op* op);
// flexible GMRES / GCR over the C ABI's vector calls (lfx_solver_flex.cu);
// work: FGMRES s, w, dx, Ax, res, v[gcrk], Pv[gcrk]; GCR dx, res, Ax, v, Pv
int fgmres_host(lfx_op* op, lfx_prec* prec, const lfx_solver_cfg& cfg,
                const std::vector<lfx_vec*>& work, lfx_vec* x, const lfx_vec* b,
                lfx_solve_info* info);
int gcr_host(lfx_op* op, lfx_prec* prec, const lfx_solver_cfg& cfg,
             const std::vector<lfx_vec*>& work, lfx_vec* x, const lfx_vec* b,
             lfx_solve_info* info);
int precondition_only_host(lfx_op* op, lfx_prec* prec, const lfx_solver_cfg& cfg,
                           const std::vector<lfx_vec*>& work, lfx_vec* x, const lfx_vec* b,
                           lfx_solve_info* info);
int jacobi_host(lfx_op* op, lfx_prec* prec, const lfx_solver_cfg& cfg, double rho_relax,
                const std::vector<lfx_vec*>& work, lfx_vec* x, const lfx_vec* b,
                lfx_solve_info* info);
int chebyshev_host(lfx_op* op, lfx_prec* prec, const lfx_solver_cfg& cfg, double lmin,
                   double lmax, const std::vector<lfx_vec*>& work, lfx_vec* x, const lfx_vec* b,
                   lfx_solve_info* info);
int prec_apply_impl(lfx_prec* p, int32_t precision, const void* x, void* y, int64_t n,
                    const int* skip);
// Small device -> host results go through pinned, device-mapped host memory
// written by a one-block kernel, not a copy engine: they never queue behind
// large field copies that other streams have in flight.
int host_alloc_mapped(lfx_ctx* ctx, void** host, void** dev, size_t bytes);
int to_host_small(lfx_ctx* ctx, void* host_dev, const void* dev, size_t bytes);
void timing_begin(lfx_ctx* ctx, int32_t precision);
void timing_end(lfx_ctx* ctx);
}  // namespace lfx
