// Batched, continuously admitted mixed-precision solves of many independent
// SPD systems (the W0 mass+diffusion and W2 Helmholtz operators are both SPD,
// with SPD Jacobi / column-tridiagonal preconditioners).
//
// Algorithm per slot: preconditioned CG whose recurrences, operator apply and
// preconditioner run in FP32, with reliable updates: the steps accumulate in
// an FP32 correction; when the FP32 recursive residual has fallen by a factor
// delta since the last true residual (or reaches the tolerance), the
// correction is added to the FP64 solution and the true residual b - A x is
// recomputed with the FP64 operator and replaces it. A slot converges only on
// that FP64 true residual, ||b - A x|| / ||b - A x0||.
//
// Batching: every kernel covers all slots -- entity columns, 8192-element
// chunks and CMA columns come from device work lists of (slot, item) pairs --
// and reads per-slot pointers and state from device tables, so one CUDA graph
// of `iters` super-iterations serves any set of admitted slots. Slots whose
// phase does not call for a kernel skip its items. Per-slot reductions sum in
// a fixed order (lanes, then warps, then chunks), with a completion ticket per
// slot, so a slot's result is bit-identical whatever else is in the batch.
// Vectors and list regions come from pools sized at creation: admitting a
// request allocates nothing, and is refused when the pools are full.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "lfx_internal.cuh"

using namespace lfx;

namespace {

enum { PH_EMPTY = 0, PH_INIT = 1, PH_RUN = 2, PH_DONE = 3 };

struct BSlot {
  // operator (gather layout shared by the FP32 and FP64 copies)
  const int4* ent_pack;
  const int32_t* grp_pack;
  const float* M32;
  const double* M64;
  int32_t gp_stride, nent, nl, ndf1;
  int32_t blk32, blk64, nch, part_off;
  int64_t n;
  // preconditioner: Jacobi diag (all rows) and, for the line kind, Thomas
  // factors [row][column] on the columns
  const float* diag;
  const float *fa, *finv, *fc;
  const int32_t *first, *ind;
  int32_t ncol, nrow;
  // vectors: x (FP64) moves only at true residuals; between them the FP32
  // xc accumulates the steps, x += xc then (a reliable update)
  const double* b;
  double* x;
  double* r64;
  float *r, *p, *z, *xc;
};

struct BState {
  int phase, flag, iter, status;
  int max_iter, fresh, pad0, pad1;
  double tol, r0, rlast, rnorm, rz, alpha, beta, true_rel;
};

constexpr double kDelta = 1e-3;  // reliable update when ||r|| drops by this factor

__device__ __forceinline__ bool ph_run(const BState& s) { return s.phase == PH_RUN; }
__device__ __forceinline__ bool ph_resid(const BState& s) {
  return s.phase == PH_INIT || (s.phase == PH_RUN && s.flag);
}
__device__ __forceinline__ bool ph_active(const BState& s) {
  return s.phase == PH_INIT || s.phase == PH_RUN;
}

// values of one batched chunk item: kBSub chunks of RCHUNK
constexpr int kBSub = 4;
inline int64_t bchunks(int64_t n) { return (n + (int64_t)kBSub * RCHUNK - 1) / ((int64_t)kBSub * RCHUNK); }

// Batched chunk kernel: items are (slot, chunk); ld/op as in chunk_kernel but
// with the slot's descriptor; fin(slot desc, state, tot) runs once per slot
// after all its chunks. A non-null gate that reads zero skips the launch; a
// non-null reset is cleared by the first thread.
template <int NR, class Pred, class Ld, class Op, class Fin>
__global__ void __launch_bounds__(RT) bchunk(const int2* list, const int* len, const BSlot* slots,
                                            BState* st, double* partials, unsigned* tickets,
                                            const int* gate, int* reset, Pred pred, Ld ld, Op op,
                                            Fin fin) {
  __shared__ double sm[RT / 32];
  __shared__ int am_last;
  if (gate && !*((volatile const int*)gate)) return;
  if (reset && blockIdx.x == 0 && threadIdx.x == 0) *reset = 0;
  const int L = *len;
  for (int u = blockIdx.x; u < L; u += gridDim.x) {
    const int2 w = list[u];
    if (w.x < 0) continue;
    BState& Sg = st[w.x];
    if (!pred(Sg)) continue;
    // local copies: the element loop's stores cannot alias them, so pointers
    // and scalars stay in registers
    const BSlot D = slots[w.x];
    const BState S = Sg;
    using V = decltype(ld(D, int64_t(0)));
    double acc[NR > 0 ? NR : 1];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = 0.0;
    // an item is kBSub consecutive 2048-value chunks, taken in order, each
    // with all its loads issued before its stores (one block reduction per
    // item: the fixed cost of an item is spread over more values)
    for (int sub = 0; sub < kBSub; ++sub) {
      const int64_t base = ((int64_t)w.y * kBSub + sub) * RCHUNK + threadIdx.x;
      if (base - threadIdx.x >= D.n) break;
      V v[RPER];
#pragma unroll
      for (int m = 0; m < RPER; ++m) {
        const int64_t i = base + (int64_t)m * RT;
        if (i < D.n) v[m] = ld(D, i);
      }
#pragma unroll
      for (int m = 0; m < RPER; ++m) {
        const int64_t i = base + (int64_t)m * RT;
        if (i < D.n) op(D, S, i, v[m], acc);
      }
    }
    if constexpr (NR > 0) {
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const double t = block_sum(acc[r], sm);
      if (threadIdx.x == 0) partials[D.part_off + (int64_t)r * D.nch + w.y] = t;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(&tickets[w.x], 1u) == (unsigned)D.nch - 1);
    __syncthreads();
    if (am_last) {
      __threadfence();
      double tot[NR > 0 ? NR : 1];
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        double a = 0.0;
        for (int i = threadIdx.x; i < D.nch; i += RT)
          a = a + __ldcg(&partials[D.part_off + (int64_t)r * D.nch + i]);
        tot[r] = block_sum(a, sm);
      }
      if (threadIdx.x == 0) {
        fin(D, Sg, tot);
        tickets[w.x] = 0u;
      }
      __syncthreads();
    }
    }
  }
}

// Batched LMA apply (register gather), items (slot, entity). RESID: y = b - A64 x
// with x = slot.x, y = slot.r64; else z = A32 p. A non-null gate that reads
// zero skips the launch.
template <int NDF2, bool RESID>
__global__ void __launch_bounds__(256) bapply(const int2* list, const int* len, const BSlot* slots,
                                              const BState* st, const int* gate) {
  using T = typename std::conditional<RESID, double, float>::type;
  if (gate && !*((volatile const int*)gate)) return;
  const int lane = threadIdx.x & 31;
  const int L = *len;
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int64_t u = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int2 wn = u < L ? list[u] : make_int2(-1, -1);
  for (; u < L; u += nwarp) {
    // the next item's list entry is loaded while this one is computed
    const int2 w = wn;
    wn = u + nwarp < L ? list[u + nwarp] : make_int2(-1, -1);
    if (w.x < 0) continue;
    if (RESID ? !ph_resid(st[w.x]) : !ph_run(st[w.x])) continue;
    // local copy: the stores below cannot alias it, so the pointers stay in
    // registers across the column loop
    const BSlot D = slots[w.x];
    const T* __restrict__ M = RESID ? (const T*)D.M64 : (const T*)D.M32;
    const int blk = RESID ? D.blk64 : D.blk32;
    const T* __restrict__ x = RESID ? (const T*)D.x : (const T*)D.p;
    T* __restrict__ y = RESID ? (T*)D.r64 : (T*)D.z;
    const int nl = D.nl;
    const size_t cell_stride = (size_t)D.ndf1 * blk;
    const int4 ep = __ldg(D.ent_pack + w.y);
    // all 32 lanes run every pass so the shuffles below see a converged warp
    for (int l0 = 0; l0 < ep.y; l0 += 32) {
      const int l = l0 + lane;
      T acc = T(0);
      for (int g = ep.z; g < ep.w; ++g) {
        // group record {cell, records, map_from row} as 16-byte vectors
        // (gp_stride is a multiple of 4 ints)
        const int4* gp4 = reinterpret_cast<const int4*>(D.grp_pack + (size_t)g * D.gp_stride);
        const int4 h0 = __ldg(gp4);
        const int c = h0.x;
        const uint32_t pk = (uint32_t)h0.y;
        int tmp[8];
        tmp[0] = h0.z;
        tmp[1] = h0.w;
        if (NDF2 > 2) {
          const int4 h1 = __ldg(gp4 + 1);
          tmp[2] = h1.x;
          tmp[3] = h1.y;
          tmp[4] = h1.z;
          tmp[5] = h1.w;
        }
        if (NDF2 > 6) {
          const int4 h2 = __ldg(gp4 + 2);
          tmp[6] = h2.x;
          tmp[7] = h2.y;
        }
        const int o0 = (pk >> 8) & 7u, o1 = (pk >> 17) & 7u;
        const int k0 = l - o0, k1 = l - o1;
        const bool v0 = (unsigned)k0 < (unsigned)nl;
        if ((pk & 3u) == 1) {
          // one record (warp-uniform branch): no second-record instructions
          const T* M0 = M + (size_t)c * cell_stride + (size_t)((pk >> 2) & 63u) * blk + (v0 ? k0 : 0);
          T a0[NDF2], b0[NDF2];
#pragma unroll
          for (int j = 0; j < NDF2; ++j) {
            a0[j] = v0 ? __ldg(M0 + j * nl) : T(0);
            b0[j] = v0 ? __ldg(x + tmp[j] + k0) : T(0);
          }
#pragma unroll
          for (int j = 0; j < NDF2; ++j)
            if (v0) acc = fmaT(a0[j], b0[j], acc);
          continue;
        }
        const bool v1 = (pk & 3u) > 1 && (unsigned)k1 < (unsigned)nl;
        // second record one level above the first: its x values are the
        // neighbouring lane's first-record values
        const bool pair = (pk & 3u) == 2 && o1 == o0 + 1;
        const T* Mc = M + (size_t)c * cell_stride;
        const T* M0 = Mc + (size_t)((pk >> 2) & 63u) * blk + (v0 ? k0 : 0);
        const T* M1 = Mc + (size_t)((pk >> 11) & 63u) * blk + (v1 ? k1 : 0);
        T a0[NDF2], b0[NDF2], a1[NDF2], b1[NDF2];
#pragma unroll
        for (int j = 0; j < NDF2; ++j) {
          a0[j] = v0 ? __ldg(M0 + j * nl) : T(0);
          b0[j] = v0 ? __ldg(x + tmp[j] + k0) : T(0);
          a1[j] = v1 ? __ldg(M1 + j * nl) : T(0);
        }
        if (pair) {
#pragma unroll
          for (int j = 0; j < NDF2; ++j) {
            const T up = __shfl_up_sync(0xffffffffu, b0[j], 1);
            b1[j] = (lane == 0) ? (v1 ? __ldg(x + tmp[j] + k1) : T(0)) : up;
          }
        } else {
#pragma unroll
          for (int j = 0; j < NDF2; ++j) b1[j] = v1 ? __ldg(x + tmp[j] + k1) : T(0);
        }
#pragma unroll
        for (int j = 0; j < NDF2; ++j) {
          if (v0) acc = fmaT(a0[j], b0[j], acc);
          if (v1) acc = fmaT(a1[j], b1[j], acc);
        }
      }
      if (l < ep.y) {
        const int row = ep.x + l;
        if (RESID)
          y[row] = (T)D.b[row] - acc;
        else
          y[row] = acc;
      }
    }
  }
}

// 16-byte asynchronous copies global -> shared and their groups
__device__ __forceinline__ void bcp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   (unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void bcp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bcp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Batched apply for 6-dof cells whose columns read at most two blocks from
// at most two cells (W2): the per-item column descriptors sit in list order
// in the batch's own pool (copied at admission), so each warp keeps the
// descriptors of its next kBFetchDepth items in flight (cp.async ring in
// shared memory) and an item waits on memory once, for its matrix rows and x
// values (matrix rows with streaming, evict-first loads). Same sums in the
// same order as bapply.
constexpr int kBFetchDepth = 4;

template <bool RESID>
__global__ void __launch_bounds__(256, RESID ? 2 : 3) bapply_fetch(const int2* list, const int* len,
                                                                   const BSlot* slots,
                                                                   const BState* st, const int* gate,
                                                                   const int* bdesc) {
  using T = typename std::conditional<RESID, double, float>::type;
  constexpr int NDF2 = 6, GS = fd_group_ints(NDF2), FS = fd_ints(NDF2), NV = FS / 4;
  __shared__ __align__(16) int ring[8][kBFetchDepth][FS];
  if (gate && !*((volatile const int*)gate)) return;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int L = *len;
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t e0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
#pragma unroll
  for (int q = 0; q < kBFetchDepth; ++q) {
    const int64_t e = e0 + q * nwarp;
    if (lane < NV && e < L) bcp_async16(&ring[wib][q][4 * lane], bdesc + e * FS + 4 * lane);
    bcp_commit();
  }
  int2 wn = e0 < L ? list[e0] : make_int2(-1, -1);
  int sl = 0;
  for (int64_t e = e0; e < L; e += nwarp) {
    bcp_wait<kBFetchDepth - 1>();
    __syncwarp();
    const int2 w = wn;
    wn = e + nwarp < L ? list[e + nwarp] : make_int2(-1, -1);
    const int* d = ring[wib][sl];
    if (w.x >= 0 && (RESID ? ph_resid(st[w.x]) : ph_run(st[w.x]))) {
      const BSlot* P = slots + w.x;
      const T* __restrict__ M = RESID ? (const T*)P->M64 : (const T*)P->M32;
      const int blk = RESID ? P->blk64 : P->blk32;
      const T* __restrict__ x = RESID ? (const T*)P->x : (const T*)P->p;
      T* __restrict__ y = RESID ? (T*)P->r64 : (T*)P->z;
      const double* __restrict__ bv = P->b;
      const int nl = P->nl;
      const size_t cell_stride = (size_t)NDF2 * blk;
      const int base = d[0], h = d[1], ng = d[2];
      for (int l0 = 0; l0 < h; l0 += 32) {
        const int l = l0 + lane;
        T acc = T(0);
        const uint32_t pk0 = (uint32_t)d[5];
        const int o0 = (pk0 >> 8) & 7u;
        const int k0 = l - o0;
        const bool v0 = (unsigned)k0 < (unsigned)nl;
        const T* M0 = M + (size_t)d[4] * cell_stride + (size_t)((pk0 >> 2) & 63u) * blk + (v0 ? k0 : 0);
        if (ng == 2) {
          const uint32_t pk1 = (uint32_t)d[5 + GS];
          const int k1 = l - (int)((pk1 >> 8) & 7u);
          const bool v1 = (unsigned)k1 < (unsigned)nl;
          const T* M1 = M + (size_t)d[4 + GS] * cell_stride + (size_t)((pk1 >> 2) & 63u) * blk +
                        (v1 ? k1 : 0);
          T a0[NDF2], b0[NDF2], a1[NDF2], b1[NDF2];
#pragma unroll
          for (int j = 0; j < NDF2; ++j) {
            a0[j] = v0 ? __ldcs(M0 + j * nl) : T(0);
            a1[j] = v1 ? __ldcs(M1 + j * nl) : T(0);
          }
#pragma unroll
          for (int j = 0; j < NDF2; ++j) {
            b0[j] = v0 ? __ldg(x + d[6 + j] + k0) : T(0);
            b1[j] = v1 ? __ldg(x + d[6 + GS + j] + k1) : T(0);
          }
#pragma unroll
          for (int j = 0; j < NDF2; ++j)
            if (v0) acc = fmaT(a0[j], b0[j], acc);
#pragma unroll
          for (int j = 0; j < NDF2; ++j)
            if (v1) acc = fmaT(a1[j], b1[j], acc);
        } else if ((pk0 & 3u) == 1) {
          T a0[NDF2], b0[NDF2];
#pragma unroll
          for (int j = 0; j < NDF2; ++j) {
            a0[j] = v0 ? __ldcs(M0 + j * nl) : T(0);
            b0[j] = v0 ? __ldg(x + d[6 + j] + k0) : T(0);
          }
#pragma unroll
          for (int j = 0; j < NDF2; ++j)
            if (v0) acc = fmaT(a0[j], b0[j], acc);
        } else {
          // one cell, two records (bottom and top of a column)
          const int o1 = (pk0 >> 17) & 7u;
          const int k1 = l - o1;
          const bool v1 = (unsigned)k1 < (unsigned)nl;
          const bool pair = o1 == o0 + 1;
          const T* M1 = M + (size_t)d[4] * cell_stride + (size_t)((pk0 >> 11) & 63u) * blk +
                        (v1 ? k1 : 0);
          T a0[NDF2], b0[NDF2], a1[NDF2], b1[NDF2];
#pragma unroll
          for (int j = 0; j < NDF2; ++j) {
            a0[j] = v0 ? __ldcs(M0 + j * nl) : T(0);
            b0[j] = v0 ? __ldg(x + d[6 + j] + k0) : T(0);
            a1[j] = v1 ? __ldcs(M1 + j * nl) : T(0);
          }
          if (pair) {
#pragma unroll
            for (int j = 0; j < NDF2; ++j) {
              const T up = __shfl_up_sync(0xffffffffu, b0[j], 1);
              b1[j] = (lane == 0) ? (v1 ? __ldg(x + d[6 + j] + k1) : T(0)) : up;
            }
          } else {
#pragma unroll
            for (int j = 0; j < NDF2; ++j) b1[j] = v1 ? __ldg(x + d[6 + j] + k1) : T(0);
          }
#pragma unroll
          for (int j = 0; j < NDF2; ++j) {
            if (v0) acc = fmaT(a0[j], b0[j], acc);
            if (v1) acc = fmaT(a1[j], b1[j], acc);
          }
        }
        if (l < h) {
          const int row = base + l;
          if (RESID)
            y[row] = (T)bv[row] - acc;
          else
            y[row] = acc;
        }
      }
    }
    __syncwarp();
    // the slot is free again: fetch the descriptor kBFetchDepth items ahead
    const int64_t en = e + kBFetchDepth * nwarp;
    if (lane < NV && en < L) bcp_async16(&ring[wib][sl][4 * lane], bdesc + en * FS + 4 * lane);
    bcp_commit();
    sl = sl + 1 == kBFetchDepth ? 0 : sl + 1;
  }
  bcp_wait<0>();
}

// Batched column-tridiagonal sweeps (the Jacobi part of the line
// preconditioner runs in the fused prec+dot chunk kernel), the rows of 64
// consecutive list items (columns, of any slots) staged through shared memory: one warp per column copies its
// rows in and out (a column's rows are contiguous dofs, so the copies
// coalesce), and each thread sweeps its column on the staged copy with the
// factors read from global memory (coalesced: [row][column]); same arithmetic
// as thomas_sweep. Admission refuses columns of more than kBRows rows.
constexpr int kBCols = 64, kBRows = 160, kBThreads = 128;

__global__ void __launch_bounds__(kBThreads) bthomas_staged(const int2* list, const int* len,
                                                             const BSlot* slots, const BState* st) {
  constexpr int LD = kBCols + 1, NW = kBThreads / 32, CPW = kBCols / NW;
  __shared__ float xs[kBRows * LD];
  // per column of the chunk: rows (0: nothing to do), first dof, indirection
  // and the slot's r and z (read once, so the copies below do not wait on
  // the list and slot records column by column)
  __shared__ int s_nrow[kBCols], s_f[kBCols];
  __shared__ const int* s_ind[kBCols];
  __shared__ const float* s_r[kBCols];
  __shared__ float* s_z[kBCols];
  __shared__ int s_maxrow;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int L = *len;
  for (int u0 = blockIdx.x * kBCols; u0 < L; u0 += gridDim.x * kBCols) {
    if (threadIdx.x == 0) s_maxrow = 0;
    __syncthreads();
    if (threadIdx.x < kBCols) {
      const int t = threadIdx.x, u = u0 + t;
      int nrow = 0;
      if (u < L) {
        const int2 w = list[u];
        if (w.x >= 0 && ph_active(st[w.x])) {
          const BSlot* D = slots + w.x;
          nrow = D->nrow;
          s_f[t] = __ldg(D->first + w.y);
          s_ind[t] = D->ind;
          s_r[t] = D->r;
          s_z[t] = D->z;
        }
      }
      s_nrow[t] = nrow;
      atomicMax(&s_maxrow, nrow);
    }
    __syncthreads();
    const int maxrow = s_maxrow;
    // stage: lane l copies row r0 + l of the warp's columns, loads first
    for (int r0 = 0; r0 < maxrow; r0 += 32) {
      const int i = r0 + lane;
      float v[CPW];
#pragma unroll
      for (int k = 0; k < CPW; ++k) {
        const int j = warp + NW * k;
        v[k] = i < s_nrow[j] ? s_r[j][s_f[j] + __ldg(s_ind[j] + i)] : 0.0f;
      }
#pragma unroll
      for (int k = 0; k < CPW; ++k) {
        const int j = warp + NW * k;
        if (i < s_nrow[j]) xs[i * LD + j] = v[k];
      }
    }
    __syncthreads();
    const int j = threadIdx.x;
    if (j < kBCols && s_nrow[j] > 0) {
      const int2 w = list[u0 + j];
      const BSlot* D = slots + w.x;
      const int nrow = s_nrow[j], nc = D->ncol, c = w.y;
      const float *fa = D->fa, *finv = D->finv, *fc = D->fc;
      float* col = xs + j;
      double d = 0.0;
      constexpr int R = 8;
      for (int i0 = 0; i0 < nrow; i0 += R) {
        double iv[R], av[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int i = i0 + q;
          if (i < nrow) {
            iv[q] = (double)__ldg(finv + (size_t)i * nc + c);
            av[q] = (double)__ldg(fa + (size_t)i * nc + c);
          }
        }
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int i = i0 + q;
          if (i < nrow) {
            const double xv = (double)col[i * LD];
            d = (i == 0) ? iv[q] * xv : iv[q] * fma(-av[q], d, xv);
            col[i * LD] = (float)d;
          }
        }
      }
      for (int i0 = nrow - 2; i0 >= 0; i0 -= R) {
        double cv[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int i = i0 - q;
          if (i >= 0) cv[q] = (double)__ldg(fc + (size_t)i * nc + c);
        }
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int i = i0 - q;
          if (i >= 0) {
            d = fma(-cv[q], d, (double)col[i * LD]);
            col[i * LD] = (float)d;
          }
        }
      }
    }
    __syncthreads();
    for (int r0 = 0; r0 < maxrow; r0 += 32) {
      const int i = r0 + lane;
#pragma unroll
      for (int k = 0; k < CPW; ++k) {
        const int jj = warp + NW * k;
        if (i < s_nrow[jj]) s_z[jj][s_f[jj] + __ldg(s_ind[jj] + i)] = xs[i * LD + jj];
      }
    }
    __syncthreads();
  }
}

}  // namespace

// host-side record of one slot
struct SlotHost {
  bool used = false;
  int64_t vec_off = 0, vec_len = 0;  // in the vector pools (elements)
  int64_t ent_off = 0, ent_len = 0, ch_off = 0, ch_len = 0, col_off = 0, col_len = 0;
  int64_t part_off = 0, part_len = 0;
  lfx_vec* x = nullptr;
  int64_t tag = 0;
};

struct lfx_batch {
  lfx_ctx* ctx = nullptr;
  int max_slots = 0, ndf = 0, iters = 4;
  int64_t cap_dofs = 0, cap_ent = 0, cap_ch = 0, cap_col = 0, cap_part = 0;
  BSlot* d_slots = nullptr;
  BSlot* h_slots = nullptr;
  BState* d_state = nullptr;
  BState* h_state = nullptr;  // pinned
  int2 *d_ent = nullptr, *d_ch = nullptr, *d_col = nullptr;
  int* d_len = nullptr;  // [3]: ent, chunk, col list lengths (high-water marks)
  int h_len[3] = {0, 0, 0};
  double* d_partials = nullptr;
  unsigned* d_tickets = nullptr;
  double* pool64 = nullptr;  // r64 per slot
  float* pool32 = nullptr;   // r, p, z, xc per slot (4 per dof)
  // per entity-list item, the column descriptor of the prefetching gather
  // (6-dof cells), copied from the slot's operator at admission
  int* d_bdesc = nullptr;
  std::vector<SlotHost> slots;
  cudaGraphExec_t graph = nullptr;
  int64_t graph_kernels = 0;
  size_t bytes = 0;
};

namespace {

// first fit in [0, cap) among the used ranges given by (off, len) of the slots
int64_t first_fit(const std::vector<SlotHost>& s, int64_t SlotHost::*off, int64_t SlotHost::*len,
                  int64_t need, int64_t cap) {
  std::vector<std::pair<int64_t, int64_t>> used;
  for (auto& x : s)
    if (x.used && x.*len) used.push_back({x.*off, x.*len});
  std::sort(used.begin(), used.end());
  int64_t at = 0;
  for (auto& u : used) {
    if (u.first - at >= need) return at;
    at = std::max(at, u.first + u.second);
  }
  return cap - at >= need ? at : -1;
}

template <class T>
int upload_region(lfx_ctx* ctx, T* dst, const std::vector<T>& src) {
  if (src.empty()) return LFX_OK;
  LFX_CK(ctx, cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice,
                              ctx->stream));
  return LFX_OK;
}

int set_lengths(lfx_batch* B) {
  int64_t e = 0, c = 0, k = 0;
  for (auto& s : B->slots)
    if (s.used) {
      e = std::max(e, s.ent_off + s.ent_len);
      c = std::max(c, s.ch_off + s.ch_len);
      k = std::max(k, s.col_off + s.col_len);
    }
  B->h_len[0] = (int)e;
  B->h_len[1] = (int)c;
  B->h_len[2] = (int)k;
  LFX_CK(B->ctx, cudaMemcpyAsync(B->d_len, B->h_len, sizeof(int) * 3, cudaMemcpyHostToDevice,
                                 B->ctx->stream));
  return LFX_OK;
}

// one super-iteration for every slot
template <int NDF2>
int launch_super(lfx_batch* B) {
  lfx_ctx* ctx = B->ctx;
  const int gridc = ctx->num_sms * 16;
  const int grida = ctx->num_sms * 16;
  BSlot* sl = B->d_slots;
  BState* st = B->d_state;
  const int* le = B->d_len;
  const int* lc = B->d_len + 1;
  const int* lk = B->d_len + 2;
  // nonzero while some slot needs a true residual this super-iteration: set
  // by admission and by step 3, cleared by step 6
  int* need = B->d_len + 3;
  double* pa = B->d_partials;
  unsigned* tk = B->d_tickets;
  auto run = [] __device__(const BState& s) { return ph_run(s); };
  auto resid = [] __device__(const BState& s) { return ph_resid(s); };
  auto active = [] __device__(const BState& s) { return ph_active(s); };
  // 1. z = A32 p
  if constexpr (NDF2 == 6)
    bapply_fetch<false><<<ctx->num_sms * 3, 256, 0, ctx->stream>>>(B->d_ent, le, sl, st, nullptr,
                                                                    B->d_bdesc);
  else
    bapply<NDF2, false><<<grida, 256, 0, ctx->stream>>>(B->d_ent, le, sl, st, nullptr);
  // 2. alpha = rz / <p, z>
  bchunk<1><<<gridc, RT, 0, ctx->stream>>>(
      B->d_ch, lc, sl, st, pa, tk, nullptr, nullptr, run,
      [] __device__(const BSlot& D, int64_t i) { return V2<float>{D.p[i], D.z[i]}; },
      [] __device__(const BSlot&, const BState&, int64_t, const V2<float>& v, double* a) {
        a[0] = fma((double)v.a, (double)v.b, a[0]);
      },
      [] __device__(const BSlot&, BState& S, const double* t) { S.alpha = S.rz / t[0]; });
  // 3. xc += alpha p, r -= alpha z (FP32); ||r||; decide on a true residual
  bchunk<1><<<gridc, RT, 0, ctx->stream>>>(
      B->d_ch, lc, sl, st, pa, tk, nullptr, nullptr, run,
      [] __device__(const BSlot& D, int64_t i) {
        return V4<float>{D.xc[i], D.p[i], D.r[i], D.z[i]};
      },
      [] __device__(const BSlot& D, const BState& S, int64_t i, const V4<float>& v, double* a) {
        D.xc[i] = fmaf((float)S.alpha, v.b, v.a);
        const float ri = fmaf((float)(-S.alpha), v.d, v.c);
        D.r[i] = ri;
        a[0] = fma((double)ri, (double)ri, a[0]);
      },
      [need] __device__(const BSlot&, BState& S, const double* t) {
        S.iter += 1;
        S.rnorm = sqrt(t[0]);
        if (S.rnorm <= kDelta * S.rlast || S.rnorm <= S.tol * S.r0 || S.iter >= S.max_iter ||
            !(S.rnorm == S.rnorm)) {
          S.flag = 1;
          *need = 1;
        }
      });
  // 3b. reliable update: x += xc (FP64), xc = 0 (new slots: xc = 0)
  bchunk<0><<<gridc, RT, 0, ctx->stream>>>(
      B->d_ch, lc, sl, st, pa, tk, need, nullptr, resid,
      [] __device__(const BSlot& D, int64_t i) { return V2<double>{D.x[i], (double)D.xc[i]}; },
      [] __device__(const BSlot& D, const BState& S, int64_t i, const V2<double>& v, double*) {
        if (S.phase != PH_INIT) D.x[i] = v.a + v.b;
        D.xc[i] = 0.0f;
      },
      [] __device__(const BSlot&, BState&, const double*) {});
  // 4. r64 = b - A64 x (new slots, and slots taking a true residual)
  if constexpr (NDF2 == 6)
    bapply_fetch<true><<<ctx->num_sms * 2, 256, 0, ctx->stream>>>(B->d_ent, le, sl, st, need,
                                                                   B->d_bdesc);
  else
    bapply<NDF2, true><<<grida, 256, 0, ctx->stream>>>(B->d_ent, le, sl, st, need);
  // 5. ||r64||, r = r64 (FP32); convergence on the true residual
  bchunk<1><<<gridc, RT, 0, ctx->stream>>>(
      B->d_ch, lc, sl, st, pa, tk, need, nullptr, resid,
      [] __device__(const BSlot& D, int64_t i) { return V1<double>{D.r64[i]}; },
      [] __device__(const BSlot& D, const BState&, int64_t i, const V1<double>& v, double* a) {
        D.r[i] = (float)v.a;
        a[0] = fma(v.a, v.a, a[0]);
      },
      [] __device__(const BSlot&, BState& S, const double* t) {
        const double nr = sqrt(t[0]);
        if (S.phase == PH_INIT) {
          S.r0 = nr;
          S.rlast = nr;
          S.true_rel = nr > 0.0 ? 1.0 : 0.0;
          if (nr < DBL_EPSILON) {
            S.phase = PH_DONE;
            S.true_rel = 0.0;
          }
          return;
        }
        S.flag = 0;
        S.rlast = nr;
        S.true_rel = nr / S.r0;
        if (S.true_rel <= S.tol) {
          S.phase = PH_DONE;
        } else if (!(nr == nr)) {
          S.phase = PH_DONE;
          S.status = LFX_NAN_DETECTED;
        } else if (S.iter >= S.max_iter) {
          S.phase = PH_DONE;
          S.status = LFX_NOT_CONVERGED;
        }
      });
  // 6. z = P r (column sweeps for the line kind), then the Jacobi rows fused
  //    with rz_new = <r, z> and beta
  if (B->cap_col > 0)
    bthomas_staged<<<ctx->num_sms * 8, kBThreads, 0, ctx->stream>>>(B->d_col, lk, sl, st);
  bchunk<1><<<gridc, RT, 0, ctx->stream>>>(
      B->d_ch, lc, sl, st, pa, tk, nullptr, need, active,
      [] __device__(const BSlot& D, int64_t i) { return V3<float>{D.r[i], D.diag[i], D.z[i]}; },
      [] __device__(const BSlot& D, const BState&, int64_t i, const V3<float>& v, double* a) {
        // rows with a positive diagonal entry are Jacobi rows; the column rows
        // (written by the sweeps) carry a zero in the Jacobi diagonal
        float zi = v.c;
        if (v.b != 0.0f) {
          zi = v.a / v.b;
          D.z[i] = zi;
        }
        a[0] = fma((double)v.a, (double)zi, a[0]);
      },
      [] __device__(const BSlot&, BState& S, const double* t) {
        S.beta = S.fresh ? 0.0 : t[0] / S.rz;
        S.rz = t[0];
      });
  // 7. p = z + beta p (p = z for a new slot); new slots start iterating
  bchunk<1><<<gridc, RT, 0, ctx->stream>>>(
      B->d_ch, lc, sl, st, pa, tk, nullptr, nullptr, active,
      [] __device__(const BSlot& D, int64_t i) { return V2<float>{D.p[i], D.z[i]}; },
      [] __device__(const BSlot& D, const BState& S, int64_t i, const V2<float>& v, double*) {
        D.p[i] = S.fresh ? v.b : fmaf((float)S.beta, v.a, v.b);
      },
      [] __device__(const BSlot&, BState& S, const double*) {
        S.fresh = 0;
        if (S.phase == PH_INIT) S.phase = PH_RUN;
      });
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

int capture(lfx_batch* B) {
  lfx_ctx* ctx = B->ctx;
  cudaGraph_t g = nullptr;
  LFX_CK(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  int rc = LFX_OK;
  for (int it = 0; it < B->iters && !rc; ++it)
    rc = B->ndf == 8 ? launch_super<8>(B) : launch_super<6>(B);
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  if (rc || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return rc ? rc : cuda_fail(ctx, e, "cudaStreamEndCapture");
  }
  e = cudaGraphInstantiate(&B->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
  B->graph_kernels = (B->cap_col > 0 ? 9 : 8) * (int64_t)B->iters;
  return LFX_OK;
}

}  // namespace

extern "C" {

int lfx_batch_create(lfx_ctx* ctx, int32_t ndf, int32_t max_slots, int64_t max_dofs,
                     int64_t max_entities, int64_t max_columns, int32_t iters_per_launch,
                     lfx_batch** out) {
  if (!ctx || !out || (ndf != 6 && ndf != 8) || max_slots < 1 || max_dofs < 1 ||
      max_entities < 1 || iters_per_launch < 1)
    return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  lfx_batch* B = new lfx_batch();
  B->ctx = ctx;
  B->ndf = ndf;
  B->max_slots = max_slots;
  B->iters = iters_per_launch;
  B->cap_dofs = max_dofs;
  B->cap_ent = max_entities;
  B->cap_ch = nchunks(max_dofs) + max_slots;
  B->cap_col = max_columns;
  B->cap_part = 2 * B->cap_ch;
  B->slots.resize(max_slots);
  int rc = dmalloc(ctx, (void**)&B->d_slots, sizeof(BSlot) * max_slots);
  if (!rc) rc = dmalloc(ctx, (void**)&B->d_state, sizeof(BState) * max_slots);
  if (!rc) rc = dmalloc(ctx, (void**)&B->d_ent, sizeof(int2) * B->cap_ent);
  if (!rc) rc = dmalloc(ctx, (void**)&B->d_ch, sizeof(int2) * B->cap_ch);
  if (!rc && B->cap_col) rc = dmalloc(ctx, (void**)&B->d_col, sizeof(int2) * B->cap_col);
  if (!rc) rc = dmalloc(ctx, (void**)&B->d_len, sizeof(int) * 4);
  if (!rc) rc = dmalloc(ctx, (void**)&B->d_partials, sizeof(double) * B->cap_part);
  if (!rc) rc = dmalloc(ctx, (void**)&B->d_tickets, sizeof(unsigned) * max_slots);
  if (!rc) rc = dmalloc(ctx, (void**)&B->pool64, sizeof(double) * max_dofs);
  if (!rc) rc = dmalloc(ctx, (void**)&B->pool32, sizeof(float) * 4 * max_dofs);
  if (!rc && ndf == 6)
    rc = dmalloc(ctx, (void**)&B->d_bdesc, sizeof(int) * fd_ints(6) * B->cap_ent);
  if (!rc && cudaMallocHost((void**)&B->h_state, sizeof(BState) * max_slots) != cudaSuccess)
    rc = LFX_OUT_OF_MEMORY;
  B->h_slots = new BSlot[max_slots];
  if (!rc) {
    memset(B->h_slots, 0, sizeof(BSlot) * max_slots);
    memset(B->h_state, 0, sizeof(BState) * max_slots);
    cudaMemsetAsync(B->d_state, 0, sizeof(BState) * max_slots, ctx->stream);
    cudaMemsetAsync(B->d_tickets, 0, sizeof(unsigned) * max_slots, ctx->stream);
    cudaMemsetAsync(B->d_len, 0, sizeof(int) * 4, ctx->stream);
    cudaMemsetAsync(B->d_slots, 0, sizeof(BSlot) * max_slots, ctx->stream);
    // list entries start out as "no slot"
    cudaMemsetAsync(B->d_ent, 0xff, sizeof(int2) * B->cap_ent, ctx->stream);
    cudaMemsetAsync(B->d_ch, 0xff, sizeof(int2) * B->cap_ch, ctx->stream);
    if (B->cap_col) cudaMemsetAsync(B->d_col, 0xff, sizeof(int2) * B->cap_col, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = LFX_CUDA_ERROR;
  }
  if (!rc) rc = capture(B);
  if (rc) {
    lfx_batch_destroy(B);
    return rc;
  }
  *out = B;
  return LFX_OK;
}

int lfx_batch_destroy(lfx_batch* B) {
  if (!B) return LFX_OK;
  lfx_ctx* ctx = B->ctx;
  if (B->graph) cudaGraphExecDestroy(B->graph);
  dfree(ctx, B->d_slots, sizeof(BSlot) * B->max_slots);
  dfree(ctx, B->d_state, sizeof(BState) * B->max_slots);
  dfree(ctx, B->d_ent, sizeof(int2) * B->cap_ent);
  dfree(ctx, B->d_ch, sizeof(int2) * B->cap_ch);
  dfree(ctx, B->d_col, sizeof(int2) * B->cap_col);
  dfree(ctx, B->d_len, sizeof(int) * 4);
  dfree(ctx, B->d_partials, sizeof(double) * B->cap_part);
  dfree(ctx, B->d_tickets, sizeof(unsigned) * B->max_slots);
  dfree(ctx, B->pool64, sizeof(double) * B->cap_dofs);
  dfree(ctx, B->pool32, sizeof(float) * 4 * B->cap_dofs);
  if (B->d_bdesc) dfree(ctx, B->d_bdesc, sizeof(int) * fd_ints(6) * B->cap_ent);
  if (B->h_state) cudaFreeHost(B->h_state);
  delete[] B->h_slots;
  delete B;
  return LFX_OK;
}

// Admits one solve A x = b into a free slot: op64 / op32 the FP64 and FP32
// copies of one operator (same layout), prec32 its FP32 Jacobi or column
// preconditioner, b and x FP64 vectors (x is the initial guess and receives
// the solution; both must stay alive until the slot is retired).
int lfx_batch_admit(lfx_batch* B, lfx_op* op64, lfx_op* op32, lfx_prec* prec32, const lfx_vec* b,
                    lfx_vec* x, double tol, int32_t max_iter, int64_t tag, int32_t* slot_out) {
  if (!B || !op64 || !op32 || !prec32 || !b || !x || !slot_out) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = B->ctx;
  *slot_out = -1;
  const lfx_lma_layout* L = op64->lay;
  if (op32->lay != L || op64->precision != LFX_R64 || op32->precision != LFX_R32)
    return fail(ctx, LFX_TYPE_MISMATCH, "batch needs FP64 and FP32 copies of one operator");
  if (L->ndf_from != B->ndf || L->ndf_to != B->ndf || L->max_nrec > 2 || !L->ent_pack)
    return fail(ctx, LFX_NOT_SUPPORTED, "operator shape does not match the batch");
  if (B->ndf == 6 && (!L->fdesc || L->fd_ints != fd_ints(6)))
    return fail(ctx, LFX_NOT_SUPPORTED,
                "batch of 6-dof cells needs columns reading at most two blocks from two cells");
  if (prec32->precision != LFX_R32 || (prec32->kind != PREC_DIAG && prec32->kind != PREC_CMA) ||
      !prec32->rdiag || prec32->rdiag_n != L->undf_to)
    return fail(ctx, LFX_NOT_SUPPORTED, "batch needs an FP32 Jacobi or column preconditioner with a diagonal");
  if (prec32->kind == PREC_CMA && prec32->nrow > kBRows)
    return fail(ctx, LFX_NOT_SUPPORTED, "batch column preconditioner: at most 160 rows per column");
  if (b->precision != LFX_R64 || x->precision != LFX_R64 || b->undf[0] != L->undf_to ||
      x->undf[0] != L->undf_to)
    return fail(ctx, LFX_TYPE_MISMATCH, "b and x must be FP64 vectors of the operator's space");
  int s = -1;
  for (int i = 0; i < B->max_slots; ++i)
    if (!B->slots[i].used) {
      s = i;
      break;
    }
  if (s < 0) return fail(ctx, LFX_OUT_OF_MEMORY, "no free batch slot");
  const int64_t n = L->undf_to;
  const int64_t nch = bchunks(n);
  const int64_t ncol = prec32->kind == PREC_CMA ? prec32->ncell_2d : 0;
  SlotHost& H = B->slots[s];
  H = SlotHost();
  H.vec_len = n;
  H.ent_len = L->nent;
  H.ch_len = nch;
  H.col_len = ncol;
  H.part_len = 2 * nch;
  H.vec_off = first_fit(B->slots, &SlotHost::vec_off, &SlotHost::vec_len, n, B->cap_dofs);
  H.ent_off = first_fit(B->slots, &SlotHost::ent_off, &SlotHost::ent_len, H.ent_len, B->cap_ent);
  H.ch_off = first_fit(B->slots, &SlotHost::ch_off, &SlotHost::ch_len, nch, B->cap_ch);
  H.col_off = ncol ? first_fit(B->slots, &SlotHost::col_off, &SlotHost::col_len, ncol, B->cap_col) : 0;
  H.part_off = first_fit(B->slots, &SlotHost::part_off, &SlotHost::part_len, 2 * nch, B->cap_part);
  if (H.vec_off < 0 || H.ent_off < 0 || H.ch_off < 0 || H.col_off < 0 || H.part_off < 0) {
    H = SlotHost();
    return fail(ctx, LFX_OUT_OF_MEMORY, "batch pools are full");
  }
  H.used = true;
  H.x = x;
  H.tag = tag;
  // descriptor
  BSlot D{};
  D.ent_pack = L->ent_pack;
  D.grp_pack = L->grp_pack;
  D.M32 = (const float*)op32->mat;
  D.M64 = (const double*)op64->mat;
  D.gp_stride = L->gp_stride;
  D.nent = L->nent;
  D.nl = L->nlayers;
  D.ndf1 = L->ndf_to;
  D.blk32 = op32->blk;
  D.blk64 = op64->blk;
  D.nch = (int32_t)nch;
  D.part_off = (int32_t)H.part_off;
  D.n = n;
  D.diag = (const float*)prec32->rdiag;
  if (prec32->kind == PREC_CMA) {
    D.fa = (const float*)prec32->fa;
    D.finv = (const float*)prec32->finv;
    D.fc = (const float*)prec32->fc;
    D.first = prec32->first_dof;
    D.ind = prec32->indirection;
    D.ncol = prec32->ncell_2d;
    D.nrow = prec32->nrow;
  }
  D.b = (const double*)b->data[0];
  D.x = (double*)x->data[0];
  D.r64 = B->pool64 + H.vec_off;
  D.r = B->pool32 + 4 * H.vec_off;
  D.p = D.r + n;
  D.z = D.p + n;
  D.xc = D.z + n;
  B->h_slots[s] = D;
  BState S{};
  S.phase = PH_INIT;
  S.fresh = 1;
  S.tol = tol;
  S.max_iter = max_iter;
  B->h_state[s] = S;
  // the line preconditioner's Jacobi diagonal must carry zeros on the column
  // rows (the fused kernel tells the two kinds of row apart by it)
  int rc = LFX_OK;
  if (prec32->kind == PREC_CMA && !prec32->jacobi_zeroed) {
    std::vector<float> d(n);
    LFX_CK(ctx, cudaMemcpy(d.data(), prec32->rdiag, n * 4, cudaMemcpyDeviceToHost));
    std::vector<int32_t> f(prec32->ncell_2d), ind(prec32->nrow);
    LFX_CK(ctx, cudaMemcpy(f.data(), prec32->first_dof, f.size() * 4, cudaMemcpyDeviceToHost));
    LFX_CK(ctx, cudaMemcpy(ind.data(), prec32->indirection, ind.size() * 4, cudaMemcpyDeviceToHost));
    // (the single-solve preconditioner reads this diagonal on the other rows only)
    for (size_t c = 0; c < f.size(); ++c)
      for (size_t i = 0; i < ind.size(); ++i) d[(size_t)f[c] + ind[i]] = 0.0f;
    LFX_CK(ctx, cudaMemcpy(prec32->rdiag, d.data(), n * 4, cudaMemcpyHostToDevice));
    prec32->jacobi_zeroed = true;
  }
  std::vector<int2> ent(H.ent_len), ch(nch), col(ncol);
  for (int64_t e = 0; e < H.ent_len; ++e) ent[e] = make_int2(s, (int)e);
  for (int64_t c = 0; c < nch; ++c) ch[c] = make_int2(s, (int)c);
  for (int64_t c = 0; c < ncol; ++c) col[c] = make_int2(s, (int)c);
  rc = upload_region(ctx, B->d_ent + H.ent_off, ent);
  if (!rc && B->d_bdesc)
    LFX_CK(ctx, cudaMemcpyAsync(B->d_bdesc + (size_t)H.ent_off * fd_ints(6), L->fdesc,
                                sizeof(int) * fd_ints(6) * H.ent_len, cudaMemcpyDeviceToDevice,
                                ctx->stream));
  if (!rc) rc = upload_region(ctx, B->d_ch + H.ch_off, ch);
  if (!rc && ncol) rc = upload_region(ctx, B->d_col + H.col_off, col);
  if (!rc) LFX_CK(ctx, cudaMemcpyAsync(B->d_slots + s, &B->h_slots[s], sizeof(BSlot),
                                       cudaMemcpyHostToDevice, ctx->stream));
  if (!rc) LFX_CK(ctx, cudaMemcpyAsync(B->d_state + s, &B->h_state[s], sizeof(BState),
                                       cudaMemcpyHostToDevice, ctx->stream));
  // the new slot takes its first residual in the next super-iteration
  if (!rc) LFX_CK(ctx, cudaMemsetAsync(B->d_len + 3, 1, sizeof(int), ctx->stream));
  if (!rc) rc = set_lengths(B);
  if (rc) {
    H = SlotHost();
    return rc;
  }
  *slot_out = s;
  return LFX_OK;
}

// Runs one replay (iters super-iterations) for every admitted slot, then
// reads the slot states. *ndone receives the number of slots that are done
// (converged or failed) and not yet retired.
int lfx_batch_step(lfx_batch* B, int32_t* ndone) {
  if (!B) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = B->ctx;
  LFX_CK(ctx, cudaGraphLaunch(B->graph, ctx->stream));
  ctx->launches += B->graph_kernels;
  LFX_CK(ctx, cudaMemcpyAsync(B->h_state, B->d_state, sizeof(BState) * B->max_slots,
                              cudaMemcpyDeviceToHost, ctx->stream));
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  int nd = 0;
  for (int s = 0; s < B->max_slots; ++s)
    if (B->slots[s].used && B->h_state[s].phase == PH_DONE) ++nd;
  if (ndone) *ndone = nd;
  return LFX_OK;
}

// Slot state: 0 empty, 1 starting, 2 iterating, 3 done.
int lfx_batch_slot_info(const lfx_batch* B, int32_t slot, int32_t* phase, int64_t* tag,
                        lfx_solve_info* info) {
  if (!B || slot < 0 || slot >= B->max_slots) return LFX_INVALID_ARGUMENT;
  const BState& S = B->h_state[slot];
  if (phase) *phase = B->slots[slot].used ? S.phase : PH_EMPTY;
  if (tag) *tag = B->slots[slot].tag;
  if (info) {
    memset(info, 0, sizeof *info);
    info->iterations = S.iter;
    info->converged = S.phase == PH_DONE && S.status == 0;
    info->initial_norm = S.r0;
    info->final_norm = S.rlast;
    info->final_rel = S.true_rel;
    info->status = S.status;
  }
  return LFX_OK;
}

// Frees a done (or any) slot for new admissions.
int lfx_batch_retire(lfx_batch* B, int32_t slot) {
  if (!B || slot < 0 || slot >= B->max_slots) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = B->ctx;
  SlotHost& H = B->slots[slot];
  if (!H.used) return LFX_OK;
  // mark its list items and state empty on the device
  std::vector<int2> none_e(H.ent_len, make_int2(-1, -1)), none_c(H.ch_len, make_int2(-1, -1)),
      none_k(H.col_len, make_int2(-1, -1));
  int rc = upload_region(ctx, B->d_ent + H.ent_off, none_e);
  if (!rc) rc = upload_region(ctx, B->d_ch + H.ch_off, none_c);
  if (!rc && H.col_len) rc = upload_region(ctx, B->d_col + H.col_off, none_k);
  B->h_state[slot] = BState{};
  if (!rc) LFX_CK(ctx, cudaMemcpyAsync(B->d_state + slot, &B->h_state[slot], sizeof(BState),
                                       cudaMemcpyHostToDevice, ctx->stream));
  H = SlotHost();
  if (!rc) rc = set_lengths(B);
  if (!rc) LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return rc;
}

}  // extern "C"
