// Many right-hand sides of one LMA operator at once, with the per-cell
// products on the tensor cores.
//
// Vectors of nrhs (16, 32 or 64) right-hand sides are stored dof-major,
// [undf][nrhs]. For one cell at one level the local product
//   Y_loc (nrhs x 8) = X_loc (nrhs x 8) . M^T (8 x 8)
// is a small GEMM: the right-hand sides are the rows of an mma.sync m16n8k8
// (TF32, or BF16, with FP32 accumulation), the cell's eight local dofs its
// columns, the local matrix its B operand. The operator must have the
// lowest-order nodal (W0) structure: ndf = 8, dofs 0..3 on the bottom and
// 4..7 on the top vertices, top = bottom + 1, so every dof lies on a vertex
// column of nlayers + 1 dofs.
//
// Summation without atomics (deterministic): the cell columns are split into
// compact patches (breadth-first over shared vertices), and every vertex
// column is owned by one patch (the patch holding most of its cells). One
// thread block per patch computes every cell column touching its owned
// vertices -- a few cells next to the patch are computed by two blocks -- and
// keeps the owned rows of a block of LB levels (2, 4 or 8, picked by
// lfx_mrhs_autotune) in shared memory. A warp walks one cell column up the
// levels of the block. The MMA's output columns are ordered (bottom, top) per
// vertex, so one lane holds both rows of a vertex: the top-vertex result of
// level k stays in its registers and joins the bottom rows of level k + 1, and
// each (cell column, vertex, level) adds once into shared memory. Cells are
// taken in colours (no two of a colour share an owned vertex) with a barrier
// between colours, so every sum has a fixed order.
//
// The solve wraps an FP32 preconditioned CG over all right-hand sides (each
// with its own step lengths; Jacobi preconditioner) in FP64 iterative
// refinement: the residual b - A x and the solution stay FP64 (RHS-major, the
// plain FP64 operator applies them), each inner solve reduces its residual by
// the inner tolerance, and a right-hand side converges on its true FP64
// residual ||b - A x|| / ||b - A x0||.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <queue>
#include <unordered_map>
#include <vector>

#include "lfx_internal.cuh"

using namespace lfx;

namespace {

constexpr int kMaxPC = 12;  // colours inside one patch, at most
constexpr int kWarps = 4;   // warps per patch block
constexpr int kDefaultPatch = 16;

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}
// D = A B with A 16x8 (rows: right-hand sides), B 8x8, FP32 accumulate from 0
__device__ __forceinline__ void mma_tf32(float* d, uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%10,%10,%10,%10};\n"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1), "f"(0.0f));
}
__device__ __forceinline__ void mma_bf16(float* d, uint32_t a01, uint32_t a23, uint32_t b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%7,%7,%7,%7};\n"
      : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
      : "r"(a01), "r"(a23), "r"(b), "f"(0.0f));
}

// Local matrices in B-fragment order, one 32-lane record per cell level
// (c2d * nl + k). B(j, n) = M(i(n), j) with the output dofs ordered (bottom,
// top) per vertex: i(2v) = v, i(2v + 1) = v + 4. Lane (g = lane / 4,
// t = lane % 4) holds B(t, g), B(t + 4, g) as TF32 (float2), or B(2t, g),
// B(2t + 1, g) as packed BF16; M(df, df2) is element
// (c * ndf + df) * blk + df2 * nl + k of the operator's matrices.
template <class TM, bool BF>
__global__ void mrhs_relayout(const TM* __restrict__ M, int64_t nc3, int nl, int blk, void* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nc3 * 32) return;
  const int lane = (int)(i & 31);
  const int64_t c3 = i >> 5;
  const int64_t c = c3 / nl;
  const int k = (int)(c3 % nl);
  const int g = lane >> 2, t = lane & 3;
  const int ig = (g >> 1) + 4 * (g & 1);
  auto at = [&](int df, int df2) {
    return (float)M[(c * 8 + df) * (int64_t)blk + (int64_t)df2 * nl + k];
  };
  if (BF) {
    reinterpret_cast<uint32_t*>(out)[i] = pack_bf16(at(ig, 2 * t), at(ig, 2 * t + 1));
  } else {
    float2 v;
    v.x = __uint_as_float(to_tf32(at(ig, t)));
    v.y = __uint_as_float(to_tf32(at(ig, t + 4)));
    reinterpret_cast<float2*>(out)[i] = v;
  }
}

struct MrhsArgs {
  const int4* pinfo;     // [npatch] {owned offset, owned count, cell offset, colours}
  const int* pcol;       // [npatch][kMaxPC + 1] first entry of each colour
  const int* own_base;   // first dof of each owned vertex column
  const int4* cells;     // per entry {c2d, xb0, xb1, xb2}, {xb3, owned slots, 0, 0}
  const void* Mf;
  int nl;
};

// TF32 rounding (half away from zero) on the integer pipe; BF16: one
// round-to-nearest-even conversion of two values into a packed pair (lo in
// the low half).
__device__ __forceinline__ uint32_t tf32_bits(float x) {
  return (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u;
}
__device__ __forceinline__ uint32_t bf16_pair(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
// W consecutive floats (W = 2, 4 or 8; aligned to W)
template <int W, class P>
__device__ __forceinline__ void ldw(P p, float (&v)[W]) {
  if constexpr (W == 2) {
    const float2 a = __ldg(reinterpret_cast<const float2*>(p));
    v[0] = a.x; v[1] = a.y;
  } else {
#pragma unroll
    for (int h = 0; h < W / 4; ++h) {
      const float4 a = __ldg(reinterpret_cast<const float4*>(p) + h);
      v[4 * h] = a.x; v[4 * h + 1] = a.y; v[4 * h + 2] = a.z; v[4 * h + 3] = a.w;
    }
  }
}
template <int W>
__device__ __forceinline__ void addw(float* r, const float (&o)[W]) {
  if constexpr (W == 2) {
    float2* q = reinterpret_cast<float2*>(r);
    float2 a = *q;
    a.x += o[0]; a.y += o[1];
    *q = a;
  } else {
#pragma unroll
    for (int h = 0; h < W / 4; ++h) {
      float4* q = reinterpret_cast<float4*>(r) + h;
      float4 a = *q;
      a.x += o[4 * h]; a.y += o[4 * h + 1]; a.z += o[4 * h + 2]; a.w += o[4 * h + 3];
      *q = a;
    }
  }
}

// One cell column over the levels [l0, l0 + nlb) of a block: MMAs per level,
// vertical carry, adds into the owned rows ys[slot][level - l0][rhs].
// Right-hand side map: with W = 2 RB, MMA row g of right-hand-side block rb
// is right-hand side W g + 2 rb and row g + 8 is W g + 2 rb + 1, so lane
// group g loads and adds the W consecutive right-hand sides W g .. W g + W - 1.
// Output columns 2t, 2t + 1 are the bottom and top rows of vertex t.
template <int RB, bool BF, int LB>
__device__ __forceinline__ void mrhs_cell(const MrhsArgs& A, const float* __restrict__ X,
                                          float* ys, int e, int l0, int nlb, int lane) {
  constexpr int NR = 16 * RB, RS = NR + 4, SLAB = (LB + 1) * RS, W = 2 * RB;
  const int g = lane >> 2, t = lane & 3;
  const int4 ca = A.cells[2 * e], cb = A.cells[2 * e + 1];
  const int nl = A.nl;
  const unsigned st = ((unsigned)cb.y >> (8 * t)) & 255u;  // owned slot of vertex t
  const size_t mrec = ((size_t)ca.x * nl + l0) * 32 + lane;

  // operands of all levels of the block, loaded before the first MMA
  uint32_t xa[LB + 1][W];
  uint32_t bm[LB][2];
  if (!BF) {
    // A columns t (bottom) and t + 4 (top): vertex t at levels k and k + 1
    const int xbt = t == 0 ? ca.y : t == 1 ? ca.z : t == 2 ? ca.w : cb.x;
    const float* xc = X + (size_t)(xbt + l0) * NR + W * g;
#pragma unroll
    for (int kk = 0; kk <= LB; ++kk) {
      float v[W];
      if (kk <= nlb) {
        ldw<W>(xc + kk * NR, v);
      } else {
#pragma unroll
        for (int w = 0; w < W; ++w) v[w] = 0.f;
      }
#pragma unroll
      for (int w = 0; w < W; ++w) xa[kk][w] = tf32_bits(v[w]);
    }
    const float2* mc = reinterpret_cast<const float2*>(A.Mf) + mrec;
#pragma unroll
    for (int kk = 0; kk < LB; ++kk) {
      const float2 v = kk < nlb ? __ldg(mc + kk * 32) : make_float2(0.f, 0.f);
      bm[kk][0] = __float_as_uint(v.x);
      bm[kk][1] = __float_as_uint(v.y);
    }
  } else {
    // A columns 2t, 2t + 1: vertices 2 (t % 2), 2 (t % 2) + 1 at level offset t / 2
    const int lo = t >> 1;
    const int x0 = (t & 1) ? ca.w : ca.y, x1 = (t & 1) ? cb.x : ca.z;
    const float* p0 = X + (size_t)(x0 + l0 + lo) * NR + W * g;
    const float* p1 = X + (size_t)(x1 + l0 + lo) * NR + W * g;
#pragma unroll
    for (int kk = 0; kk < LB; ++kk) {
      float v0[W], v1[W];
      if (kk < nlb) {
        ldw<W>(p0 + kk * NR, v0);
        ldw<W>(p1 + kk * NR, v1);
      } else {
#pragma unroll
        for (int w = 0; w < W; ++w) v0[w] = v1[w] = 0.f;
      }
#pragma unroll
      for (int w = 0; w < W; ++w) xa[kk][w] = bf16_pair(v0[w], v1[w]);
    }
    const uint32_t* mc = reinterpret_cast<const uint32_t*>(A.Mf) + mrec;
#pragma unroll
    for (int kk = 0; kk < LB; ++kk) bm[kk][0] = kk < nlb ? __ldg(mc + kk * 32) : 0u;
  }

  float carry[W];  // top rows of the level below (row kk)
  float* yr = ys + st * SLAB + W * g;
#pragma unroll
  for (int kk = 0; kk < LB; ++kk) {
    if (kk >= nlb) break;  // warp-uniform
    float d[RB][4];
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
      if (!BF)
        mma_tf32(d[rb], xa[kk][2 * rb], xa[kk][2 * rb + 1], xa[kk + 1][2 * rb],
                 xa[kk + 1][2 * rb + 1], bm[kk][0], bm[kk][1]);
      else
        mma_bf16(d[rb], xa[kk][2 * rb], xa[kk][2 * rb + 1], bm[kk][0]);
    }
    float o[W];
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
      o[2 * rb] = d[rb][0];
      o[2 * rb + 1] = d[rb][2];
      if (kk > 0) {
        o[2 * rb] += carry[2 * rb];
        o[2 * rb + 1] += carry[2 * rb + 1];
      }
      carry[2 * rb] = d[rb][1];
      carry[2 * rb + 1] = d[rb][3];
    }
    if (st != 255u) {
      addw<W>(yr + kk * RS, o);
      // top rows of the block's last level: row nlb, carried to the next block
      if (kk == nlb - 1) addw<W>(yr + (kk + 1) * RS, carry);
    }
  }
}

template <int RB, bool BF, int LB>
__global__ void __launch_bounds__(kWarps * 32) mrhs_apply_k(MrhsArgs A, const float* __restrict__ X,
                                                          float* __restrict__ Y) {
  constexpr int NR = 16 * RB, RS = NR + 4, SLAB = (LB + 1) * RS, C4 = NR / 4;
  extern __shared__ float4 ys4[];
  float* ys = reinterpret_cast<float*>(ys4);
  const int p = blockIdx.x;
  const int4 pi = A.pinfo[p];
  const int nown = pi.y, nl = A.nl;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int* pc = A.pcol + (size_t)p * (kMaxPC + 1);
  for (int i = threadIdx.x; i < nown * SLAB; i += blockDim.x) ys[i] = 0.f;
  for (int l0 = 0; l0 < nl; l0 += LB) {
    const int nlb = min(LB, nl - l0);
    for (int q = 0; q < pi.w; ++q) {
      __syncthreads();  // zeroing / the previous colour's adds are done
      const int e1 = pi.z + pc[q + 1];
      for (int e = pi.z + pc[q] + warp; e < e1; e += kWarps)
        mrhs_cell<RB, BF, LB>(A, X, ys, e, l0, nlb, lane);
    }
    __syncthreads();
    const bool last = l0 + nlb >= nl;
    const int rows = nlb + (last ? 1 : 0);
    // flush: one warp per owned vertex column, lanes over (row, float4)
    for (int sl = warp; sl < nown; sl += kWarps) {
      const float* src = ys + sl * SLAB;
      float* dst = Y + (size_t)(A.own_base[pi.x + sl] + l0) * NR;
      for (int i = lane; i < rows * C4; i += 32) {
        const int rr = i / C4, c4 = i % C4;
        *reinterpret_cast<float4*>(dst + (size_t)rr * NR + 4 * c4) =
            *reinterpret_cast<const float4*>(src + rr * RS + 4 * c4);
      }
    }
    if (last) break;
    __syncthreads();
    // row nlb (top of the block) becomes row 0 of the next block
    for (int i = threadIdx.x; i < nown * RS; i += blockDim.x) {
      float* b = ys + (i / RS) * SLAB + (i % RS);
      b[0] = b[nlb * RS];
#pragma unroll
      for (int r = 1; r <= LB; ++r) b[r * RS] = 0.f;
    }
  }
}

// ------------------------------------------------ dof-major vector kernels
// A thread handles four consecutive right-hand sides of a row (16-byte
// accesses): NR / 4 threads per row, RPB = 1024 / NR rows per block pass.

template <int NR>
struct MvShape {
  static constexpr int TPR = NR / 4;      // threads per row
  static constexpr int RPB = 256 / TPR;   // rows per block pass
};

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }

// Sums acc over the rows of the block, then over all blocks in block order
// (the last block to finish, by ticket), into tot[r * NR + col]. Returns true
// in that last block, with tot complete. acc[r][j] belongs to column
// 4 (threadIdx.x % TPR) + j.
template <int NR, int NRED>
__device__ bool mv_finish(const double (&acc)[NRED][4], double* partials, unsigned* ticket,
                          double* tot) {
  using S = MvShape<NR>;
  __shared__ double sm[S::RPB * NR];
  __shared__ int am_last;
  const int G = gridDim.x;
  const int c4 = threadIdx.x % S::TPR, rr = threadIdx.x / S::TPR;
#pragma unroll
  for (int r = 0; r < NRED; ++r) {
#pragma unroll
    for (int j = 0; j < 4; ++j) sm[rr * NR + 4 * c4 + j] = acc[r][j];
    __syncthreads();
    if (threadIdx.x < NR) {
      double s = 0.0;
      for (int q = 0; q < S::RPB; ++q) s = s + sm[q * NR + threadIdx.x];
      partials[((size_t)r * NR + threadIdx.x) * G + blockIdx.x] = s;
    }
    __syncthreads();
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = atomicAdd(ticket, 1u) == (unsigned)G - 1;
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int pr = w; pr < NRED * NR; pr += 8) {
    double s = 0.0;
    for (int b = lane; b < G; b += 32) s = s + __ldcg(partials + (size_t)pr * G + b);
    s = warp_butterfly(s);
    if (lane == 0) tot[pr] = s;
  }
  if (threadIdx.x == 0) *ticket = 0u;
  __syncthreads();
  return true;
}

struct MvState {
  double rz[64], alpha[64], beta[64], r0[64], rn[64];
  int active[64], iters[64];
  int nactive;
};

__device__ void count_active(MvState* S, int nr) {
  if (threadIdx.x == 0) {
    int n = 0;
    for (int c = 0; c < nr; ++c) n += S->active[c];
    S->nactive = n;
  }
}

#define LFX_MV_ROWS(NR)                                                      \
  const int c4 = threadIdx.x % MvShape<NR>::TPR;                             \
  for (int64_t row = (int64_t)blockIdx.x * MvShape<NR>::RPB +                \
                     threadIdx.x / MvShape<NR>::TPR;                         \
       row < n; row += (int64_t)gridDim.x * MvShape<NR>::RPB)

// x = 0, p = z = D^-1 r; rz = <r, z>, r0 = ||r|| per right-hand side
template <int NR>
__global__ void __launch_bounds__(256) mv_init(int64_t n, const float* __restrict__ dinv,
                                               const float* __restrict__ r, float* __restrict__ p,
                                               float* __restrict__ x, const int* act_out,
                                               MvState* S, double* partials, unsigned* ticket) {
  __shared__ double tot[2 * NR];
  double acc[2][4] = {};
  LFX_MV_ROWS(NR) {
    const size_t i = (size_t)row * NR + 4 * c4;
    const float4 rv = ld4(r + i);
    const float d = dinv[row];
    const float4 zv = make_float4(rv.x * d, rv.y * d, rv.z * d, rv.w * d);
    st4(p + i, zv);
    st4(x + i, make_float4(0.f, 0.f, 0.f, 0.f));
    const float ra[4] = {rv.x, rv.y, rv.z, rv.w}, za[4] = {zv.x, zv.y, zv.z, zv.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      acc[0][j] = fma((double)ra[j], (double)ra[j], acc[0][j]);
      acc[1][j] = fma((double)ra[j], (double)za[j], acc[1][j]);
    }
  }
  if (!mv_finish<NR, 2>(acc, partials, ticket, tot)) return;
  if (threadIdx.x < NR) {
    const int c = threadIdx.x;
    const double r0 = sqrt(tot[c]);
    S->r0[c] = r0;
    S->rn[c] = r0;
    S->rz[c] = tot[NR + c];
    S->alpha[c] = 0.0;
    S->beta[c] = 0.0;
    S->active[c] = act_out[c] && r0 > 0.0 && tot[NR + c] > 0.0;
  }
  __syncthreads();
  count_active(S, NR);
}

// alpha = rz / <p, q>
template <int NR>
__global__ void __launch_bounds__(256) mv_alpha(int64_t n, const float* __restrict__ p,
                                                const float* __restrict__ q, MvState* S,
                                                double* partials, unsigned* ticket) {
  __shared__ double tot[NR];
  double acc[1][4] = {};
  LFX_MV_ROWS(NR) {
    const size_t i = (size_t)row * NR + 4 * c4;
    const float4 pv = ld4(p + i), qv = ld4(q + i);
    acc[0][0] = fma((double)pv.x, (double)qv.x, acc[0][0]);
    acc[0][1] = fma((double)pv.y, (double)qv.y, acc[0][1]);
    acc[0][2] = fma((double)pv.z, (double)qv.z, acc[0][2]);
    acc[0][3] = fma((double)pv.w, (double)qv.w, acc[0][3]);
  }
  if (!mv_finish<NR, 1>(acc, partials, ticket, tot)) return;
  if (threadIdx.x < NR) {
    const int c = threadIdx.x;
    S->alpha[c] = (S->active[c] && tot[c] != 0.0) ? S->rz[c] / tot[c] : 0.0;
  }
}

// x += alpha p, r -= alpha q; ||r||, rz_new = <r, D^-1 r>; beta; inner
// convergence ||r|| <= tol ||r0||
template <int NR>
__global__ void __launch_bounds__(256) mv_update(int64_t n, const float* __restrict__ dinv,
                                                 const float* __restrict__ p,
                                                 const float* __restrict__ q, float* __restrict__ x,
                                                 float* __restrict__ r, double tol, MvState* S,
                                                 double* partials, unsigned* ticket) {
  __shared__ double tot[2 * NR];
  float a[4];
  {
    const int c0 = 4 * (threadIdx.x % MvShape<NR>::TPR);
#pragma unroll
    for (int j = 0; j < 4; ++j) a[j] = (float)S->alpha[c0 + j];
  }
  double acc[2][4] = {};
  LFX_MV_ROWS(NR) {
    const size_t i = (size_t)row * NR + 4 * c4;
    const float4 pv = ld4(p + i), qv = ld4(q + i), xv = ld4(x + i), rv = ld4(r + i);
    const float d = dinv[row];
    st4(x + i, make_float4(fmaf(a[0], pv.x, xv.x), fmaf(a[1], pv.y, xv.y), fmaf(a[2], pv.z, xv.z),
                           fmaf(a[3], pv.w, xv.w)));
    const float rn[4] = {fmaf(-a[0], qv.x, rv.x), fmaf(-a[1], qv.y, rv.y),
                         fmaf(-a[2], qv.z, rv.z), fmaf(-a[3], qv.w, rv.w)};
    st4(r + i, make_float4(rn[0], rn[1], rn[2], rn[3]));
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      acc[0][j] = fma((double)rn[j], (double)rn[j], acc[0][j]);
      acc[1][j] = fma((double)rn[j], (double)(rn[j] * d), acc[1][j]);
    }
  }
  if (!mv_finish<NR, 2>(acc, partials, ticket, tot)) return;
  if (threadIdx.x < NR) {
    const int c = threadIdx.x;
    if (S->active[c]) {
      const double rn = sqrt(tot[c]);
      S->rn[c] = rn;
      S->beta[c] = tot[NR + c] / S->rz[c];
      S->rz[c] = tot[NR + c];
      S->iters[c] += 1;
      if (!(rn > tol * S->r0[c]) || !(tot[NR + c] > 0.0)) S->active[c] = 0;
    } else {
      S->beta[c] = 0.0;
    }
  }
  __syncthreads();
  count_active(S, NR);
}

// p = D^-1 r + beta p
template <int NR>
__global__ void __launch_bounds__(256) mv_direction(int64_t n, const float* __restrict__ dinv,
                                                    const float* __restrict__ r,
                                                    float* __restrict__ p, const MvState* S) {
  float b[4];
  {
    const int c0 = 4 * (threadIdx.x % MvShape<NR>::TPR);
#pragma unroll
    for (int j = 0; j < 4; ++j) b[j] = (float)S->beta[c0 + j];
  }
  LFX_MV_ROWS(NR) {
    const size_t i = (size_t)row * NR + 4 * c4;
    const float4 rv = ld4(r + i), pv = ld4(p + i);
    const float d = dinv[row];
    st4(p + i, make_float4(fmaf(b[0], pv.x, rv.x * d), fmaf(b[1], pv.y, rv.y * d),
                           fmaf(b[2], pv.z, rv.z * d), fmaf(b[3], pv.w, rv.w * d)));
  }
}
#undef LFX_MV_ROWS

// r[row][col] = (float) R[col * ld + row] (RHS-major FP64 to dof-major FP32)
template <int NR>
__global__ void mv_from_rhs_major(int64_t n, const double* __restrict__ R, int64_t ld,
                                  float* __restrict__ r) {
  constexpr int TW = NR < 32 ? NR : 32;
  __shared__ float tile[TW][33];
  const int64_t row0 = (int64_t)blockIdx.x * 32;
  const int col0 = blockIdx.y * TW;
  for (int j = threadIdx.y; j < TW; j += blockDim.y) {
    const int64_t row = row0 + threadIdx.x;
    if (row < n) tile[j][threadIdx.x] = (float)R[(size_t)(col0 + j) * ld + row];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int64_t row = row0 + j;
    if (row < n && threadIdx.x < TW) r[(size_t)row * NR + col0 + threadIdx.x] = tile[threadIdx.x][j];
  }
}

// X[col * ld + row] += x[row][col]
template <int NR>
__global__ void mv_add_to_rhs_major(int64_t n, const float* __restrict__ x, double* __restrict__ X,
                                    int64_t ld) {
  constexpr int TW = NR < 32 ? NR : 32;
  __shared__ float tile[TW][33];
  const int64_t row0 = (int64_t)blockIdx.x * 32;
  const int col0 = blockIdx.y * TW;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int64_t row = row0 + j;
    if (row < n && threadIdx.x < TW) tile[threadIdx.x][j] = x[(size_t)row * NR + col0 + threadIdx.x];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < TW; j += blockDim.y) {
    const int64_t row = row0 + threadIdx.x;
    if (row < n) X[(size_t)(col0 + j) * ld + row] += (double)tile[j][threadIdx.x];
  }
}

__global__ void k_dinv(int64_t n, const double* __restrict__ d, float* __restrict__ dinv) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dinv[i] = (float)(1.0 / d[i]);
}

// ------------------------------------------------ block CG
// Breakdown-free block preconditioned CG on all 64 right-hand sides at once
// (the block Krylov method of the reference's block_gcr_solve family,
// sci_iterative_solver_mod.f90:1461-1628, in its CG form):
//   Z = D^-1 R, P = orth(Z)
//   loop: Q = A P; alpha = (P^T Q)^-1 P^T R; X += P alpha; R -= Q alpha;
//         beta = -(P^T Q)^-1 Q^T D^-1 R; P = orth(D^-1 R + P beta)
// orth(W) = W T with T from a pivoted Cholesky factorisation of W^T W that
// stops at pivots below kBcgDrop times the largest one: directions the block
// no longer spans (right-hand sides that have converged, or become
// dependent) are dropped, so the method does not break down. The products
// with the tall n x 64 blocks run as 32-row chunks staged in shared memory,
// each thread holding a 4 x 4 (Gram) or 2 x 4 (update) register tile; the
// Gram sums are FP32 within a chunk, FP64 across chunks and blocks, in a
// fixed order; the 64 x 64 algebra runs in FP64 in one block.
constexpr int kBS = 64;          // right-hand sides of a block solve
constexpr int kBcgRows = 32;     // rows per staged chunk
// W is FP32 and its Gram sums carry relative errors near 1e-6 of the largest
// entry, so directions whose pivot falls below 1e-5 of the largest are noise
// and are dropped (the kept part of W then has a condition number under
// about 300, and W T is orthonormal to a few parts in a thousand)
constexpr double kBcgDrop = 1e-5;

struct BcgSmall {
  double C[2 * kBS * kBS];  // [v][i][j]: v = 0 P^T Q, v = 1 P^T R (gram of P with Q, R)
  double E[kBS * kBS];      // Q^T D^-1 R
  double G[kBS * kBS];      // W^T W
  double L1[kBS * kBS];     // inverse of the Cholesky factor of the active block of P^T Q
  double r0[kBS], rn[kBS];
  float coef[kBS * kBS];    // alpha, beta or T [k][j] for the next row update
  int active[kBS];          // right-hand sides the solve works on
  int rank, done, iters, fail;
};

// ---- The same Gram on the 5th-generation tensor cores (tcgen05).
// D (64 x 64 NV) = U^T [V_0 .. V_NV-1] accumulates in tensor memory (TMEM,
// FP32): A = U^T (64 x K) and B = V^T (64 NV x K) are both K-major in shared
// memory (kind::tf32 takes K-major operands only), in the canonical
// no-swizzle layout: core matrices of 8 MN-rows x 16 bytes (4 K values),
// MN-rows 16 bytes apart, MN groups of 8 rows 128 bytes apart (stride byte
// offset), K groups of 4 values MN/8 x 128 bytes apart (leading byte offset).
// Each FP32 value is split into TF32 parts hi + lo and a product taken as
// hi hi + hi lo + lo hi (three kind::tf32 MMAs of M = 64, K = 8 per K step),
// which keeps about FP32 accuracy. Two 32-row stages: the block stages the
// next chunk while the tensor core works on the last one; one elected thread
// issues the MMAs and commits them to the stage's mbarrier. Every mbarrier
// wait is bounded; a wait that runs out sets st->fail = 2 and the block
// stops issuing work (the final wait is bounded too before TMEM is freed).
constexpr int kTcRows = 32;
constexpr int kTcThreads = 128;
constexpr unsigned long long kTcWaitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// shared-memory matrix descriptor: start, leading (K group) and stride (MN
// group) byte offsets, version 1, no swizzle
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor: FP32 accumulate, A and B TF32, both K-major, M = 64
template <int N>
__host__ __device__ constexpr uint32_t idesc_tf32_k() {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(64 >> 4) << 24);
}
__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}
__device__ __forceinline__ unsigned long long tc_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// wait for the mbarrier phase of the given parity, for at most kTcWaitNs
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity) {
  const unsigned long long t0 = tc_clock();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (tc_clock() - t0 > kTcWaitNs) return false;
  }
}
__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
// stage rows row0 .. row0 + 31 (the K dimension) of an n x MN block made of
// 64-column row-major sources (columns 0..63 from s0, 64.. from s1) as the
// K-major operand (MN x 32), TF32 hi and lo parts; rows past n are zero. A
// thread takes four consecutive rows of one column: the warp's loads of a row
// are coalesced and its 16-byte stores fill 512 contiguous bytes.
__device__ __forceinline__ void tc_stage(unsigned char* hi, unsigned char* lo, int MN,
                                         const float* s0, const float* s1, int64_t row0,
                                         int64_t n, const float* __restrict__ scale) {
  for (int e = threadIdx.x; e < (kTcRows / 4) * MN; e += kTcThreads) {
    const int m = e % MN, kq = e / MN;
    const float* src = m < kBS ? s0 + m : s1 + (m - kBS);
    float v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int64_t k = row0 + 4 * kq + q;
      v[q] = 0.f;
      if (k < n) {
        v[q] = __ldg(src + (size_t)k * kBS);
        if (scale) v[q] *= __ldg(scale + k);
      }
    }
    const float4 h = make_float4(tf32_round(v[0]), tf32_round(v[1]), tf32_round(v[2]), tf32_round(v[3]));
    const float4 l = make_float4(tf32_round(v[0] - h.x), tf32_round(v[1] - h.y),
                                 tf32_round(v[2] - h.z), tf32_round(v[3] - h.w));
    const size_t off = ((size_t)kq * (MN / 8) + m / 8) * 128 + (size_t)(m % 8) * 16;
    *reinterpret_cast<float4*>(hi + off) = h;
    *reinterpret_cast<float4*>(lo + off) = l;
  }
}

template <int NV>
__global__ void __launch_bounds__(kTcThreads) bcg_gram_tc(int64_t n, const float* __restrict__ U,
                                                         const float* __restrict__ V0,
                                                         const float* __restrict__ V1,
                                                         const float* __restrict__ vscale,
                                                         double* __restrict__ partials,
                                                         BcgSmall* st) {
  constexpr int N = kBS * NV, LBA = kBS / 8 * 128, LBB = N / 8 * 128;
  constexpr int ABYTES = kTcRows * kBS * 4, BBYTES = kTcRows * N * 4;
  constexpr int STAGE = 2 * ABYTES + 2 * BBYTES;
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  __shared__ int s_abort;
  if (st->done) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base)),
                 "r"((uint32_t)N)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])) : "memory");
    s_abort = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  constexpr uint32_t IDESC = idesc_tf32_k<N>();
  int j = 0;  // chunks of this block so far
  for (int64_t c = blockIdx.x; c * kTcRows < n; c += gridDim.x, ++j) {
    const int sidx = j & 1;
    unsigned char* base = tc_smem + (size_t)sidx * STAGE;
    if (j >= 2) {
      // the MMAs that last read this stage have completed
      if (threadIdx.x == 0 && !tc_wait(smem_u32(&mbar[sidx]), (uint32_t)((j / 2 - 1) & 1))) {
        s_abort = 1;
        st->fail = 2;
      }
      __syncthreads();
      if (s_abort) break;
    }
    tc_stage(base, base + ABYTES, kBS, U, U, c * kTcRows, n, nullptr);
    tc_stage(base + 2 * ABYTES, base + 2 * ABYTES + BBYTES, N, V0, NV > 1 ? V1 : V0,
             c * kTcRows, n, vscale);
    // generic-proxy writes of the operands become visible to the tensor core
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_hi = smem_u32(base), a_lo = a_hi + ABYTES;
      const uint32_t b_hi = a_hi + 2 * ABYTES, b_lo = b_hi + BBYTES;
#pragma unroll
      for (int kg = 0; kg < kTcRows / 8; ++kg) {
        // K step kg: K groups 2 kg and 2 kg + 1
        const uint64_t ah = umma_desc(a_hi + 2 * kg * LBA, LBA, 128);
        const uint64_t al = umma_desc(a_lo + 2 * kg * LBA, LBA, 128);
        const uint64_t bh = umma_desc(b_hi + 2 * kg * LBB, LBB, 128);
        const uint64_t bl = umma_desc(b_lo + 2 * kg * LBB, LBB, 128);
        tc_mma(tmem, ah, bh, IDESC, (j > 0 || kg > 0) ? 1u : 0u);
        tc_mma(tmem, ah, bl, IDESC, 1u);
        tc_mma(tmem, al, bh, IDESC, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mbar[sidx]))
                   : "memory");
    }
  }
  // the last commit covers every MMA of the block
  if (j > 0 && threadIdx.x == 0 &&
      !tc_wait(smem_u32(&mbar[(j - 1) & 1]), (uint32_t)(((j - 1) / 2) & 1))) {
    s_abort = 1;
    st->fail = 2;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  double* out = partials + (size_t)blockIdx.x * NV * kBS * kBS;
  // M = 64: row m sits in TMEM lane (m % 16) + 32 (m / 16); warp w reads
  // lanes 32 w .. 32 w + 31, whose first 16 hold rows 16 w .. 16 w + 15
#pragma unroll
  for (int c0 = 0; c0 < N; c0 += 32) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
        "%28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    if (lane < 16) {
      const int m = 16 * warp + lane;
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        const int jj = c0 + q, v = jj / kBS, jc = jj % kBS;
        out[((size_t)v * kBS + m) * kBS + jc] =
            (j > 0 && !s_abort) ? (double)__uint_as_float(r[q]) : 0.0;
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"((uint32_t)N)
                 : "memory");
}

template <int NV>
constexpr size_t tc_gram_smem() {
  return 2 * (2 * (size_t)kTcRows * kBS * 4 + 2 * (size_t)kTcRows * kBS * NV * 4);
}

// out[e] = sum over the blocks, in block order, of partials[b][e]
__global__ void bcg_reduce(int nb, int ne, const double* __restrict__ partials,
                           double* __restrict__ out, const BcgSmall* st) {
  if (st->done) return;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  // block order, as before; eight loads in flight ahead of the additions
  double s = 0.0;
  int b = 0;
  for (; b + 8 <= nb; b += 8) {
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = __ldg(partials + (size_t)(b + q) * ne + e);
#pragma unroll
    for (int q = 0; q < 8; ++q) s = s + v[q];
  }
  for (; b < nb; ++b) s = s + __ldg(partials + (size_t)b * ne + e);
  out[e] = s;
}

// ---- The same products with the tall blocks streamed. A block takes the
// 32-row chunks c = blockIdx.x + i gridDim.x of its operands (each chunk of
// an n x 64 row-major FP32 block is one contiguous 8 KB run) through a ring
// of S stages in shared memory: thread 0 moves a chunk's operands with
// cp.async.bulk copies completing on the stage's mbarrier, S - 1 chunks
// ahead of the compute, so the bytes in flight cost no registers. Every wait
// is bounded (kTcWaitNs); the block decides together (__syncthreads_and)
// and, on a time-out, sets st->fail = 2, waits (bounded) for the copies it
// issued and stops. Sums: FP32 within a chunk, FP64 across chunks and blocks, in a fixed order.
constexpr int kChunkBytes = kBcgRows * kBS * 4;  // one operand's chunk
template <int NA, int S>
struct ChunkRing {
  static constexpr int STAGE = NA * kChunkBytes;
  static constexpr size_t BYTES = (size_t)S * STAGE + (size_t)S * 8;
};
__device__ __forceinline__ bool chunk_try(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool chunk_wait(uint64_t* bar, unsigned parity) {
  if (chunk_try(bar, parity)) return true;
  const unsigned long long t0 = tc_clock();
  while (!chunk_try(bar, parity))
    if (tc_clock() - t0 > kTcWaitNs) return false;
  return true;
}
// thread 0: chunk c of the NA operands into stage buffer dst, on bar
template <int NA>
__device__ __forceinline__ void chunk_issue(const float* const (&src)[NA], int64_t c, int64_t n,
                                            unsigned char* dst, uint64_t* bar) {
  const int64_t row0 = c * kBcgRows;
  const int rows = (int)(n - row0 < (int64_t)kBcgRows ? n - row0 : (int64_t)kBcgRows);
  const unsigned bytes = (unsigned)rows * kBS * 4;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes * NA)
               : "memory");
#pragma unroll
  for (int a = 0; a < NA; ++a)
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst + a * kChunkBytes)),
        "l"(src[a] + (size_t)row0 * kBS), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// the ring's set-up and its bounded drain after a time-out (chunks from..to-1:
// the one whose wait ran out and those issued after it)
template <int S>
__device__ __forceinline__ void chunk_ring_init(uint64_t* bar) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar + i)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}
template <int S>
__device__ __forceinline__ void chunk_ring_drain(uint64_t* bar, int from, int to) {
  if (threadIdx.x == 0)
    for (int i = from; i < to; ++i) chunk_wait(bar + i % S, (unsigned)((i / S) & 1));
}

template <int NV>
__global__ void __launch_bounds__(256, 2) bcg_gram_s(int64_t n, const float* __restrict__ U,
                                                  const float* __restrict__ V0,
                                                  const float* __restrict__ V1,
                                                  const float* __restrict__ vscale,
                                                  double* __restrict__ partials, BcgSmall* st) {
  constexpr int NA = 1 + NV, S = 4;
  using RG = ChunkRing<NA, S>;
  extern __shared__ __align__(16) unsigned char ring_smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(ring_smem + S * RG::STAGE);
  if (st->done) return;
  const float* src[NA];
  src[0] = U;
  src[1] = V0;
  if (NV > 1) src[NA - 1] = V1;
  const int64_t nchunk = (n + kBcgRows - 1) / kBcgRows;
  const int nmine = blockIdx.x < nchunk ? (int)((nchunk - 1 - blockIdx.x) / gridDim.x + 1) : 0;
  chunk_ring_init<S>(bar);
  if (threadIdx.x == 0)
    for (int i = 0; i < S && i < nmine; ++i)
      chunk_issue<NA>(src, blockIdx.x + (int64_t)i * gridDim.x, n, ring_smem + i * RG::STAGE, bar + i);
  const int i0 = 4 * (threadIdx.x / 16), j0 = 4 * (threadIdx.x % 16);
  double acc[NV][4][4];
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[v][a][b] = 0.0;
  bool failed = false;
  for (int i = 0; i < nmine; ++i) {
    const int stg = i % S;
    const bool ok = chunk_wait(bar + stg, (unsigned)((i / S) & 1));
    if (!__syncthreads_and(ok)) {
      if (threadIdx.x == 0) st->fail = 2;
      chunk_ring_drain<S>(bar, i, nmine < i + S ? nmine : i + S);
      failed = true;
      break;
    }
    const int64_t c = blockIdx.x + (int64_t)i * gridDim.x, row0 = c * kBcgRows;
    const int rows = (int)(n - row0 < (int64_t)kBcgRows ? n - row0 : (int64_t)kBcgRows);
    const float (*Us)[kBS] = reinterpret_cast<const float (*)[kBS]>(ring_smem + stg * RG::STAGE);
    float a[NV][4][4];
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) a[v][x][y] = 0.f;
    // the row scales of this chunk: one load a lane, then shuffles (the
    // two-operand form measured faster this way; the one-operand form keeps
    // a load per row)
    const int lane = threadIdx.x & 31;
    const float sc_lane = (NV == 2 && vscale && lane < rows) ? __ldg(vscale + row0 + lane) : 1.f;
    for (int r = 0; r < rows; ++r) {
      const float4 u = *reinterpret_cast<const float4*>(&Us[r][i0]);
      const float uu[4] = {u.x, u.y, u.z, u.w};
      const float sc = !vscale ? 1.f
                       : NV == 2 ? __shfl_sync(0xffffffffu, sc_lane, r)
                                 : __ldg(vscale + row0 + r);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const float (*Vs)[kBS] =
            reinterpret_cast<const float (*)[kBS]>(ring_smem + stg * RG::STAGE + (1 + v) * kChunkBytes);
        float4 w = *reinterpret_cast<const float4*>(&Vs[r][j0]);
        if (vscale) {
          w.x *= sc; w.y *= sc; w.z *= sc; w.w *= sc;
        }
        const float ww[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int y = 0; y < 4; ++y) a[v][x][y] = fmaf(uu[x], ww[y], a[v][x][y]);
      }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[v][x][y] += (double)a[v][x][y];
    __syncthreads();  // the stage is read: it takes chunk i + S
    if (threadIdx.x == 0 && i + S < nmine)
      chunk_issue<NA>(src, blockIdx.x + (int64_t)(i + S) * gridDim.x, n, ring_smem + stg * RG::STAGE,
                      bar + stg);
  }
  double* out = partials + (size_t)blockIdx.x * NV * kBS * kBS;
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y)
        out[((size_t)v * kBS + i0 + x) * kBS + j0 + y] = failed ? 0.0 : acc[v][x][y];
}

// Y (+)= B C streamed: mode 0 (P, Q, X, R): X += P C, R -= Q C and the column
// sums of R^2; mode 1 (P, R): W = D^-1 R + P C; mode 2 (W): P = W C
template <int MODE>
struct UpdOps {
  static constexpr int NA = MODE == 0 ? 4 : MODE == 1 ? 2 : 1;
  static constexpr int S = MODE == 0 ? 3 : 4;
};
template <int MODE>
__global__ void __launch_bounds__(256) bcg_update_s(int64_t n, const float* __restrict__ A0,
                                                    const float* __restrict__ A1, float* Y0,
                                                    float* Y1, const float* __restrict__ dinv,
                                                    const BcgSmall* st, int skip_p,
                                                    double* __restrict__ partials) {
  constexpr int NA = UpdOps<MODE>::NA, S = UpdOps<MODE>::S;
  using RG = ChunkRing<NA, S>;
  extern __shared__ __align__(16) unsigned char ring_smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(ring_smem + S * RG::STAGE);
  __shared__ __align__(16) float Cs[kBS][kBS];
  if (st->done) return;
  for (int e = threadIdx.x; e < kBS * kBS; e += blockDim.x) Cs[e / kBS][e % kBS] = st->coef[e];
  // streamed operands: mode 0 P, Q, X, R; mode 1 P, R; mode 2 W
  const float* src[NA];
  src[0] = A0;
  if (MODE == 0) {
    src[1] = A1;
    src[2] = Y0;
    src[3] = Y1;
  } else if (MODE == 1) {
    src[1] = A1;
  }
  const int64_t nchunk = (n + kBcgRows - 1) / kBcgRows;
  const int nmine = blockIdx.x < nchunk ? (int)((nchunk - 1 - blockIdx.x) / gridDim.x + 1) : 0;
  chunk_ring_init<S>(bar);
  if (threadIdx.x == 0)
    for (int i = 0; i < S && i < nmine; ++i)
      chunk_issue<NA>(src, blockIdx.x + (int64_t)i * gridDim.x, n, ring_smem + i * RG::STAGE, bar + i);
  // thread: column c of the output for the 8 rows 8 rg .. 8 rg + 7 of each
  // chunk, with column c of the coefficients in registers; the operand rows
  // are read four values at a time, every lane of a warp at the same address
  // (one shared-memory wavefront). Each output is one fmaf chain over
  // k = 0..63, as before the tiling changed.
  const int c = 32 * ((threadIdx.x >> 5) & 1) + (threadIdx.x & 31), rg = threadIdx.x >> 6;
  float cr[kBS];
  __syncthreads();  // Cs is written
#pragma unroll
  for (int k = 0; k < kBS; ++k) cr[k] = Cs[k][c];
  // the squared-residual sums of row pairs 4 rg + i, in the order of the
  // earlier two-rows-a-thread form (row 2q, then 2q + 1, chunk by chunk)
  double nrm[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = 0; i < nmine; ++i) {
    const int stg = i % S;
    const bool ok = chunk_wait(bar + stg, (unsigned)((i / S) & 1));
    if (!__syncthreads_and(ok)) {
      if (threadIdx.x == 0) const_cast<BcgSmall*>(st)->fail = 2;
      chunk_ring_drain<S>(bar, i, nmine < i + S ? nmine : i + S);
      break;
    }
    const int64_t ch = blockIdx.x + (int64_t)i * gridDim.x, row0 = ch * kBcgRows;
    const int rows = (int)(n - row0 < (int64_t)kBcgRows ? n - row0 : (int64_t)kBcgRows);
    const unsigned char* stage = ring_smem + stg * RG::STAGE;
    const float (*As0)[kBS] = reinterpret_cast<const float (*)[kBS]>(stage);
    const float (*As1)[kBS] = reinterpret_cast<const float (*)[kBS]>(stage + kChunkBytes);
    if (MODE == 1 && rows == kBcgRows) {
      // a full chunk: the thread's 8 rows with their fmaf chains
      // interleaved (independent chains, each still over k = 0..63 in
      // order; measured faster for this mode only)
      const int rb = 8 * rg;
      float d[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) d[q] = 0.f;
      if (!skip_p) {
#pragma unroll
        for (int k = 0; k < kBS; k += 4) {
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const float4 a0 = *reinterpret_cast<const float4*>(&As0[rb + q][k]);
            d[q] = fmaf(a0.x, cr[k], d[q]);
            d[q] = fmaf(a0.y, cr[k + 1], d[q]);
            d[q] = fmaf(a0.z, cr[k + 2], d[q]);
            d[q] = fmaf(a0.w, cr[k + 3], d[q]);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int r = rb + q;
        const float rv = As1[r][c];
        const float dv = __ldg(dinv + row0 + r);
        Y0[(size_t)(row0 + r) * kBS + c] = fmaf(rv, dv, d[q]);
      }
    } else
#pragma unroll 1
    for (int i8 = 0; i8 < 8; ++i8) {
      const int r = 8 * rg + i8;
      if (r >= rows) break;
      const size_t o = (size_t)(row0 + r) * kBS + c;
      float d0 = 0.f, d1 = 0.f;
      if (!skip_p) {
#pragma unroll
        for (int k = 0; k < kBS; k += 4) {
          const float4 a0 = *reinterpret_cast<const float4*>(&As0[r][k]);
          d0 = fmaf(a0.x, cr[k], d0);
          d0 = fmaf(a0.y, cr[k + 1], d0);
          d0 = fmaf(a0.z, cr[k + 2], d0);
          d0 = fmaf(a0.w, cr[k + 3], d0);
          if (MODE == 0) {
            const float4 a1 = *reinterpret_cast<const float4*>(&As1[r][k]);
            d1 = fmaf(a1.x, cr[k], d1);
            d1 = fmaf(a1.y, cr[k + 1], d1);
            d1 = fmaf(a1.z, cr[k + 2], d1);
            d1 = fmaf(a1.w, cr[k + 3], d1);
          }
        }
      }
      if (MODE == 0) {
        const float x = reinterpret_cast<const float*>(stage + 2 * kChunkBytes)[r * kBS + c];
        const float rv = reinterpret_cast<const float*>(stage + 3 * kChunkBytes)[r * kBS + c];
        Y0[o] = x + d0;
        const float rn = rv - d1;
        Y1[o] = rn;
        const double rd = (double)rn;
        switch (i8 >> 1) {
          case 0: nrm[0] = fma(rd, rd, nrm[0]); break;
          case 1: nrm[1] = fma(rd, rd, nrm[1]); break;
          case 2: nrm[2] = fma(rd, rd, nrm[2]); break;
          default: nrm[3] = fma(rd, rd, nrm[3]); break;
        }
      } else if (MODE == 1) {
        const float rv = As1[r][c];
        const float dv = __ldg(dinv + row0 + r);
        Y0[o] = fmaf(rv, dv, d0);
      } else {
        Y0[o] = d0;
      }
    }
    __syncthreads();  // the stage is read: it takes chunk i + S
    if (threadIdx.x == 0 && i + S < nmine)
      chunk_issue<NA>(src, blockIdx.x + (int64_t)(i + S) * gridDim.x, n, ring_smem + stg * RG::STAGE,
                      bar + stg);
  }
  if (MODE == 0) {
    // column sums of R^2 in a fixed order, in the ring's memory (every
    // chunk has been consumed)
    __syncthreads();
    double (*red)[kBS] = reinterpret_cast<double (*)[kBS]>(ring_smem);
#pragma unroll
    for (int j = 0; j < 4; ++j) red[4 * rg + j][c] = nrm[j];
    __syncthreads();
    if (threadIdx.x < kBS) {
      double s = 0.0;
      for (int q = 0; q < 16; ++q) s = s + red[q][threadIdx.x];
      partials[(size_t)blockIdx.x * kBS + threadIdx.x] = s;
    }
  }
}

// column norms ||R_j|| of the initial residual (r0) and, for the columns not
// active, R_j = 0 so the block leaves them alone
__global__ void __launch_bounds__(256) bcg_mask(int64_t n, float* R, const int* act) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n * kBS;
       e += (int64_t)gridDim.x * blockDim.x)
    if (!act[e % kBS]) R[e] = 0.f;
}

// The 64 x 64 algebra of one step, in FP64, one block of 256 threads.
// mode 0 (alpha): L = chol(active r x r block of P^T Q); L1 = L^-1 (kept for
//   mode 1); alpha = L1^T (L1 P^T R)
// mode 1 (beta): rn = sqrt(column sums) (convergence: done when every active
//   right-hand side has rn <= tol r0); beta = -L1^T (L1 Q^T D^-1 R)
// mode 2 (orth): pivoted Cholesky of W^T W -> rank and T (P = W T)
// mode 3 (norms of the initial residual into r0)
// The kernel's whole shared state is one dynamic buffer laid out here (no
// static shared variables beside it): three 64 x 65 FP64 matrices, then the
// pivot order and two flags.
constexpr size_t kBcgMatBytes = sizeof(double) * kBS * (kBS + 1);
constexpr size_t kBcgSmallSmem = 3 * kBcgMatBytes + sizeof(int) * (kBS + 4);

// Linv = L^-1 for the r x r lower factor L(i, k): thread j < r forms column
// j (rows below j by forward substitution, the dot products in four partial
// sums); rows and columns past r are zero
template <class Lf>
__device__ __forceinline__ void lower_inverse(int r, Lf L, double (*Linv)[kBS + 1]) {
  const int t = threadIdx.x;
  if (t < kBS) {
    const int j = t;
    for (int i = 0; i < kBS; ++i) Linv[i][j] = 0.0;
    if (j < r) {
      Linv[j][j] = 1.0 / L(j, j);
      for (int i = j + 1; i < r; ++i) {
        double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
        int k = j;
        for (; k + 3 < i; k += 4) {
          v0 = fma(L(i, k), Linv[k][j], v0);
          v1 = fma(L(i, k + 1), Linv[k + 1][j], v1);
          v2 = fma(L(i, k + 2), Linv[k + 2][j], v2);
          v3 = fma(L(i, k + 3), Linv[k + 3][j], v3);
        }
        for (; k < i; ++k) v0 = fma(L(i, k), Linv[k][j], v0);
        Linv[i][j] = -((v0 + v1) + (v2 + v3)) / L(i, i);
      }
    }
  }
  __syncthreads();
}

// Out = op(A) B for 64 x 64 operands, op(A) = A or A^T; each thread a 4 x 4
// tile, k in increasing order
template <bool TRANS>
__device__ __forceinline__ void small_mm(const double (*A)[kBS + 1], const double (*B)[kBS + 1],
                                         double (*Out)[kBS + 1], double scale) {
  const int i0 = 4 * (threadIdx.x / 16), j0 = 4 * (threadIdx.x % 16);
  double acc[4][4];
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) acc[x][y] = 0.0;
  for (int k = 0; k < kBS; ++k) {
    double a[4], bv[4];
#pragma unroll
    for (int x = 0; x < 4; ++x) a[x] = TRANS ? A[k][i0 + x] : A[i0 + x][k];
#pragma unroll
    for (int y = 0; y < 4; ++y) bv[y] = B[k][j0 + y];
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
      for (int y = 0; y < 4; ++y) acc[x][y] = fma(a[x], bv[y], acc[x][y]);
  }
  __syncthreads();  // Out may alias B
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) Out[i0 + x][j0 + y] = scale * acc[x][y];
  __syncthreads();
}

__global__ void __launch_bounds__(256) bcg_small(int mode, BcgSmall* st, double tol) {
  extern __shared__ __align__(16) unsigned char bcg_dyn[];
  double (*M)[kBS + 1] = reinterpret_cast<double (*)[kBS + 1]>(bcg_dyn);
  double (*Bm)[kBS + 1] = reinterpret_cast<double (*)[kBS + 1]>(bcg_dyn + kBcgMatBytes);
  double (*Y)[kBS + 1] = reinterpret_cast<double (*)[kBS + 1]>(bcg_dyn + 2 * kBcgMatBytes);
  int* perm = reinterpret_cast<int*>(bcg_dyn + 3 * kBcgMatBytes);
  int& s_r = perm[kBS];
  int& s_stop = perm[kBS + 1];
  const int t = threadIdx.x;
  if (st->done) return;
  if (mode == 3) {
    // the column sums of R^2 were reduced into rn
    if (t < kBS) {
      st->r0[t] = sqrt(st->rn[t]);
      st->rn[t] = st->r0[t];
    }
    return;
  }
  if (mode == 0 || mode == 1) {
    const int r = st->rank;
    if (mode == 0) {
      // Cholesky of the r x r active block of P^T Q (column by column)
      for (int e = t; e < kBS * kBS; e += blockDim.x) M[e / kBS][e % kBS] = st->C[e];
      __syncthreads();
      // two barriers a step: every thread takes the pivot's root from the
      // diagonal itself (written back only in the update phase, which does
      // not read it), the column is divided, then the trailing triangle is
      // updated by a 16 x 16 thread grid (no index division)
      const int ti = t >> 4, tj = t & 15;
      bool stop = false;
      for (int k = 0; k < r; ++k) {
        const double d = M[k][k];
        if (!(d > 0.0)) {
          stop = true;  // every thread reads the same d
          break;
        }
        const double sk = sqrt(d);
        for (int i = k + 1 + t; i < r; i += blockDim.x) M[i][k] /= sk;
        __syncthreads();
        if (t == 0) M[k][k] = sk;
        for (int i = k + 1 + ti; i < r; i += 16) {
          const double lik = M[i][k];
          for (int j = k + 1 + tj; j <= i; j += 16) M[i][j] -= lik * M[j][k];
        }
        __syncthreads();
      }
      if (stop) {
        if (t == 0) { st->fail = 1; st->done = 1; }
        return;
      }
      // L1 = L^-1, kept for mode 1
      lower_inverse(r, [&](int i, int k) { return M[i][k]; }, Bm);
      for (int e = t; e < kBS * kBS; e += blockDim.x) st->L1[e] = Bm[e / kBS][e % kBS];
      // right-hand sides: P^T R
      for (int e = t; e < kBS * kBS; e += blockDim.x) M[e / kBS][e % kBS] = st->C[kBS * kBS + e];
      __syncthreads();
    } else {
      if (t < kBS) st->rn[t] = sqrt(st->rn[t]);
      __syncthreads();
      if (t == 0) {
        int done = 1;
        for (int j = 0; j < kBS; ++j)
          if (st->active[j] && st->rn[j] > tol * st->r0[j]) done = 0;
        st->iters += 1;
        s_stop = done;
      }
      __syncthreads();
      if (s_stop) {
        if (t == 0) st->done = 1;
        return;
      }
      for (int e = t; e < kBS * kBS; e += blockDim.x) {
        Bm[e / kBS][e % kBS] = st->L1[e];
        M[e / kBS][e % kBS] = st->E[e];
      }
      __syncthreads();
    }
    // rows past r of the right-hand sides do not take part
    for (int e = t; e < kBS * kBS; e += blockDim.x)
      if (e / kBS >= r) M[e / kBS][e % kBS] = 0.0;
    __syncthreads();
    // Y = L1 B, then the coefficients L1^T Y (negated for beta)
    small_mm<false>(Bm, M, Y, 1.0);
    small_mm<true>(Bm, Y, Y, mode == 0 ? 1.0 : -1.0);
    for (int e = t; e < kBS * kBS; e += blockDim.x) st->coef[e] = (float)Y[e / kBS][e % kBS];
    return;
  }
  // mode 2: pivoted Cholesky of G = W^T W, stopping at pivots below
  // kBcgDrop times the largest diagonal entry. The pivoting is by index:
  // rows and columns stay where they are and perm[i] names the row of step
  // i, so L[i][j] = M[perm[i]][perm[j]] (i >= j) once the loop is done. (A
  // form that swapped rows and columns in place, in one thread inside the
  // loop over steps, lost the pivot's square root on the B200 while the same
  // statements with a constant step index did not; the index form has no
  // such swaps.) Warp 0 finds each pivot: the largest remaining diagonal
  // entry, the first in step order on a tie.
  for (int e = t; e < kBS * kBS; e += blockDim.x) M[e / kBS][e % kBS] = st->G[e];
  if (t < kBS) perm[t] = t;
  if (t == 0) s_r = 0;
  __syncthreads();
  double dmax = 0.0;
  for (int i = 0; i < kBS; ++i) dmax = fmax(dmax, M[i][i]);
  const int ti = t >> 4, tj = t & 15;
  for (int k = 0; k < kBS; ++k) {
    if (t < 32) {
      // lane l looks at steps k + l and k + l + 32
      double bv = -INFINITY;
      int bi = kBS;  // none (every candidate NaN): the factorisation stops
      for (int i = k + t; i < kBS; i += 32) {
        const double dv = M[perm[i]][perm[i]];
        if (dv > bv) { bv = dv; bi = i; }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
      }
      if (t == 0) {
        const int p = bi < kBS ? bi : k;
        const int pk = perm[p];
        const int stop = bi >= kBS || !(M[pk][pk] > kBcgDrop * dmax) || !(dmax > 0.0);
        if (!stop) {
          perm[p] = perm[k];
          perm[k] = pk;
          M[pk][pk] = sqrt(M[pk][pk]);
          s_r = k + 1;
        }
        s_stop = stop;
      }
    }
    __syncthreads();
    if (s_stop) break;
    const int pk = perm[k];
    for (int i = k + 1 + t; i < kBS; i += blockDim.x) M[perm[i]][pk] /= M[pk][pk];
    __syncthreads();
    // the trailing square by a 16 x 16 thread grid (no index division)
    const int m = kBS - k - 1;
    for (int a = ti; a < m; a += 16) {
      const int pi = perm[k + 1 + a];
      const double lik = M[pi][pk];
      for (int b = tj; b < m; b += 16) {
        const int pj = perm[k + 1 + b];
        M[pi][pj] -= lik * M[pj][pk];
      }
    }
    __syncthreads();
  }
  const int r = s_r;
  // Linv = L^-1 (r x r, lower; L[i][k] = M[perm[i]][perm[k]])
  lower_inverse(r, [&](int i, int k) { return M[perm[i]][perm[k]]; }, Bm);
  // T[perm[i]][j] = Linv[j][i] (i <= j < r), zero elsewhere
  for (int e = t; e < kBS * kBS; e += blockDim.x) st->coef[e] = 0.f;
  __syncthreads();
  for (int e = t; e < r * r; e += blockDim.x) {
    const int i = e / r, j = e % r;
    if (i <= j) st->coef[perm[i] * kBS + j] = (float)Bm[j][i];
  }
  if (t == 0) {
    st->rank = r;
    if (r == 0) st->done = 1;
  }
}

}  // namespace

struct lfx_mrhs {
  lfx_ctx* ctx = nullptr;
  int32_t kind = LFX_MRHS_TF32, nrhs = 64, nl = 0, ncell_2d = 0;
  int64_t undf = 0;
  int32_t npatch = 0, own_max = 0, max_colours = 0;
  int64_t nent = 0;
  int4* pinfo = nullptr;
  int* pcol = nullptr;
  int* own_base = nullptr;
  int4* cells = nullptr;
  void* Mf = nullptr;
  size_t Mf_bytes = 0;
  int32_t lb = 4;  // levels per block of the apply (2, 4 or 8)
  size_t pinfo_b = 0, pcol_b = 0, own_b = 0, cells_b = 0;
  // solve work space, allocated by the first solve
  float *x32 = nullptr, *r32 = nullptr, *p32 = nullptr, *q32 = nullptr, *dinv = nullptr;
  double* R64 = nullptr;
  double* nrm = nullptr;      // [nrhs] device
  double* h_nrm = nullptr;    // [nrhs] pinned
  int* d_act = nullptr;       // [nrhs]
  MvState* S = nullptr;
  MvState* h_S = nullptr;     // pinned
  double* partials = nullptr;
  unsigned* ticket = nullptr;
  int grid = 0;
  size_t work_bytes = 0;
  // block CG: W, the small algebra state and the Gram partials
  float* w32 = nullptr;
  BcgSmall* bcg = nullptr;
  BcgSmall* h_bcg = nullptr;  // pinned
  double* bpart = nullptr;
  int bgrid = 0;
  int gram_tc = 0;  // block CG Gram products on the tcgen05 tensor cores (1) or the FP32 cores (0)
};

namespace {

size_t mrhs_smem(const lfx_mrhs* m, int lb) {
  return (size_t)m->own_max * (lb + 1) * (m->nrhs + 4) * sizeof(float);
}

template <int RB, bool BF, int LB>
int launch_t(lfx_mrhs* m, const float* x, float* y) {
  lfx_ctx* ctx = m->ctx;
  MrhsArgs A{m->pinfo, m->pcol, m->own_base, m->cells, m->Mf, m->nl};
  const size_t smem = mrhs_smem(m, LB);
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(mrhs_apply_k<RB, BF, LB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return fail(ctx, LFX_NOT_SUPPORTED, "apply shared memory exceeds the device limit");
  mrhs_apply_k<RB, BF, LB><<<m->npatch, kWarps * 32, smem, ctx->stream>>>(A, x, y);
  ctx->launches++;
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

template <int RB, bool BF>
int launch_lb(lfx_mrhs* m, int lb, const float* x, float* y) {
  switch (lb) {
    case 2: return launch_t<RB, BF, 2>(m, x, y);
    case 8: return launch_t<RB, BF, 8>(m, x, y);
    default: return launch_t<RB, BF, 4>(m, x, y);
  }
}

int mrhs_launch_lb(lfx_mrhs* m, int lb, const float* x, float* y) {
  const bool bf = m->kind == LFX_MRHS_BF16;
  switch (m->nrhs) {
    case 16: return bf ? launch_lb<1, true>(m, lb, x, y) : launch_lb<1, false>(m, lb, x, y);
    case 32: return bf ? launch_lb<2, true>(m, lb, x, y) : launch_lb<2, false>(m, lb, x, y);
    default: return bf ? launch_lb<4, true>(m, lb, x, y) : launch_lb<4, false>(m, lb, x, y);
  }
}

int mrhs_launch(lfx_mrhs* m, const float* x, float* y) { return mrhs_launch_lb(m, m->lb, x, y); }

void mrhs_free(lfx_mrhs* m) {
  lfx_ctx* ctx = m->ctx;
  dfree(ctx, m->pinfo, m->pinfo_b);
  dfree(ctx, m->pcol, m->pcol_b);
  dfree(ctx, m->own_base, m->own_b);
  dfree(ctx, m->cells, m->cells_b);
  dfree(ctx, m->Mf, m->Mf_bytes);
  const size_t v32 = (size_t)m->undf * m->nrhs * 4;
  dfree(ctx, m->x32, v32);
  dfree(ctx, m->r32, v32);
  dfree(ctx, m->p32, v32);
  dfree(ctx, m->q32, v32);
  dfree(ctx, m->dinv, (size_t)m->undf * 4);
  dfree(ctx, m->R64, (size_t)m->undf * m->nrhs * 8);
  dfree(ctx, m->nrm, sizeof(double) * 64);
  dfree(ctx, m->d_act, sizeof(int) * 64);
  dfree(ctx, m->S, sizeof(MvState));
  dfree(ctx, m->partials, sizeof(double) * 2 * 64 * m->grid);
  dfree(ctx, m->ticket, sizeof(unsigned));
  if (m->h_nrm) cudaFreeHost(m->h_nrm);
  if (m->h_S) cudaFreeHost(m->h_S);
  dfree(ctx, m->w32, v32);
  dfree(ctx, m->bcg, sizeof(BcgSmall));
  dfree(ctx, m->bpart, sizeof(double) * 2 * kBS * kBS * m->bgrid);
  if (m->h_bcg) cudaFreeHost(m->h_bcg);
}

}  // namespace

int lfx_mrhs_create(const lfx_op* op, int32_t kind, int32_t nrhs, int32_t cells_per_patch,
                    lfx_mrhs** out) {
  if (!op || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  lfx_ctx* ctx = op->ctx;
  const lfx_lma_layout* L = op->lay;
  if (kind != LFX_MRHS_TF32 && kind != LFX_MRHS_BF16)
    return fail(ctx, LFX_INVALID_ARGUMENT, "kind must be LFX_MRHS_TF32 or LFX_MRHS_BF16");
  if (nrhs != 16 && nrhs != 32 && nrhs != 64)
    return fail(ctx, LFX_INVALID_ARGUMENT, "nrhs must be 16, 32 or 64");
  if (cells_per_patch < 0 || cells_per_patch > 256)
    return fail(ctx, LFX_INVALID_ARGUMENT, "cells_per_patch must be in [0, 256]");
  const int P = cells_per_patch ? cells_per_patch : kDefaultPatch;
  if (L->ndf_to != 8 || L->ndf_from != 8 || L->undf_to != L->undf_from)
    return fail(ctx, LFX_NOT_SUPPORTED, "multi-RHS apply needs a square ndf = 8 (W0) operator");
  const int nc = L->ncell_2d, nl = L->nlayers;
  std::vector<int32_t> mt((size_t)nc * 8), mf((size_t)nc * 8);
  LFX_CK(ctx, cudaMemcpy(mt.data(), L->map_to, mt.size() * 4, cudaMemcpyDeviceToHost));
  LFX_CK(ctx, cudaMemcpy(mf.data(), L->map_from, mf.size() * 4, cudaMemcpyDeviceToHost));
  if (mt != mf) return fail(ctx, LFX_NOT_SUPPORTED, "multi-RHS apply needs map_to == map_from");
  // vertex columns
  std::unordered_map<int32_t, int32_t> vid;
  std::vector<int32_t> vbase;
  std::vector<int32_t> cv((size_t)nc * 4);
  for (int c = 0; c < nc; ++c)
    for (int v = 0; v < 4; ++v) {
      const int32_t b = mt[(size_t)c * 8 + v];
      if (mt[(size_t)c * 8 + 4 + v] != b + 1)
        return fail(ctx, LFX_NOT_SUPPORTED,
                    "multi-RHS apply needs W0 dofs: top vertex dof = bottom dof + 1");
      if (b < 0 || (int64_t)b + nl >= L->undf_to)
        return fail(ctx, LFX_INVALID_ARGUMENT, "dofmap entry out of range");
      auto it = vid.find(b);
      int id;
      if (it == vid.end()) {
        id = (int)vbase.size();
        vid.emplace(b, id);
        vbase.push_back(b);
      } else {
        id = it->second;
      }
      cv[(size_t)c * 4 + v] = id;
    }
  const int nv = (int)vbase.size();
  if ((int64_t)nv * (nl + 1) != L->undf_to)
    return fail(ctx, LFX_NOT_SUPPORTED, "multi-RHS apply needs every dof on a vertex column");
  std::vector<int32_t> voff(nv + 1, 0), vcells;
  for (int c = 0; c < nc; ++c)
    for (int v = 0; v < 4; ++v) voff[cv[(size_t)c * 4 + v] + 1]++;
  for (int i = 0; i < nv; ++i) voff[i + 1] += voff[i];
  vcells.resize(voff[nv]);
  {
    std::vector<int32_t> fill(voff.begin(), voff.end() - 1);
    for (int c = 0; c < nc; ++c)
      for (int v = 0; v < 4; ++v) vcells[fill[cv[(size_t)c * 4 + v]]++] = c;
  }
  // compact patches: breadth-first over cells sharing a vertex
  std::vector<int32_t> patch(nc, -1);
  int npatch = 0;
  {
    std::vector<int32_t> queue;
    for (int s = 0; s < nc; ++s) {
      if (patch[s] >= 0) continue;
      queue.clear();
      queue.push_back(s);
      patch[s] = npatch;
      int taken = 1;
      for (size_t h = 0; h < queue.size() && taken < P; ++h) {
        const int c = queue[h];
        for (int v = 0; v < 4 && taken < P; ++v) {
          const int id = cv[(size_t)c * 4 + v];
          for (int k = voff[id]; k < voff[id + 1] && taken < P; ++k) {
            const int n2 = vcells[k];
            if (patch[n2] < 0) {
              patch[n2] = npatch;
              queue.push_back(n2);
              ++taken;
            }
          }
        }
      }
      ++npatch;
    }
  }
  // owner of a vertex column: the patch holding most of its cells (ties: the
  // patch of its lowest cell)
  std::vector<int32_t> owner(nv);
  for (int i = 0; i < nv; ++i) {
    int best = -1, bestn = 0;
    for (int k = voff[i]; k < voff[i + 1]; ++k) {
      const int pk = patch[vcells[k]];
      int n = 0;
      for (int k2 = voff[i]; k2 < voff[i + 1]; ++k2) n += patch[vcells[k2]] == pk;
      if (n > bestn || (n == bestn && pk < best)) {
        best = pk;
        bestn = n;
      }
    }
    owner[i] = best;
  }
  std::vector<std::vector<int32_t>> pown(npatch);
  for (int i = 0; i < nv; ++i) pown[owner[i]].push_back(i);
  std::vector<int4> h_pinfo(npatch);
  std::vector<int> h_pcol((size_t)npatch * (kMaxPC + 1), 0);
  std::vector<int> h_own;
  std::vector<int4> h_cells;
  int own_max = 0, max_col = 0;
  std::vector<int32_t> slot_of(nv, -1);
  for (int p = 0; p < npatch; ++p) {
    const auto& ov = pown[p];
    if (ov.size() > 254) return fail(ctx, LFX_NOT_SUPPORTED, "patch owns too many vertex columns");
    for (size_t s = 0; s < ov.size(); ++s) slot_of[ov[s]] = (int)s;
    std::vector<int32_t> need;
    for (int id : ov)
      for (int k = voff[id]; k < voff[id + 1]; ++k) need.push_back(vcells[k]);
    std::sort(need.begin(), need.end());
    need.erase(std::unique(need.begin(), need.end()), need.end());
    // greedy colours: cells sharing an owned vertex differ
    std::vector<uint32_t> used(ov.size(), 0u);
    std::vector<int> colour(need.size());
    int ncol = 0;
    for (size_t i = 0; i < need.size(); ++i) {
      uint32_t forbid = 0u;
      for (int v = 0; v < 4; ++v) {
        const int s = slot_of[cv[(size_t)need[i] * 4 + v]];
        if (s >= 0) forbid |= used[s];
      }
      int col = 0;
      while (forbid & (1u << col)) ++col;
      if (col >= kMaxPC) return fail(ctx, LFX_NOT_SUPPORTED, "patch needs too many colours");
      colour[i] = col;
      ncol = std::max(ncol, col + 1);
      for (int v = 0; v < 4; ++v) {
        const int s = slot_of[cv[(size_t)need[i] * 4 + v]];
        if (s >= 0) used[s] |= 1u << col;
      }
    }
    h_pinfo[p] = make_int4((int)h_own.size(), (int)ov.size(), (int)(h_cells.size() / 2), ncol);
    int* pc = h_pcol.data() + (size_t)p * (kMaxPC + 1);
    int n = 0;
    for (int col = 0; col < ncol; ++col) {
      pc[col] = n;
      for (size_t i = 0; i < need.size(); ++i) {
        if (colour[i] != col) continue;
        const int c = need[i];
        unsigned sp = 0u;
        for (int v = 0; v < 4; ++v) {
          const int s = slot_of[cv[(size_t)c * 4 + v]];
          sp |= (unsigned)(s >= 0 ? s : 255) << (8 * v);
        }
        const int32_t* mc = mt.data() + (size_t)c * 8;
        h_cells.push_back(make_int4(c, mc[0], mc[1], mc[2]));
        h_cells.push_back(make_int4(mc[3], (int)sp, 0, 0));
        ++n;
      }
    }
    pc[ncol] = n;
    for (int id : ov) h_own.push_back(vbase[id]);
    for (int id : ov) slot_of[id] = -1;
    own_max = std::max(own_max, (int)ov.size());
    max_col = std::max(max_col, ncol);
  }

  auto* m = new lfx_mrhs();
  m->ctx = ctx;
  m->kind = kind;
  m->nrhs = nrhs;
  m->nl = nl;
  m->ncell_2d = nc;
  m->undf = L->undf_to;
  m->npatch = npatch;
  m->own_max = own_max;
  m->max_colours = max_col;
  m->nent = (int64_t)h_cells.size() / 2;
  int rc = LFX_OK;
  if (mrhs_smem(m, 2) > 227 * 1024) rc = fail(ctx, LFX_NOT_SUPPORTED, "patch too large for shared memory");
  m->lb = mrhs_smem(m, 4) <= 227 * 1024 ? 4 : 2;
  auto up = [&](void** dst, size_t* held, const void* src, size_t bytes) {
    if (rc) return;
    rc = dmalloc(ctx, dst, bytes);
    if (!rc) *held = bytes;
    if (!rc && cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
      rc = fail(ctx, LFX_CUDA_ERROR, "upload of the patch tables failed");
  };
  up((void**)&m->pinfo, &m->pinfo_b, h_pinfo.data(), h_pinfo.size() * sizeof(int4));
  up((void**)&m->pcol, &m->pcol_b, h_pcol.data(), h_pcol.size() * sizeof(int));
  up((void**)&m->own_base, &m->own_b, h_own.data(), h_own.size() * sizeof(int));
  up((void**)&m->cells, &m->cells_b, h_cells.data(), h_cells.size() * sizeof(int4));
  const int64_t nc3 = (int64_t)nc * nl;
  m->Mf_bytes = (size_t)nc3 * 32 * (kind == LFX_MRHS_BF16 ? 4 : 8);
  if (!rc) rc = dmalloc(ctx, &m->Mf, m->Mf_bytes);
  if (!rc) {
    const int64_t nthr = nc3 * 32;
    const int blocks = (int)((nthr + 255) / 256);
    const bool bf = kind == LFX_MRHS_BF16;
    if (op->precision == LFX_R64) {
      if (bf)
        mrhs_relayout<double, true><<<blocks, 256, 0, ctx->stream>>>((const double*)op->mat, nc3, nl, op->blk, m->Mf);
      else
        mrhs_relayout<double, false><<<blocks, 256, 0, ctx->stream>>>((const double*)op->mat, nc3, nl, op->blk, m->Mf);
    } else {
      if (bf)
        mrhs_relayout<float, true><<<blocks, 256, 0, ctx->stream>>>((const float*)op->mat, nc3, nl, op->blk, m->Mf);
      else
        mrhs_relayout<float, false><<<blocks, 256, 0, ctx->stream>>>((const float*)op->mat, nc3, nl, op->blk, m->Mf);
    }
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      rc = fail(ctx, LFX_CUDA_ERROR, "matrix relayout failed");
  }
  if (rc) {
    mrhs_free(m);
    delete m;
    return rc;
  }
  *out = m;
  return LFX_OK;
}

int lfx_mrhs_destroy(lfx_mrhs* m) {
  if (!m) return LFX_OK;
  mrhs_free(m);
  delete m;
  return LFX_OK;
}

int lfx_mrhs_info(const lfx_mrhs* m, int32_t* npatch, int64_t* cell_entries, int32_t* max_owned,
                  int32_t* max_colours, int64_t* matrix_bytes) {
  if (!m) return LFX_INVALID_ARGUMENT;
  if (npatch) *npatch = m->npatch;
  if (cell_entries) *cell_entries = m->nent * m->nl;
  if (max_owned) *max_owned = m->own_max;
  if (max_colours) *max_colours = m->max_colours;
  if (matrix_bytes) *matrix_bytes = (int64_t)m->Mf_bytes;
  return LFX_OK;
}

int lfx_mrhs_apply(lfx_mrhs* m, const float* x, float* y) {
  if (!m || !x || !y || x == y) return LFX_INVALID_ARGUMENT;
  return mrhs_launch(m, x, y);
}

int lfx_mrhs_time_apply(lfx_mrhs* m, const float* x, float* y, int32_t reps, float* us) {
  if (!m || !x || !y || x == y || reps < 1 || !us) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = m->ctx;
  int rc = mrhs_launch(m, x, y);  // warm
  if (rc) return rc;
  cudaEvent_t e0, e1;
  LFX_CK(ctx, cudaEventCreate(&e0));
  LFX_CK(ctx, cudaEventCreate(&e1));
  cudaEventRecord(e0, ctx->stream);
  for (int r = 0; r < reps && !rc; ++r) rc = mrhs_launch(m, x, y);
  cudaEventRecord(e1, ctx->stream);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess && !rc)
    rc = fail(ctx, LFX_CUDA_ERROR, "multi-RHS apply timing failed");
  float ms = 0.f;
  if (!rc) cudaEventElapsedTime(&ms, e0, e1);
  *us = 1e3f * ms / reps;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

// Times the apply with 2, 4 and 8 levels per block (those whose shared
// memory fits) over reps applies each and keeps the fastest.
int lfx_mrhs_autotune(lfx_mrhs* m, int32_t reps, int32_t* lb, float* us) {
  if (!m || reps < 1) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = m->ctx;
  const size_t bytes = (size_t)m->undf * m->nrhs * sizeof(float);
  float *x = nullptr, *y = nullptr;
  int rc = dmalloc(ctx, (void**)&x, bytes);
  if (!rc) rc = dmalloc(ctx, (void**)&y, bytes);
  if (!rc) LFX_CK(ctx, cudaMemsetAsync(x, 0, bytes, ctx->stream));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (!rc) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
  }
  int best = m->lb;
  float best_us = 0.f;
  for (int cand : {2, 4, 8}) {
    if (rc) break;
    if (mrhs_smem(m, cand) > 227 * 1024) continue;
    rc = mrhs_launch_lb(m, cand, x, y);  // warm
    cudaEventRecord(e0, ctx->stream);
    for (int r = 0; r < reps && !rc; ++r) rc = mrhs_launch_lb(m, cand, x, y);
    cudaEventRecord(e1, ctx->stream);
    if (!rc && cudaStreamSynchronize(ctx->stream) != cudaSuccess)
      rc = fail(ctx, LFX_CUDA_ERROR, "multi-RHS apply timing failed");
    float ms = 0.f;
    if (!rc) cudaEventElapsedTime(&ms, e0, e1);
    const float t = 1e3f * ms / reps;
    if (!rc && (best_us == 0.f || t < best_us)) {
      best_us = t;
      best = cand;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  dfree(ctx, x, bytes);
  dfree(ctx, y, bytes);
  if (rc) return rc;
  m->lb = best;
  if (lb) *lb = best;
  if (us) *us = best_us;
  return LFX_OK;
}

namespace {

int ensure_work(lfx_mrhs* m) {
  if (m->x32) return LFX_OK;
  lfx_ctx* ctx = m->ctx;
  const size_t v32 = (size_t)m->undf * m->nrhs * 4;
  m->grid = ctx->num_sms * 4;
  int rc = dmalloc(ctx, (void**)&m->x32, v32);
  if (!rc) rc = dmalloc(ctx, (void**)&m->r32, v32);
  if (!rc) rc = dmalloc(ctx, (void**)&m->p32, v32);
  if (!rc) rc = dmalloc(ctx, (void**)&m->q32, v32);
  if (!rc) rc = dmalloc(ctx, (void**)&m->dinv, (size_t)m->undf * 4);
  if (!rc) rc = dmalloc(ctx, (void**)&m->R64, (size_t)m->undf * m->nrhs * 8);
  if (!rc) rc = dmalloc(ctx, (void**)&m->nrm, sizeof(double) * 64);
  if (!rc) rc = dmalloc(ctx, (void**)&m->d_act, sizeof(int) * 64);
  if (!rc) rc = dmalloc(ctx, (void**)&m->S, sizeof(MvState));
  if (!rc) rc = dmalloc(ctx, (void**)&m->partials, sizeof(double) * 2 * 64 * m->grid);
  if (!rc) rc = dmalloc(ctx, (void**)&m->ticket, sizeof(unsigned));
  if (!rc && cudaMallocHost(&m->h_nrm, sizeof(double) * 64) != cudaSuccess)
    rc = fail(ctx, LFX_OUT_OF_MEMORY, "pinned allocation failed");
  if (!rc && cudaMallocHost(&m->h_S, sizeof(MvState)) != cudaSuccess)
    rc = fail(ctx, LFX_OUT_OF_MEMORY, "pinned allocation failed");
  if (!rc) LFX_CK(ctx, cudaMemsetAsync(m->ticket, 0, sizeof(unsigned), ctx->stream));
  if (!rc) LFX_CK(ctx, cudaMemsetAsync(m->S, 0, sizeof(MvState), ctx->stream));
  return rc;
}

// R = B - A64 X per right-hand side, and ||R|| into m->h_nrm
int outer_residual(lfx_mrhs* m, lfx_op* op64, const double* b, double* x, int64_t ld) {
  lfx_ctx* ctx = m->ctx;
  const int64_t n = m->undf;
  for (int r = 0; r < m->nrhs; ++r) {
    int rc = op_apply_impl(op64, x + (size_t)r * ld, m->R64 + (size_t)r * n, b + (size_t)r * ld,
                           nullptr);
    if (rc) return rc;
    const double* R = m->R64 + (size_t)r * n;
    double* out = m->nrm + r;
    rc = launch_chunks<1>(
        ctx, n, [=] __device__(int64_t i) { return V1<double>{R[i]}; },
        [=] __device__(int64_t, const V1<double>& v, double* acc) {
          acc[0] = fma(v.a, v.a, acc[0]);
        },
        [=] __device__(const double* tot) { *out = sqrt(tot[0]); });
    if (rc) return rc;
  }
  LFX_CK(ctx, cudaMemcpyAsync(m->h_nrm, m->nrm, sizeof(double) * m->nrhs, cudaMemcpyDeviceToHost,
                              ctx->stream));
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return LFX_OK;
}

template <int NR>
int inner_solve(lfx_mrhs* m, const int* act, double tol, int max_inner, int* inner_its) {
  lfx_ctx* ctx = m->ctx;
  const int64_t n = m->undf;
  const int G = m->grid;
  const dim3 tb(32, 8), tg((unsigned)((n + 31) / 32), NR < 32 ? 1 : NR / 32);
  mv_from_rhs_major<NR><<<tg, tb, 0, ctx->stream>>>(n, m->R64, n, m->r32);
  LFX_CK(ctx, cudaMemcpyAsync(m->d_act, act, sizeof(int) * NR, cudaMemcpyHostToDevice, ctx->stream));
  mv_init<NR><<<G, 256, 0, ctx->stream>>>(n, m->dinv, m->r32, m->p32, m->x32, m->d_act, m->S,
                                          m->partials, m->ticket);
  ctx->launches += 2;
  LFX_CK(ctx, cudaGetLastError());
  int it = 0;
  constexpr int kCheck = 8;
  while (it < max_inner) {
    const int nb = std::min(kCheck, max_inner - it);
    for (int s = 0; s < nb; ++s) {
      int rc = mrhs_launch(m, m->p32, m->q32);
      if (rc) return rc;
      mv_alpha<NR><<<G, 256, 0, ctx->stream>>>(n, m->p32, m->q32, m->S, m->partials, m->ticket);
      mv_update<NR><<<G, 256, 0, ctx->stream>>>(n, m->dinv, m->p32, m->q32, m->x32, m->r32, tol,
                                                m->S, m->partials, m->ticket);
      mv_direction<NR><<<G, 256, 0, ctx->stream>>>(n, m->dinv, m->r32, m->p32, m->S);
      ctx->launches += 3;
    }
    LFX_CK(ctx, cudaGetLastError());
    it += nb;
    LFX_CK(ctx, cudaMemcpyAsync(&m->h_S->nactive, &m->S->nactive, sizeof(int),
                                cudaMemcpyDeviceToHost, ctx->stream));
    LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
    if (m->h_S->nactive == 0) break;
  }
  *inner_its = it;
  return LFX_OK;
}

// partials of U^T [V0 (V1)] (rows of V scaled by vscale when given) on the
// tensor cores or the FP32 cores, then the fixed-order reduction into out
template <int NV>
int gram(lfx_mrhs* m, const float* U, const float* V0, const float* V1, const float* vscale,
         BcgSmall* st, double* out) {
  lfx_ctx* ctx = m->ctx;
  const int64_t n = m->undf;
  if (m->gram_tc) {
    static bool attr = false;
    if (!attr) {
      LFX_CK(ctx, cudaFuncSetAttribute(bcg_gram_tc<NV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)tc_gram_smem<NV>()));
      attr = true;
    }
    bcg_gram_tc<NV><<<m->bgrid, kTcThreads, tc_gram_smem<NV>(), ctx->stream>>>(n, U, V0, V1,
                                                                               vscale, m->bpart, st);
  } else {
    constexpr size_t smem = ChunkRing<1 + NV, 4>::BYTES;
    static bool sattr = false;
    if (!sattr) {
      LFX_CK(ctx, cudaFuncSetAttribute(bcg_gram_s<NV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
      sattr = true;
    }
    bcg_gram_s<NV><<<m->bgrid, 256, smem, ctx->stream>>>(n, U, V0, V1, vscale, m->bpart, st);
  }
  const int ne = NV * kBS * kBS;
  bcg_reduce<<<(ne + 255) / 256, 256, 0, ctx->stream>>>(m->bgrid, ne, m->bpart, out, st);
  ctx->launches += 2;
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

int ensure_bcg(lfx_mrhs* m) {
  if (m->bcg) return LFX_OK;
  lfx_ctx* ctx = m->ctx;
  LFX_CK(ctx, cudaFuncSetAttribute(bcg_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)kBcgSmallSmem));
  m->bgrid = ctx->num_sms * 2;
  int rc = dmalloc(ctx, (void**)&m->w32, (size_t)m->undf * m->nrhs * 4);
  if (!rc) rc = dmalloc(ctx, (void**)&m->bcg, sizeof(BcgSmall));
  if (!rc) rc = dmalloc(ctx, (void**)&m->bpart, sizeof(double) * 2 * kBS * kBS * m->bgrid);
  if (!rc && cudaMallocHost((void**)&m->h_bcg, sizeof(BcgSmall)) != cudaSuccess)
    rc = fail(ctx, LFX_OUT_OF_MEMORY, "pinned allocation failed");
  return rc;
}

// the streamed update kernel of a mode with its shared memory set: returns a
// callable taking the kernel's arguments
template <int MODE>
auto upd_launch(lfx_ctx* ctx, int G) {
  using RG = ChunkRing<UpdOps<MODE>::NA, UpdOps<MODE>::S>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(bcg_update_s<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)RG::BYTES);
    attr = true;
  }
  return [ctx, G](int64_t n, const float* A0, const float* A1, float* Y0, float* Y1,
                  const float* dinv, const BcgSmall* st, int skip_p, double* partials) {
    bcg_update_s<MODE><<<G, 256, RG::BYTES, ctx->stream>>>(n, A0, A1, Y0, Y1, dinv, st, skip_p,
                                                            partials);
  };
}

// One inner block-CG solve of A X = R (R from the outer residual, X = 0),
// each active right-hand side reduced by tol, at most max_inner iterations.
int bcg_inner(lfx_mrhs* m, const int* act, double tol, int max_inner, int* inner_its,
              int* failed) {
  lfx_ctx* ctx = m->ctx;
  const int64_t n = m->undf;
  const int G = m->bgrid;
  BcgSmall* st = m->bcg;
  const dim3 tb(32, 8), tg((unsigned)((n + 31) / 32), kBS / 32);
  mv_from_rhs_major<kBS><<<tg, tb, 0, ctx->stream>>>(n, m->R64, n, m->r32);
  LFX_CK(ctx, cudaMemsetAsync(st, 0, sizeof(BcgSmall), ctx->stream));
  LFX_CK(ctx, cudaMemcpyAsync(st->active, act, sizeof(int) * kBS, cudaMemcpyHostToDevice,
                              ctx->stream));
  LFX_CK(ctx, cudaMemsetAsync(m->x32, 0, (size_t)n * kBS * 4, ctx->stream));
  bcg_mask<<<ctx->num_sms * 8, 256, 0, ctx->stream>>>(n, m->r32, st->active);
  // r0: column norms of R (the update kernel's norm pass, products left out)
  upd_launch<0>(ctx, G)(n, m->p32, m->q32, m->x32, m->r32, m->dinv, st, 1,
                                            m->bpart);
  bcg_reduce<<<1, kBS, 0, ctx->stream>>>(G, kBS, m->bpart, st->rn, st);
  bcg_small<<<1, 256, kBcgSmallSmem, ctx->stream>>>(3, st, tol);
  // P = orth(D^-1 R)
  upd_launch<1>(ctx, G)(n, m->p32, m->r32, m->w32, nullptr, m->dinv, st, 1,
                                            nullptr);
  int rc = gram<1>(m, m->w32, m->w32, nullptr, nullptr, st, st->G);
  if (rc) return rc;
  bcg_small<<<1, 256, kBcgSmallSmem, ctx->stream>>>(2, st, tol);
  upd_launch<2>(ctx, G)(n, m->w32, nullptr, m->p32, nullptr, nullptr, st, 0,
                                            nullptr);
  ctx->launches += 10;
  LFX_CK(ctx, cudaGetLastError());
  int it = 0;
  while (it < max_inner) {
    // Q = A P; alpha
    rc = mrhs_launch(m, m->p32, m->q32);
    if (!rc) rc = gram<2>(m, m->p32, m->q32, m->r32, nullptr, st, st->C);
    if (rc) return rc;
    bcg_small<<<1, 256, kBcgSmallSmem, ctx->stream>>>(0, st, tol);
    // X += P alpha, R -= Q alpha, ||R_j||
    upd_launch<0>(ctx, G)(n, m->p32, m->q32, m->x32, m->r32, m->dinv, st, 0,
                                              m->bpart);
    bcg_reduce<<<1, kBS, 0, ctx->stream>>>(G, kBS, m->bpart, st->rn, st);
    // beta (and convergence)
    rc = gram<1>(m, m->q32, m->r32, nullptr, m->dinv, st, st->E);
    if (rc) return rc;
    bcg_small<<<1, 256, kBcgSmallSmem, ctx->stream>>>(1, st, tol);
    // P = orth(D^-1 R + P beta)
    upd_launch<1>(ctx, G)(n, m->p32, m->r32, m->w32, nullptr, m->dinv, st, 0,
                                              nullptr);
    rc = gram<1>(m, m->w32, m->w32, nullptr, nullptr, st, st->G);
    if (rc) return rc;
    bcg_small<<<1, 256, kBcgSmallSmem, ctx->stream>>>(2, st, tol);
    upd_launch<2>(ctx, G)(n, m->w32, nullptr, m->p32, nullptr, nullptr, st,
                                              0, nullptr);
    ctx->launches += 13;
    LFX_CK(ctx, cudaGetLastError());
    ++it;
    LFX_CK(ctx, cudaMemcpyAsync(&m->h_bcg->rank, &st->rank, 4 * sizeof(int),
                                cudaMemcpyDeviceToHost, ctx->stream));
    LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
    if (m->h_bcg->done) break;
  }
  *inner_its = m->h_bcg->iters;
  *failed = m->h_bcg->fail;
  return LFX_OK;
}

template <int NR>
int add_correction(lfx_mrhs* m, double* x, int64_t ld) {
  lfx_ctx* ctx = m->ctx;
  const int64_t n = m->undf;
  const dim3 tb(32, 8), tg((unsigned)((n + 31) / 32), NR < 32 ? 1 : NR / 32);
  mv_add_to_rhs_major<NR><<<tg, tb, 0, ctx->stream>>>(n, m->x32, x, ld);
  ctx->launches++;
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

}  // namespace

int lfx_mrhs_set_gram(lfx_mrhs* m, int32_t tensor) {
  if (!m || (tensor != 0 && tensor != 1)) return LFX_INVALID_ARGUMENT;
  m->gram_tc = tensor;
  return LFX_OK;
}

int lfx_mrhs_gram(lfx_mrhs* m, const float* U, const float* V0, const float* V1, int32_t nv,
                  int32_t tensor, double* out) {
  if (!m || !U || !V0 || !out || (nv != 1 && nv != 2) || (nv == 2 && !V1) ||
      (tensor != 0 && tensor != 1))
    return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = m->ctx;
  if (m->nrhs != kBS) return fail(ctx, LFX_NOT_SUPPORTED, "Gram products of 64 columns only");
  int rc = ensure_work(m);
  if (!rc) rc = ensure_bcg(m);
  if (rc) return rc;
  LFX_CK(ctx, cudaMemsetAsync(m->bcg, 0, sizeof(BcgSmall), ctx->stream));
  const int keep = m->gram_tc;
  m->gram_tc = tensor;
  rc = nv == 1 ? gram<1>(m, U, V0, nullptr, nullptr, m->bcg, out)
               : gram<2>(m, U, V0, V1, nullptr, m->bcg, out);
  m->gram_tc = keep;
  if (rc) return rc;
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  int h_fail = 0;
  LFX_CK(ctx, cudaMemcpy(&h_fail, &m->bcg->fail, sizeof(int), cudaMemcpyDeviceToHost));
  if (h_fail) return fail(ctx, LFX_TIMEOUT, "a tensor-core wait ran out");
  return LFX_OK;
}

int lfx_mrhs_solve(lfx_mrhs* m, lfx_op* op64, const lfx_vec* diag, const double* b, double* x,
                   int64_t ld, const lfx_mrhs_cfg* cfg, lfx_solve_info* info) {
  if (!m || !op64 || !diag || !b || !x || !cfg || !info) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = m->ctx;
  if (op64->precision != LFX_R64 || op64->lay->undf_to != m->undf || op64->lay->undf_from != m->undf)
    return fail(ctx, LFX_INVALID_ARGUMENT, "op64 must be the FP64 operator of the same space");
  if (diag->precision != LFX_R64 || diag->data.size() != 1 || diag->undf[0] != m->undf)
    return fail(ctx, LFX_INVALID_ARGUMENT, "diag must be one FP64 field of undf values");
  if (ld < m->undf) return fail(ctx, LFX_INVALID_ARGUMENT, "ld must be at least undf");
  if (!(cfg->r_tol > 0.0) || !(cfg->inner_tol > 0.0) || !(cfg->inner_tol < 1.0) ||
      cfg->max_outer < 1 || cfg->max_inner < 1 ||
      (cfg->method != LFX_MRHS_PER_RHS_CG && cfg->method != LFX_MRHS_BLOCK_CG))
    return fail(ctx, LFX_INVALID_ARGUMENT, "bad tolerances, iteration limits or method");
  const bool block = cfg->method == LFX_MRHS_BLOCK_CG;
  if (block && m->nrhs != kBS)
    return fail(ctx, LFX_NOT_SUPPORTED, "block CG runs 64 right-hand sides");
  int rc = ensure_work(m);
  if (!rc && block) rc = ensure_bcg(m);
  if (rc) return rc;
  std::vector<int> bcg_its(m->nrhs, 0);
  const int nr = m->nrhs;
  const int64_t n = m->undf;
  k_dinv<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(n, (const double*)diag->data[0],
                                                                m->dinv);
  LFX_CK(ctx, cudaGetLastError());
  LFX_CK(ctx, cudaMemsetAsync(m->S, 0, sizeof(MvState), ctx->stream));
  std::vector<double> r0(nr), rn(nr);
  std::vector<int> act(64, 0), outer_n(nr, 0);
  rc = outer_residual(m, op64, b, x, ld);
  if (rc) return rc;
  for (int r = 0; r < nr; ++r) r0[r] = rn[r] = m->h_nrm[r];
  int outer = 0, inner_total = 0;
  for (;;) {
    int nact = 0;
    for (int r = 0; r < nr; ++r) {
      const bool conv = r0[r] == 0.0 || rn[r] <= cfg->r_tol * r0[r];
      act[r] = !conv && std::isfinite(rn[r]);
      nact += act[r];
    }
    if (nact == 0 || outer >= cfg->max_outer) break;
    int its = 0, bfail = 0;
    if (block) {
      rc = bcg_inner(m, act.data(), cfg->inner_tol, cfg->max_inner, &its, &bfail);
      for (int r = 0; r < nr; ++r)
        if (act[r]) bcg_its[r] += its;
    } else {
      rc = nr == 16 ? inner_solve<16>(m, act.data(), cfg->inner_tol, cfg->max_inner, &its)
           : nr == 32 ? inner_solve<32>(m, act.data(), cfg->inner_tol, cfg->max_inner, &its)
                      : inner_solve<64>(m, act.data(), cfg->inner_tol, cfg->max_inner, &its);
    }
    if (!rc) rc = nr == 16 ? add_correction<16>(m, x, ld)
                  : nr == 32 ? add_correction<32>(m, x, ld)
                             : add_correction<64>(m, x, ld);
    if (rc) return rc;
    inner_total += its;
    for (int r = 0; r < nr; ++r) outer_n[r] += act[r];
    ++outer;
    rc = outer_residual(m, op64, b, x, ld);
    if (rc) return rc;
    for (int r = 0; r < nr; ++r) rn[r] = m->h_nrm[r];
  }
  LFX_CK(ctx, cudaMemcpyAsync(m->h_S, m->S, sizeof(MvState), cudaMemcpyDeviceToHost, ctx->stream));
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  rc = lfx_ctx_check_device_error(ctx);
  for (int r = 0; r < nr; ++r) {
    lfx_solve_info& I = info[r];
    memset(&I, 0, sizeof I);
    I.initial_norm = r0[r];
    I.final_norm = rn[r];
    I.final_rel = r0[r] > 0.0 ? rn[r] / r0[r] : 0.0;
    I.converged = r0[r] == 0.0 || rn[r] <= cfg->r_tol * r0[r];
    I.outer_iterations = outer_n[r];
    I.inner_iterations = block ? bcg_its[r] : m->h_S->iters[r];
    I.iterations = I.inner_iterations;
    I.applies = inner_total;
    I.status = I.converged ? LFX_OK : (std::isfinite(rn[r]) ? LFX_NOT_CONVERGED : LFX_NAN_DETECTED);
  }
  return rc;
}
