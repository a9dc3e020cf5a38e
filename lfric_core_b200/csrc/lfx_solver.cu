// Device-resident Krylov solvers: cg_solve, bicgstab_solve and gmres_solve of
// components/science/source/solver/sci_iterative_solver_mod.f90 (:495-592,
// :645-779, :830-1003), plus FP64 iterative refinement around a reduced-
// precision inner solve.
//
// Every scalar of the recurrences lives in device memory and is updated by the
// last block of the fused reduction kernel that produces it (see
// chunk_kernel), so an iteration issues no host round trip. Kernels take a
// "done" flag and return at once when it is set. The kernel sequence of one
// GMRES restart cycle, or of 8 CG / BiCGStab iterations, is captured once into
// a CUDA graph (per solution / right-hand-side buffer pair) and replayed; the
// host reads the flag once per replay. Vector updates that the reference
// performs as separate builtins are fused when the fusion does not change a
// single rounding (e.g. t = r; t += a v  ==>  t = fma(a, v, r)).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <functional>

#include <type_traits>

#include "lfx_internal.cuh"

namespace lfx {
int drain_timing(lfx_ctx* ctx);
}
using namespace lfx;

namespace {

constexpr int MAX_GCRK = 64;
constexpr double EPS_RDEF = DBL_EPSILON;  // constants_mod.F90:167

struct DevState {
  int done, converged, iter, status;
  int applies, monitor, max_iter, askip;  // askip: skip the rest of a GMRES cycle
  int m, inner_mode;                      // m: Krylov vectors used by the cycle
  int x_zero, x_nonzero;                  // initial guess all zero / not (residual skip flags)
  double r_tol, a_tol;
  double r_nrm_0, r_nrm, rz, alpha, neg_alpha, beta;
  // bicgstab
  double rho, rho_old, omega, coef, tt, ts, sc_err, err;
  // gmres
  double gbeta, gbeta0, inv_beta, res_norm, inv_hn;
};

struct VecPtrs {
  const void* p[MAX_GCRK];
};

struct GraphEntry {
  const void* x = nullptr;
  const void* b = nullptr;
  bool timed = false;
  int variant = 0;  // bodies that differ for the same vectors (one-cycle runs)
  cudaGraphExec_t exec = nullptr;
  std::vector<TimedPair> ev;  // apply-timing events recorded by the graph
  int64_t kernels = 0;
};

}  // namespace

struct lfx_solver {
  lfx_ctx* ctx = nullptr;
  int kind = 0;
  lfx_op* op = nullptr;
  lfx_prec* prec = nullptr;
  lfx_solver_cfg cfg{};
  int32_t precision = LFX_R64;
  int64_t n = 0;
  std::vector<void*> work;  // owned device vectors of n elements
  DevState* d_state = nullptr;
  DevState* h_state = nullptr;      // pinned, mapped into the device's address space
  DevState* h_state_dev = nullptr;  // its device address
  double* d_gm = nullptr;       // gmres: H, negH, g, u, cs, sn, basis scales
  bool inner_mode = false;      // GMRES used as the inner solve of a refinement
  bool zero_x0 = false;         // the next apply starts from x = 0 (set by the refinement)
  std::vector<GraphEntry> graphs;
  int pending = -1;  // graph launched last, whose timings are not collected yet
  std::vector<lfx_vec*> hv;  // work vectors of the host-driven solvers
  double rho_relax = 1.0, lmin = 0.0, lmax = 0.0;  // Jacobi / Chebyshev
  // refined solver
  lfx_solver* inner = nullptr;
  double inner_rtol = 0.0;
  lfx_vec *r32 = nullptr, *d32 = nullptr;
  double* d_r64 = nullptr;
};

namespace {

size_t esz(int32_t p) { return p == LFX_R64 ? 8 : 4; }
size_t gm_doubles(int K) { return 2 * (size_t)(K + 1) * K + 2 * (size_t)(K + 1) + 3 * (size_t)K + 8; }

int read_state(lfx_solver* s) {
  lfx_ctx* ctx = s->ctx;
  int rc = to_host_small(ctx, s->h_state_dev, s->d_state, sizeof(DevState));
  if (rc) return rc;
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return LFX_OK;
}

// the initial state travels as a kernel argument (no copy engine involved)
__global__ void put_state(DevState* d, DevState h) { *d = h; }

int init_state(lfx_solver* s) {
  DevState h{};
  h.r_tol = s->cfg.r_tol;
  h.a_tol = s->cfg.a_tol;
  h.max_iter = s->cfg.max_iter;
  h.monitor = s->cfg.monitor_convergence ? 1 : 0;
  h.inner_mode = s->inner_mode ? 1 : 0;
  h.m = s->cfg.gcrk;
  *s->h_state = h;
  put_state<<<1, 1, 0, s->ctx->stream>>>(s->d_state, h);
  s->ctx->launches++;
  LFX_CK(s->ctx, cudaGetLastError());
  return LFX_OK;
}

// Runs `body` (a fixed sequence of launches on the context stream) through a
// CUDA graph cached per (x, b) pair, then reads the device state (wait) or
// leaves the graph queued (!wait: the caller reads the state later and then
// calls collect_timing).
// flags[0] (nonzero = true) stays set and flags[1] stays clear while every
// x[i] is zero; any nonzero entry clears the first and sets the second
template <class T>
__global__ void __launch_bounds__(256) zero_check(int64_t n, const T* __restrict__ x, int* flags) {
  for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256)
    if (x[i] != T(0)) {
      flags[0] = 0;
      flags[1] = 1;
    }
}

// r = b - A x, where a zero initial guess (checked on the device) skips the
// apply and copies b: b - A 0 = b exactly, so the bits are those of the
// apply; a nonzero x costs one extra read of x
template <class T>
int residual_from(lfx_solver* s, lfx_op* op, const T* x, T* r, const T* b, int* flags) {
  lfx_ctx* ctx = s->ctx;
  const int64_t n = s->n;
  LFX_CK(ctx, cudaMemsetAsync(flags, 0x01, sizeof(int), ctx->stream));
  LFX_CK(ctx, cudaMemsetAsync(flags + 1, 0, sizeof(int), ctx->stream));
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((n + 1023) / 1024, ctx->num_sms * 8));
  zero_check<T><<<grid, 256, 0, ctx->stream>>>(n, x, flags);
  ctx->launches++;
  LFX_CK(ctx, cudaGetLastError());
  // (not in the per-apply timings: it may idle)
  const bool timed = ctx->time_applies;
  ctx->time_applies = false;
  int rc = op_apply_impl(op, x, r, b, flags);  // idles when x == 0
  ctx->time_applies = timed;
  if (rc) return rc;
  return launch_chunks<0>(
      ctx, n, [=] __device__(int64_t i) { return V1<T>{b[i]}; },
      [=] __device__(int64_t i, const V1<T>& v, double*) { r[i] = v.a; }, NoFin{},
      flags + 1);  // idles when x != 0
}

// adds the apply timings of the last launched graph (finished) to the context
void collect_timing(lfx_solver* s) {
  lfx_ctx* ctx = s->ctx;
  const int pi = s->pending;
  s->pending = -1;
  if (pi < 0 || pi >= (int)s->graphs.size() || !ctx->time_applies) return;
  GraphEntry* ge = &s->graphs[pi];
  for (auto& p : ge->ev) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      const int k = p.prec == LFX_R32 ? 1 : 0;
      ctx->timed_ms[k] += ms;
      ctx->timed_launches[k] += 1;
    }
  }
}

int run_graph(lfx_solver* s, const void* x, const void* b, const std::function<int()>& body,
              bool wait = true, int variant = 0) {
  lfx_ctx* ctx = s->ctx;
  GraphEntry* ge = nullptr;
  for (auto& g : s->graphs)
    if (g.x == x && g.b == b && g.timed == ctx->time_applies && g.variant == variant) ge = &g;
  if (!ge) {
    GraphEntry g;
    g.variant = variant;
    g.x = x;
    g.b = b;
    g.timed = ctx->time_applies;
    cudaGraph_t graph = nullptr;
    LFX_CK(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    std::vector<TimedPair> ev;
    ctx->capture_ev = &ev;
    const int64_t l0 = ctx->launches;
    int rc = body();
    ctx->capture_ev = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    if (rc || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      for (auto& p : ev) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
      }
      return rc ? rc : cuda_fail(ctx, e, "cudaStreamEndCapture");
    }
    e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
    g.ev = std::move(ev);
    g.kernels = ctx->launches - l0;  // kernels in one replay (capture launched none)
    ctx->launches = l0;
    s->graphs.push_back(std::move(g));
    ge = &s->graphs.back();
  }
  LFX_CK(ctx, cudaGraphLaunch(ge->exec, ctx->stream));
  ctx->launches += ge->kernels;
  s->pending = (int)(ge - s->graphs.data());
  if (!wait) return LFX_OK;
  int rc = read_state(s);
  if (rc) return rc;
  collect_timing(s);
  return LFX_OK;
}

void free_graphs(lfx_solver* s) {
  for (auto& g : s->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto& p : g.ev) {
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
  }
  s->graphs.clear();
  s->pending = -1;
}

template <class T, int N>
struct Pack {
  T v[N];
};

// Classical Gram-Schmidt, inner products: h(j) = <v_j, w>, j < NR, one pass.
template <class T, int NR>
int cgs_dots(lfx_ctx* ctx, int64_t n, const VecPtrs& vp, const T* w, double* hcol, double* nhcol,
             const int* skip) {
  return launch_chunks<NR>(
      ctx, n,
      [=] __device__(int64_t i) {
        Pack<T, NR + 1> q;
#pragma unroll
        for (int j = 0; j < NR; ++j) q.v[j] = ((const T*)vp.p[j])[i];
        q.v[NR] = w[i];
        return q;
      },
      [=] __device__(int64_t, const Pack<T, NR + 1>& q, double* a) {
#pragma unroll
        for (int j = 0; j < NR; ++j) a[j] = fma((double)q.v[j], (double)q.v[NR], a[j]);
      },
      [=] __device__(const double* t) {
        for (int j = 0; j < NR; ++j) {
          hcol[j] = t[j];
          nhcol[j] = -t[j];
        }
      },
      skip);
}

// Classical Gram-Schmidt, update: w -= sum_j h(j) v_j (in order) and ||w||;
// fin receives the norm.
template <class T, int NR, class Fin>
int cgs_update(lfx_ctx* ctx, int64_t n, const VecPtrs& vp, T* w, const double* nhcol, Fin fin,
               const int* skip) {
  return launch_chunks<1>(
      ctx, n,
      [=] __device__(int64_t i) {
        Pack<T, NR + 1> q;
#pragma unroll
        for (int j = 0; j < NR; ++j) q.v[j] = ((const T*)vp.p[j])[i];
        q.v[NR] = w[i];
        return q;
      },
      [=] __device__(int64_t i, const Pack<T, NR + 1>& q, double* a) {
        T wi = q.v[NR];
#pragma unroll
        for (int j = 0; j < NR; ++j) wi = fmaT((T)nhcol[j], q.v[j], wi);
        w[i] = wi;
        a[0] = fma((double)wi, (double)wi, a[0]);
      },
      fin, skip);
}

// FP32 classical Gram-Schmidt of the inner solve, streamed as float4 quads:
// every thread walks its quads of the NR basis vectors and w in a grid-stride
// loop (all loads of a quad issued together), adds each quad's products,
// formed in FP32, into FP64 running sums, and the block reduces once at the
// end. The last block to finish sums the block partials warp by warp in block
// order, so the result is fixed for a given grid (the grid depends only on n
// and the GPU's SM count). The n % 4 tail goes to block 0.
constexpr int kCgsThreads = 256;

__device__ __forceinline__ float quad_dot(const float4& a, const float4& b) {
  float s = a.x * b.x;
  s = fmaf(a.y, b.y, s);
  s = fmaf(a.z, b.z, s);
  return fmaf(a.w, b.w, s);
}

// block sums of acc[0..NR) into partials[r * grid + block]; returns true in
// every thread of the last block, whose tot[0..NR) (valid in all its threads)
// then holds the grand totals
template <int NR>
__device__ __forceinline__ bool cgs_reduce(double (&acc)[NR], double* partials, unsigned* ticket,
                                           double (&tot)[NR]) {
  __shared__ double sm[kCgsThreads / 32][NR];
  __shared__ double st[NR];
  __shared__ int am_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    const double v = warp_butterfly(acc[r]);
    if (lane == 0) sm[warp][r] = v;
  }
  __syncthreads();
  if (threadIdx.x < NR) {
    double t = sm[0][threadIdx.x];
#pragma unroll
    for (int q = 1; q < kCgsThreads / 32; ++q) t = t + sm[q][threadIdx.x];
    partials[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = t;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  for (int r = warp; r < NR; r += kCgsThreads / 32) {
    double a = 0.0;
    for (int i = lane; i < (int)gridDim.x; i += 32) a = a + __ldcg(&partials[(int64_t)r * gridDim.x + i]);
    a = warp_butterfly(a);
    if (lane == 0) st[r] = a;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < NR; ++r) tot[r] = st[r];
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

// grid-stride steps per loop trip of the float4 Gram-Schmidt kernels: with
// few basis vectors a thread has too few loads in flight per step
template <int NR>
struct CgsUnroll {
  static constexpr int U = NR <= 2 ? 4 : (NR <= 5 ? 2 : 1);
};

// sig (nullable): the basis is stored unnormalised, v_j = sig[j] u_j, and the
// true vector is sig[prev] w; then hcol receives the true inner products
// <v_j, sig[prev] w> and nhcol the update coefficients -sig[j]^2 <u_j, w>
template <int NR>
__global__ void __launch_bounds__(kCgsThreads) cgs_dots_f4(int64_t n, VecPtrs vp,
                                                           const float* __restrict__ w,
                                                           double* hcol, double* nhcol,
                                                           const double* sig, int prev,
                                                           double* partials, unsigned* ticket,
                                                           const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  double acc[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) acc[r] = 0.0;
  const int64_t n4 = n >> 2;
  const float4* w4 = reinterpret_cast<const float4*>(w);
  // CgsUnroll<NR>::U grid-stride steps per trip, loads first (the same
  // element order per thread as one step per trip)
  constexpr int U = CgsUnroll<NR>::U;
  const int64_t stride = (int64_t)gridDim.x * kCgsThreads;
  for (int64_t q0 = (int64_t)blockIdx.x * kCgsThreads + threadIdx.x; q0 < n4; q0 += U * stride) {
    float4 v[U][NR], wq[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t q = q0 + u * stride;
      if (q < n4) {
#pragma unroll
        for (int r = 0; r < NR; ++r) v[u][r] = __ldg(reinterpret_cast<const float4*>(vp.p[r]) + q);
        wq[u] = __ldg(w4 + q);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (q0 + u * stride < n4) {
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] += (double)quad_dot(v[u][r], wq[u]);
      }
  }
  if (blockIdx.x == 0 && threadIdx.x < (n & 3)) {
    const int64_t i = 4 * n4 + threadIdx.x;
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] += (double)(((const float*)vp.p[r])[i] * w[i]);
  }
  double tot[NR];
  if (cgs_reduce<NR>(acc, partials, ticket, tot) && threadIdx.x == 0) {
    for (int r = 0; r < NR; ++r) {
      if (sig) {
        hcol[r] = sig[r] * sig[prev] * tot[r];
        nhcol[r] = -(sig[r] * sig[r]) * tot[r];
      } else {
        hcol[r] = tot[r];
        nhcol[r] = -tot[r];
      }
    }
  }
}

// out = w + sum_j nhcol[j] v_j (out may be w) and fin(||out||^2)
template <int NR, class Fin>
__global__ void __launch_bounds__(kCgsThreads) cgs_update_f4(int64_t n, VecPtrs vp,
                                                             const float* w, float* out,
                                                             const double* nhcol, Fin fin,
                                                             double* partials, unsigned* ticket,
                                                             const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  float c[NR];
#pragma unroll
  for (int r = 0; r < NR; ++r) c[r] = (float)nhcol[r];
  double acc[1] = {0.0};
  const int64_t n4 = n >> 2;
  const float4* w4 = reinterpret_cast<const float4*>(w);
  float4* o4 = reinterpret_cast<float4*>(out);
  constexpr int U = CgsUnroll<NR>::U;
  const int64_t stride = (int64_t)gridDim.x * kCgsThreads;
  for (int64_t q0 = (int64_t)blockIdx.x * kCgsThreads + threadIdx.x; q0 < n4; q0 += U * stride) {
    float4 v[U][NR], wq[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t q = q0 + u * stride;
      if (q < n4) {
#pragma unroll
        for (int r = 0; r < NR; ++r) v[u][r] = __ldg(reinterpret_cast<const float4*>(vp.p[r]) + q);
        wq[u] = w4[q];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t q = q0 + u * stride;
      if (q < n4) {
        float4 o = wq[u];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          o.x = fmaf(c[r], v[u][r].x, o.x);
          o.y = fmaf(c[r], v[u][r].y, o.y);
          o.z = fmaf(c[r], v[u][r].z, o.z);
          o.w = fmaf(c[r], v[u][r].w, o.w);
        }
        o4[q] = o;
        acc[0] += (double)quad_dot(o, o);
      }
    }
  }
  if (blockIdx.x == 0 && threadIdx.x < (n & 3)) {
    const int64_t i = 4 * n4 + threadIdx.x;
    float wi = w[i];
#pragma unroll
    for (int r = 0; r < NR; ++r) wi = fmaf(c[r], ((const float*)vp.p[r])[i], wi);
    out[i] = wi;
    acc[0] += (double)(wi * wi);
  }
  double tot[1];
  if (cgs_reduce<1>(acc, partials, ticket, tot) && threadIdx.x == 0) fin(tot);
}

// blocks of a float4 Gram-Schmidt kernel resident on the GPU at once
template <class K>
int resident_blocks(const lfx_ctx* ctx, K kernel) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kCgsThreads, 0);
  return ctx->num_sms * std::max(per_sm, 1);
}

bool quad_aligned(const VecPtrs& vp, int nr, const void* w) {
  if ((uintptr_t)w & 15) return false;
  for (int r = 0; r < nr; ++r)
    if ((uintptr_t)vp.p[r] & 15) return false;
  return true;
}

template <int NR, class Fin>
int cgs_step_f4(lfx_ctx* ctx, int64_t n, const VecPtrs& vp, float* w, float* out, double* hcol,
                double* nhcol, const double* sig, int prev, Fin fin, const int* skip) {
  // one resident wave, and at most one block per 2048 values (the partials
  // scratch holds nchunks(n) values per sum)
  static int gd = 0, gu = 0;
  if (!gd) gd = resident_blocks(ctx, cgs_dots_f4<NR>);
  if (!gu) gu = resident_blocks(ctx, cgs_update_f4<NR, Fin>);
  const int64_t cap = std::max<int64_t>(1, nchunks(n));
  cgs_dots_f4<NR><<<(int)std::min<int64_t>(gd, cap), kCgsThreads, 0, ctx->stream>>>(
      n, vp, w, hcol, nhcol, sig, prev, ctx->d_partials, ctx->d_ticket, skip);
  cgs_update_f4<NR, Fin><<<(int)std::min<int64_t>(gu, cap), kCgsThreads, 0, ctx->stream>>>(
      n, vp, w, out, nhcol, fin, ctx->d_partials, ctx->d_ticket, skip);
  ctx->launches += 2;
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

template <class T, class Fin>
int cgs_step(lfx_ctx* ctx, int64_t n, int nr, const VecPtrs& vp, T* w, double* hcol,
             double* nhcol, Fin fin, const int* skip) {
  int rc = LFX_INVALID_ARGUMENT;
  if constexpr (std::is_same<T, float>::value) {
    if (quad_aligned(vp, nr, w)) {
      switch (nr) {
#define CGS_F4(N) \
  case N: return cgs_step_f4<N>(ctx, n, vp, w, w, hcol, nhcol, nullptr, 0, fin, skip);
        CGS_F4(1) CGS_F4(2) CGS_F4(3) CGS_F4(4) CGS_F4(5) CGS_F4(6)
        CGS_F4(7) CGS_F4(8) CGS_F4(9) CGS_F4(10) CGS_F4(11) CGS_F4(12)
#undef CGS_F4
      }
    }
  }
  switch (nr) {
#define CGS_CASE(N)                                                          \
  case N:                                                                    \
    rc = cgs_dots<T, N>(ctx, n, vp, w, hcol, nhcol, skip);                   \
    if (!rc) rc = cgs_update<T, N>(ctx, n, vp, w, nhcol, fin, skip);         \
    break;
    CGS_CASE(1) CGS_CASE(2) CGS_CASE(3) CGS_CASE(4) CGS_CASE(5) CGS_CASE(6)
    CGS_CASE(7) CGS_CASE(8) CGS_CASE(9) CGS_CASE(10) CGS_CASE(11) CGS_CASE(12)
#undef CGS_CASE
  }
  return rc;
}
constexpr int kMaxCgs = 12;

// Gram-Schmidt step of the inner solve over an unnormalised FP32 basis
// (v_j = sig[j] u_j; the true vector is sig[nr - 1] w): out = w - sum_j
// sig[j]^2 <u_j, w> u_j, the next basis vector unnormalised, whose scale
// sig[nr] = sig[nr - 1] / ||sig[nr - 1] out|| the norm's fin sets.
template <class Fin>
int cgs_step_lazy(lfx_ctx* ctx, int64_t n, int nr, const VecPtrs& vp, float* w, float* out,
                  double* hcol, double* nhcol, const double* sig, Fin fin, const int* skip) {
  switch (nr) {
#define CGS_LZ(N) \
  case N: return cgs_step_f4<N>(ctx, n, vp, w, out, hcol, nhcol, sig, N - 1, fin, skip);
    CGS_LZ(1) CGS_LZ(2) CGS_LZ(3) CGS_LZ(4) CGS_LZ(5) CGS_LZ(6)
    CGS_LZ(7) CGS_LZ(8) CGS_LZ(9) CGS_LZ(10) CGS_LZ(11) CGS_LZ(12)
#undef CGS_LZ
  }
  return LFX_INVALID_ARGUMENT;
}

template <class T>
int norm_kernel(lfx_ctx* ctx, int64_t n, const T* v, double* out, const int* skip) {
  return launch_chunks<1>(
      ctx, n, [=] __device__(int64_t i) { return V1<T>{v[i]}; },
      [=] __device__(int64_t, const V1<T>& q, double* a) { a[0] = fma((double)q.a, (double)q.a, a[0]); },
      [=] __device__(const double* t) { *out = sqrt(t[0]); }, skip);
}

// ------------------------------------------------------------------ CG
template <class T>
int cg_run(lfx_solver* s, T* x, const T* b) {
  lfx_ctx* ctx = s->ctx;
  DevState* S = s->d_state;
  const int64_t n = s->n;
  T* r = (T*)s->work[0];
  T* p = (T*)s->work[1];
  T* z = (T*)s->work[2];
  const int* done = &S->done;
  int rc;
  // r = b - A x   (apply, scale(-1), axpy(1, b): one rounding, b - Ax)
  if ((rc = op_apply_impl(s->op, x, r, b, nullptr))) return rc;
  rc = launch_chunks<1>(
      ctx, n, [=] __device__(int64_t i) { return V1<T>{r[i]}; },
      [=] __device__(int64_t, const V1<T>& q, double* a) { a[0] = fma((double)q.a, (double)q.a, a[0]); },
      [=] __device__(const double* t) {
        S->applies = 1;
        S->r_nrm_0 = sqrt(t[0]);
        if (S->r_nrm_0 < EPS_RDEF) {  // :531
          S->done = 1;
          S->converged = 1;
          S->r_nrm = S->r_nrm_0;
        }
      });
  if (rc) return rc;
  if ((rc = prec_apply_impl(s->prec, s->precision, r, z, n, done))) return rc;
  rc = launch_chunks<1>(
      ctx, n, [=] __device__(int64_t i) { return V2<T>{r[i], z[i]}; },
      [=] __device__(int64_t i, const V2<T>& q, double* a) {
        p[i] = q.b;
        a[0] = fma((double)q.a, (double)q.b, a[0]);
      },
      [=] __device__(const double* t) { S->rz = t[0]; }, done);
  if (rc) return rc;
  const bool diag_prec = s->prec->kind == PREC_DIAG;
  const T* dg = (const T*)s->prec->rdiag;
  auto batch = [&]() -> int {
    int q;
    for (int it = 0; it < 8; ++it) {
      if ((q = op_apply_impl(s->op, p, z, nullptr, done))) return q;  // z = A p
      q = launch_chunks<1>(
          ctx, n, [=] __device__(int64_t i) { return V2<T>{p[i], z[i]}; },
          [=] __device__(int64_t, const V2<T>& v, double* a) {
            a[0] = fma((double)v.a, (double)v.b, a[0]);
          },
          [=] __device__(const double* t) {
            S->applies += 1;
            S->alpha = S->rz / t[0];
            S->neg_alpha = -S->alpha;
          },
          done);
      if (q) return q;
      // x += alpha p ; r -= alpha z ; ||r||
      q = launch_chunks<1>(
          ctx, n, [=] __device__(int64_t i) { return V4<T>{x[i], p[i], r[i], z[i]}; },
          [=] __device__(int64_t i, const V4<T>& v, double* a) {
            x[i] = fmaT((T)S->alpha, v.b, v.a);
            const T ri = fmaT((T)S->neg_alpha, v.d, v.c);
            r[i] = ri;
            a[0] = fma((double)ri, (double)ri, a[0]);
          },
          [=] __device__(const double* t) {
            S->iter += 1;
            S->r_nrm = sqrt(t[0]);
            if (S->monitor) {
              if (S->r_nrm / S->r_nrm_0 <= S->r_tol || S->r_nrm <= S->a_tol) {  // :563
                S->done = 1;
                S->converged = 1;
              } else if (isnan(S->r_nrm)) {
                S->done = 1;
                S->status = LFX_NAN_DETECTED;
              }
            }
            if (S->iter >= S->max_iter) S->done = 1;
          },
          done);
      if (q) return q;
      // z = P r ; rz_new = <r, z> ; beta ; p = beta p + z
      auto fin_beta = [=] __device__(const double* t) {
        S->beta = t[0] / S->rz;
        S->rz = t[0];
      };
      if (diag_prec) {
        q = launch_chunks<1>(
            ctx, n, [=] __device__(int64_t i) { return V2<T>{r[i], dg[i]}; },
            [=] __device__(int64_t i, const V2<T>& v, double* a) {
              const T zi = v.a / v.b;
              z[i] = zi;
              a[0] = fma((double)v.a, (double)zi, a[0]);
            },
            fin_beta, done);
      } else {
        if ((q = prec_apply_impl(s->prec, s->precision, r, z, n, done))) return q;
        q = launch_chunks<1>(
            ctx, n, [=] __device__(int64_t i) { return V2<T>{r[i], z[i]}; },
            [=] __device__(int64_t, const V2<T>& v, double* a) {
              a[0] = fma((double)v.a, (double)v.b, a[0]);
            },
            fin_beta, done);
      }
      if (q) return q;
      q = launch_chunks<0>(
          ctx, n, [=] __device__(int64_t i) { return V2<T>{p[i], z[i]}; },
          [=] __device__(int64_t i, const V2<T>& v, double*) { p[i] = fmaT((T)S->beta, v.a, v.b); },
          NoFin{}, done);
      if (q) return q;
    }
    return LFX_OK;
  };
  // no host round trip before the first graph: its kernels idle if the
  // initial residual already ended the solve (device flags)
  do {
    if ((rc = run_graph(s, x, b, batch))) return rc;
  } while (!s->h_state->done);
  return LFX_OK;
}

// ------------------------------------------------------------------ BiCGStab
template <class T>
int bicgstab_run(lfx_solver* s, T* x, const T* b) {
  lfx_ctx* ctx = s->ctx;
  DevState* S = s->d_state;
  const int64_t n = s->n;
  T *r = (T*)s->work[0], *r0 = (T*)s->work[1], *p = (T*)s->work[2], *v = (T*)s->work[3];
  T *t = (T*)s->work[4], *sv = (T*)s->work[5], *y = (T*)s->work[6], *z = (T*)s->work[7];
  const int* done = &S->done;
  int rc;
  // v = A x ; r = b - v ; r0 = r ; sc_err = ||r|| ; v = p = 0
  if ((rc = op_apply_impl(s->op, x, r, b, nullptr))) return rc;
  rc = launch_chunks<1>(
      ctx, n, [=] __device__(int64_t i) { return V1<T>{r[i]}; },
      [=] __device__(int64_t i, const V1<T>& q, double* a) {
        r0[i] = q.a;
        v[i] = T(0);
        p[i] = T(0);
        a[0] = fma((double)q.a, (double)q.a, a[0]);
      },
      [=] __device__(const double* tt) {
        S->applies = 1;
        S->r_nrm_0 = sqrt(tt[0]);
        S->sc_err = S->r_nrm_0;
        if (S->sc_err < EPS_RDEF) {  // :692
          S->done = 1;
          S->converged = 1;
          S->r_nrm = S->sc_err;
        } else {
          S->sc_err = fmax(S->sc_err, S->a_tol);
        }
        S->alpha = 1.0;
        S->omega = 1.0;
        S->rho_old = 1.0;
      });
  if (rc) return rc;
  auto batch = [&]() -> int {
    int q;
    for (int it = 0; it < 8; ++it) {
      // rho = <r, r0> ; beta = (rho/rho_old)(alpha/omega)
      q = launch_chunks<1>(
          ctx, n, [=] __device__(int64_t i) { return V2<T>{r[i], r0[i]}; },
          [=] __device__(int64_t, const V2<T>& w, double* a) {
            a[0] = fma((double)w.a, (double)w.b, a[0]);
          },
          [=] __device__(const double* tt) {
            S->rho = tt[0];
            S->beta = (S->rho / S->rho_old) * (S->alpha / S->omega);
            S->coef = -(S->beta * S->omega);
          },
          done);
      if (q) return q;
      // t = r - beta*omega v
      q = launch_chunks<0>(
          ctx, n, [=] __device__(int64_t i) { return V2<T>{v[i], r[i]}; },
          [=] __device__(int64_t i, const V2<T>& w, double*) { t[i] = fmaT((T)S->coef, w.a, w.b); },
          NoFin{}, done);
      if (q) return q;
      if ((q = prec_apply_impl(s->prec, s->precision, t, y, n, done))) return q;
      q = launch_chunks<0>(
          ctx, n, [=] __device__(int64_t i) { return V2<T>{p[i], y[i]}; },
          [=] __device__(int64_t i, const V2<T>& w, double*) { p[i] = fmaT((T)S->beta, w.a, w.b); },
          NoFin{}, done);
      if (q) return q;
      if ((q = op_apply_impl(s->op, p, v, nullptr, done))) return q;
      q = launch_chunks<1>(
          ctx, n, [=] __device__(int64_t i) { return V2<T>{r0[i], v[i]}; },
          [=] __device__(int64_t, const V2<T>& w, double* a) {
            a[0] = fma((double)w.a, (double)w.b, a[0]);
          },
          [=] __device__(const double* tt) {
            S->alpha = S->rho / tt[0];
            S->neg_alpha = -S->alpha;
          },
          done);
      if (q) return q;
      q = launch_chunks<0>(
          ctx, n, [=] __device__(int64_t i) { return V2<T>{v[i], r[i]}; },
          [=] __device__(int64_t i, const V2<T>& w, double*) {
            sv[i] = fmaT((T)S->neg_alpha, w.a, w.b);
          },
          NoFin{}, done);
      if (q) return q;
      if ((q = prec_apply_impl(s->prec, s->precision, sv, z, n, done))) return q;
      if ((q = op_apply_impl(s->op, z, t, nullptr, done))) return q;
      q = launch_chunks<2>(
          ctx, n, [=] __device__(int64_t i) { return V2<T>{t[i], sv[i]}; },
          [=] __device__(int64_t, const V2<T>& w, double* a) {
            a[0] = fma((double)w.a, (double)w.a, a[0]);
            a[1] = fma((double)w.a, (double)w.b, a[1]);
          },
          [=] __device__(const double* tt) {
            S->applies += 2;
            S->tt = tt[0];
            S->ts = tt[1];
            S->omega = S->ts / S->tt;
          },
          done);
      if (q) return q;
      // x += omega z ; x += alpha p ; r = s - omega t ; ||r||
      q = launch_chunks<1>(
          ctx, n,
          [=] __device__(int64_t i) {
            return V3<T>{x[i], z[i], p[i]};
          },
          [=] __device__(int64_t i, const V3<T>& w, double* a) {
            const T om = (T)S->omega;
            const T xi = fmaT(om, w.b, w.a);
            x[i] = fmaT((T)S->alpha, w.c, xi);
            const T ri = fmaT(-om, t[i], sv[i]);
            r[i] = ri;
            a[0] = fma((double)ri, (double)ri, a[0]);
          },
          [=] __device__(const double* tt) {
            S->rho_old = S->rho;
            S->iter += 1;
            S->r_nrm = sqrt(tt[0]);
            S->err = S->r_nrm / S->sc_err;
            if (S->monitor) {
              if (S->err < S->r_tol) {  // :760
                S->done = 1;
                S->converged = 1;
              } else if (isnan(S->err)) {
                S->done = 1;
                S->status = LFX_NAN_DETECTED;
              }
            }
            if (S->iter >= S->max_iter) S->done = 1;
          },
          done);
      if (q) return q;
    }
    return LFX_OK;
  };
  // no host round trip before the first graph: its kernels idle if the
  // initial residual already ended the solve (device flags)
  do {
    if ((rc = run_graph(s, x, b, batch))) return rc;
  } while (!s->h_state->done);
  return LFX_OK;
}

// ------------------------------------------------------------------ GMRES
// Givens rotations and back substitution (:930-953) by one thread. In inner
// mode the rotations were already applied column by column as the Arnoldi
// process ran, and only the back substitution over the m vectors is left.
// x += sum_k u[k] v_k over the cycle's m basis vectors, 16 bytes per thread
// per pass (the reference's order per element, so the same bits as the
// scalar form); all pointers 16-byte aligned; the n % W tail in block 0
template <class T>
__global__ void __launch_bounds__(256) gmres_xupdate(int64_t n, VecPtrs vp, const double* u,
                                                     const int* mptr, T* x, const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  using Q = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
  constexpr int W = 16 / sizeof(T);
  const int m = *mptr;
  const int64_t nq = n / W;
  Q* xq = reinterpret_cast<Q*>(x);
  for (int64_t q = (int64_t)blockIdx.x * 256 + threadIdx.x; q < nq; q += (int64_t)gridDim.x * 256) {
    T xv[W];
    const Q a = xq[q];
    memcpy(xv, &a, 16);
#pragma unroll 4
    for (int k = 0; k < m; ++k) {
      const Q b = __ldg(reinterpret_cast<const Q*>(vp.p[k]) + q);
      T vv[W];
      memcpy(vv, &b, 16);
      const T uk = (T)u[k];
#pragma unroll
      for (int e = 0; e < W; ++e) xv[e] = fmaT(uk, vv[e], xv[e]);
    }
    Q o;
    memcpy(&o, xv, 16);
    xq[q] = o;
  }
  if (blockIdx.x == 0 && threadIdx.x < n - nq * W) {
    const int64_t i = nq * W + threadIdx.x;
    T xi = x[i];
    for (int k = 0; k < m; ++k) xi = fmaT((T)u[k], ((const T*)vp.p[k])[i], xi);
    x[i] = xi;
  }
}

// sig (nullable): scales of an unnormalised basis, folded into u
__global__ void gmres_finish_cycle(DevState* S, double* gm, int K, const double* sig,
                                   int count_cycle) {
  if (S->done) return;
  double* h = gm;                  // H(i,j) at (i-1) + (K+1)(j-1)
  double* g = gm + 2 * (K + 1) * K;
  double* u = g + (K + 1);
#define H(i, j) h[((i) - 1) + (K + 1) * ((j) - 1)]
  const int m = S->inner_mode ? S->m : K;
  if (!S->inner_mode) {
    for (int iv = 1; iv <= K; ++iv) {
      const double nrm = sqrt(fma(H(iv, iv), H(iv, iv), H(iv + 1, iv) * H(iv + 1, iv)));
      const double si = H(iv + 1, iv) / nrm;
      const double ci = H(iv, iv) / nrm;
      const double p = fma(ci, g[iv - 1], si * g[iv]);
      const double q = fma(-si, g[iv - 1], ci * g[iv]);
      g[iv - 1] = p;
      g[iv] = q;
      for (int ivj = iv; ivj <= K; ++ivj) {
        const double h1 = fma(ci, H(iv, ivj), si * H(iv + 1, ivj));
        const double h2 = fma(-si, H(iv, ivj), ci * H(iv + 1, ivj));
        H(iv, ivj) = h1;
        H(iv + 1, ivj) = h2;
      }
    }
  }
  u[m - 1] = g[m - 1] / H(m, m);
  for (int iv = m - 1; iv >= 1; --iv) {
    double a = g[iv - 1];
    for (int ivj = iv + 1; ivj <= m; ++ivj) a = fma(-H(iv, ivj), u[ivj - 1], a);
    u[iv - 1] = a / H(iv, iv);
  }
  if (sig)
    for (int iv = 0; iv < m; ++iv) u[iv] = u[iv] * sig[iv];
  S->m = m;
  if (count_cycle) S->iter += 1;  // the cycle ends without its own residual
#undef H
}

// one_cycle: queue the initial residual and exactly one restart cycle, without
// the cycle's closing residual, and return without waiting (the refinement
// reads the state after its own residual, in the same synchronisation; a NaN
// in the cycle reaches that FP64 residual through the solution update)
template <class T>
int gmres_run(lfx_solver* s, T* x, const T* b, bool one_cycle = false) {
  lfx_ctx* ctx = s->ctx;
  DevState* S = s->d_state;
  const int64_t n = s->n;
  const int K = s->cfg.gcrk;
  T* sv = (T*)s->work[0];
  T* w = (T*)s->work[1];
  T* res = (T*)s->work[2];
  T* V[MAX_GCRK];
  for (int k = 0; k < K; ++k) V[k] = (T*)s->work[3 + k];
  double* h = s->d_gm;
  double* nh = h + (K + 1) * K;
  double* g = nh + (K + 1) * K;
  double* u = g + (K + 1);
  double* cs = u + K;
  double* sn = cs + K;
  double* sig = sn + K;
  const int* done = &S->done;
  const int* askip = &S->askip;
  // the inner solve's FP32 basis is kept unnormalised (v_j = sig[j] u_j), so
  // no pass rescales it: the preconditioner writes u_0 and each Gram-Schmidt
  // update writes the next u_j directly
  bool lazy = false;
  if constexpr (std::is_same<T, float>::value) {
    lazy = s->inner_mode && K <= kMaxCgs && ((uintptr_t)w & 15) == 0;
    for (int k = 0; k < K; ++k) lazy = lazy && ((uintptr_t)V[k] & 15) == 0;
  }
  int rc;
  // res = b - A x ; sc_err = ||res||. When the refinement's inner solve
  // starts from x = 0, res = b exactly and the apply is skipped.
  const bool zero_x0 = s->zero_x0;
  s->zero_x0 = false;
  if (!zero_x0 && (rc = residual_from<T>(s, s->op, x, res, b, &S->x_zero))) return rc;
  const T* r0src = zero_x0 ? b : res;
  rc = launch_chunks<1>(
      ctx, n, [=] __device__(int64_t i) { return V1<T>{r0src[i]}; },
      [=] __device__(int64_t i, const V1<T>& q, double* a) {
        if (zero_x0) res[i] = q.a;
        a[0] = fma((double)q.a, (double)q.a, a[0]);
      },
      [=] __device__(const double* t) {
        S->applies = zero_x0 ? 0 : 1;
        S->r_nrm_0 = sqrt(t[0]);
        S->sc_err = S->r_nrm_0;
        if (S->sc_err < EPS_RDEF) {  // :866
          S->done = 1;
          S->askip = 1;
          S->converged = 1;
          S->r_nrm = S->sc_err;
        } else if (S->monitor) {
          S->sc_err = fmax(S->sc_err, S->a_tol);
        }
      });
  if (rc) return rc;
  VecPtrs vp{};
  for (int k = 0; k < K; ++k) vp.p[k] = V[k];
  auto cycle = [&]() -> int {
    int q;
    // s = P res ; beta = ||s|| ; v1 = s / beta ; g = (beta, 0, ...)
    T* s0 = lazy ? V[0] : sv;
    if ((q = prec_apply_impl(s->prec, s->precision, res, s0, n, done))) return q;
    q = launch_chunks<1>(
        ctx, n, [=] __device__(int64_t i) { return V1<T>{s0[i]}; },
        [=] __device__(int64_t, const V1<T>& v, double* a) { a[0] = fma((double)v.a, (double)v.a, a[0]); },
        [=] __device__(const double* t) {
          S->gbeta = sqrt(t[0]);
          if (S->iter == 0) S->gbeta0 = S->gbeta;
          S->inv_beta = 1.0 / S->gbeta;
          sig[0] = S->inv_beta;
          S->m = K;
          for (int k = 0; k <= K; ++k) g[k] = 0.0;
          g[0] = S->gbeta;
        },
        done);
    if (q) return q;
    if (!lazy) {
      T* v0 = V[0];
      q = launch_chunks<0>(
          ctx, n, [=] __device__(int64_t i) { return V1<T>{sv[i]}; },
          [=] __device__(int64_t i, const V1<T>& v, double*) { v0[i] = (T)S->inv_beta * v.a; },
          NoFin{}, done);
      if (q) return q;
    }
    for (int iv = 1; iv <= K; ++iv) {
      if ((q = op_apply_impl(s->op, V[iv - 1], sv, nullptr, askip))) return q;  // s = A v
      if ((q = prec_apply_impl(s->prec, s->precision, sv, w, n, askip))) return q;  // w = P s
      double* col = &h[(K + 1) * (iv - 1)];  // H(:, iv)
      const int ivc = iv;
      // last step of the orthogonalisation: H(iv+1, iv) = ||w||, and in inner
      // mode the column's Givens rotation and the in-cycle convergence test
      const bool lz = lazy;
      auto fin_norm = [=] __device__(const double* t) {
        const double hn = lz ? sig[ivc - 1] * sqrt(t[0]) : sqrt(t[0]);
        col[ivc] = hn;  // H(iv+1, iv)
        S->inv_hn = 1.0 / hn;
        sig[ivc] = lz ? sig[ivc - 1] * S->inv_hn : S->inv_hn;
        S->applies += 1;
        if (S->inner_mode) {
          for (int j = 1; j < ivc; ++j) {
            const double h1 = fma(cs[j - 1], col[j - 1], sn[j - 1] * col[j]);
            const double h2 = fma(-sn[j - 1], col[j - 1], cs[j - 1] * col[j]);
            col[j - 1] = h1;
            col[j] = h2;
          }
          const double a0 = col[ivc - 1], a1 = col[ivc];
          const double nrm = sqrt(fma(a0, a0, a1 * a1));
          const double ci = a0 / nrm, si = a1 / nrm;
          cs[ivc - 1] = ci;
          sn[ivc - 1] = si;
          col[ivc - 1] = fma(ci, a0, si * a1);
          col[ivc] = 0.0;
          const double gp = g[ivc - 1], gq = g[ivc];
          g[ivc - 1] = fma(ci, gp, si * gq);
          g[ivc] = fma(-si, gp, ci * gq);
          if (fabs(g[ivc]) <= S->r_tol * S->gbeta0 || ivc == K) {
            S->m = ivc;
            S->askip = 1;
          }
        }
      };
      if (lazy) {
        VecPtrs vpi{};
        for (int k = 0; k < iv; ++k) vpi.p[k] = V[k];
        float* out = (float*)(iv < K ? V[iv] : w);
        q = cgs_step_lazy(ctx, n, iv, vpi, (float*)w, out, col, &nh[(K + 1) * (iv - 1)], sig,
                          fin_norm, askip);
        if (q) return q;
      } else if (s->inner_mode && K <= kMaxCgs) {
        // inner solve: classical Gram-Schmidt, two passes per step
        VecPtrs vpi{};
        for (int k = 0; k < iv; ++k) vpi.p[k] = V[k];
        q = cgs_step<T>(ctx, n, iv, vpi, w, col, &nh[(K + 1) * (iv - 1)], fin_norm, askip);
        if (q) return q;
      } else {
      // modified Gram-Schmidt (the reference's): h(j,iv) = <v_j, w> ; w -= h(j,iv) v_j
      {
        const T* vj = V[0];
        double* hj = &h[0 + (K + 1) * (iv - 1)];
        double* nhj = &nh[0 + (K + 1) * (iv - 1)];
        q = launch_chunks<1>(
            ctx, n, [=] __device__(int64_t i) { return V2<T>{vj[i], w[i]}; },
            [=] __device__(int64_t, const V2<T>& v, double* a) {
              a[0] = fma((double)v.a, (double)v.b, a[0]);
            },
            [=] __device__(const double* t) {
              *hj = t[0];
              *nhj = -t[0];
            },
            askip);
        if (q) return q;
      }
      for (int j = 2; j <= iv; ++j) {
        const T* vprev = V[j - 2];
        const T* vj = V[j - 1];
        const double* nhp = &nh[(j - 2) + (K + 1) * (iv - 1)];
        double* hj = &h[(j - 1) + (K + 1) * (iv - 1)];
        double* nhj = &nh[(j - 1) + (K + 1) * (iv - 1)];
        q = launch_chunks<1>(
            ctx, n, [=] __device__(int64_t i) { return V3<T>{vprev[i], w[i], vj[i]}; },
            [=] __device__(int64_t i, const V3<T>& v, double* a) {
              const T wi = fmaT((T)*nhp, v.a, v.b);
              w[i] = wi;
              a[0] = fma((double)v.c, (double)wi, a[0]);
            },
            [=] __device__(const double* t) {
              *hj = t[0];
              *nhj = -t[0];
            },
            askip);
        if (q) return q;
      }
      {
        const T* vl = V[iv - 1];
        const double* nhp = &nh[(iv - 1) + (K + 1) * (iv - 1)];
        q = launch_chunks<1>(
            ctx, n, [=] __device__(int64_t i) { return V2<T>{vl[i], w[i]}; },
            [=] __device__(int64_t i, const V2<T>& v, double* a) {
              const T wi = fmaT((T)*nhp, v.a, v.b);
              w[i] = wi;
              a[0] = fma((double)wi, (double)wi, a[0]);
            },
            fin_norm, askip);
        if (q) return q;
      }
      }
      if (iv < K && !lazy) {
        T* vn = V[iv];
        q = launch_chunks<0>(
            ctx, n, [=] __device__(int64_t i) { return V1<T>{w[i]}; },
            [=] __device__(int64_t i, const V1<T>& v, double*) { vn[i] = (T)S->inv_hn * v.a; },
            NoFin{}, askip);
        if (q) return q;
      }
    }
    gmres_finish_cycle<<<1, 1, 0, ctx->stream>>>(S, h, K, lazy ? sig : nullptr, one_cycle);
    ctx->launches++;
    LFX_CK(ctx, cudaGetLastError());
    // x += sum_iv u(iv) v_iv over the m vectors of the cycle, one pass, the
    // reference's order per element
    bool al = ((uintptr_t)x & 15) == 0;
    for (int k = 0; k < K; ++k) al = al && ((uintptr_t)V[k] & 15) == 0;
    if (al) {
      const int grid = (int)std::max<int64_t>(
          1, std::min<int64_t>((n + 256 * 4 - 1) / (256 * 4), (int64_t)ctx->num_sms * 8));
      gmres_xupdate<T><<<grid, 256, 0, ctx->stream>>>(n, vp, u, &S->m, x, done);
      ctx->launches++;
      LFX_CK(ctx, cudaGetLastError());
    } else {
    q = launch_chunks<0>(
        ctx, n, [=] __device__(int64_t i) { return V1<T>{x[i]}; },
        [=] __device__(int64_t i, const V1<T>& v, double*) {
          T xi = v.a;
          const int m = S->m;
          for (int k = 0; k < m; ++k) xi = fmaT((T)u[k], ((const T*)vp.p[k])[i], xi);
          x[i] = xi;
        },
        NoFin{}, done);
    if (q) return q;
    }
    // a single queued cycle is followed at once by the caller's own (FP64)
    // residual, the only one it reads: this cycle's residual is not formed
    if (one_cycle) return LFX_OK;
    if ((q = op_apply_impl(s->op, x, res, b, done))) return q;  // res = b - A x
    q = launch_chunks<1>(
        ctx, n, [=] __device__(int64_t i) { return V1<T>{res[i]}; },
        [=] __device__(int64_t, const V1<T>& v, double* a) { a[0] = fma((double)v.a, (double)v.a, a[0]); },
        [=] __device__(const double* t) {
          S->applies += 1;
          S->iter += 1;
          S->res_norm = sqrt(t[0]);
          S->r_nrm = S->res_norm;
          S->err = S->res_norm / S->sc_err;
          if (S->monitor) {
            if (S->err < S->r_tol) {  // :970
              S->done = 1;
              S->converged = 1;
            } else if (isnan(S->err)) {
              S->done = 1;
              S->status = LFX_NAN_DETECTED;
            }
          }
          if (S->iter >= S->max_iter) S->done = 1;
          S->askip = S->done;
        },
        done);
    return q;
  };
  if (one_cycle) return run_graph(s, x, b, cycle, false, 1);
  // no host round trip before the first graph: its kernels idle if the
  // initial residual already ended the solve (device flags)
  do {
    if ((rc = run_graph(s, x, b, cycle))) return rc;
  } while (!s->h_state->done);
  return LFX_OK;
}

void fill_info(lfx_solver* s, lfx_solve_info* info) {
  const DevState& h = *s->h_state;
  info->iterations = h.iter;
  info->converged = h.converged;
  info->initial_norm = h.r_nrm_0;
  info->final_norm = h.r_nrm;
  info->final_rel = s->kind == LFX_SOLVER_CG ? (h.r_nrm_0 > 0 ? h.r_nrm / h.r_nrm_0 : 0.0) : h.err;
  if (h.converged && h.iter == 0) info->final_rel = 0.0;
  info->applies = h.applies;
  info->status = h.status;
}

int free_solver(lfx_solver* s) {
  if (!s) return LFX_OK;
  lfx_ctx* ctx = s->ctx;
  free_graphs(s);
  for (void* p : s->work) dfree(ctx, p, s->n * esz(s->precision));
  dfree(ctx, s->d_state, sizeof(DevState));
  if (s->h_state) cudaFreeHost(s->h_state);
  if (s->d_gm) dfree(ctx, s->d_gm, sizeof(double) * gm_doubles(s->cfg.gcrk));
  if (s->r32) lfx_vec_destroy(s->r32);
  if (s->d32) lfx_vec_destroy(s->d32);
  if (s->d_r64) dfree(ctx, s->d_r64, s->n * 8);
  for (lfx_vec* v : s->hv) lfx_vec_destroy(v);
  delete s;
  return LFX_OK;
}

// a solver whose scalar recurrences run on the host over the vector C ABI
// (lfx_solver_flex.cu), with nvec work vectors
int create_host_solver(lfx_ctx* ctx, int kind, lfx_op* op, lfx_prec* prec,
                       const lfx_solver_cfg& cfg, int nvec, lfx_solver** out) {
  if (op->lay->undf_to != op->lay->undf_from)
    return fail(ctx, LFX_INVALID_ARGUMENT, "Krylov solve needs a square operator");
  if (prec->kind != PREC_NULL && prec->precision != op->precision)
    return fail(ctx, LFX_TYPE_MISMATCH, "operator and preconditioner precision differ");
  lfx_solver* s = new lfx_solver();
  s->ctx = ctx;
  s->kind = kind;
  s->op = op;
  s->prec = prec;
  s->cfg = cfg;
  s->precision = op->precision;
  s->n = op->lay->undf_to;
  int64_t n = s->n;
  int rc = LFX_OK;
  for (int i = 0; i < nvec && !rc; ++i) {
    lfx_vec* v = nullptr;
    rc = lfx_vec_create(ctx, 1, &n, s->precision, &v);
    if (!rc) s->hv.push_back(v);
  }
  if (rc) {
    free_solver(s);
    return rc;
  }
  *out = s;
  return LFX_OK;
}

int alloc_common(lfx_solver* s, int nwork) {
  lfx_ctx* ctx = s->ctx;
  int rc = dmalloc(ctx, (void**)&s->d_state, sizeof(DevState));
  if (rc) return rc;
  rc = host_alloc_mapped(ctx, (void**)&s->h_state, (void**)&s->h_state_dev, sizeof(DevState));
  if (rc) return rc;
  for (int k = 0; k < nwork; ++k) {
    void* p = nullptr;
    rc = dmalloc(ctx, &p, s->n * esz(s->precision));
    if (rc) return rc;
    s->work.push_back(p);
  }
  // up to gcrk simultaneous sums (classical Gram-Schmidt of the inner solve)
  return ensure_partials(ctx, s->n, std::max(4, s->cfg.gcrk + 1));
}

// ------------------------------------------------------------------ refinement
int refined_run(lfx_solver* s, lfx_vec* xv, const lfx_vec* bv, lfx_solve_info* info) {
  lfx_ctx* ctx = s->ctx;
  const int64_t n = s->n;
  double* x = (double*)xv->data[0];
  const double* b = (const double*)bv->data[0];
  double* r = s->d_r64;
  float* r32 = (float*)s->r32->data[0];
  float* d32 = (float*)s->d32->data[0];
  double* sc = ctx->d_scalars;
  int rc;
  auto resid_norm = [&](double* out) -> int {
    int q = op_apply_impl(s->op, x, r, b, nullptr);
    if (q) return q;
    q = norm_kernel(ctx, n, (const double*)r, sc, nullptr);
    if (!q) q = to_host_small(ctx, ctx->h_scalars_dev, sc, 8);
    if (q) return q;
    LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
    *out = ctx->h_scalars[0];
    return LFX_OK;
  };
  // an FP32 GMRES inner solve runs one restart cycle per refinement step,
  // queued with the step's FP64 residual (one host round trip per step)
  const bool fast = s->inner->kind == LFX_SOLVER_GMRES && s->inner->inner_mode &&
                    s->inner->precision == LFX_R32;
  double r0 = 0.0, rn = 0.0;
  {
    // the first residual skips its apply when x starts at zero
    int q = residual_from<double>(s, s->op, x, r, b, &s->d_state->x_zero);
    if (!q) q = norm_kernel(ctx, n, (const double*)r, sc, nullptr);
    if (!q) q = to_host_small(ctx, ctx->h_scalars_dev, sc, 8);
    if (q) return q;
    LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
    r0 = ctx->h_scalars[0];
  }
  memset(info, 0, sizeof *info);
  info->initial_norm = r0;
  info->applies = 1;
  rn = r0;
  if (r0 < EPS_RDEF) {
    info->converged = 1;
    info->final_norm = r0;
    return LFX_OK;
  }
  for (int k = 1; k <= s->cfg.max_iter; ++k) {
    // r32 = r / ||r|| ; d32 = 0
    const double inv = 1.0 / rn;
    rc = launch_chunks<0>(
        ctx, n, [=] __device__(int64_t i) { return V1<double>{r[i]}; },
        [=] __device__(int64_t i, const V1<double>& v, double*) {
          r32[i] = (float)(v.a * inv);
          d32[i] = 0.0f;
        },
        NoFin{});
    if (rc) return rc;
    lfx_solve_info ii{};
    lfx_solver* in = s->inner;
    if (fast) {
      // one inner GMRES cycle, queued; its state comes back with the
      // residual norm below, in one synchronisation
      if ((rc = init_state(in))) return rc;
      in->zero_x0 = true;  // d32 was just zeroed
      if ((rc = gmres_run<float>(in, d32, r32, true))) return rc;
      if ((rc = to_host_small(ctx, in->h_state_dev, in->d_state, sizeof(DevState)))) return rc;
    } else {
      in->zero_x0 = in->kind == LFX_SOLVER_GMRES;  // d32 was just zeroed
      rc = lfx_solver_apply(in, s->d32, s->r32, &ii);
      if (rc && rc != LFX_NOT_CONVERGED) return rc;
      info->inner_iterations += ii.iterations;
      info->applies += ii.applies;
    }
    // x += ||r|| d
    const double scale = rn;
    rc = launch_chunks<0>(
        ctx, n, [=] __device__(int64_t i) { return V2<double>{x[i], (double)d32[i]}; },
        [=] __device__(int64_t i, const V2<double>& v, double*) { x[i] = fma(scale, v.b, v.a); },
        NoFin{});
    if (rc) return rc;
    if ((rc = resid_norm(&rn))) return rc;
    if (fast) {
      collect_timing(in);
      fill_info(in, &ii);
      if (ii.status == LFX_NAN_DETECTED) {
        info->status = LFX_NAN_DETECTED;
        return fail(ctx, LFX_NAN_DETECTED, "NaN in the inner solve");
      }
      info->inner_iterations += ii.iterations;
      info->applies += ii.applies;
    }
    info->applies += 1;
    info->outer_iterations = k;
    info->iterations = k;
    info->final_norm = rn;
    info->final_rel = rn / r0;
    if (std::isnan(rn)) {
      info->status = LFX_NAN_DETECTED;
      return fail(ctx, LFX_NAN_DETECTED, "NaN in refined residual");
    }
    if (rn / r0 <= s->cfg.r_tol || rn <= s->cfg.a_tol) {
      info->converged = 1;
      break;
    }
  }
  return LFX_OK;
}

}  // namespace

extern "C" {

int lfx_solver_create(lfx_ctx* ctx, int32_t kind, lfx_op* op, lfx_prec* prec,
                      const lfx_solver_cfg* cfg, lfx_solver** out) {
  if (!ctx || !op || !prec || !cfg || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  if (kind < LFX_SOLVER_CG || kind > LFX_SOLVER_CHEBYSHEV)
    return fail(ctx, LFX_INVALID_ARGUMENT, "unknown solver kind");
  if (op->lay->undf_to != op->lay->undf_from)
    return fail(ctx, LFX_INVALID_ARGUMENT, "Krylov solve needs a square operator");
  if (prec->kind != PREC_NULL && prec->precision != op->precision)
    return fail(ctx, LFX_TYPE_MISMATCH, "operator and preconditioner precision differ");
  if ((prec->kind == PREC_DIAG || (prec->kind == PREC_CMA && prec->rdiag)) &&
      prec->rdiag_n != op->lay->undf_to)
    return fail(ctx, LFX_TYPE_MISMATCH, "preconditioner diagonal does not match the operator");
  if (prec->kind == PREC_CMA && prec->max_row >= op->lay->undf_to)
    return fail(ctx, LFX_TYPE_MISMATCH, "CMA rows fall outside the operator's space");
  if (cfg->max_iter < 1) return fail(ctx, LFX_INVALID_ARGUMENT, "max_iter must be positive");
  if (kind >= LFX_SOLVER_GMRES && (cfg->gcrk < 1 || cfg->gcrk > MAX_GCRK))
    return fail(ctx, LFX_INVALID_ARGUMENT, "gcrk must be in 1..64");
  if (kind == LFX_SOLVER_FGMRES || kind == LFX_SOLVER_GCR)
    return create_host_solver(ctx, kind, op, prec, *cfg,
                              (kind == LFX_SOLVER_FGMRES ? 5 : 3) + 2 * cfg->gcrk, out);
  if (kind > LFX_SOLVER_GCR)
    return fail(ctx, LFX_INVALID_ARGUMENT,
                "precondition-only, Jacobi and Chebyshev solvers have their own constructors");
  lfx_solver* s = new lfx_solver();
  s->ctx = ctx;
  s->kind = kind;
  s->op = op;
  s->prec = prec;
  s->cfg = *cfg;
  s->precision = op->precision;
  s->n = op->lay->undf_to;
  int nwork = kind == LFX_SOLVER_CG ? 3 : kind == LFX_SOLVER_BICGSTAB ? 8 : 3 + cfg->gcrk;
  int rc = alloc_common(s, nwork);
  if (!rc && kind == LFX_SOLVER_GMRES)
    rc = dmalloc(ctx, (void**)&s->d_gm, sizeof(double) * gm_doubles(cfg->gcrk));
  if (rc) {
    free_solver(s);
    return rc;
  }
  *out = s;
  return LFX_OK;
}

int lfx_refined_solver_create(lfx_ctx* ctx, lfx_op* op64, lfx_solver* inner, double inner_rtol,
                              const lfx_solver_cfg* cfg, lfx_solver** out) {
  if (!ctx || !op64 || !inner || !cfg || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  if (op64->precision != LFX_R64) return fail(ctx, LFX_TYPE_MISMATCH, "outer operator must be FP64");
  if (inner->precision != LFX_R32 || inner->n != op64->lay->undf_to)
    return fail(ctx, LFX_TYPE_MISMATCH, "inner solver must be FP32 on the same space");
  lfx_solver* s = new lfx_solver();
  s->ctx = ctx;
  s->kind = 100;
  s->op = op64;
  s->cfg = *cfg;
  s->precision = LFX_R64;
  s->n = op64->lay->undf_to;
  s->inner = inner;
  s->inner_rtol = inner_rtol;
  int64_t n = s->n;
  int rc = dmalloc(ctx, (void**)&s->d_r64, n * 8);
  if (!rc) rc = lfx_vec_create(ctx, 1, &n, LFX_R32, &s->r32);
  if (!rc) rc = lfx_vec_create(ctx, 1, &n, LFX_R32, &s->d32);
  if (!rc) rc = dmalloc(ctx, (void**)&s->d_state, sizeof(DevState));
  if (!rc)
    rc = host_alloc_mapped(ctx, (void**)&s->h_state, (void**)&s->h_state_dev, sizeof(DevState));
  if (!rc) rc = ensure_partials(ctx, n, 4);
  if (rc) {
    free_solver(s);
    return rc;
  }
  // the inner GMRES runs in "inner mode": rotations applied as the Arnoldi
  // process goes, and the cycle ends as soon as the residual estimate meets
  // the inner tolerance (the outer FP64 residual decides convergence)
  inner->cfg.r_tol = inner_rtol;
  inner->inner_mode = inner->kind == LFX_SOLVER_GMRES;
  free_graphs(inner);
  *out = s;
  return LFX_OK;
}

int lfx_solver_apply(lfx_solver* s, lfx_vec* x, const lfx_vec* b, lfx_solve_info* info) {
  if (!s || !x || !b) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = s->ctx;
  lfx_solve_info local{};
  if (!info) info = &local;
  memset(info, 0, sizeof *info);
  if (x->precision != s->precision || b->precision != s->precision)
    return fail(ctx, LFX_TYPE_MISMATCH, "solver and vector precision differ");
  if (x->data.size() != 1 || b->data.size() != 1)
    return fail(ctx, LFX_NOT_SUPPORTED, "device solves take single-field vectors");
  if (x->undf[0] != s->n || b->undf[0] != s->n)
    return fail(ctx, LFX_TYPE_MISMATCH, "vector length does not match the operator");
  if (x->data[0] == b->data[0]) return fail(ctx, LFX_INVALID_ARGUMENT, "x and b must differ");
  int rc;
  if (s->kind >= LFX_SOLVER_FGMRES && s->kind <= LFX_SOLVER_CHEBYSHEV) {
    switch (s->kind) {
      case LFX_SOLVER_FGMRES: rc = fgmres_host(s->op, s->prec, s->cfg, s->hv, x, b, info); break;
      case LFX_SOLVER_GCR: rc = gcr_host(s->op, s->prec, s->cfg, s->hv, x, b, info); break;
      case LFX_SOLVER_PRECONDITION_ONLY:
        rc = precondition_only_host(s->op, s->prec, s->cfg, s->hv, x, b, info);
        break;
      case LFX_SOLVER_JACOBI:
        rc = jacobi_host(s->op, s->prec, s->cfg, s->rho_relax, s->hv, x, b, info);
        break;
      default:
        rc = chebyshev_host(s->op, s->prec, s->cfg, s->lmin, s->lmax, s->hv, x, b, info);
        break;
    }
    if (!rc) rc = lfx_ctx_check_device_error(ctx);
    if (rc) {
      info->status = rc;
      return rc;
    }
    if (info->status == LFX_NAN_DETECTED) return fail(ctx, LFX_NAN_DETECTED, "NaN in residual");
    // as the reference: GCR logs non-convergence as an error in both branches;
    // Chebyshev, which has no convergence test, logs its final residual as an
    // error whenever fail_on_non_converged is set
    if (s->kind == LFX_SOLVER_CHEBYSHEV && s->cfg.monitor_convergence &&
        s->cfg.fail_on_non_converged) {
      info->status = LFX_NOT_CONVERGED;
      return fail(ctx, LFX_NOT_CONVERGED, "chebyshev with fail_on_non_converged");
    }
    const bool must_fail = s->kind == LFX_SOLVER_GCR || s->cfg.fail_on_non_converged;
    if (!info->converged && s->cfg.monitor_convergence && must_fail) {
      info->status = LFX_NOT_CONVERGED;
      return fail(ctx, LFX_NOT_CONVERGED, "solver did not converge");
    }
    return LFX_OK;
  }
  if (s->kind == 100) {
    rc = refined_run(s, x, b, info);
  } else {
    if ((rc = init_state(s))) return rc;
    if (s->kind == LFX_SOLVER_CG)
      rc = s->precision == LFX_R64 ? cg_run<double>(s, (double*)x->data[0], (const double*)b->data[0])
                                   : cg_run<float>(s, (float*)x->data[0], (const float*)b->data[0]);
    else if (s->kind == LFX_SOLVER_BICGSTAB)
      rc = s->precision == LFX_R64
               ? bicgstab_run<double>(s, (double*)x->data[0], (const double*)b->data[0])
               : bicgstab_run<float>(s, (float*)x->data[0], (const float*)b->data[0]);
    else
      rc = s->precision == LFX_R64
               ? gmres_run<double>(s, (double*)x->data[0], (const double*)b->data[0])
               : gmres_run<float>(s, (float*)x->data[0], (const float*)b->data[0]);
    if (!rc) rc = read_state(s);
    if (!rc) fill_info(s, info);
  }
  if (ctx->time_applies) drain_timing(ctx);
  if (!rc) rc = lfx_ctx_check_device_error(ctx);
  if (rc) {
    info->status = rc;
    return rc;
  }
  if (info->status == LFX_NAN_DETECTED) return fail(ctx, LFX_NAN_DETECTED, "NaN in residual");
  if (!info->converged && s->cfg.monitor_convergence && s->cfg.fail_on_non_converged) {
    info->status = LFX_NOT_CONVERGED;
    return fail(ctx, LFX_NOT_CONVERGED, "solver did not converge");
  }
  return LFX_OK;
}

int lfx_solver_destroy(lfx_solver* s) { return free_solver(s); }

int lfx_precondition_only_solver_create(lfx_ctx* ctx, lfx_op* op, lfx_prec* prec,
                                        int32_t monitor_convergence, lfx_solver** out) {
  if (!ctx || !op || !prec || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  lfx_solver_cfg cfg{};
  cfg.max_iter = 1;
  cfg.monitor_convergence = monitor_convergence;
  return create_host_solver(ctx, LFX_SOLVER_PRECONDITION_ONLY, op, prec, cfg, 2, out);
}

int lfx_jacobi_solver_create(lfx_ctx* ctx, lfx_op* op, lfx_prec* prec, double r_tol, double a_tol,
                             int32_t max_iter, int32_t monitor_convergence,
                             int32_t fail_on_non_converged, double rho_relax, lfx_solver** out) {
  if (!ctx || !op || !prec || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  if (max_iter < 1) return fail(ctx, LFX_INVALID_ARGUMENT, "max_iter must be positive");
  lfx_solver_cfg cfg{r_tol, a_tol, max_iter, 1, monitor_convergence, fail_on_non_converged};
  int rc = create_host_solver(ctx, LFX_SOLVER_JACOBI, op, prec, cfg, 2, out);
  if (!rc) (*out)->rho_relax = rho_relax;
  return rc;
}

int lfx_chebyshev_solver_create(lfx_ctx* ctx, lfx_op* op, lfx_prec* prec, double r_tol,
                                double a_tol, int32_t max_iter, int32_t monitor_convergence,
                                int32_t fail_on_non_converged, double lmin, double lmax,
                                lfx_solver** out) {
  if (!ctx || !op || !prec || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  if (max_iter < 1) return fail(ctx, LFX_INVALID_ARGUMENT, "max_iter must be positive");
  if (!(lmax > lmin)) return fail(ctx, LFX_INVALID_ARGUMENT, "lmax must exceed lmin");
  lfx_solver_cfg cfg{r_tol, a_tol, max_iter, 1, monitor_convergence, fail_on_non_converged};
  int rc = create_host_solver(ctx, LFX_SOLVER_CHEBYSHEV, op, prec, cfg, 4, out);
  if (!rc) {
    (*out)->lmin = lmin;
    (*out)->lmax = lmax;
  }
  return rc;
}

// The tolerances are read from the solver's device state at every solve, so
// changing them keeps the captured graphs valid.
int lfx_solver_set_tolerance(lfx_solver* s, double r_tol, double a_tol) {
  if (!s || !(r_tol >= 0.0) || !(a_tol >= 0.0)) return LFX_INVALID_ARGUMENT;
  s->cfg.r_tol = r_tol;
  s->cfg.a_tol = a_tol;
  return LFX_OK;
}

}  // extern "C"
