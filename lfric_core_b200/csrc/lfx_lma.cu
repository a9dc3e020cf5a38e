// LMA operator apply: the reference's matrix_vector_kernel over a cell
// colouring (sci_mass_matrix_operator_alg_mod.x90:98,
// matrix_vector_kernel_mod.F90:107-140), recast as a race-free gather.
//
// The reference visits colours in turn and, per cell column, adds
// M(ik+k, df, df2) * x(map2(df2)+k) into lhs(map1(df)+k) for df2 (outer) and
// df (inner). Cells of one colour share no dof, so every output dof receives
// its contributions in the order (colour of the cell, df2, df). The device
// computes each output dof in one lane, walking its contributing cells in
// that same order, so the FP64 result equals the coloured scatter bit for
// bit, with one launch and no atomics.
//
// Device layout of the local matrices: [cell][df][df2][k] (k fastest), each
// (cell, df) block padded to a multiple of 16 bytes. A warp owns one dof
// column ("entity") at a time; the (cell, df) blocks it needs are each read
// exactly once. The main kernel (lma_tma) streams those blocks into shared
// memory with bulk asynchronous copies (cp.async.bulk, completion on an
// mbarrier) several entities ahead of the computation, so HBM reads are
// large, aligned and always in flight; the lanes then combine them with x
// gathered from L2.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "lfx_internal.cuh"

using namespace lfx;

namespace {

struct LayoutArgs {
  int32_t nent, nlayers, ndf1, ndf2, blk;
  const int32_t* ent_base;
  const int32_t* ent_h;
  const int32_t* ent_grp;
  const int32_t* grp_cell;
  const uint32_t* grp_rec;
  const int32_t* map_from;
  const int4* ent_pack;
  const int32_t* grp_pack;
  int32_t gp_stride;
  const int32_t* desc;
  const int32_t* fdesc;
};

LayoutArgs args_of(const lfx_lma_layout* L, int blk) {
  return LayoutArgs{L->nent,     L->nlayers,  L->ndf_to,   L->ndf_from, blk,
                    L->ent_base, L->ent_h,    L->ent_grp,  L->grp_cell, L->grp_rec,
                    L->map_from, L->ent_pack, L->grp_pack, L->gp_stride, L->desc,
                    L->fdesc};
}

// packed group record: bits 0-1 nrec (1..3); record r at bit 2+9r: df (6 bits), off (3 bits)
__host__ __device__ inline int rec_n(uint32_t p) { return p & 3u; }
__host__ __device__ inline int rec_df(uint32_t p, int r) { return (p >> (2 + 9 * r)) & 63u; }
__host__ __device__ inline int rec_off(uint32_t p, int r) { return (p >> (8 + 9 * r)) & 7u; }

// elements per (cell, df) block: ndf2*nl rounded up to 16 bytes
int block_elems(int ndf2, int nl, size_t esz) {
  const size_t b = (size_t)ndf2 * nl * esz;
  return (int)(((b + 15) / 16 * 16) / esz);
}

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// 4- or 8-byte asynchronous copy global -> shared, and an mbarrier arrival
// that fires once all of this thread's earlier copies have landed (the
// pending count is raised first, so the phase waits for them)
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src),
               "n"(BYTES)
               : "memory");
}
__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.shared.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// ---------------------------------------------------------------- kernels

// Generic gather (any ndf, up to three records per group).
template <class T>
__global__ void __launch_bounds__(256) lma_gather(LayoutArgs A, const T* __restrict__ M,
                                                  const T* __restrict__ x, T* __restrict__ y,
                                                  const T* __restrict__ b, const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  const int ndf2 = A.ndf2;
  const int nl = A.nlayers;
  const int lane = threadIdx.x & 31;
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const size_t cell_stride = (size_t)A.ndf1 * A.blk;
  for (int64_t e = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < A.nent; e += nwarp) {
    const int base = A.ent_base[e], h = A.ent_h[e];
    const int g0 = A.ent_grp[e], g1 = A.ent_grp[e + 1];
    for (int l = lane; l < h; l += 32) {
      T acc = T(0);
      for (int g = g0; g < g1; ++g) {
        const int c = A.grp_cell[g];
        const uint32_t pk = A.grp_rec[g];
        const int nrec = rec_n(pk);
        const T* Mc = M + (size_t)c * cell_stride;
        const int* mf = A.map_from + (size_t)c * ndf2;
        for (int j = 0; j < ndf2; ++j) {
          const int xb = mf[j];
          for (int r = 0; r < nrec; ++r) {
            const int k = l - rec_off(pk, r);
            if (k >= 0 && k < nl)
              acc = fmaT(Mc[(size_t)rec_df(pk, r) * A.blk + j * nl + k], x[xb + k], acc);
          }
        }
      }
      if (b)
        y[base + l] = b[base + l] - acc;
      else
        y[base + l] = acc;
    }
  }
}

// One group record {cell, records, map_from row} read as 16-byte vectors
// (gp_stride is a multiple of 4 ints).
template <int NDF2>
__device__ __forceinline__ void gather_record(const LayoutArgs& A, int g, int& c, uint32_t& pk,
                                              int* mf) {
  const int4* gp4 = reinterpret_cast<const int4*>(A.grp_pack + (size_t)g * A.gp_stride);
  const int4 h0 = __ldg(gp4);
  c = h0.x;
  pk = (uint32_t)h0.y;
  int tmp[12];
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
#pragma unroll
  for (int j = 0; j < NDF2; ++j) mf[j] = tmp[j];
}

// One cell group's contribution to output row l of an entity column (groups of
// at most two records): all loads of the group are issued before the FMA
// chain that consumes them; matrix rows, read once per apply, with streaming
// (evict-first) loads so that x stays in L2. The warp must be converged (pair
// shuffles).
template <class T, int NDF2>
__device__ __forceinline__ T group_acc(const LayoutArgs& A, const T* __restrict__ M,
                                       const T* __restrict__ x, size_t cell_stride, int l,
                                       int lane, int c, uint32_t pk, const int* mf, T acc) {
  const int nl = A.nlayers;
  const int k0 = l - rec_off(pk, 0), k1 = l - rec_off(pk, 1);
  const bool v0 = (unsigned)k0 < (unsigned)nl;
  if (rec_n(pk) == 1) {
    // one record (warp-uniform branch): no second-record instructions
    const T* M0 = M + (size_t)c * cell_stride + (size_t)rec_df(pk, 0) * A.blk + (v0 ? k0 : 0);
    T a0[NDF2], b0[NDF2];
#pragma unroll
    for (int j = 0; j < NDF2; ++j) {
      a0[j] = v0 ? __ldcs(M0 + j * nl) : T(0);
      b0[j] = v0 ? __ldg(x + mf[j] + k0) : T(0);
    }
#pragma unroll
    for (int j = 0; j < NDF2; ++j)
      if (v0) acc = fmaT(a0[j], b0[j], acc);
    return acc;
  }
  const bool v1 = rec_n(pk) > 1 && (unsigned)k1 < (unsigned)nl;
  // second record one level above the first (bottom/top vertex or face): its
  // x values are the neighbouring lane's first-record values
  const bool pair = rec_n(pk) == 2 && rec_off(pk, 1) == rec_off(pk, 0) + 1;
  const T* Mc = M + (size_t)c * cell_stride;
  const T* M0 = Mc + (size_t)rec_df(pk, 0) * A.blk + (v0 ? k0 : 0);
  const T* M1 = Mc + (size_t)rec_df(pk, 1) * A.blk + (v1 ? k1 : 0);
  T a0[NDF2], b0[NDF2], a1[NDF2], b1[NDF2];
#pragma unroll
  for (int j = 0; j < NDF2; ++j) {
    a0[j] = v0 ? __ldcs(M0 + j * nl) : T(0);
    b0[j] = v0 ? __ldg(x + mf[j] + k0) : T(0);
    a1[j] = v1 ? __ldcs(M1 + j * nl) : T(0);
  }
  if (pair) {
#pragma unroll
    for (int j = 0; j < NDF2; ++j) {
      const T up = __shfl_up_sync(0xffffffffu, b0[j], 1);
      b1[j] = (lane == 0) ? (v1 ? __ldg(x + mf[j] + k1) : T(0)) : up;
    }
  } else {
#pragma unroll
    for (int j = 0; j < NDF2; ++j) b1[j] = v1 ? __ldg(x + mf[j] + k1) : T(0);
  }
#pragma unroll
  for (int j = 0; j < NDF2; ++j) {
    if (v0) acc = fmaT(a0[j], b0[j], acc);
    if (v1) acc = fmaT(a1[j], b1[j], acc);
  }
  return acc;
}

// Register path (no shared memory) for groups of at most two records.
template <class T, int NDF2>
__global__ void __launch_bounds__(256) lma_gather2(LayoutArgs A, const T* __restrict__ M,
                                                   const T* __restrict__ x, T* __restrict__ y,
                                                   const T* __restrict__ b, const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  const int lane = threadIdx.x & 31;
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const size_t cell_stride = (size_t)A.ndf1 * A.blk;
  for (int64_t e = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < A.nent; e += nwarp) {
    const int4 ep = __ldg(A.ent_pack + e);
    const int base = ep.x, h = ep.y, g0 = ep.z, g1 = ep.w;
    // all 32 lanes run every pass (lanes past the column's top just carry no
    // valid record) so that the shuffles see a converged warp
    for (int l0 = 0; l0 < h; l0 += 32) {
      const int l = l0 + lane;
      T acc = T(0);
      for (int g = g0; g < g1; ++g) {
        int c;
        uint32_t pk;
        int mf[NDF2];
        gather_record<NDF2>(A, g, c, pk, mf);
        acc = group_acc<T, NDF2>(A, M, x, cell_stride, l, lane, c, pk, mf, acc);
      }
      if (l < h) {
        if (b)
          y[base + l] = b[base + l] - acc;
        else
          y[base + l] = acc;
      }
    }
  }
}

// Per-column descriptor of lma_fetch (columns reading at most two (cell, df)
// blocks from at most two cells): ints {base, h, groups, 0}, then per group
// {cell, record, map_from row} padded to a multiple of 4 ints.

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The register gather with its column descriptors prefetched: each warp keeps
// the descriptors of its next kFetchDepth columns in flight (16-byte cp.async
// into a per-warp ring in shared memory), so a column waits on memory once,
// for its matrix rows and x values, which all lanes issue before the first
// FMA. Columns of two one-record groups (horizontal W2 faces) load both
// groups at once; a column of one group goes through group_acc. Same sums in
// the same order (and bits) as lma_gather2.
constexpr int kFetchDepth = 4;

template <class T, int NDF2, int MINB>
__global__ void __launch_bounds__(256, MINB) lma_fetch(LayoutArgs A, const T* __restrict__ M,
                                                 const T* __restrict__ x, T* __restrict__ y,
                                                 const T* __restrict__ b, const int* skip) {
  constexpr int GS = fd_group_ints(NDF2), FS = fd_ints(NDF2), NV = FS / 4;
  __shared__ __align__(16) int ring[8][kFetchDepth][FS];
  if (skip && *((volatile const int*)skip)) return;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nl = A.nlayers;
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t e0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const size_t cell_stride = (size_t)A.ndf1 * A.blk;
  const int4* fd = reinterpret_cast<const int4*>(A.fdesc);
#pragma unroll
  for (int s = 0; s < kFetchDepth; ++s) {
    const int64_t e = e0 + s * nwarp;
    if (lane < NV && e < A.nent) cp_async16(&ring[wib][s][4 * lane], fd + e * NV + lane);
    cp_async_commit();
  }
  int s = 0;
  for (int64_t e = e0; e < A.nent; e += nwarp) {
    cp_async_wait<kFetchDepth - 1>();
    __syncwarp();
    // fields are read from the ring where they are used (fewer live registers)
    const int* d = ring[wib][s];
    const int4 hd = *reinterpret_cast<const int4*>(d);
    const int base = hd.x, h = hd.y, ng = hd.z;
    for (int l0 = 0; l0 < h; l0 += 32) {
      const int l = l0 + lane;
      T acc = T(0);
      if (ng == 2) {
        // two cells, one record each: every load of both before the FMAs
        const uint32_t pk0 = (uint32_t)d[5], pk1 = (uint32_t)d[5 + GS];
        const int k0 = l - rec_off(pk0, 0), k1 = l - rec_off(pk1, 0);
        const bool v0 = (unsigned)k0 < (unsigned)nl, v1 = (unsigned)k1 < (unsigned)nl;
        const T* M0 = M + (size_t)d[4] * cell_stride + (size_t)rec_df(pk0, 0) * A.blk + (v0 ? k0 : 0);
        const T* M1 = M + (size_t)d[4 + GS] * cell_stride + (size_t)rec_df(pk1, 0) * A.blk + (v1 ? k1 : 0);
        T a0[NDF2], b0[NDF2], a1[NDF2], b1[NDF2];
#pragma unroll
        for (int j = 0; j < NDF2; ++j) {
          a0[j] = v0 ? __ldcs(M0 + j * nl) : T(0);
          a1[j] = v1 ? __ldcs(M1 + j * nl) : T(0);
        }
#pragma unroll
        for (int j = 0; j < NDF2; ++j) {
          b0[j] = v0 ? __ldg(x + (d[6 + j] + k0)) : T(0);
          b1[j] = v1 ? __ldg(x + (d[6 + GS + j] + k1)) : T(0);
        }
#pragma unroll
        for (int j = 0; j < NDF2; ++j)
          if (v0) acc = fmaT(a0[j], b0[j], acc);
#pragma unroll
        for (int j = 0; j < NDF2; ++j)
          if (v1) acc = fmaT(a1[j], b1[j], acc);
      } else if (ng == 1) {
        int mf[NDF2];
#pragma unroll
        for (int j = 0; j < NDF2; ++j) mf[j] = d[6 + j];
        acc = group_acc<T, NDF2>(A, M, x, cell_stride, l, lane, d[4], (uint32_t)d[5], mf, acc);
      }
      if (l < h) {
        if (b)
          y[base + l] = b[base + l] - acc;
        else
          y[base + l] = acc;
      }
    }
    __syncwarp();
    // the slot is free again: fetch the descriptor kFetchDepth columns ahead
    const int64_t en = e + kFetchDepth * nwarp;
    if (lane < NV && en < A.nent) cp_async16(&ring[wib][s][4 * lane], fd + en * NV + lane);
    cp_async_commit();
    s = s + 1 == kFetchDepth ? 0 : s + 1;
  }
  cp_async_wait<0>();
}

// Shared-memory layout of one warp in lma_tma: S stages, each holding up to
// MAXB (cell, df) blocks, the stage's mbarrier and the entity's metadata.
struct TmaMeta {
  int base, h, ng, nblk;
  int grp[8 * 10];  // per group: pk, mf[ndf2] (at most 8 groups, ndf2 <= 8)
};

constexpr unsigned kWaitLimit = 1u << 26;  // bounded mbarrier spin (~seconds)

// Bulk-copy pipelined gather for groups of at most two records, at most
// MAXG groups per entity and NDF2 <= 8. err receives 1 if a stage wait ran
// out (then the kernel stops issuing, drains what it issued and returns).
template <class T, int NDF2>
__global__ void __launch_bounds__(256) lma_tma(LayoutArgs A, const T* __restrict__ M,
                                               const T* __restrict__ x, T* __restrict__ y,
                                               const T* __restrict__ b, const int* skip,
                                               int stages, int maxb, int* err) {
  if (skip && *((volatile const int*)skip)) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int nl = A.nlayers;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const size_t stage_bytes = (size_t)maxb * A.blk * sizeof(T);
  const size_t warp_bytes = stages * (stage_bytes + sizeof(TmaMeta) + 16);
  unsigned char* wsm = smem_raw + wib * warp_bytes;
  T* buf = (T*)wsm;                                              // [stages][maxb*blk]
  TmaMeta* meta = (TmaMeta*)(wsm + stages * stage_bytes);        // [stages]
  uint64_t* bar = (uint64_t*)(wsm + stages * (stage_bytes + sizeof(TmaMeta)));  // [stages]
  const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const size_t cell_stride = (size_t)A.ndf1 * A.blk;
  const unsigned blk_bytes = (unsigned)(A.blk * sizeof(T));

  // lane 0: read entity i's metadata into stage s and start its block copies
  auto issue = [&](int64_t e, int s) {
    const int4 ep = __ldg(A.ent_pack + e);
    TmaMeta& mt = meta[s];
    mt.base = ep.x;
    mt.h = ep.y;
    mt.ng = ep.w - ep.z;
    int nb = 0;
    for (int g = 0; g < mt.ng; ++g) {
      const int32_t* gp = A.grp_pack + (size_t)(ep.z + g) * A.gp_stride;
      const int c = __ldg(gp);
      const int pk = __ldg(gp + 1);
      mt.grp[g * 10] = pk;
#pragma unroll
      for (int j = 0; j < NDF2; ++j) mt.grp[g * 10 + 1 + j] = __ldg(gp + 2 + j);
      nb += rec_n((uint32_t)pk);
    }
    mt.nblk = nb;
    fence_proxy_async();
    mbar_expect_tx(&bar[s], (unsigned)nb * blk_bytes);
    int q = 0;
    for (int g = 0; g < mt.ng; ++g) {
      const uint32_t pk = (uint32_t)mt.grp[g * 10];
      const int c = __ldg(A.grp_pack + (size_t)(ep.z + g) * A.gp_stride);
      for (int r = 0; r < rec_n(pk); ++r, ++q)
        bulk_load(buf + (size_t)s * maxb * A.blk + (size_t)q * A.blk,
                  M + (size_t)c * cell_stride + (size_t)rec_df(pk, r) * A.blk, blk_bytes, &bar[s]);
    }
  };

  if (lane == 0) {
    for (int s = 0; s < stages; ++s) mbar_init(&bar[s], 1);
    fence_proxy_async();
  }
  __syncwarp();
  // prologue: fill the pipeline
  if (lane == 0)
    for (int s = 0; s < stages; ++s) {
      const int64_t e = warp0 + (int64_t)s * nwarp;
      if (e < A.nent) issue(e, s);
    }
  __syncwarp();
  int64_t it = 0;
  bool failed = false;
  int64_t e = warp0;
  for (; e < A.nent; e += nwarp, ++it) {
    const int s = (int)(it % stages);
    const unsigned parity = (unsigned)((it / stages) & 1);
    unsigned spins = 0;
    while (!mbar_try_wait(&bar[s], parity)) {
      if (++spins > kWaitLimit) {
        failed = true;
        break;
      }
    }
    if (__any_sync(0xffffffffu, failed)) {
      if (lane == 0) atomicExch(err, 1);
      break;
    }
    const TmaMeta& mt = meta[s];
    const T* sb = buf + (size_t)s * maxb * A.blk;
    for (int l = lane; l < mt.h; l += 32) {
      T acc = T(0);
      int q = 0;
      for (int g = 0; g < mt.ng; ++g) {
        const uint32_t pk = (uint32_t)mt.grp[g * 10];
        const int* mf = &mt.grp[g * 10 + 1];
        const int k0 = l - rec_off(pk, 0), k1 = l - rec_off(pk, 1);
        const bool v0 = (unsigned)k0 < (unsigned)nl;
        const bool v1 = rec_n(pk) > 1 && (unsigned)k1 < (unsigned)nl;
        const T* s0 = sb + (size_t)q * A.blk + (v0 ? k0 : 0);
        const T* s1 = v1 ? sb + (size_t)(q + 1) * A.blk + k1 : sb;
        T b0[NDF2], b1[NDF2];
#pragma unroll
        for (int j = 0; j < NDF2; ++j) {
          b0[j] = v0 ? __ldg(x + mf[j] + k0) : T(0);
          b1[j] = v1 ? __ldg(x + mf[j] + k1) : T(0);
        }
#pragma unroll
        for (int j = 0; j < NDF2; ++j) {
          if (v0) acc = fmaT(s0[j * nl], b0[j], acc);
          if (v1) acc = fmaT(s1[j * nl], b1[j], acc);
        }
        q += rec_n(pk);
      }
      if (b)
        y[mt.base + l] = b[mt.base + l] - acc;
      else
        y[mt.base + l] = acc;
    }
    __syncwarp();
    if (lane == 0) {
      const int64_t en = e + (int64_t)stages * nwarp;
      if (en < A.nent) issue(en, s);
    }
    __syncwarp();
  }
  if (failed && lane == 0) {
    // drain: the stages of iterations it .. it+stages-1 may still have copies
    // in flight; wait (bounded) for each before the shared memory is released
    for (int k = 0; k < stages; ++k) {
      const int64_t ik = it + k;
      if (warp0 + ik * nwarp >= A.nent) break;
      const int s = (int)(ik % stages);
      const unsigned parity = (unsigned)((ik / stages) & 1);
      unsigned spins = 0;
      while (!mbar_try_wait(&bar[s], parity) && ++spins < kWaitLimit) {
      }
    }
  }
}

// Pipelined gather for columns of at most 32 NP dofs, groups of at most two
// records. Each warp walks its entity columns with `stages` in flight; a
// stage holds the column's descriptor, its (cell, df) matrix blocks (bulk
// copies) and, per record, lane and level, the x values the FMAs need
// (4/8-byte cp.async), all tracked by the stage's mbarrier. Descriptors are
// loaded one coalesced request per column, two columns ahead. The compute
// reads shared memory only, in lma_gather2's order (same bits). err receives
// 1 if a stage wait ran out (the kernel then drains and returns).
template <class T, int NDF2, int IPL, int NP>
__global__ void __launch_bounds__(256) lma_pipe(LayoutArgs A, const T* __restrict__ M,
                                                const T* __restrict__ x, T* __restrict__ y,
                                                const T* __restrict__ b, const int* skip,
                                                int stages, int maxb, int* err) {
  if (skip && *((volatile const int*)skip)) return;
  constexpr int GS = 2 + NDF2;
  constexpr int DS = 32 * IPL;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int nl = A.nlayers;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const size_t mat_b = (size_t)maxb * A.blk * sizeof(T);
  const size_t xs_b = (size_t)maxb * NDF2 * 32 * NP * sizeof(T);
  const size_t stage_b = mat_b + xs_b + DS * 4 + 16;
  unsigned char* wsm = smem_raw + (size_t)wib * stages * stage_b;
  auto mat_of = [&](int s) { return (T*)(wsm + s * stage_b); };
  auto xs_of = [&](int s) { return (T*)(wsm + s * stage_b + mat_b); };
  auto meta_of = [&](int s) { return (int*)(wsm + s * stage_b + mat_b + xs_b); };
  auto bar_of = [&](int s) { return (uint64_t*)(wsm + s * stage_b + mat_b + xs_b + DS * 4); };
  const int64_t warp0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  if (warp0 >= A.nent) return;  // whole warp: no barrier of this warp is used
  const size_t cell_stride = (size_t)A.ndf1 * A.blk;
  const unsigned blk_bytes = (unsigned)(A.blk * sizeof(T));

  // descriptor of column e, lane i holding ints IPL i .. IPL i + IPL - 1
  auto load_desc = [&](int64_t e, int (&d)[IPL]) {
    if (e < A.nent) {
      const int* src = A.desc + (size_t)e * DS + lane * IPL;
      if (IPL == 2) {
        const int2 v = __ldg(reinterpret_cast<const int2*>(src));
        d[0] = v.x;
        d[IPL - 1] = v.y;
      } else {
        d[0] = __ldg(src);
      }
    }
  };
  // int k of a descriptor held across the warp (k warp-uniform)
  auto D = [&](const int (&d)[IPL], int k) {
    const int v = (IPL == 2 && (k & 1)) ? d[IPL - 1] : d[0];
    return __shfl_sync(0xffffffffu, v, k / IPL);
  };

  // whole warp: start column e's copies into stage s
  auto issue = [&](int s, const int (&d)[IPL]) {
    int* mt = meta_of(s);
#pragma unroll
    for (int i = 0; i < IPL; ++i) mt[lane * IPL + i] = d[i];
    const int h = D(d, 1), ng = D(d, 2), nb = D(d, 3);
    T* xs = xs_of(s);
    int q = 0;
    const T* src = M;  // this lane's matrix block (lane < nb)
    for (int g = 0; g < ng; ++g) {
      const int c = D(d, 4 + g * GS);
      const uint32_t pk = (uint32_t)D(d, 5 + g * GS);
      int mf[NDF2];
#pragma unroll
      for (int j = 0; j < NDF2; ++j) mf[j] = D(d, 6 + g * GS + j);
      for (int r = 0; r < rec_n(pk); ++r, ++q) {
        if (lane == q) src = M + (size_t)c * cell_stride + (size_t)rec_df(pk, r) * A.blk;
        const int off = rec_off(pk, r);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const int l = lane + 32 * p, k = l - off;
          if (l < h && (unsigned)k < (unsigned)nl) {
#pragma unroll
            for (int j = 0; j < NDF2; ++j)
              cp_async<sizeof(T)>(xs + ((size_t)(q * NDF2 + j) * NP + p) * 32 + lane,
                                  x + mf[j] + k);
          }
        }
      }
    }
    cp_async_mbar_arrive(bar_of(s));
    __syncwarp();
    if (lane == 0) mbar_expect_tx(bar_of(s), (unsigned)nb * blk_bytes);
    __syncwarp();
    if (lane < nb) {
      fence_proxy_async();
      bulk_load(mat_of(s) + (size_t)lane * A.blk, src, blk_bytes, bar_of(s));
    }
  };

  if (lane == 0) {
    for (int s = 0; s < stages; ++s) mbar_init(bar_of(s), 1);
    fence_proxy_async();
  }
  __syncwarp();
  int d0[IPL] = {}, d1[IPL] = {};
  for (int s = 0; s < stages; ++s) {
    const int64_t e = warp0 + (int64_t)s * nwarp;
    if (e >= A.nent) break;
    int d[IPL] = {};
    load_desc(e, d);
    issue(s, d);
  }
  load_desc(warp0 + (int64_t)stages * nwarp, d0);
  load_desc(warp0 + (int64_t)(stages + 1) * nwarp, d1);
  int64_t it = 0;
  bool failed = false;
  for (int64_t e = warp0; e < A.nent; e += nwarp, ++it) {
    const int s = (int)(it % stages);
    const unsigned parity = (unsigned)((it / stages) & 1);
    unsigned spins = 0;
    while (!mbar_try_wait(bar_of(s), parity)) {
      if (++spins > kWaitLimit) {
        failed = true;
        break;
      }
    }
    if (__any_sync(0xffffffffu, failed)) {
      failed = true;
      if (lane == 0) atomicExch(err, 1);
      break;
    }
    const int* mt = meta_of(s);
    const T* ms = mat_of(s);
    const T* xs = xs_of(s);
    const int base = mt[0], h = mt[1], ng = mt[2];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const int l = lane + 32 * p;
      if (l < h) {
        T acc = T(0);
        int q = 0;
        for (int g = 0; g < ng; ++g) {
          const uint32_t pk = (uint32_t)mt[5 + g * GS];
          const int k0 = l - rec_off(pk, 0), k1 = l - rec_off(pk, 1);
          const bool v0 = (unsigned)k0 < (unsigned)nl;
          const bool v1 = rec_n(pk) > 1 && (unsigned)k1 < (unsigned)nl;
          const T* s0 = ms + (size_t)q * A.blk + (v0 ? k0 : 0);
          const T* s1 = v1 ? ms + (size_t)(q + 1) * A.blk + k1 : ms;
          const T* x0 = xs + ((size_t)q * NDF2 * NP + p) * 32 + lane;
          const T* x1 = xs + ((size_t)(q + 1) * NDF2 * NP + p) * 32 + lane;
#pragma unroll
          for (int j = 0; j < NDF2; ++j) {
            if (v0) acc = fmaT(s0[j * nl], x0[j * NP * 32], acc);
            if (v1) acc = fmaT(s1[j * nl], x1[j * NP * 32], acc);
          }
          q += rec_n(pk);
        }
        if (b)
          y[base + l] = b[base + l] - acc;
        else
          y[base + l] = acc;
      }
    }
    __syncwarp();
    if (e + (int64_t)stages * nwarp < A.nent) issue(s, d0);
#pragma unroll
    for (int i = 0; i < IPL; ++i) d0[i] = d1[i];
    load_desc(e + (int64_t)(stages + 2) * nwarp, d1);
  }
  if (failed && lane == 0) {
    // drain: stages of iterations it .. it+stages-1 may still have copies in
    // flight; wait (bounded) for each before the shared memory is released
    for (int k = 0; k < stages; ++k) {
      const int64_t ik = it + k;
      if (warp0 + ik * nwarp >= A.nent) break;
      const int s = (int)(ik % stages);
      const unsigned parity = (unsigned)((ik / stages) & 1);
      unsigned spins = 0;
      while (!mbar_try_wait(bar_of(s), parity) && ++spins < kWaitLimit) {
      }
    }
  }
}

// mm_diagonal (sci_mm_diagonal_kernel_mod.F90:117-122): per cell, layer k
// outer and df inner, diag += M(ik, df, df). In gather form a dof takes its
// records of one cell in increasing k (decreasing off), then increasing df.
template <class T>
__global__ void lma_diag(LayoutArgs A, int max_off, const T* __restrict__ M, T* __restrict__ d) {
  const int nl = A.nlayers, ndf = A.ndf1;
  const int lane = threadIdx.x & 31;
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const size_t cell_stride = (size_t)ndf * A.blk;
  for (int64_t e = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < A.nent; e += nwarp) {
    const int base = A.ent_base[e], h = A.ent_h[e];
    for (int l = lane; l < h; l += 32) {
      T acc = T(0);
      for (int g = A.ent_grp[e]; g < A.ent_grp[e + 1]; ++g) {
        const uint32_t pk = A.grp_rec[g];
        const T* Mc = M + (size_t)A.grp_cell[g] * cell_stride;
        for (int o = max_off; o >= 0; --o)
          for (int r = 0; r < rec_n(pk); ++r) {
            if (rec_off(pk, r) != o) continue;
            const int k = l - o, df = rec_df(pk, r);
            if (k >= 0 && k < nl) acc = acc + Mc[(size_t)df * A.blk + df * nl + k];
          }
      }
      d[base + l] = acc;
    }
  }
}

// transpose_matrix_vector (transpose_matrix_vector_kernel_mod.F90:128-144):
// per layer k and from-space dof df, s = sum_j M(ik, j, df) x(map_to(j)+k) and
// lhs += s. Gather over the from-space layout; records of one cell in
// increasing k, then increasing df. blk is the stored matrix's block stride.
template <class T>
__global__ void lma_gather_t(LayoutArgs A, int max_off, int blk, const T* __restrict__ M,
                             const T* __restrict__ x, const int32_t* __restrict__ map_to,
                             T* __restrict__ y) {
  // here A.ndf1 is the from-space ndf (output), A.ndf2 the to-space ndf
  const int nl = A.nlayers, ndf_in = A.ndf2;
  const int lane = threadIdx.x & 31;
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const size_t cell_stride = (size_t)ndf_in * blk;  // stored as [c][j(to)][df(from)][k]
  for (int64_t e = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < A.nent; e += nwarp) {
    const int base = A.ent_base[e], h = A.ent_h[e];
    for (int l = lane; l < h; l += 32) {
      T acc = T(0);
      for (int g = A.ent_grp[e]; g < A.ent_grp[e + 1]; ++g) {
        const uint32_t pk = A.grp_rec[g];
        const int c = A.grp_cell[g];
        const T* Mc = M + (size_t)c * cell_stride;
        const int* mt = map_to + (size_t)c * ndf_in;
        for (int o = max_off; o >= 0; --o)
          for (int r = 0; r < rec_n(pk); ++r) {
            if (rec_off(pk, r) != o) continue;
            const int k = l - o, df = rec_df(pk, r);
            if (k < 0 || k >= nl) continue;
            T s = T(0);
            for (int j = 0; j < ndf_in; ++j)
              s = fmaT(Mc[(size_t)j * blk + df * nl + k], x[mt[j] + k], s);
            acc = acc + s;
          }
      }
      y[base + l] = acc;
    }
  }
}

// Fortran (nc3, ndf1, ndf2) FP64 -> [c][df] blocks of blk elements, [df2][k] inside
template <class T>
__global__ void relayout(const double* __restrict__ src, T* __restrict__ dst, int64_t ncell,
                         int nl, int ndf1, int ndf2, int blk) {
  const int64_t total = ncell * ndf1 * blk;
  const int64_t nc3 = ncell * nl;
  for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d < total;
       d += (int64_t)gridDim.x * blockDim.x) {
    const int in = (int)(d % blk);
    const int64_t cd = d / blk;
    const int df = (int)(cd % ndf1);
    const int64_t c = cd / ndf1;
    if (in >= ndf2 * nl) {
      dst[d] = T(0);
      continue;
    }
    const int df2 = in / nl, k = in % nl;
    dst[d] = (T)src[(c * nl + k) + nc3 * (df + (int64_t)ndf1 * df2)];
  }
}

// ---------------------------------------------------------------- cell scatter
// The reference's own loop shape, one colour at a time: a warp takes one cell
// column (lane = level), loads the cell's local matrices and x values once,
// and adds M(df, df2) x(df2) into every dof of the cell in the reference's
// order (df2 outer, df inner), directly into y. The first cell on a dof
// column (in colour order) starts from zero, later ones from the stored sum,
// and in the residual form (b given) the last one writes b - sum;
// a column holding two records of the same cell at consecutive offsets (the
// bottom and top faces or vertices of a cell column) is summed by the lane
// of the output level, which takes the upper record's terms from the lane
// below. Cells of one colour share no dof, so a launch per colour is
// race-free, and every dof receives its terms in the coloured order of the
// reference (the bits of the gather kernels). With a symmetric operator the
// matrix is read from its packed upper triangle, so each entry crosses HBM
// once.
template <int NDF>
__host__ __device__ constexpr int pidx(int i, int j) {
  return i <= j ? i * NDF - i * (i - 1) / 2 + (j - i) : j * NDF - j * (j - 1) / 2 + (i - j);
}

// cells: the launch's colour in the colour-loop order (cell ids); q0: the
// position of its first cell in that order. Descriptors and the packed
// matrix copy are stored in that order (so a colour's launch streams one
// contiguous run of each); the full matrix copy stays in cell order.
struct CellArgs {
  int nl, blk, cstride, dints;
  const int* cells;
  int ncells;
  const int* desc;
  int q0;
};

template <class T, int NDF, bool SYM, bool RESID, bool CANON>
__global__ void __launch_bounds__(256) lma_cells(CellArgs C, const T* __restrict__ M,
                                                 const T* __restrict__ x, T* __restrict__ y,
                                                 const T* __restrict__ b, const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  const int lane = threadIdx.x & 31;
  const int ci = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (ci >= C.ncells) return;  // whole warps
  const int q = C.q0 + ci;
  const int c = SYM ? q : __ldg(C.cells + ci);  // the matrix block
  const int* dsc = C.desc + (size_t)q * C.dints;
  int mf[NDF];
#pragma unroll
  for (int j = 0; j < NDF; ++j) mf[j] = __ldg(dsc + j);
  const uint32_t flags = (uint32_t)__ldg(dsc + NDF), part = (uint32_t)__ldg(dsc + NDF + 1);
  const int nl = C.nl;
  const bool v = lane < nl;
  const T* Mc = M + (size_t)c * C.cstride + (v ? lane : 0);
  constexpr int NP = SYM ? NDF * (NDF + 1) / 2 : NDF * NDF;
  T m[NP], xv[NDF], yo[NDF];
  // the matrix is read once per apply: streaming (evict-first) loads keep x
  // and the partial sums of y in L2 for the later colours
#pragma unroll
  for (int p = 0; p < NP; ++p)
    m[p] = v ? __ldcs(Mc + (SYM ? p * nl : (p / NDF) * C.blk + (p % NDF) * nl)) : T(0);
#pragma unroll
  for (int j = 0; j < NDF; ++j) xv[j] = v ? __ldg(x + mf[j] + lane) : T(0);
  // the launch of colour k > 0 may start while colour k - 1 finishes
  // (programmatic dependent launch): its matrix and x loads above overlap that
  // tail, and it waits here, before touching y, until colour k - 1 has
  // completed (a no-op for a launch without the dependency)
  asm volatile("griddepcontrol.wait;" ::: "memory");
#pragma unroll
  for (int df = 0; df < NDF; ++df) {
    const bool lower = is_lower<NDF, CANON>(flags, df), upper = is_upper<NDF, CANON>(flags, df);
    const bool opens = (flags >> df) & 1u;
    const bool live = lower ? lane <= nl : v;
    yo[df] = (!upper && !opens && live) ? y[mf[df] + lane] : T(0);
  }
#define MV(i, j) m[SYM ? pidx<NDF>(i, j) : (i) * NDF + (j)]
#pragma unroll
  for (int df = 0; df < NDF; ++df) {
    if (is_upper<NDF, CANON>(flags, df)) continue;  // upper record: summed with its lower one
    if (is_lower<NDF, CANON>(flags, df)) {
      const int bsel = partner<NDF, CANON>(part, df);
#pragma unroll
      for (int bb = df + 1; bb < NDF; ++bb) {
        if (bb != bsel) continue;
        T acc = yo[df];
#pragma unroll
        for (int j = 0; j < NDF; ++j) {
          const T mb = __shfl_up_sync(0xffffffffu, MV(bb, j), 1);
          const T xb = __shfl_up_sync(0xffffffffu, xv[j], 1);
          if (v) acc = fmaT(MV(df, j), xv[j], acc);
          if (lane >= 1 && lane <= nl) acc = fmaT(mb, xb, acc);
        }
        if (lane <= nl) {
          // the last cell on the column writes b - A x in the residual form
          const int row = mf[df] + lane;
          y[row] = (RESID && ((flags >> (24 + df)) & 1u)) ? b[row] - acc : acc;
        }
      }
    } else {
      T acc = yo[df];
#pragma unroll
      for (int j = 0; j < NDF; ++j) acc = fmaT(MV(df, j), xv[j], acc);
      if (v) {
        // the last cell on the column writes b - A x in the residual form
        const int row = mf[df] + lane;
        y[row] = (RESID && ((flags >> (24 + df)) & 1u)) ? b[row] - acc : acc;
      }
    }
  }
#undef MV
}

// The cell scatter for columns of more than 31 levels: a cell column is split
// into nseg segments of L <= 31 levels, one warp each. In segment sg, lane l
// (1 <= l <= L) holds level k = sg * L + l - 1 and writes the dofs of that
// level (and the bottom face of a pair, whose upper-record terms come from
// the lane below); lane 0 holds the level just below the segment only to
// supply those terms to lane 1 and writes nothing. Every dof therefore gets
// the terms of lma_cells in the same order (the same bits).
template <class T, int NDF, bool SYM, bool RESID, bool CANON>
__global__ void __launch_bounds__(256) lma_cells_seg(CellArgs C, int nseg, int L,
                                                     const T* __restrict__ M,
                                                     const T* __restrict__ x, T* __restrict__ y,
                                                     const T* __restrict__ b, const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  const int lane = threadIdx.x & 31;
  const int64_t wg = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (wg >= (int64_t)C.ncells * nseg) return;  // whole warps
  const int ci = (int)(wg / nseg), sg = (int)(wg % nseg);
  const int q = C.q0 + ci;
  const int c = SYM ? q : __ldg(C.cells + ci);  // the matrix block
  const int* dsc = C.desc + (size_t)q * C.dints;
  int mf[NDF];
#pragma unroll
  for (int j = 0; j < NDF; ++j) mf[j] = __ldg(dsc + j);
  const uint32_t flags = (uint32_t)__ldg(dsc + NDF), part = (uint32_t)__ldg(dsc + NDF + 1);
  const int nl = C.nl;
  const int k = sg * L + lane - 1;           // this lane's level
  const bool own = lane >= 1 && lane <= L;   // lanes that write
  const bool v = k >= 0 && k < nl && lane <= L;  // a cell level this warp needs
  const T* Mc = M + (size_t)c * C.cstride + (v ? k : 0);
  constexpr int NP = SYM ? NDF * (NDF + 1) / 2 : NDF * NDF;
  T m[NP], xv[NDF], yo[NDF];
#pragma unroll
  for (int p = 0; p < NP; ++p)
    m[p] = v ? __ldcs(Mc + (SYM ? p * nl : (p / NDF) * C.blk + (p % NDF) * nl)) : T(0);
#pragma unroll
  for (int j = 0; j < NDF; ++j) xv[j] = v ? __ldg(x + mf[j] + k) : T(0);
  asm volatile("griddepcontrol.wait;" ::: "memory");
#pragma unroll
  for (int df = 0; df < NDF; ++df) {
    const bool lower = is_lower<NDF, CANON>(flags, df), upper = is_upper<NDF, CANON>(flags, df);
    const bool opens = (flags >> df) & 1u;
    const bool live = own && (lower ? k <= nl : v);
    yo[df] = (!upper && !opens && live) ? y[mf[df] + k] : T(0);
  }
#define MV(i, j) m[SYM ? pidx<NDF>(i, j) : (i) * NDF + (j)]
#pragma unroll
  for (int df = 0; df < NDF; ++df) {
    if (is_upper<NDF, CANON>(flags, df)) continue;  // upper record: summed with its lower one
    if (is_lower<NDF, CANON>(flags, df)) {
      const int bsel = partner<NDF, CANON>(part, df);
#pragma unroll
      for (int bb = df + 1; bb < NDF; ++bb) {
        if (bb != bsel) continue;
        T acc = yo[df];
#pragma unroll
        for (int j = 0; j < NDF; ++j) {
          const T mb = __shfl_up_sync(0xffffffffu, MV(bb, j), 1);
          const T xb = __shfl_up_sync(0xffffffffu, xv[j], 1);
          if (v) acc = fmaT(MV(df, j), xv[j], acc);
          if (own && k >= 1 && k <= nl) acc = fmaT(mb, xb, acc);
        }
        if (own && k <= nl) {
          const int row = mf[df] + k;
          y[row] = (RESID && ((flags >> (24 + df)) & 1u)) ? b[row] - acc : acc;
        }
      }
    } else {
      T acc = yo[df];
#pragma unroll
      for (int j = 0; j < NDF; ++j) acc = fmaT(MV(df, j), xv[j], acc);
      if (own && v) {
        const int row = mf[df] + k;
        y[row] = (RESID && ((flags >> (24 + df)) & 1u)) ? b[row] - acc : acc;
      }
    }
  }
#undef MV
}

// The cell scatter with each warp's next cells staged ahead: a warp walks
// the colour's cells with stride (warps in the grid) and keeps the local
// matrices and descriptors of its next S cells in flight (16-byte cp.async
// into a per-warp ring in shared memory), so HBM sees every warp's upcoming
// matrix blocks at once; lanes then read their level's entries from shared
// memory. Same arithmetic as lma_cells.
constexpr int kCellWarps = 4;

template <class T, int NDF, bool SYM, int S, bool RESID, bool CANON>
__global__ void __launch_bounds__(32 * kCellWarps) lma_cells_pipe(CellArgs C, const T* __restrict__ M,
                                                                 const T* __restrict__ x,
                                                                 T* __restrict__ y,
                                                                 const T* __restrict__ b,
                                                                 int stage_bytes,
                                                                 const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  extern __shared__ __align__(16) unsigned char cell_ring[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned char* ring = cell_ring + (size_t)wib * S * stage_bytes;
  const int mat_bytes = C.cstride * (int)sizeof(T);
  const int nq = mat_bytes / 16, dq = C.dints / 4;
  auto issue = [&](int64_t i, int s) {
    if (i < C.ncells) {
      const int cq = C.q0 + (int)i;
      const int c = SYM ? cq : __ldg(C.cells + i);  // the matrix block
      const char* src = reinterpret_cast<const char*>(M + (size_t)c * C.cstride);
      unsigned char* dst = ring + (size_t)s * stage_bytes;
      for (int q = lane; q < nq; q += 32) cp_async16(dst + 16 * q, src + 16 * q);
      const char* ds = reinterpret_cast<const char*>(C.desc + (size_t)cq * C.dints);
      if (lane < dq) cp_async16(dst + mat_bytes + 16 * lane, ds + 16 * lane);
    }
    cp_async_commit();
  };
#pragma unroll
  for (int s = 0; s < S; ++s) issue(gw + s * nw, s);
  const int nl = C.nl;
  const bool v = lane < nl;
  int s = 0;
  for (int64_t i = gw; i < C.ncells; i += nw) {
    cp_async_wait<S - 1>();
    __syncwarp();
    const unsigned char* st = ring + (size_t)s * stage_bytes;
    const T* sm = reinterpret_cast<const T*>(st) + (v ? lane : 0);
    const int* dsc = reinterpret_cast<const int*>(st + mat_bytes);
    int mf[NDF];
#pragma unroll
    for (int j = 0; j < NDF; ++j) mf[j] = dsc[j];
    const uint32_t flags = (uint32_t)dsc[NDF], part = (uint32_t)dsc[NDF + 1];
    constexpr int NP = SYM ? NDF * (NDF + 1) / 2 : NDF * NDF;
    T m[NP], xv[NDF], yo[NDF];
#pragma unroll
    for (int j = 0; j < NDF; ++j) xv[j] = v ? __ldg(x + mf[j] + lane) : T(0);
#pragma unroll
    for (int df = 0; df < NDF; ++df) {
      const bool lower = is_lower<NDF, CANON>(flags, df), upper = is_upper<NDF, CANON>(flags, df);
      const bool opens = (flags >> df) & 1u;
      const bool live = lower ? lane <= nl : v;
      yo[df] = (!upper && !opens && live) ? y[mf[df] + lane] : T(0);
    }
#pragma unroll
    for (int p = 0; p < NP; ++p)
      m[p] = v ? sm[SYM ? p * nl : (p / NDF) * C.blk + (p % NDF) * nl] : T(0);
    __syncwarp();
    // the stage is free again: fetch the cell S ahead
    issue(i + (int64_t)S * nw, s);
    s = s + 1 == S ? 0 : s + 1;
#define MV(i, j) m[SYM ? pidx<NDF>(i, j) : (i) * NDF + (j)]
#pragma unroll
    for (int df = 0; df < NDF; ++df) {
      if (is_upper<NDF, CANON>(flags, df)) continue;
      if (is_lower<NDF, CANON>(flags, df)) {
        const int bsel = partner<NDF, CANON>(part, df);
#pragma unroll
        for (int bb = df + 1; bb < NDF; ++bb) {
          if (bb != bsel) continue;
          T acc = yo[df];
#pragma unroll
          for (int j = 0; j < NDF; ++j) {
            const T mb = __shfl_up_sync(0xffffffffu, MV(bb, j), 1);
            const T xb = __shfl_up_sync(0xffffffffu, xv[j], 1);
            if (v) acc = fmaT(MV(df, j), xv[j], acc);
            if (lane >= 1 && lane <= nl) acc = fmaT(mb, xb, acc);
          }
          if (lane <= nl) {
            // the last cell on the column writes b - A x in the residual form
            const int row = mf[df] + lane;
            y[row] = (RESID && ((flags >> (24 + df)) & 1u)) ? b[row] - acc : acc;
          }
        }
      } else {
        T acc = yo[df];
#pragma unroll
        for (int j = 0; j < NDF; ++j) acc = fmaT(MV(df, j), xv[j], acc);
        if (v) {
          // the last cell on the column writes b - A x in the residual form
          const int row = mf[df] + lane;
          y[row] = (RESID && ((flags >> (24 + df)) & 1u)) ? b[row] - acc : acc;
        }
      }
    }
#undef MV
  }
  cp_async_wait<0>();
}

// The cell scatter as ONE persistent launch over all colours (kernel 6).
// Every warp of the grid walks its cells (stride: warps in the grid) colour
// after colour, through a ring of S stages in shared memory:
//   - S cells ahead, lane 0 moves the cell's matrix block and descriptor
//     with two cp.async.bulk copies completing on the stage's mbarrier;
//   - D cells ahead (D < S, so the descriptor has landed), every lane copies
//     its level's x values and partial sums of y for that cell with 4/8-byte
//     cp.async (zero-filled where the reference adds nothing), one commit
//     group per cell;
//   - the cell itself is summed from shared memory with the arithmetic of
//     lma_cells (the same bits).
// Colours are separated by a grid-wide barrier (the launch is cooperative:
// all blocks are resident). The matrix stream and the x copies run on across
// the barrier; the partial sums of y of a cell of the next colour are read
// only after it (a cell whose y would have been copied before the barrier is
// marked and reads y from L2 when its turn comes). Every wait is bounded by
// limit_ns; a time-out writes LFX_TIMEOUT to err, the grid leaves at the next
// barrier, and each warp first waits (bounded) for the copies it issued.
constexpr int kRingMaxCol = 16;  // colours of one ring launch, at most

struct CellRingArgs {
  int nl, blk, cstride, dints;
  const int* cells;  // colour-loop order -> cell (the full-storage matrix)
  const int* desc;
  int ncol, stages;
  unsigned* bar;  // [0] arrivals, [1] generation
  int* err;
  unsigned long long limit_ns;
  int cs[kRingMaxCol + 1];  // first position of each colour in the colour-loop order
};

__device__ __forceinline__ unsigned long long ring_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool ring_wait_ns(uint64_t* bar, unsigned parity,
                                             unsigned long long limit) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = ring_clock();
  while (!mbar_try_wait(bar, parity))
    if (ring_clock() - t0 > limit) return false;
  return true;
}
// BYTES-byte asynchronous copy that writes zeros instead when !on
template <int BYTES>
__device__ __forceinline__ void cp_async_zf(void* dst, const void* src, bool on) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(smem_u32(dst)), "l"(src),
               "n"(BYTES), "r"(on ? BYTES : 0)
               : "memory");
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
// grid-wide barrier; false when a block reported an error or the wait ran out
__device__ bool ring_grid_sync(const CellRingArgs& R, int* bad) {
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = *(volatile int*)R.err == 0;
    if (ok) {
      const unsigned gen = ld_acquire_u32(R.bar + 1);
      __threadfence();
      const unsigned arrived = atomicAdd(R.bar, 1u);
      if (arrived == gridDim.x - 1) {
        R.bar[0] = 0u;
        __threadfence();
        atomicExch(R.bar + 1, gen + 1u);
      } else {
        const unsigned long long t0 = ring_clock();
        while (ld_acquire_u32(R.bar + 1) == gen) {
          if (*(volatile int*)R.err) {
            ok = 0;
            break;
          }
          if (ring_clock() - t0 > R.limit_ns) {
            atomicExch(R.err, (int)LFX_TIMEOUT);
            ok = 0;
            break;
          }
        }
      }
      __threadfence();
    }
    *bad = !ok;
  }
  __syncthreads();
  return !*(volatile int*)bad;
}

template <class T, int NDF, bool SYM, int D, bool RESID, bool CANON>
__global__ void __launch_bounds__(256) lma_cells_ring(CellRingArgs R, const T* __restrict__ M,
                                                      const T* __restrict__ x, T* __restrict__ y,
                                                      const T* __restrict__ b, const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  extern __shared__ __align__(128) unsigned char ring_smem[];
  __shared__ int bad;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nwb = blockDim.x >> 5;
  const int S = R.stages, nl = R.nl;
  const int gw = blockIdx.x * nwb + wib, nw = gridDim.x * nwb;
  const unsigned mat_bytes = (unsigned)R.cstride * sizeof(T), dsc_bytes = (unsigned)R.dints * 4;
  // stage: matrix block, descriptor, x[NDF][32], y[NDF][32]
  const unsigned stage_bytes = mat_bytes + dsc_bytes + 2u * NDF * 32u * sizeof(T);
  unsigned char* ring = ring_smem + (size_t)wib * S * stage_bytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring_smem + (size_t)nwb * S * stage_bytes) + wib * S;
  if (lane == 0) {
    for (int s = 0; s < S; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();

  // a cursor over this warp's cells: colour k, position q in the colour loop
  auto advance = [&](int& k, int& q) {
    q += nw;
    while (k < R.ncol && q >= R.cs[k + 1]) {
      ++k;
      if (k < R.ncol) q = R.cs[k] + gw;
    }
  };
  auto first = [&](int& k, int& q) {
    k = 0;
    q = R.cs[0] + gw;
    while (k < R.ncol && q >= R.cs[k + 1]) {
      ++k;
      if (k < R.ncol) q = R.cs[k] + gw;
    }
  };
  // far copy (lane 0): matrix block and descriptor of the cell at (fk, fq)
  int fk, fq;
  unsigned nfar = 0;  // cells far-issued (lane 0's count)
  auto far_issue = [&]() {
    const unsigned s = nfar % (unsigned)S;
    unsigned char* st = ring + (size_t)s * stage_bytes;
    const int c = SYM ? fq : __ldg(R.cells + fq);
    fence_proxy_async();
    mbar_expect_tx(&bars[s], mat_bytes + dsc_bytes);
    bulk_load(st, M + (size_t)c * R.cstride, mat_bytes, &bars[s]);
    bulk_load(st + mat_bytes, R.desc + (size_t)fq * R.dints, dsc_bytes, &bars[s]);
    ++nfar;
    advance(fk, fq);
  };
  first(fk, fq);
  if (lane == 0)
    for (int i = 0; i < S && fk < R.ncol; ++i) far_issue();
  // near copy (all lanes): x and y of the cell at (nk, nq), after its
  // descriptor has landed; y only while the consumer is in the same colour
  int nk, nq;
  first(nk, nq);
  unsigned nnear = 0;    // cells near-issued (their descriptors waited for)
  unsigned ydefer = 0u;  // per stage: y of this cell not copied (read from L2 later)
  bool ok = true;
  const bool v = lane < nl;
  auto near_issue = [&](int kc) {
    if (nk < R.ncol) {
      const unsigned s = nnear % (unsigned)S;
      unsigned char* st = ring + (size_t)s * stage_bytes;
      if (!ring_wait_ns(&bars[s], (nnear / (unsigned)S) & 1u, R.limit_ns)) {
        ok = false;
        cp_async_commit();
        return;
      }
      const int* dsc = reinterpret_cast<const int*>(st + mat_bytes);
      const uint32_t flags = (uint32_t)dsc[NDF];
      T* xs = reinterpret_cast<T*>(st + mat_bytes + dsc_bytes);
      T* ys = xs + NDF * 32;
#pragma unroll
      for (int j = 0; j < NDF; ++j) {
        const int mf = dsc[j];
        cp_async_zf<sizeof(T)>(xs + j * 32 + lane, x + mf + (v ? lane : 0), v);
      }
      if (nk == kc) {
#pragma unroll
        for (int df = 0; df < NDF; ++df) {
          const bool lower = is_lower<NDF, CANON>(flags, df), upper = is_upper<NDF, CANON>(flags, df);
          const bool opens = (flags >> df) & 1u;
          const bool live = lower ? lane <= nl : v;
          const bool on = !upper && !opens && live;
          cp_async_zf<sizeof(T)>(ys + df * 32 + lane, y + dsc[df] + (on ? lane : 0), on);
        }
        ydefer &= ~(1u << s);
      } else {
        ydefer |= 1u << s;
      }
      ++nnear;
      advance(nk, nq);
    }
    cp_async_commit();
  };
  for (int i = 0; i < D; ++i) near_issue(0);

  unsigned ncons = 0;
  for (int kc = 0; kc < R.ncol; ++kc) {
    if (kc > 0) {
      if (!ok) atomicExch(R.err, (int)LFX_TIMEOUT);
      if (!ring_grid_sync(R, &bad)) break;
    }
    for (int q = R.cs[kc] + gw; q < R.cs[kc + 1] && ok; q += nw) {
      near_issue(kc);
      if (!ok) break;
      cp_async_wait<D>();
      __syncwarp();
      const unsigned s = ncons % (unsigned)S;
      const unsigned char* st = ring + (size_t)s * stage_bytes;
      const T* sm = reinterpret_cast<const T*>(st) + (v ? lane : 0);
      const int* dsc = reinterpret_cast<const int*>(st + mat_bytes);
      const T* xs = reinterpret_cast<const T*>(st + mat_bytes + dsc_bytes);
      const T* ys = xs + NDF * 32;
      int mf[NDF];
#pragma unroll
      for (int j = 0; j < NDF; ++j) mf[j] = dsc[j];
      const uint32_t flags = (uint32_t)dsc[NDF], part = (uint32_t)dsc[NDF + 1];
      constexpr int NP = SYM ? NDF * (NDF + 1) / 2 : NDF * NDF;
      T m[NP], xv[NDF], yo[NDF];
#pragma unroll
      for (int j = 0; j < NDF; ++j) xv[j] = xs[j * 32 + lane];
      if ((ydefer >> s) & 1u) {
#pragma unroll
        for (int df = 0; df < NDF; ++df) {
          const bool lower = is_lower<NDF, CANON>(flags, df), upper = is_upper<NDF, CANON>(flags, df);
          const bool opens = (flags >> df) & 1u;
          const bool live = lower ? lane <= nl : v;
          yo[df] = (!upper && !opens && live) ? __ldcg(y + mf[df] + lane) : T(0);
        }
      } else {
#pragma unroll
        for (int df = 0; df < NDF; ++df) yo[df] = ys[df * 32 + lane];
      }
#pragma unroll
      for (int p = 0; p < NP; ++p)
        m[p] = v ? sm[SYM ? p * nl : (p / NDF) * R.blk + (p % NDF) * nl] : T(0);
      __syncwarp();
      // every lane has read the stage: lane 0 refills it S cells ahead
      if (lane == 0 && fk < R.ncol) far_issue();
      ++ncons;
#define MV(i, j) m[SYM ? pidx<NDF>(i, j) : (i) * NDF + (j)]
#pragma unroll
      for (int df = 0; df < NDF; ++df) {
        if (is_upper<NDF, CANON>(flags, df)) continue;
        if (is_lower<NDF, CANON>(flags, df)) {
          const int bsel = partner<NDF, CANON>(part, df);
#pragma unroll
          for (int bb = df + 1; bb < NDF; ++bb) {
            if (bb != bsel) continue;
            T acc = yo[df];
#pragma unroll
            for (int j = 0; j < NDF; ++j) {
              const T mb = __shfl_up_sync(0xffffffffu, MV(bb, j), 1);
              const T xb = __shfl_up_sync(0xffffffffu, xv[j], 1);
              if (v) acc = fmaT(MV(df, j), xv[j], acc);
              if (lane >= 1 && lane <= nl) acc = fmaT(mb, xb, acc);
            }
            if (lane <= nl) {
              const int row = mf[df] + lane;
              __stcg(y + row, (RESID && ((flags >> (24 + df)) & 1u)) ? __ldg(b + row) - acc : acc);
            }
          }
        } else {
          T acc = yo[df];
#pragma unroll
          for (int j = 0; j < NDF; ++j) acc = fmaT(MV(df, j), xv[j], acc);
          if (v) {
            const int row = mf[df] + lane;
            __stcg(y + row, (RESID && ((flags >> (24 + df)) & 1u)) ? __ldg(b + row) - acc : acc);
          }
        }
      }
#undef MV
    }
  }
  if (!ok) atomicExch(R.err, (int)LFX_TIMEOUT);
  // leave with nothing in flight: this warp's per-lane copies, then (lane 0,
  // bounded, at least 2 s) the bulk copies it issued and nobody waited for
  cp_async_wait<0>();
  if (lane == 0) {
    const unsigned long long drain = R.limit_ns > 2000000000ull ? R.limit_ns : 2000000000ull;
    for (unsigned i = nnear; i < nfar; ++i)
      ring_wait_ns(&bars[i % (unsigned)S], (i / (unsigned)S) & 1u, drain);
  }
  __syncwarp();
}

// level-major copy of the FP32 packed triangles: dst[(q nl + k) 4 npv + p]
// = src[q sblk + p nl + k], zero in the padding p >= np
__global__ void relayout_level_major(const float* __restrict__ src, float* __restrict__ dst,
                                     int64_t ncol, int nl, int np, int npv, int sblk) {
  const int w = 4 * npv;
  const int64_t total = ncol * nl * w;
  for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d < total;
       d += (int64_t)gridDim.x * blockDim.x) {
    const int p = (int)(d % w);
    const int64_t qk = d / w;
    const int k = (int)(qk % nl);
    const int64_t q = qk / nl;
    dst[d] = p < np ? src[q * sblk + (int64_t)p * nl + k] : 0.f;
  }
}

// packed upper triangle [q][p][k] (block stride sblk; block q holds the q-th
// cell of the colour loop, order[q]) from the Fortran (nc3, ndf, ndf) FP64
// stencil
template <class T>
__global__ void relayout_sym(const double* __restrict__ src, T* __restrict__ dst, int64_t ncell,
                             int nl, int ndf, int sblk, const int* __restrict__ order) {
  const int np = ndf * (ndf + 1) / 2;
  const int64_t total = ncell * sblk;
  const int64_t nc3 = ncell * nl;
  for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d < total;
       d += (int64_t)gridDim.x * blockDim.x) {
    const int in = (int)(d % sblk);
    const int64_t c = order[d / sblk];  // block q holds the q-th cell of the colour loop
    if (in >= np * nl) {
      dst[d] = T(0);
      continue;
    }
    int p = in / nl, i = 0;
    const int k = in % nl;
    while (p >= ndf - i) {
      p -= ndf - i;
      ++i;
    }
    const int j = i + p;
    dst[d] = (T)src[(c * nl + k) + nc3 * (i + (int64_t)ndf * j)];
  }
}

// *bad = 1 unless every local matrix equals its transpose bit for bit
__global__ void sym_check(const double* __restrict__ src, int64_t nc3, int ndf, int* bad) {
  const int64_t total = nc3 * ndf * ndf;
  for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d < total;
       d += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = d % nc3;
    const int ij = (int)(d / nc3), i = ij % ndf, j = ij / ndf;
    if (i < j && __double_as_longlong(src[r + nc3 * (i + (int64_t)ndf * j)]) !=
                     __double_as_longlong(src[r + nc3 * (j + (int64_t)ndf * i)]))
      *bad = 1;
  }
}

struct HostRec {
  int32_t start, cell, df;
};

// Builds the gather layout of the space described by `map` (ndf dofs per
// cell, [c][df] 1-based) for a colouring given as rank[c]. When mf0 (the
// 0-based from-space map, ndf_from per cell) is given, the packed records of
// the fast kernels are built too.
int build_layout(lfx_ctx* ctx, lfx_lma_layout* L, int32_t ncell, int32_t nl, int32_t ndf,
                 const int32_t* map, int64_t undf, const std::vector<int32_t>& rank,
                 const int32_t* mf0, int32_t ndf_from, const std::vector<int32_t>* colour) {
  std::vector<HostRec> recs;
  recs.reserve((size_t)ncell * ndf);
  for (int32_t c = 0; c < ncell; ++c)
    for (int32_t df = 0; df < ndf; ++df) {
      int32_t s = map[(size_t)c * ndf + df] - 1;
      if (s < 0 || (int64_t)s + nl > undf)
        return fail(ctx, LFX_INVALID_ARGUMENT, "dofmap entry out of range");
      recs.push_back({s, c, df});
    }
  std::stable_sort(recs.begin(), recs.end(),
                   [](const HostRec& a, const HostRec& b) { return a.start < b.start; });
  std::vector<int32_t> ent_base, ent_h, ent_grp, grp_cell;
  std::vector<uint32_t> grp_rec;
  // cell-scatter plan: only for square operators on one dofmap (colour given)
  bool cs = colour != nullptr && ndf <= 8;
  std::vector<uint32_t> cs_flags(cs ? (size_t)ncell : 0, 0u), cs_part(cs ? (size_t)ncell : 0, 0u);
  size_t i = 0;
  int64_t covered = 0;
  int max_off = 0, max_h = 0, max_groups = 0, max_blocks = 0;
  while (i < recs.size()) {
    const int32_t base = recs[i].start;
    int32_t end = base + nl;
    size_t j = i + 1;
    while (j < recs.size() && recs[j].start < end) {
      end = std::max(end, recs[j].start + nl);
      ++j;
    }
    // records i..j-1 form one entity column [base, end)
    std::vector<HostRec> er(recs.begin() + i, recs.begin() + j);
    std::stable_sort(er.begin(), er.end(), [&](const HostRec& a, const HostRec& b) {
      if (rank[a.cell] != rank[b.cell]) return rank[a.cell] < rank[b.cell];
      return a.df < b.df;
    });
    ent_base.push_back(base);
    ent_h.push_back(end - base);
    max_h = std::max(max_h, end - base);
    covered += end - base;
    ent_grp.push_back((int32_t)grp_cell.size());
    size_t q = 0;
    int ng = 0, nb = 0;
    while (q < er.size()) {
      size_t r = q;
      uint32_t pk = 0;
      int n = 0;
      while (r < er.size() && er[r].cell == er[q].cell) {
        int off = er[r].start - base;
        if (n >= 3 || off > 7 || er[r].df > 63)
          return fail(ctx, LFX_NOT_SUPPORTED,
                      "dofmap pattern not supported (more than 3 local dofs of one cell on a "
                      "dof column, or vertical offset > 7)");
        pk |= ((uint32_t)er[r].df & 63u) << (2 + 9 * n);
        pk |= ((uint32_t)off & 7u) << (8 + 9 * n);
        max_off = std::max(max_off, off);
        ++n;
        ++r;
      }
      pk |= (uint32_t)n;
      L->max_nrec = std::max(L->max_nrec, n);
      if (cs) {
        // every cell on the column must carry the first cell's record pattern
        // (one record, or two at consecutive offsets), in distinct colours
        const uint32_t pat = pk & ~((63u << 2) | (63u << 11) | (63u << 20));
        const uint32_t pat0 = grp_cell.size() > (size_t)ent_grp.back()
                                  ? grp_rec[ent_grp.back()] & ~((63u << 2) | (63u << 11) | (63u << 20))
                                  : pat;
        if (n > 2 || pat != pat0 || (n == 2 && rec_off(pk, 1) != rec_off(pk, 0) + 1)) cs = false;
        for (int32_t g = ent_grp.back(); cs && g < (int32_t)grp_cell.size(); ++g)
          if ((*colour)[grp_cell[g]] == (*colour)[er[q].cell]) cs = false;
        if (cs) {
          const int32_t c = er[q].cell;
          const bool first = (int32_t)grp_cell.size() == ent_grp.back();
          const bool last = r == er.size();
          const int a = rec_df(pk, 0);
          if (first) cs_flags[c] |= 1u << a;
          if (last) cs_flags[c] |= 1u << (24 + a);
          if (n == 2) {
            const int bb = rec_df(pk, 1);
            if (first) cs_flags[c] |= 1u << bb;
            if (last) cs_flags[c] |= 1u << (24 + bb);
            cs_flags[c] |= (1u << (8 + a)) | (1u << (16 + bb));
            cs_part[c] |= (uint32_t)bb << (4 * a);
          }
        }
      }
      grp_cell.push_back(er[q].cell);
      grp_rec.push_back(pk);
      ++ng;
      nb += n;
      q = r;
    }
    max_groups = std::max(max_groups, ng);
    max_blocks = std::max(max_blocks, nb);
    i = j;
  }
  ent_grp.push_back((int32_t)grp_cell.size());
  L->nent = (int32_t)ent_base.size();
  L->ngrp = (int32_t)grp_cell.size();
  L->max_h = max_h;
  L->max_off = max_off;
  L->max_groups = max_groups;
  L->max_blocks = max_blocks;
  L->full_cover = covered == undf;
  int rc = 0;
  auto up = [&](void** dst, const void* src, size_t bytes) {
    if (rc) return;
    rc = dmalloc(ctx, dst, bytes);
    if (!rc && bytes && cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
      rc = fail(ctx, LFX_CUDA_ERROR, "upload of LMA layout failed");
  };
  up((void**)&L->ent_base, ent_base.data(), ent_base.size() * 4);
  up((void**)&L->ent_h, ent_h.data(), ent_h.size() * 4);
  up((void**)&L->ent_grp, ent_grp.data(), ent_grp.size() * 4);
  up((void**)&L->grp_cell, grp_cell.data(), grp_cell.size() * 4);
  up((void**)&L->grp_rec, grp_rec.data(), grp_rec.size() * 4);
  if (cs && mf0) {
    // cells in colour-loop order, the start of each colour, per cell descriptors
    std::vector<int32_t> order(ncell);
    for (int32_t c = 0; c < ncell; ++c) order[rank[c]] = c;
    int32_t ncol = 0;
    for (int32_t c = 0; c < ncell; ++c) ncol = std::max(ncol, (*colour)[c] + 1);
    L->colour_start.assign(ncol + 1, 0);
    for (int32_t c = 0; c < ncell; ++c) L->colour_start[(*colour)[c] + 1]++;
    for (int32_t k = 0; k < ncol; ++k) L->colour_start[k + 1] += L->colour_start[k];
    L->cs_ints = (ndf + 2 + 3) / 4 * 4;
    std::vector<int32_t> d((size_t)ncell * L->cs_ints, 0);
    for (int32_t c = 0; c < ncell; ++c) {
      int32_t* row = &d[(size_t)rank[c] * L->cs_ints];  // in colour-loop order
      for (int j = 0; j < ndf; ++j) row[j] = mf0[(size_t)c * ndf + j];
      row[ndf] = (int32_t)cs_flags[c];
      row[ndf + 1] = (int32_t)cs_part[c];
    }
    up((void**)&L->cs_cells, order.data(), order.size() * 4);
    up((void**)&L->cs_desc, d.data(), d.size() * 4);
    L->cs_ok = rc == 0;
    // one vertical-pair structure for every cell (the reference element's)?
    constexpr uint32_t kStructBits = 0x00FFFF00u;
    L->cs_uniform = ncell > 0;
    for (int32_t c = 1; c < ncell && L->cs_uniform; ++c)
      L->cs_uniform = (cs_flags[c] & kStructBits) == (cs_flags[0] & kStructBits) &&
                      cs_part[c] == cs_part[0];
    if (L->cs_uniform) {
      L->cs_struct_flags = cs_flags[0] & kStructBits;
      L->cs_struct_part = cs_part[0];
    }
  }
  if (mf0) {
    std::vector<int4> ep(L->nent);
    for (int32_t e = 0; e < L->nent; ++e) ep[e] = make_int4(ent_base[e], ent_h[e], ent_grp[e], ent_grp[e + 1]);
    L->gp_stride = (2 + ndf_from + 3) / 4 * 4;
    std::vector<int32_t> gp((size_t)L->ngrp * L->gp_stride, 0);
    for (int32_t g = 0; g < L->ngrp; ++g) {
      int32_t* row = &gp[(size_t)g * L->gp_stride];
      row[0] = grp_cell[g];
      row[1] = (int32_t)grp_rec[g];
      for (int j = 0; j < ndf_from; ++j) row[2 + j] = mf0[(size_t)grp_cell[g] * ndf_from + j];
    }
    up((void**)&L->ent_pack, ep.data(), ep.size() * sizeof(int4));
    up((void**)&L->grp_pack, gp.data(), gp.size() * 4);
    // one-load descriptors for the pipelined gather (groups of at most two
    // records, at most 64 ints, columns of at most 96 dofs)
    const int gs = 2 + ndf_from;
    const int need = 4 + max_groups * gs;
    if (L->max_nrec <= 2 && need <= 64 && max_h <= 96) {
      L->desc_ipl = need <= 32 ? 1 : 2;
      const int ds = 32 * L->desc_ipl;
      std::vector<int32_t> d((size_t)L->nent * ds, 0);
      for (int32_t e = 0; e < L->nent; ++e) {
        int32_t* row = &d[(size_t)e * ds];
        row[0] = ent_base[e];
        row[1] = ent_h[e];
        row[2] = ent_grp[e + 1] - ent_grp[e];
        int nb = 0;
        for (int32_t g = ent_grp[e]; g < ent_grp[e + 1]; ++g) {
          int32_t* gr = row + 4 + (g - ent_grp[e]) * gs;
          gr[0] = grp_cell[g];
          gr[1] = (int32_t)grp_rec[g];
          for (int j = 0; j < ndf_from; ++j) gr[2 + j] = mf0[(size_t)grp_cell[g] * ndf_from + j];
          nb += rec_n(grp_rec[g]);
        }
        row[3] = nb;
      }
      up((void**)&L->desc, d.data(), d.size() * 4);
    }
    // descriptors of the prefetching gather (at most two blocks from at most
    // two cells per column)
    if (max_blocks <= 2 && max_groups <= 2 && (ndf_from == 1 || ndf_from == 6 || ndf_from == 8)) {
      const int gs = fd_group_ints(ndf_from), fs = fd_ints(ndf_from);
      L->fd_ints = fs;
      std::vector<int32_t> d((size_t)L->nent * fs, 0);
      for (int32_t e = 0; e < L->nent; ++e) {
        int32_t* row = &d[(size_t)e * fs];
        row[0] = ent_base[e];
        row[1] = ent_h[e];
        row[2] = ent_grp[e + 1] - ent_grp[e];
        for (int32_t g = ent_grp[e]; g < ent_grp[e + 1]; ++g) {
          int32_t* gr = row + 4 + (g - ent_grp[e]) * gs;
          gr[0] = grp_cell[g];
          gr[1] = (int32_t)grp_rec[g];
          for (int j = 0; j < ndf_from; ++j) gr[2 + j] = mf0[(size_t)grp_cell[g] * ndf_from + j];
        }
      }
      up((void**)&L->fdesc, d.data(), d.size() * 4);
    }
  }
  return rc;
}

void free_layout(lfx_ctx* ctx, lfx_lma_layout* L) {
  if (!L) return;
  dfree(ctx, L->ent_base, (size_t)L->nent * 4);
  dfree(ctx, L->ent_h, (size_t)L->nent * 4);
  dfree(ctx, L->ent_grp, (size_t)(L->nent + 1) * 4);
  dfree(ctx, L->grp_cell, (size_t)L->ngrp * 4);
  dfree(ctx, L->grp_rec, (size_t)L->ngrp * 4);
  dfree(ctx, L->ent_pack, (size_t)L->nent * sizeof(int4));
  dfree(ctx, L->grp_pack, (size_t)L->ngrp * L->gp_stride * 4);
  dfree(ctx, L->desc, (size_t)L->nent * 32 * L->desc_ipl * 4);
  dfree(ctx, L->fdesc, (size_t)L->nent * L->fd_ints * 4);
  dfree(ctx, L->cs_cells, (size_t)L->ncell_2d * 4);
  dfree(ctx, L->cs_desc, (size_t)L->ncell_2d * L->cs_ints * 4);
  dfree(ctx, L->map_from, (size_t)L->ncell_2d * L->ndf_from * 4);
  dfree(ctx, L->map_to, (size_t)L->ncell_2d * L->ndf_to * 4);
  free_layout(ctx, L->tlay);
  delete L;
}

int upload_matrix(lfx_ctx* ctx, lfx_op* op, const double* stencil) {
  const lfx_lma_layout* L = op->lay;
  const size_t esz = op->precision == LFX_R64 ? 8 : 4;
  op->blk = block_elems(L->ndf_from, L->nlayers, esz);
  const int64_t total_in = (int64_t)L->ncell_2d * L->ndf_to * L->ndf_from * L->nlayers;
  const int64_t total = (int64_t)L->ncell_2d * L->ndf_to * op->blk;
  double* raw = nullptr;
  int rc = dmalloc(ctx, (void**)&raw, (size_t)total_in * 8);
  if (rc) return rc;
  rc = dmalloc(ctx, &op->mat, (size_t)total * esz);
  if (rc) {
    dfree(ctx, raw, (size_t)total_in * 8);
    return rc;
  }
  op->mat_bytes = (size_t)total * esz;
  // the stencil may be host or device memory (unified addressing)
  LFX_CK(ctx, cudaMemcpyAsync(raw, stencil, (size_t)total_in * 8, cudaMemcpyDefault, ctx->stream));
  const int grid = ctx->num_sms * 16;
  if (op->precision == LFX_R64)
    relayout<double><<<grid, 256, 0, ctx->stream>>>(raw, (double*)op->mat, L->ncell_2d, L->nlayers,
                                                     L->ndf_to, L->ndf_from, op->blk);
  else
    relayout<float><<<grid, 256, 0, ctx->stream>>>(raw, (float*)op->mat, L->ncell_2d, L->nlayers,
                                                    L->ndf_to, L->ndf_from, op->blk);
  LFX_CK(ctx, cudaGetLastError());
  if (L->cs_ok) {
    // bitwise symmetric local matrices: keep the packed upper triangle too
    int* bad = nullptr;
    int hbad = 1;
    rc = dmalloc(ctx, (void**)&bad, 4);
    if (!rc) {
      cudaMemsetAsync(bad, 0, 4, ctx->stream);
      sym_check<<<grid, 256, 0, ctx->stream>>>(raw, (int64_t)L->ncell_2d * L->nlayers, L->ndf_to, bad);
      LFX_CK(ctx, cudaGetLastError());
      LFX_CK(ctx, cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, ctx->stream));
      LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
      dfree(ctx, bad, 4);
    }
    if (!rc && !hbad) {
      const int np = L->ndf_to * (L->ndf_to + 1) / 2;
      const size_t b = (size_t)np * L->nlayers * esz;
      op->sblk = (int)(((b + 15) / 16 * 16) / esz);
      op->smat_bytes = (size_t)L->ncell_2d * op->sblk * esz;
      rc = dmalloc(ctx, &op->smat, op->smat_bytes);
      if (!rc) {
        if (op->precision == LFX_R64)
          relayout_sym<double><<<grid, 256, 0, ctx->stream>>>(raw, (double*)op->smat, L->ncell_2d,
                                                               L->nlayers, L->ndf_to, op->sblk,
                                                               L->cs_cells);
        else
          relayout_sym<float><<<grid, 256, 0, ctx->stream>>>(raw, (float*)op->smat, L->ncell_2d,
                                                              L->nlayers, L->ndf_to, op->sblk,
                                                              L->cs_cells);
        LFX_CK(ctx, cudaGetLastError());
      } else {
        op->smat_bytes = 0;
      }
    }
  }
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, raw, (size_t)total_in * 8);
  return rc;
}

int gather_grid(const lfx_ctx* ctx, int32_t nent) {
  int64_t g = ((int64_t)nent + 7) / 8;
  int64_t cap = (int64_t)ctx->num_sms * 16;
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}

// launch shape of lma_tma: warps per block and pipeline stages, with the
// dynamic shared memory they need (0 warps when the operator does not fit)
struct TmaShape {
  int warps = 0, stages = 0;
  size_t smem = 0;
};
constexpr size_t kTmaSmemMax = 96 * 1024;

bool tma_ok(const lfx_op* op) {
  const lfx_lma_layout* L = op->lay;
  // the kernel is instantiated for ndf_from 1, 6 and 8 only; its metadata
  // holds at most 8 groups of at most 2 records
  if (L->max_nrec > 2 || L->max_groups > 8) return false;
  return L->ndf_from == 1 || L->ndf_from == 6 || L->ndf_from == 8;
}

TmaShape tma_shape(const lfx_op* op, int stages, int warps) {
  TmaShape t;
  if (!tma_ok(op) || stages < 1 || warps < 1) return t;
  const size_t esz = op->precision == LFX_R64 ? 8 : 4;
  const size_t stage = (size_t)op->lay->max_blocks * op->blk * esz;
  const size_t per_warp = stages * (stage + sizeof(TmaMeta) + 16);
  if (per_warp * warps > kTmaSmemMax) return t;
  t.warps = warps;
  t.stages = stages;
  t.smem = per_warp * warps;
  return t;
}

TmaShape tma_default(const lfx_op* op) {
  for (int stages = 4; stages >= 2; --stages)
    for (int warps = 4; warps >= 1; warps >>= 1) {
      TmaShape t = tma_shape(op, stages, warps);
      if (t.warps) return t;
    }
  return TmaShape{};
}

// pipelined gather (kernel 4): needs the one-load descriptors
bool pipe_ok(const lfx_op* op) {
  const lfx_lma_layout* L = op->lay;
  if (!L->desc || L->max_nrec > 2 || L->max_h > 96 || L->max_blocks > 32) return false;
  return L->ndf_from == 1 || L->ndf_from == 6 || L->ndf_from == 8;
}

TmaShape pipe_shape(const lfx_op* op, int stages, int warps) {
  TmaShape t;
  if (!pipe_ok(op) || stages < 1 || warps < 1) return t;
  const lfx_lma_layout* L = op->lay;
  const size_t esz = op->precision == LFX_R64 ? 8 : 4;
  const int np = (L->max_h + 31) / 32;
  const size_t stage = (size_t)L->max_blocks * op->blk * esz +
                       (size_t)L->max_blocks * L->ndf_from * 32 * np * esz +
                       (size_t)32 * L->desc_ipl * 4 + 16;
  const size_t per_warp = stages * stage;
  if (per_warp * warps > kTmaSmemMax) return t;
  t.warps = warps;
  t.stages = stages;
  t.smem = per_warp * warps;
  return t;
}

TmaShape pipe_default(const lfx_op* op) {
  for (int stages = 4; stages >= 2; --stages)
    for (int warps = 4; warps >= 1; warps >>= 1) {
      TmaShape t = pipe_shape(op, stages, warps);
      if (t.warps) return t;
    }
  return TmaShape{};
}

template <class T, int N, int IPL, int NP>
void launch_pipe_t(lfx_ctx* ctx, const lfx_op* op, const LayoutArgs& A, const TmaShape& ts,
                   const void* x, void* y, const void* b, const int* skip) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(lma_pipe<T, N, IPL, NP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kTmaSmemMax);
    attr = true;
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lma_pipe<T, N, IPL, NP>, 32 * ts.warps,
                                                ts.smem);
  if (per_sm < 1) per_sm = 1;
  const int grid = (int)std::min<int64_t>(((int64_t)A.nent + ts.warps - 1) / ts.warps,
                                          (int64_t)ctx->num_sms * per_sm);
  lma_pipe<T, N, IPL, NP><<<grid, 32 * ts.warps, ts.smem, ctx->stream>>>(
      A, (const T*)op->mat, (const T*)x, (T*)y, (const T*)b, skip, ts.stages,
      op->lay->max_blocks, ctx->d_err);
}

template <class T, int N, int IPL>
void launch_pipe_np(lfx_ctx* ctx, const lfx_op* op, const LayoutArgs& A, const TmaShape& ts,
                    const void* x, void* y, const void* b, const int* skip) {
  switch ((op->lay->max_h + 31) / 32) {
    case 1: launch_pipe_t<T, N, IPL, 1>(ctx, op, A, ts, x, y, b, skip); return;
    case 2: launch_pipe_t<T, N, IPL, 2>(ctx, op, A, ts, x, y, b, skip); return;
    default: launch_pipe_t<T, N, IPL, 3>(ctx, op, A, ts, x, y, b, skip); return;
  }
}

template <class T>
void launch_pipe(lfx_ctx* ctx, const lfx_op* op, const LayoutArgs& A, const TmaShape& ts,
                 const void* x, void* y, const void* b, const int* skip) {
  const bool two = op->lay->desc_ipl == 2;
  switch (op->lay->ndf_from) {
    case 1: launch_pipe_np<T, 1, 1>(ctx, op, A, ts, x, y, b, skip); return;
    case 6:
      if (two) launch_pipe_np<T, 6, 2>(ctx, op, A, ts, x, y, b, skip);
      else launch_pipe_np<T, 6, 1>(ctx, op, A, ts, x, y, b, skip);
      return;
    default:
      if (two) launch_pipe_np<T, 8, 2>(ctx, op, A, ts, x, y, b, skip);
      else launch_pipe_np<T, 8, 1>(ctx, op, A, ts, x, y, b, skip);
      return;
  }
}

template <class T, int N>
void launch_tma(lfx_ctx* ctx, const lfx_op* op, const LayoutArgs& A, const TmaShape& ts,
                const void* x, void* y, const void* b, const int* skip) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(lma_tma<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kTmaSmemMax);
    attr = true;
  }
  // persistent warps: one resident wave of blocks, each warp walking its
  // entity columns with `stages` of them in flight
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lma_tma<T, N>, 32 * ts.warps, ts.smem);
  if (per_sm < 1) per_sm = 1;
  const int grid = (int)std::min<int64_t>(((int64_t)A.nent + ts.warps - 1) / ts.warps,
                                          (int64_t)ctx->num_sms * per_sm);
  lma_tma<T, N><<<grid, 32 * ts.warps, ts.smem, ctx->stream>>>(
      A, (const T*)op->mat, (const T*)x, (T*)y, (const T*)b, skip, ts.stages,
      op->lay->max_blocks, ctx->d_err);
}

// descriptor-prefetch gather (kernel 3): columns of at most two blocks from
// at most two cells, ndf_from 1, 6 or 8
bool fetch_ok(const lfx_op* op) {
  const lfx_lma_layout* L = op->lay;
  return L->fdesc && L->max_blocks <= 2 && L->max_groups <= 2 &&
         (L->ndf_from == 1 || L->ndf_from == 6 || L->ndf_from == 8);
}

// one resident wave of blocks: each warp walks its columns with the
// descriptors of the next kFetchDepth in flight. variant 0 caps registers for
// 3 blocks of 256 per SM, variant 1 for 4 (FP32) / 2 (FP64).
template <class T, int N, int MINB>
void launch_fetch_t(lfx_ctx* ctx, const lfx_op* op, const LayoutArgs& A, const void* x, void* y,
                    const void* b, const int* skip) {
  static int per_sm = 0;
  if (!per_sm) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lma_fetch<T, N, MINB>, 256, 0);
    if (per_sm < 1) per_sm = 1;
  }
  const int grid = (int)std::min<int64_t>(((int64_t)A.nent + 7) / 8, (int64_t)ctx->num_sms * per_sm);
  lma_fetch<T, N, MINB><<<grid, 256, 0, ctx->stream>>>(A, (const T*)op->mat, (const T*)x, (T*)y,
                                                        (const T*)b, skip);
}

template <class T, int N>
void launch_fetch(lfx_ctx* ctx, const lfx_op* op, const LayoutArgs& A, int variant, const void* x,
                  void* y, const void* b, const int* skip) {
  if (variant == 1)
    launch_fetch_t<T, N, sizeof(T) == 8 ? 2 : 4>(ctx, op, A, x, y, b, skip);
  else
    launch_fetch_t<T, N, 3>(ctx, op, A, x, y, b, skip);
}

// cell scatter (kernel 5): one dofmap, the plan built, ndf 1, 6 or 8
bool cells_ok(const lfx_op* op) {
  const lfx_lma_layout* L = op->lay;
  return L->cs_ok && (L->ndf_to == 1 || L->ndf_to == 6 || L->ndf_to == 8);
}

// shared memory of one stage of lma_cells_pipe: a cell's matrix block and
// its descriptor
size_t cells_stage_bytes(const lfx_op* op) {
  const size_t esz = op->precision == LFX_R64 ? 8 : 4;
  const size_t m = op->smat ? (size_t)op->sblk * esz : (size_t)op->lay->ndf_to * op->blk * esz;
  return m + (size_t)op->lay->cs_ints * 4;
}
constexpr size_t kCellSmemMax = 200 * 1024;

// stages: 0 one cell per warp (lma_cells), 2 or 3 the staged pipeline
template <class T, int N, bool SYM, int S, bool RESID, bool CANON>
void launch_cells_t(lfx_ctx* ctx, const lfx_op* op, const void* x, void* y, const void* b,
                    const int* skip) {
  const lfx_lma_layout* L = op->lay;
  CellArgs C{L->nlayers, op->blk, SYM ? op->sblk : N * op->blk, L->cs_ints, nullptr, 0, L->cs_desc, 0};
  const T* M = (const T*)(SYM ? op->smat : op->mat);
  const int sb = (int)cells_stage_bytes(op);
  const size_t smem = (size_t)kCellWarps * S * sb;
  int per_sm = 1;
  if constexpr (S > 0) {
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(lma_cells_pipe<T, N, SYM, S, RESID, CANON>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCellSmemMax);
      attr = true;
    }
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lma_cells_pipe<T, N, SYM, S, RESID, CANON>,
                                                  32 * kCellWarps, smem);
    if (per_sm < 1) per_sm = 1;
  }
  // one launch per colour, in the reference's colour order
  for (size_t k = 0; k + 1 < L->colour_start.size(); ++k) {
    C.cells = L->cs_cells + L->colour_start[k];
    C.q0 = L->colour_start[k];
    C.ncells = L->colour_start[k + 1] - L->colour_start[k];
    if (C.ncells <= 0) continue;
    if constexpr (S > 0) {
      const int grid = (int)std::min<int64_t>(((int64_t)C.ncells + kCellWarps - 1) / kCellWarps,
                                              (int64_t)ctx->num_sms * per_sm);
      lma_cells_pipe<T, N, SYM, S, RESID, CANON><<<grid, 32 * kCellWarps, smem, ctx->stream>>>(
          C, M, (const T*)x, (T*)y, (const T*)b, sb, skip);
    } else {
      // colours after the first launch as programmatic dependents of the
      // previous colour (they wait in the kernel before reading y); a column
      // of more than 31 levels takes nseg warps of L levels each
      const int nl = L->nlayers;
      const int nseg = nl + 1 <= 32 ? 1 : (nl + 1 + 30) / 31;
      const int seg_l = (nl + 1 + nseg - 1) / nseg;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)(((int64_t)C.ncells * nseg * 32 + 255) / 256));
      cfg.blockDim = dim3(256);
      cfg.dynamicSmemBytes = 0;
      cfg.stream = ctx->stream;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      at[0].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = at;
      cfg.numAttrs = k > 0 ? 1 : 0;
      if (nseg == 1)
        cudaLaunchKernelEx(&cfg, lma_cells<T, N, SYM, RESID, CANON>, C, M, (const T*)x, (T*)y,
                           (const T*)b, skip);
      else
        cudaLaunchKernelEx(&cfg, lma_cells_seg<T, N, SYM, RESID, CANON>, C, nseg, seg_l, M,
                           (const T*)x, (T*)y, (const T*)b, skip);
    }
    ctx->launches++;
  }
  ctx->launches--;  // counted once by the caller
}

template <class T, int N, int S, bool CANON>
void launch_cells_c(lfx_ctx* ctx, const lfx_op* op, const void* x, void* y, const void* b,
                    const int* skip) {
  // the residual form is its own instantiation: the plain apply keeps its
  // register count (and occupancy)
  if (op->smat) {
    if (b)
      launch_cells_t<T, N, true, S, true, CANON>(ctx, op, x, y, b, skip);
    else
      launch_cells_t<T, N, true, S, false, CANON>(ctx, op, x, y, b, skip);
  } else {
    if (b)
      launch_cells_t<T, N, false, S, true, CANON>(ctx, op, x, y, b, skip);
    else
      launch_cells_t<T, N, false, S, false, CANON>(ctx, op, x, y, b, skip);
  }
}

// operators whose cells carry their space's reference pair structure take
// the instantiation with the pair tests at compile time (same arithmetic,
// same bits)
template <class T, int N, int S>
void launch_cells_s(lfx_ctx* ctx, const lfx_op* op, const void* x, void* y, const void* b,
                    const int* skip) {
  if constexpr (N == 6 || N == 8) {
    if (layout_canon(op->lay, N)) {
      launch_cells_c<T, N, S, true>(ctx, op, x, y, b, skip);
      return;
    }
  }
  launch_cells_c<T, N, S, false>(ctx, op, x, y, b, skip);
}

template <class T, int N>
void launch_cells(lfx_ctx* ctx, const lfx_op* op, int stages, const void* x, void* y,
                  const void* b, const int* skip) {
  switch (stages) {
    case 2: launch_cells_s<T, N, 2>(ctx, op, x, y, b, skip); return;
    case 3: launch_cells_s<T, N, 3>(ctx, op, x, y, b, skip); return;
    default: launch_cells_s<T, N, 0>(ctx, op, x, y, b, skip); return;
  }
}

// a staged cell scatter with `stages` stages fits the shared memory
bool cells_stages_ok(const lfx_op* op, int stages) {
  if (stages == 0) return true;
  if (stages != 2 && stages != 3) return false;
  if (op->lay->nlayers + 1 > 32) return false;  // the staged walk keeps one warp per column
  return (size_t)kCellWarps * stages * cells_stage_bytes(op) <= kCellSmemMax;
}

// ---- the persistent ring cell scatter (kernel 6): `stages` ring stages per
// warp (4 or 6; x and y copied stages / 2 cells ahead), `warps` per block
// (4 or 8)
constexpr size_t kRingSmemMax = 220 * 1024;

size_t ring_stage_bytes(const lfx_op* op) {
  const size_t esz = op->precision == LFX_R64 ? 8 : 4;
  const lfx_lma_layout* L = op->lay;
  const size_t m = op->smat ? (size_t)op->sblk * esz : (size_t)L->ndf_to * op->blk * esz;
  return m + (size_t)L->cs_ints * 4 + 2 * (size_t)L->ndf_to * 32 * esz;
}
size_t ring_smem_bytes(const lfx_op* op, int stages, int warps) {
  return (size_t)warps * stages * (ring_stage_bytes(op) + 8);
}
bool ring_ok(const lfx_op* op, int stages, int warps) {
  const lfx_lma_layout* L = op->lay;
  if (!cells_ok(op) || (L->ndf_to != 6 && L->ndf_to != 8)) return false;
  if (L->nlayers + 1 > 32) return false;  // one warp per cell column
  if (L->colour_start.size() < 2 || L->colour_start.size() > (size_t)kRingMaxCol + 1) return false;
  if (stages != 4 && stages != 6) return false;
  if (warps != 4 && warps != 8) return false;
  return ring_smem_bytes(op, stages, warps) <= kRingSmemMax;
}

template <class T, int N, bool SYM, int D, bool RESID, bool CANON>
void launch_ring_t(lfx_ctx* ctx, const lfx_op* op, int stages, int warps, const void* x, void* y,
                   const void* b, const int* skip) {
  const lfx_lma_layout* L = op->lay;
  CellRingArgs R{};
  R.nl = L->nlayers;
  R.blk = op->blk;
  R.cstride = SYM ? op->sblk : N * op->blk;
  R.dints = L->cs_ints;
  R.cells = L->cs_cells;
  R.desc = L->cs_desc;
  R.ncol = (int)L->colour_start.size() - 1;
  R.stages = stages;
  R.bar = reinterpret_cast<unsigned*>(ctx->d_err + 2);
  R.err = ctx->d_err;
  R.limit_ns = 2000000000ull;
  for (int k = 0; k <= R.ncol; ++k) R.cs[k] = L->colour_start[k];
  const size_t smem = ring_smem_bytes(op, stages, warps);
  auto kern = lma_cells_ring<T, N, SYM, D, RESID, CANON>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRingSmemMax);
    attr = true;
  }
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * warps, smem);
  if (per_sm < 1) per_sm = 1;
  // every block resident (cooperative launch): the colours meet at grid barriers
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(ctx->num_sms * per_sm));
  cfg.blockDim = dim3((unsigned)(32 * warps));
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, R, (const T*)(SYM ? op->smat : op->mat), (const T*)x, (T*)y,
                     (const T*)b, skip);
}

template <class T, int N, bool SYM, int D>
void launch_ring_d(lfx_ctx* ctx, const lfx_op* op, int stages, int warps, const void* x, void* y,
                   const void* b, const int* skip) {
  const bool canon = layout_canon(op->lay, N);
  if (b) {
    if (canon) launch_ring_t<T, N, SYM, D, true, true>(ctx, op, stages, warps, x, y, b, skip);
    else launch_ring_t<T, N, SYM, D, true, false>(ctx, op, stages, warps, x, y, b, skip);
  } else {
    if (canon) launch_ring_t<T, N, SYM, D, false, true>(ctx, op, stages, warps, x, y, b, skip);
    else launch_ring_t<T, N, SYM, D, false, false>(ctx, op, stages, warps, x, y, b, skip);
  }
}

template <class T, int N>
void launch_ring(lfx_ctx* ctx, const lfx_op* op, int stages, int warps, const void* x, void* y,
                 const void* b, const int* skip) {
  if (op->smat) {
    if (stages == 6) launch_ring_d<T, N, true, 3>(ctx, op, stages, warps, x, y, b, skip);
    else launch_ring_d<T, N, true, 2>(ctx, op, stages, warps, x, y, b, skip);
  } else {
    if (stages == 6) launch_ring_d<T, N, false, 3>(ctx, op, stages, warps, x, y, b, skip);
    else launch_ring_d<T, N, false, 2>(ctx, op, stages, warps, x, y, b, skip);
  }
}

// the first ring shape that fits: 6 stages of 8 warps, else fewer
TmaShape ring_default(const lfx_op* op) {
  TmaShape ts;
  for (int w : {8, 4})
    for (int st : {6, 4})
      if (!ts.warps && ring_ok(op, st, w)) {
        ts.warps = w;
        ts.stages = st;
      }
  return ts;
}

// kernel: 0 bulk-copy pipelined (shape ts), 1 register gather, 2 generic,
// 3 register gather with prefetched descriptors, 4 copy-staged pipeline (shape ts),
// 5 cell scatter, 6 the cell scatter as one persistent launch (shape ts)
template <class T>
void launch_apply_t(lfx_ctx* ctx, const lfx_op* op, int kernel, const TmaShape& ts,
                    const void* x, void* y, const void* b, const int* skip) {
  const lfx_lma_layout* L = op->lay;
  const LayoutArgs A = args_of(L, op->blk);
  if (kernel == 6) {
    if (L->ndf_to == 6)
      launch_ring<T, 6>(ctx, op, ts.stages, ts.warps, x, y, b, skip);
    else
      launch_ring<T, 8>(ctx, op, ts.stages, ts.warps, x, y, b, skip);
    return;
  }
  if (kernel == 5) {
    switch (L->ndf_to) {
      case 1: launch_cells<T, 1>(ctx, op, ts.stages, x, y, b, skip); return;
      case 6: launch_cells<T, 6>(ctx, op, ts.stages, x, y, b, skip); return;
      default: launch_cells<T, 8>(ctx, op, ts.stages, x, y, b, skip); return;
    }
  }
  if (kernel == 4) {
    launch_pipe<T>(ctx, op, A, ts, x, y, b, skip);
    return;
  }
  if (kernel == 0) {
    switch (L->ndf_from) {
      case 1: launch_tma<T, 1>(ctx, op, A, ts, x, y, b, skip); return;
      case 6: launch_tma<T, 6>(ctx, op, A, ts, x, y, b, skip); return;
      default: launch_tma<T, 8>(ctx, op, A, ts, x, y, b, skip); return;
    }
  }
  const int grid = gather_grid(ctx, L->nent);
  if (kernel == 1) {
    switch (L->ndf_from) {
      case 1: lma_gather2<T, 1><<<grid, 256, 0, ctx->stream>>>(A, (const T*)op->mat, (const T*)x, (T*)y, (const T*)b, skip); return;
      case 6: lma_gather2<T, 6><<<grid, 256, 0, ctx->stream>>>(A, (const T*)op->mat, (const T*)x, (T*)y, (const T*)b, skip); return;
      default: lma_gather2<T, 8><<<grid, 256, 0, ctx->stream>>>(A, (const T*)op->mat, (const T*)x, (T*)y, (const T*)b, skip); return;
    }
  }
  if (kernel == 3) {
    switch (L->ndf_from) {
      case 1: launch_fetch<T, 1>(ctx, op, A, ts.stages, x, y, b, skip); return;
      case 6: launch_fetch<T, 6>(ctx, op, A, ts.stages, x, y, b, skip); return;
      default: launch_fetch<T, 8>(ctx, op, A, ts.stages, x, y, b, skip); return;
    }
  }
  lma_gather<T><<<grid, 256, 0, ctx->stream>>>(A, (const T*)op->mat, (const T*)x, (T*)y,
                                               (const T*)b, skip);
}

// the register gather needs at most two records per group and ndf_from 1, 6 or 8
bool gather2_ok(const lfx_op* op) {
  const lfx_lma_layout* L = op->lay;
  return L->max_nrec <= 2 && (L->ndf_from == 1 || L->ndf_from == 6 || L->ndf_from == 8);
}

void launch_apply(lfx_ctx* ctx, const lfx_op* op, int kernel, const TmaShape& ts, const void* x,
                  void* y, const void* b, const int* skip) {
  if (op->precision == LFX_R64)
    launch_apply_t<double>(ctx, op, kernel, ts, x, y, b, skip);
  else
    launch_apply_t<float>(ctx, op, kernel, ts, x, y, b, skip);
}

// the configuration an apply of this operator uses
void pick_apply(const lfx_ctx* ctx, const lfx_op* op, int* kernel, TmaShape* ts) {
  *ts = TmaShape{};
  if (ctx->lma_kernel == 0 && tma_ok(op)) {
    *kernel = 0;
    *ts = tma_default(op);
    if (ts->warps) return;
  }
  if (ctx->lma_kernel == 3 && fetch_ok(op)) {
    *kernel = 3;
    return;
  }
  if (ctx->lma_kernel == 5 && cells_ok(op)) {
    *kernel = 5;
    return;
  }
  if (ctx->lma_kernel == 6) {
    *ts = ring_default(op);
    if (ts->warps) {
      *kernel = 6;
      return;
    }
  }
  if ((ctx->lma_kernel == 1 || ctx->lma_kernel == 3) && gather2_ok(op)) {
    *kernel = 1;
    return;
  }
  if (ctx->lma_kernel == 4 && pipe_ok(op)) {
    *kernel = 4;
    *ts = pipe_default(op);
    if (ts->warps) return;
  }
  if (ctx->lma_kernel < 0 && op->tune_kernel >= 0) {
    *kernel = op->tune_kernel;
    if (*kernel == 0) *ts = tma_shape(op, op->tune_stages, op->tune_warps);
    if (*kernel == 4) *ts = pipe_shape(op, op->tune_stages, op->tune_warps);
    if (*kernel == 3 || *kernel == 5) ts->stages = op->tune_stages;
    if (*kernel == 6) {
      ts->stages = op->tune_stages;
      ts->warps = op->tune_warps;
    }
    if ((*kernel != 0 && *kernel != 4) || ts->warps) return;
  }
  // untuned: the prefetching gather where it fits (fastest measured on W2
  // and W3 columns), else the register gather, else the generic one
  *kernel = fetch_ok(op) ? 3 : (gather2_ok(op) ? 1 : 2);
}

}  // namespace

namespace lfx {

// y = A x (b == nullptr) or y = b - A x; x, y, b raw device arrays of the op's
// precision; skip: optional device flag that turns the launch into a no-op.
int op_apply_impl(lfx_op* op, const void* x, void* y, const void* b, const int* skip) {
  lfx_ctx* ctx = op->ctx;
  const lfx_lma_layout* L = op->lay;
  const size_t esz = op->precision == LFX_R64 ? 8 : 4;
  if (!L->full_cover) {
    if (b)
      LFX_CK(ctx, cudaMemcpyAsync(y, b, L->undf_to * esz, cudaMemcpyDeviceToDevice, ctx->stream));
    else
      LFX_CK(ctx, cudaMemsetAsync(y, 0, L->undf_to * esz, ctx->stream));
  }
  int kernel = 2;
  TmaShape ts;
  pick_apply(ctx, op, &kernel, &ts);
  timing_begin(ctx, op->precision);
  ctx->launches++;
  launch_apply(ctx, op, kernel, ts, x, y, b, skip);
  timing_end(ctx);
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

size_t op_level_major_bytes(const lfx_op* op) {
  if (op->precision != LFX_R32 || !op->smat) return 0;
  const int np = op->lay->ndf_to * (op->lay->ndf_to + 1) / 2;
  return (size_t)op->lay->ncell_2d * op->lay->nlayers * ((np + 3) / 4) * 16;
}

int op_level_major(lfx_op* op) {
  lfx_ctx* ctx = op->ctx;
  if (op->precision != LFX_R32 || !op->smat)
    return fail(ctx, LFX_NOT_SUPPORTED, "level-major copy: FP32 operators with a packed copy only");
  if (op->lmat) return LFX_OK;
  const lfx_lma_layout* L = op->lay;
  const int np = L->ndf_to * (L->ndf_to + 1) / 2;
  const size_t bytes = op_level_major_bytes(op);
  int rc = dmalloc(ctx, &op->lmat, bytes);
  if (rc) return rc;
  op->lmat_bytes = bytes;
  op->lnpv = (np + 3) / 4;
  const int64_t total = (int64_t)(bytes / 4);
  const int grid = (int)std::min<int64_t>((total + 255) / 256, (int64_t)ctx->num_sms * 16);
  relayout_level_major<<<grid, 256, 0, ctx->stream>>>((const float*)op->smat, (float*)op->lmat,
                                                      L->ncell_2d, L->nlayers, np, op->lnpv,
                                                      op->sblk);
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

}  // namespace lfx

// out = fma(a, y, x) elementwise: operator_x_plus_ay on the stored copies
// (the padding between blocks is zero in both, and stays zero)
template <class T>
__global__ void lma_x_plus_ay(int64_t n, const T* __restrict__ x, T a, const T* __restrict__ y,
                              T* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = fmaT(a, y[i], x[i]);
}

int x_plus_ay_copy(lfx_ctx* ctx, int32_t precision, const void* x, double a, const void* y,
                   void* out, size_t bytes) {
  const size_t esz = precision == LFX_R64 ? 8 : 4;
  const int64_t n = (int64_t)(bytes / esz);
  const int grid = ctx->num_sms * 8;
  if (precision == LFX_R64)
    lma_x_plus_ay<double><<<grid, 256, 0, ctx->stream>>>(n, (const double*)x, a, (const double*)y,
                                                          (double*)out);
  else
    lma_x_plus_ay<float><<<grid, 256, 0, ctx->stream>>>(n, (const float*)x, (float)a,
                                                         (const float*)y, (float*)out);
  ctx->launches++;
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

extern "C" {

int lfx_lma_create(lfx_ctx* ctx, int32_t ncell_2d, int32_t nlayers, int32_t ndf_to,
                   int32_t ndf_from, const int32_t* map_to, const int32_t* map_from,
                   int64_t undf_to, int64_t undf_from, const double* local_stencil,
                   int32_t ncolours, const int32_t* ncells_per_colour,
                   const int32_t* cells_in_colour, int32_t max_cells_per_colour,
                   int32_t precision, lfx_op** out) {
  if (!ctx || !out || !map_to || !map_from || !local_stencil || !ncells_per_colour ||
      !cells_in_colour)
    return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  if (ncell_2d < 1 || nlayers < 1 || ndf_to < 1 || ndf_from < 1 || ndf_to > 63 || ndf_from > 63)
    return fail(ctx, LFX_INVALID_ARGUMENT, "bad operator dimensions");
  if (undf_to >= (1LL << 31) || undf_from >= (1LL << 31))
    return fail(ctx, LFX_NOT_SUPPORTED, "more than 2^31 dofs per field");
  if (precision != LFX_R64 && precision != LFX_R32)
    return fail(ctx, LFX_INVALID_ARGUMENT, "precision must be 64 or 32");
  // colour rank of every cell: the position of its kernel call in the
  // reference's colour loop
  std::vector<int32_t> rank(ncell_2d, -1), colour(ncell_2d, -1);
  int32_t pos = 0;
  for (int32_t col = 0; col < ncolours; ++col) {
    if (ncells_per_colour[col] < 0 || ncells_per_colour[col] > max_cells_per_colour)
      return fail(ctx, LFX_INVALID_ARGUMENT, "bad ncells_per_colour");
    for (int32_t i = 0; i < ncells_per_colour[col]; ++i) {
      int32_t cell = cells_in_colour[col + (int64_t)ncolours * i];
      if (cell < 1 || cell > ncell_2d || rank[cell - 1] >= 0)
        return fail(ctx, LFX_INVALID_ARGUMENT, "colouring does not list every cell exactly once");
      rank[cell - 1] = pos++;
      colour[cell - 1] = col;
    }
  }
  if (pos != ncell_2d)
    return fail(ctx, LFX_INVALID_ARGUMENT, "colouring does not list every cell exactly once");
  // 0-based maps
  std::vector<int32_t> mf((size_t)ncell_2d * ndf_from), mt((size_t)ncell_2d * ndf_to);
  for (size_t i = 0; i < mf.size(); ++i) {
    mf[i] = map_from[i] - 1;
    if (mf[i] < 0 || (int64_t)mf[i] + nlayers > undf_from)
      return fail(ctx, LFX_INVALID_ARGUMENT, "from-space dofmap entry out of range");
  }
  for (size_t i = 0; i < mt.size(); ++i) mt[i] = map_to[i] - 1;
  lfx_lma_layout* L = new lfx_lma_layout();
  L->ncell_2d = ncell_2d;
  L->nlayers = nlayers;
  L->ndf_to = ndf_to;
  L->ndf_from = ndf_from;
  L->undf_to = undf_to;
  L->undf_from = undf_from;
  // one dofmap on both sides: the cell-scatter plan can be built
  const bool one_map = ndf_to == ndf_from && undf_to == undf_from &&
                       std::equal(map_to, map_to + (size_t)ncell_2d * ndf_to, map_from);
  int rc = build_layout(ctx, L, ncell_2d, nlayers, ndf_to, map_to, undf_to, rank, mf.data(),
                        ndf_from, one_map ? &colour : nullptr);
  if (!rc) rc = dmalloc(ctx, (void**)&L->map_from, mf.size() * 4);
  if (!rc) rc = dmalloc(ctx, (void**)&L->map_to, mt.size() * 4);
  if (!rc) cudaMemcpy(L->map_from, mf.data(), mf.size() * 4, cudaMemcpyHostToDevice);
  if (!rc) cudaMemcpy(L->map_to, mt.data(), mt.size() * 4, cudaMemcpyHostToDevice);
  if (rc) {
    free_layout(ctx, L);
    return rc;
  }
  lfx_op* op = new lfx_op();
  op->ctx = ctx;
  op->lay = L;
  op->precision = precision;
  rc = upload_matrix(ctx, op, local_stencil);
  if (rc) {
    lfx_op_destroy(op);
    return rc;
  }
  L->rank = std::move(rank);
  *out = op;
  return LFX_OK;
}

int lfx_lma_create_like(const lfx_op* src, const double* local_stencil, int32_t precision,
                        lfx_op** out) {
  if (!src || !out || !local_stencil) return LFX_INVALID_ARGUMENT;
  if (precision != LFX_R64 && precision != LFX_R32) return LFX_INVALID_ARGUMENT;
  lfx_op* op = new lfx_op();
  op->ctx = src->ctx;
  op->lay = src->lay;
  op->lay->refcount++;
  op->precision = precision;
  int rc = upload_matrix(src->ctx, op, local_stencil);
  if (rc) {
    lfx_op_destroy(op);
    return rc;
  }
  *out = op;
  return LFX_OK;
}

int lfx_lma_sum(const lfx_op* x, double a, const lfx_op* y, lfx_op** out) {
  if (!x || !y || !out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  lfx_ctx* ctx = x->ctx;
  if (y->ctx != ctx || y->lay != x->lay || y->precision != x->precision)
    return fail(ctx, LFX_TYPE_MISMATCH,
                "lfx_lma_sum: operators must share one layout (lfx_lma_create_like) and precision");
  lfx_op* op = new lfx_op();
  op->ctx = ctx;
  op->lay = x->lay;
  op->lay->refcount++;
  op->precision = x->precision;
  op->blk = x->blk;
  int rc = dmalloc(ctx, &op->mat, x->mat_bytes);
  if (!rc) {
    op->mat_bytes = x->mat_bytes;
    rc = x_plus_ay_copy(ctx, x->precision, x->mat, a, y->mat, op->mat, x->mat_bytes);
  }
  // the packed upper triangles, when both operators have them (the sum of
  // two bitwise symmetric operators is bitwise symmetric)
  if (!rc && x->smat && y->smat && x->sblk == y->sblk) {
    rc = dmalloc(ctx, &op->smat, x->smat_bytes);
    if (!rc) {
      op->smat_bytes = x->smat_bytes;
      op->sblk = x->sblk;
      rc = x_plus_ay_copy(ctx, x->precision, x->smat, a, y->smat, op->smat, x->smat_bytes);
    }
  }
  if (rc) {
    lfx_op_destroy(op);
    return rc;
  }
  *out = op;
  return LFX_OK;
}

int lfx_op_destroy(lfx_op* op) {
  if (!op) return LFX_OK;
  lfx_ctx* ctx = op->ctx;
  dfree(ctx, op->mat, op->mat_bytes);
  dfree(ctx, op->smat, op->smat_bytes);
  dfree(ctx, op->lmat, op->lmat_bytes);
  if (op->lay && --op->lay->refcount == 0) free_layout(ctx, op->lay);
  delete op;
  return LFX_OK;
}

int lfx_op_apply(lfx_op* op, const lfx_vec* x, lfx_vec* y) {
  if (!op || !x || !y) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = op->ctx;
  if (x->precision != op->precision || y->precision != op->precision)
    return fail(ctx, LFX_TYPE_MISMATCH, "operator and vector precision differ");
  if (x->undf[0] != op->lay->undf_from || y->undf[0] != op->lay->undf_to)
    return fail(ctx, LFX_TYPE_MISMATCH, "vector length does not match the operator's space");
  if (x->data[0] == y->data[0]) return fail(ctx, LFX_INVALID_ARGUMENT, "x and y must differ");
  return op_apply_impl(op, x->data[0], y->data[0], nullptr, nullptr);
}

// Times `reps` applies of one launch configuration on scratch vectors.
int lfx_op_time_apply(lfx_op* op, int32_t kernel, int32_t stages, int32_t warps, int32_t reps,
                      float* us) {
  if (!op || !us || reps < 1 || kernel < 0 || kernel > 6) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = op->ctx;
  const lfx_lma_layout* L = op->lay;
  TmaShape ts;
  if (kernel == 0 || kernel == 4) {
    ts = kernel == 0 ? tma_shape(op, stages, warps) : pipe_shape(op, stages, warps);
    if (!ts.warps) return fail(ctx, LFX_NOT_SUPPORTED, "configuration does not fit this operator");
  }
  if (kernel == 1 && !gather2_ok(op))
    return fail(ctx, LFX_NOT_SUPPORTED, "register gather does not fit this operator");
  if (kernel == 3) {
    if (!fetch_ok(op) || stages < 0 || stages > 1)
      return fail(ctx, LFX_NOT_SUPPORTED, "prefetching gather does not fit this operator");
    ts.stages = stages;
  }
  if (kernel == 5) {
    if (!cells_ok(op) || !cells_stages_ok(op, stages))
      return fail(ctx, LFX_NOT_SUPPORTED, "cell scatter does not fit this operator");
    ts.stages = stages;
  }
  if (kernel == 6) {
    if (!ring_ok(op, stages, warps))
      return fail(ctx, LFX_NOT_SUPPORTED, "persistent cell scatter does not fit this operator");
    ts.stages = stages;
    ts.warps = warps;
  }
  const size_t esz = op->precision == LFX_R64 ? 8 : 4;
  // consecutive applies take different x and y (enough pairs to hold twice
  // the L2), so each apply reads x from and writes y to HBM as in a solve
  // whose vectors change, rather than finding them in L2
  const size_t pair = (L->undf_from + L->undf_to) * esz;
  const size_t l2 = (size_t)std::max(ctx->l2_bytes, 1);
  const int npair = (int)std::min<size_t>(8, std::max<size_t>(2, (2 * l2 + pair - 1) / pair));
  void* x[8] = {};
  void* y[8] = {};
  int rc = LFX_OK;
  for (int i = 0; i < npair && !rc; ++i) {
    rc = dmalloc(ctx, &x[i], L->undf_from * esz);
    if (!rc) rc = dmalloc(ctx, &y[i], L->undf_to * esz);
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (!rc) {
    for (int i = 0; i < npair; ++i) cudaMemsetAsync(x[i], 0, L->undf_from * esz, ctx->stream);
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    launch_apply(ctx, op, kernel, ts, x[0], y[0], nullptr, nullptr);  // warm
    cudaEventRecord(e0, ctx->stream);
    for (int r = 0; r < reps; ++r)
      launch_apply(ctx, op, kernel, ts, x[(r + 1) % npair], y[(r + 1) % npair], nullptr, nullptr);
    cudaEventRecord(e1, ctx->stream);
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
      rc = fail(ctx, LFX_CUDA_ERROR, "apply timing failed");
    float ms = 0.f;
    if (!rc) cudaEventElapsedTime(&ms, e0, e1);
    *us = 1e3f * ms / reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  for (int i = 0; i < npair; ++i) {
    if (x[i]) dfree(ctx, x[i], L->undf_from * esz);
    if (y[i]) dfree(ctx, y[i], L->undf_to * esz);
  }
  if (!rc) rc = lfx_ctx_check_device_error(ctx);
  return rc;
}

// Storage of the local matrices: bytes of the full [cell][df][df2][k] copy
// and of the packed upper triangle (0 when the operator is not symmetric or
// not on one dofmap); the cell scatter reads the packed copy when it exists.
int lfx_op_storage(const lfx_op* op, int64_t* full_bytes, int64_t* packed_bytes) {
  if (!op) return LFX_INVALID_ARGUMENT;
  if (full_bytes) *full_bytes = (int64_t)op->mat_bytes;
  if (packed_bytes) *packed_bytes = op->smat ? (int64_t)op->smat_bytes : 0;
  return LFX_OK;
}

// Keeps one launch configuration for later applies of this operator (as the
// autotuner would), after checking that it fits.
int lfx_op_set_apply(lfx_op* op, int32_t kernel, int32_t stages, int32_t warps) {
  if (!op) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = op->ctx;
  bool ok = false;
  switch (kernel) {
    case 0: ok = tma_shape(op, stages, warps).warps > 0; break;
    case 1: ok = gather2_ok(op); break;
    case 2: ok = true; break;
    case 3: ok = fetch_ok(op) && (stages == 0 || stages == 1); break;
    case 4: ok = pipe_shape(op, stages, warps).warps > 0; break;
    case 5: ok = cells_ok(op) && cells_stages_ok(op, stages); break;
    case 6: ok = ring_ok(op, stages, warps); break;
    default: return fail(ctx, LFX_INVALID_ARGUMENT, "no such apply kernel");
  }
  if (!ok) return fail(ctx, LFX_NOT_SUPPORTED, "configuration does not fit this operator");
  op->tune_kernel = kernel;
  op->tune_stages = stages;
  op->tune_warps = warps;
  return LFX_OK;
}

// Picks the fastest apply configuration for this operator by timing the
// candidates (register gather, the prefetching gather at two register caps, the
// cell scatter per colour and as one persistent launch, bulk-copy
// pipeline with 2..8 stages and 1..8 warps per block that fit the shared
// memory) and keeps it for later applies.
int lfx_op_autotune(lfx_op* op, int32_t reps, int32_t* kernel, int32_t* stages, int32_t* warps,
                    float* us) {
  if (!op) return LFX_INVALID_ARGUMENT;
  int bk = -1, bs = 0, bw = 0;
  float best = 3.4e38f;
  auto consider = [&](int k, int s, int w) -> int {
    float t = 0.f;
    int rc = lfx_op_time_apply(op, k, s, w, reps, &t);
    if (rc == LFX_NOT_SUPPORTED) return LFX_OK;
    if (rc) return rc;
    if (t < best) {
      best = t;
      bk = k;
      bs = s;
      bw = w;
    }
    return LFX_OK;
  };
  int rc = LFX_OK;
  if (gather2_ok(op)) {
    rc = consider(1, 0, 0);
    if (!rc && fetch_ok(op)) rc = consider(3, 0, 0);
    if (!rc && fetch_ok(op)) rc = consider(3, 1, 0);
    for (int st : {0, 2, 3})
      if (!rc && cells_ok(op) && cells_stages_ok(op, st)) rc = consider(5, st, 0);
    for (int st : {4, 6})
      for (int w : {4, 8})
        if (!rc && ring_ok(op, st, w)) rc = consider(6, st, w);
  } else {
    rc = consider(2, 0, 0);
  }
  if (!rc && tma_ok(op))
    for (int s : {2, 3, 4, 6, 8})
      for (int w : {1, 2, 4, 8})
        if (!rc && tma_shape(op, s, w).warps) rc = consider(0, s, w);
  if (!rc && pipe_ok(op))
    for (int s : {2, 3, 4, 6})
      for (int w : {2, 4, 8})
        if (!rc && pipe_shape(op, s, w).warps) rc = consider(4, s, w);
  if (rc) return rc;
  op->tune_kernel = bk;
  op->tune_stages = bs;
  op->tune_warps = bw;
  op->tune_us = best;
  if (kernel) *kernel = bk;
  if (stages) *stages = bs;
  if (warps) *warps = bw;
  if (us) *us = best;
  return LFX_OK;
}

int lfx_lma_diagonal(lfx_op* op, lfx_vec* diag) {
  if (!op || !diag) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = op->ctx;
  const lfx_lma_layout* L = op->lay;
  if (L->ndf_to != L->ndf_from || L->undf_to != L->undf_from)
    return fail(ctx, LFX_INVALID_ARGUMENT, "diagonal needs a square operator");
  if (diag->precision != op->precision || diag->undf[0] != L->undf_to)
    return fail(ctx, LFX_TYPE_MISMATCH, "diagonal vector does not match the operator");
  if (!L->full_cover)
    LFX_CK(ctx, cudaMemsetAsync(diag->data[0], 0, L->undf_to * diag->elem(), ctx->stream));
  const LayoutArgs A = args_of(L, op->blk);
  ctx->launches++;
  if (op->precision == LFX_R64)
    lma_diag<double><<<gather_grid(ctx, L->nent), 256, 0, ctx->stream>>>(
        A, L->max_off, (const double*)op->mat, (double*)diag->data[0]);
  else
    lma_diag<float><<<gather_grid(ctx, L->nent), 256, 0, ctx->stream>>>(
        A, L->max_off, (const float*)op->mat, (float*)diag->data[0]);
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

int lfx_op_apply_transpose(lfx_op* op, const lfx_vec* x, lfx_vec* y) {
  if (!op || !x || !y) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = op->ctx;
  lfx_lma_layout* L = op->lay;
  if (x->precision != op->precision || y->precision != op->precision)
    return fail(ctx, LFX_TYPE_MISMATCH, "operator and vector precision differ");
  if (x->undf[0] != L->undf_to || y->undf[0] != L->undf_from)
    return fail(ctx, LFX_TYPE_MISMATCH, "vector length does not match the operator's space");
  if (!L->tlay) {
    // from-space layout: entities of map_from, records ordered by colour
    std::vector<int32_t> mf((size_t)L->ncell_2d * L->ndf_from);
    LFX_CK(ctx, cudaMemcpy(mf.data(), L->map_from, mf.size() * 4, cudaMemcpyDeviceToHost));
    for (auto& v : mf) v += 1;
    lfx_lma_layout* T = new lfx_lma_layout();
    T->ncell_2d = L->ncell_2d;
    T->nlayers = L->nlayers;
    T->ndf_to = L->ndf_from;  // output side of the transpose
    T->ndf_from = L->ndf_to;
    T->undf_to = L->undf_from;
    T->undf_from = L->undf_to;
    int rc = build_layout(ctx, T, L->ncell_2d, L->nlayers, L->ndf_from, mf.data(), L->undf_from,
                          L->rank, nullptr, 0, nullptr);
    if (rc) {
      free_layout(ctx, T);
      return rc;
    }
    L->tlay = T;
  }
  lfx_lma_layout* T = L->tlay;
  if (!T->full_cover)
    LFX_CK(ctx, cudaMemsetAsync(y->data[0], 0, T->undf_to * y->elem(), ctx->stream));
  LayoutArgs A = args_of(T, op->blk);
  ctx->launches++;
  if (op->precision == LFX_R64)
    lma_gather_t<double><<<gather_grid(ctx, T->nent), 256, 0, ctx->stream>>>(
        A, T->max_off, op->blk, (const double*)op->mat, (const double*)x->data[0], L->map_to,
        (double*)y->data[0]);
  else
    lma_gather_t<float><<<gather_grid(ctx, T->nent), 256, 0, ctx->stream>>>(
        A, T->max_off, op->blk, (const float*)op->mat, (const float*)x->data[0], L->map_to,
        (float*)y->data[0]);
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

}  // extern "C"
