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
// Device layout of the local matrices: [cell][df][df2][k] (k fastest), so a
// warp that owns one dof column reads each (cell, df, df2) run of nlayers
// values as one contiguous segment, and each (cell, df) block of
// ndf2*nlayers values exactly once.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "lfx_internal.cuh"

using namespace lfx;

namespace {

struct LayoutArgs {
  int32_t nent, nlayers, ndf1, ndf2;
  const int32_t* ent_base;
  const int32_t* ent_h;
  const int32_t* ent_grp;
  const int32_t* grp_cell;
  const uint32_t* grp_rec;
  const int32_t* map_from;
};

LayoutArgs args_of(const lfx_lma_layout* L) {
  return LayoutArgs{L->nent,     L->nlayers,  L->ndf_to,   L->ndf_from, L->ent_base,
                    L->ent_h,    L->ent_grp,  L->grp_cell, L->grp_rec,  L->map_from};
}

// packed group record: bits 0-1 nrec (1..3); record r at bit 2+9r: df (6 bits), off (3 bits)
__host__ __device__ inline int rec_n(uint32_t p) { return p & 3u; }
__host__ __device__ inline int rec_df(uint32_t p, int r) { return (p >> (2 + 9 * r)) & 63u; }
__host__ __device__ inline int rec_off(uint32_t p, int r) { return (p >> (8 + 9 * r)) & 7u; }

template <class T, int NDF2>
__global__ void __launch_bounds__(256) lma_gather(LayoutArgs A, const T* __restrict__ M,
                                                  const T* __restrict__ x, T* __restrict__ y,
                                                  const T* __restrict__ b, const int* skip) {
  if (skip && *((volatile const int*)skip)) return;
  const int ndf2 = NDF2 > 0 ? NDF2 : A.ndf2;
  const int nl = A.nlayers;
  const int lane = threadIdx.x & 31;
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const size_t cell_stride = (size_t)A.ndf1 * ndf2 * nl;
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
        const int k0 = l - rec_off(pk, 0), k1 = l - rec_off(pk, 1), k2 = l - rec_off(pk, 2);
        const bool v0 = k0 >= 0 && k0 < nl;
        const bool v1 = nrec > 1 && k1 >= 0 && k1 < nl;
        const bool v2 = nrec > 2 && k2 >= 0 && k2 < nl;
        const T* M0 = Mc + (size_t)rec_df(pk, 0) * ndf2 * nl + k0;
        const T* M1 = Mc + (size_t)rec_df(pk, 1) * ndf2 * nl + k1;
        const T* M2 = Mc + (size_t)rec_df(pk, 2) * ndf2 * nl + k2;
#pragma unroll
        for (int j = 0; j < (NDF2 > 0 ? NDF2 : 1); ++j) {
          // NDF2 == 0 falls through to the runtime loop below
          if (NDF2 == 0) break;
          const int xb = mf[j];
          if (v0) acc = fmaT(__ldg(M0 + j * nl), __ldg(x + xb + k0), acc);
          if (v1) acc = fmaT(__ldg(M1 + j * nl), __ldg(x + xb + k1), acc);
          if (v2) acc = fmaT(__ldg(M2 + j * nl), __ldg(x + xb + k2), acc);
        }
        if (NDF2 == 0) {
          for (int j = 0; j < ndf2; ++j) {
            const int xb = mf[j];
            if (v0) acc = fmaT(M0[j * nl], x[xb + k0], acc);
            if (v1) acc = fmaT(M1[j * nl], x[xb + k1], acc);
            if (v2) acc = fmaT(M2[j * nl], x[xb + k2], acc);
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

// mm_diagonal (sci_mm_diagonal_kernel_mod.F90:117-122): per cell, layer k
// outer and df inner, diag += M(ik, df, df). In gather form a dof takes its
// records of one cell in increasing k (decreasing off), then increasing df.
template <class T>
__global__ void lma_diag(LayoutArgs A, int max_off, const T* __restrict__ M, T* __restrict__ d) {
  const int nl = A.nlayers, ndf = A.ndf1;
  const int lane = threadIdx.x & 31;
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const size_t cell_stride = (size_t)ndf * ndf * nl;
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
            if (k >= 0 && k < nl) acc = acc + Mc[((size_t)df * ndf + df) * nl + k];
          }
      }
      d[base + l] = acc;
    }
  }
}

// transpose_matrix_vector (transpose_matrix_vector_kernel_mod.F90:128-144):
// per layer k and from-space dof df, s = sum_j M(ik, j, df) x(map_to(j)+k) and
// lhs += s. Gather over the from-space layout; records of one cell in
// increasing k, then increasing df.
template <class T>
__global__ void lma_gather_t(LayoutArgs A, int max_off, const T* __restrict__ M,
                             const T* __restrict__ x, const int32_t* __restrict__ map_to,
                             T* __restrict__ y) {
  // here A.ndf1 is the from-space ndf (output), A.ndf2 the to-space ndf
  const int nl = A.nlayers, ndf_out = A.ndf1, ndf_in = A.ndf2;
  const int lane = threadIdx.x & 31;
  const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const size_t cell_stride = (size_t)ndf_out * ndf_in * nl;
  for (int64_t e = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; e < A.nent; e += nwarp) {
    const int base = A.ent_base[e], h = A.ent_h[e];
    for (int l = lane; l < h; l += 32) {
      T acc = T(0);
      for (int g = A.ent_grp[e]; g < A.ent_grp[e + 1]; ++g) {
        const uint32_t pk = A.grp_rec[g];
        const int c = A.grp_cell[g];
        const T* Mc = M + (size_t)c * cell_stride;  // [c][j(to)][df(from)][k]
        const int* mt = map_to + (size_t)c * ndf_in;
        for (int o = max_off; o >= 0; --o)
          for (int r = 0; r < rec_n(pk); ++r) {
            if (rec_off(pk, r) != o) continue;
            const int k = l - o, df = rec_df(pk, r);
            if (k < 0 || k >= nl) continue;
            T s = T(0);
            for (int j = 0; j < ndf_in; ++j)
              s = fmaT(Mc[((size_t)j * ndf_out + df) * nl + k], x[mt[j] + k], s);
            acc = acc + s;
          }
      }
      y[base + l] = acc;
    }
  }
}

// Fortran (nc3, ndf1, ndf2) FP64 -> [c][df][df2][k] in T
template <class T>
__global__ void relayout(const double* __restrict__ src, T* __restrict__ dst, int64_t ncell,
                         int nl, int ndf1, int ndf2) {
  const int64_t total = ncell * ndf1 * ndf2 * nl;
  const int64_t nc3 = ncell * nl;
  for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d < total;
       d += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = d;
    const int k = (int)(r % nl);
    r /= nl;
    const int df2 = (int)(r % ndf2);
    r /= ndf2;
    const int df = (int)(r % ndf1);
    const int64_t c = r / ndf1;
    dst[d] = (T)src[(c * nl + k) + nc3 * (df + (int64_t)ndf1 * df2)];
  }
}

struct HostRec {
  int32_t start, cell, df;
};

// Builds the gather layout of the space described by `map` (ndf dofs per
// cell, [c][df] 1-based) for a colouring given as rank[c].
int build_layout(lfx_ctx* ctx, lfx_lma_layout* L, int32_t ncell, int32_t nl, int32_t ndf,
                 const int32_t* map, int64_t undf, const std::vector<int32_t>& rank) {
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
  size_t i = 0;
  int64_t covered = 0;
  int max_off = 0, max_h = 0;
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
      grp_cell.push_back(er[q].cell);
      grp_rec.push_back(pk);
      q = r;
    }
    i = j;
  }
  ent_grp.push_back((int32_t)grp_cell.size());
  L->nent = (int32_t)ent_base.size();
  L->ngrp = (int32_t)grp_cell.size();
  L->max_h = max_h;
  L->max_off = max_off;
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
  return rc;
}

void free_layout(lfx_ctx* ctx, lfx_lma_layout* L) {
  if (!L) return;
  dfree(ctx, L->ent_base, (size_t)L->nent * 4);
  dfree(ctx, L->ent_h, (size_t)L->nent * 4);
  dfree(ctx, L->ent_grp, (size_t)(L->nent + 1) * 4);
  dfree(ctx, L->grp_cell, (size_t)L->ngrp * 4);
  dfree(ctx, L->grp_rec, (size_t)L->ngrp * 4);
  dfree(ctx, L->map_from, (size_t)L->ncell_2d * L->ndf_from * 4);
  dfree(ctx, L->map_to, (size_t)L->ncell_2d * L->ndf_to * 4);
  free_layout(ctx, L->tlay);
  delete L;
}

int upload_matrix(lfx_ctx* ctx, lfx_op* op, const double* stencil) {
  const lfx_lma_layout* L = op->lay;
  const int64_t total = (int64_t)L->ncell_2d * L->ndf_to * L->ndf_from * L->nlayers;
  const size_t esz = op->precision == LFX_R64 ? 8 : 4;
  double* raw = nullptr;
  int rc = dmalloc(ctx, (void**)&raw, (size_t)total * 8);
  if (rc) return rc;
  rc = dmalloc(ctx, &op->mat, (size_t)total * esz);
  if (rc) {
    dfree(ctx, raw, (size_t)total * 8);
    return rc;
  }
  op->mat_bytes = (size_t)total * esz;
  LFX_CK(ctx, cudaMemcpyAsync(raw, stencil, (size_t)total * 8, cudaMemcpyHostToDevice, ctx->stream));
  const int grid = ctx->num_sms * 16;
  if (op->precision == LFX_R64)
    relayout<double><<<grid, 256, 0, ctx->stream>>>(raw, (double*)op->mat, L->ncell_2d, L->nlayers,
                                                     L->ndf_to, L->ndf_from);
  else
    relayout<float><<<grid, 256, 0, ctx->stream>>>(raw, (float*)op->mat, L->ncell_2d, L->nlayers,
                                                    L->ndf_to, L->ndf_from);
  LFX_CK(ctx, cudaGetLastError());
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, raw, (size_t)total * 8);
  return LFX_OK;
}

int gather_grid(const lfx_ctx* ctx, int32_t nent) {
  int64_t g = ((int64_t)nent + 7) / 8;
  int64_t cap = (int64_t)ctx->num_sms * 16;
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
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
  const LayoutArgs A = args_of(L);
  const int grid = gather_grid(ctx, L->nent);
  timing_begin(ctx, op->precision);
  ctx->launches++;
#define LAUNCH(T, N)                                                                   \
  lma_gather<T, N><<<grid, 256, 0, ctx->stream>>>(A, (const T*)op->mat, (const T*)x, (T*)y, \
                                                  (const T*)b, skip)
  if (op->precision == LFX_R64) {
    switch (L->ndf_from) {
      case 1: LAUNCH(double, 1); break;
      case 6: LAUNCH(double, 6); break;
      case 8: LAUNCH(double, 8); break;
      default: LAUNCH(double, 0); break;
    }
  } else {
    switch (L->ndf_from) {
      case 1: LAUNCH(float, 1); break;
      case 6: LAUNCH(float, 6); break;
      case 8: LAUNCH(float, 8); break;
      default: LAUNCH(float, 0); break;
    }
  }
#undef LAUNCH
  timing_end(ctx);
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

}  // namespace lfx

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
  std::vector<int32_t> rank(ncell_2d, -1);
  int32_t pos = 0;
  for (int32_t col = 0; col < ncolours; ++col) {
    if (ncells_per_colour[col] < 0 || ncells_per_colour[col] > max_cells_per_colour)
      return fail(ctx, LFX_INVALID_ARGUMENT, "bad ncells_per_colour");
    for (int32_t i = 0; i < ncells_per_colour[col]; ++i) {
      int32_t cell = cells_in_colour[col + (int64_t)ncolours * i];
      if (cell < 1 || cell > ncell_2d || rank[cell - 1] >= 0)
        return fail(ctx, LFX_INVALID_ARGUMENT, "colouring does not list every cell exactly once");
      rank[cell - 1] = pos++;
    }
  }
  if (pos != ncell_2d)
    return fail(ctx, LFX_INVALID_ARGUMENT, "colouring does not list every cell exactly once");
  lfx_lma_layout* L = new lfx_lma_layout();
  L->ncell_2d = ncell_2d;
  L->nlayers = nlayers;
  L->ndf_to = ndf_to;
  L->ndf_from = ndf_from;
  L->undf_to = undf_to;
  L->undf_from = undf_from;
  int rc = build_layout(ctx, L, ncell_2d, nlayers, ndf_to, map_to, undf_to, rank);
  // 0-based maps on the device
  std::vector<int32_t> mf((size_t)ncell_2d * ndf_from), mt((size_t)ncell_2d * ndf_to);
  for (size_t i = 0; i < mf.size(); ++i) {
    mf[i] = map_from[i] - 1;
    if (mf[i] < 0 || (int64_t)mf[i] + nlayers > undf_from)
      rc = rc ? rc : fail(ctx, LFX_INVALID_ARGUMENT, "from-space dofmap entry out of range");
  }
  for (size_t i = 0; i < mt.size(); ++i) mt[i] = map_to[i] - 1;
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

int lfx_op_destroy(lfx_op* op) {
  if (!op) return LFX_OK;
  lfx_ctx* ctx = op->ctx;
  dfree(ctx, op->mat, op->mat_bytes);
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
  const LayoutArgs A = args_of(L);
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
                          L->rank);
    if (rc) {
      free_layout(ctx, T);
      return rc;
    }
    L->tlay = T;
  }
  lfx_lma_layout* T = L->tlay;
  if (!T->full_cover)
    LFX_CK(ctx, cudaMemsetAsync(y->data[0], 0, T->undf_to * y->elem(), ctx->stream));
  LayoutArgs A = args_of(T);
  // the stored matrix is [c][df_to][df_from][k]; lma_gather_t indexes it as
  // [c][j(in)][df(out)][k] with in = to-space, out = from-space
  if (op->precision == LFX_R64)
    lma_gather_t<double><<<gather_grid(ctx, T->nent), 256, 0, ctx->stream>>>(
        A, T->max_off, (const double*)op->mat, (const double*)x->data[0], L->map_to,
        (double*)y->data[0]);
  else
    lma_gather_t<float><<<gather_grid(ctx, T->nent), 256, 0, ctx->stream>>>(
        A, T->max_off, (const float*)op->mat, (const float*)x->data[0], L->map_to,
        (float*)y->data[0]);
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

}  // extern "C"
