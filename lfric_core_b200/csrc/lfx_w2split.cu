// W2 split / combine (split_w2_field_kernel_mod.F90, combine_w2_field_kernel_mod.F90)
// for the lowest-order spaces: W2 (6 dofs per cell: W, S, E, N, B, T faces)
// to and from its horizontal part W2h (4) and vertical part W2v (2).
//
// As in the reference, each cell copies its W and S faces and, where the face
// selectors say so (face_selector_ew / _ns = 2), its E and/or N face; a face
// that two cells copy receives the same value twice. The vertical part copies
// the column's nlayers + 1 face values. The per-cell face lists are resolved
// at creation; one thread per (cell, level) copies the level of every listed
// face, so the consecutive levels of a face column move as coalesced runs.
#include <algorithm>
#include <vector>

#include "lfx_internal.cuh"

using namespace lfx;

struct lfx_w2_split {
  lfx_ctx* ctx = nullptr;
  int32_t ncell_2d = 0, nlayers = 0;
  int64_t max_w2 = 0, max_w2h = 0, max_w2v = 0;  // largest 0-based dof touched + 1
  int4* d_h = nullptr;    // [ncell][4] pairs packed as {w2 base, w2h base} x 2 in two int4
  int* d_nh = nullptr;    // [ncell] horizontal faces copied
  int2* d_v = nullptr;    // [ncell] {w2 base of B, w2v base}
};

namespace {

// dir 0: uvw -> (uv, w); dir 1: (uv, w) -> uvw
template <class T, int DIR>
__global__ void w2_split_k(int ncell, int nl, const int4* __restrict__ hp, const int* __restrict__ nh,
                           const int2* __restrict__ vp, T* __restrict__ uvw, T* __restrict__ uv,
                           T* __restrict__ w) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int per = nl + 1;
  if (t >= (int64_t)ncell * per) return;
  const int c = (int)(t / per), k = (int)(t % per);
  if (k < nl) {
    const int n = nh[c];
    const int4 a = hp[2 * c], b = hp[2 * c + 1];
    const int w2b[4] = {a.x, a.z, b.x, b.z};
    const int whb[4] = {a.y, a.w, b.y, b.w};
    for (int f = 0; f < n; ++f) {
      if (DIR == 0)
        uv[whb[f] + k] = uvw[w2b[f] + k];
      else
        uvw[w2b[f] + k] = uv[whb[f] + k];
    }
  }
  const int2 v = vp[c];
  if (DIR == 0)
    w[v.y + k] = uvw[v.x + k];
  else
    uvw[v.x + k] = w[v.y + k];
}

template <class T>
int launch(lfx_w2_split* s, int dir, T* uvw, T* uv, T* w) {
  lfx_ctx* ctx = s->ctx;
  const int64_t n = (int64_t)s->ncell_2d * (s->nlayers + 1);
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (dir == 0)
    w2_split_k<T, 0><<<grid, 256, 0, ctx->stream>>>(s->ncell_2d, s->nlayers, s->d_h, s->d_nh,
                                                     s->d_v, uvw, uv, w);
  else
    w2_split_k<T, 1><<<grid, 256, 0, ctx->stream>>>(s->ncell_2d, s->nlayers, s->d_h, s->d_nh,
                                                     s->d_v, uvw, uv, w);
  ctx->launches++;
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

int run(lfx_w2_split* s, int dir, const lfx_vec* uvw, const lfx_vec* uv, const lfx_vec* w) {
  if (!s || !uvw || !uv || !w) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = s->ctx;
  if (uvw->precision != uv->precision || uvw->precision != w->precision)
    return fail(ctx, LFX_TYPE_MISMATCH, "W2, W2h and W2v fields differ in precision");
  if (uvw->data.size() != 1 || uv->data.size() != 1 || w->data.size() != 1)
    return fail(ctx, LFX_NOT_SUPPORTED, "single-field vectors only");
  if (uvw->undf[0] < s->max_w2 || uv->undf[0] < s->max_w2h || w->undf[0] < s->max_w2v)
    return fail(ctx, LFX_TYPE_MISMATCH, "a field is shorter than its dofmap");
  if (uvw->precision == LFX_R64)
    return launch<double>(s, dir, (double*)uvw->data[0], (double*)uv->data[0], (double*)w->data[0]);
  return launch<float>(s, dir, (float*)uvw->data[0], (float*)uv->data[0], (float*)w->data[0]);
}

}  // namespace

extern "C" {

int lfx_w2_split_create(lfx_ctx* ctx, int32_t ncell_2d, int32_t nlayers, const int32_t* map_w2,
                        const int32_t* map_w2h, const int32_t* map_w2v, const int32_t* map_w3_2d,
                        int64_t undf_w3_2d, const int32_t* face_selector_ew,
                        const int32_t* face_selector_ns, lfx_w2_split** out) {
  if (!ctx || !map_w2 || !map_w2h || !map_w2v || !map_w3_2d || !face_selector_ew ||
      !face_selector_ns || !out)
    return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  if (ncell_2d < 1 || nlayers < 1) return fail(ctx, LFX_INVALID_ARGUMENT, "bad mesh sizes");
  std::vector<int4> h((size_t)ncell_2d * 2);
  std::vector<int> nh(ncell_2d);
  std::vector<int2> v(ncell_2d);
  int64_t m2 = 0, mh = 0, mv = 0;
  for (int c = 0; c < ncell_2d; ++c) {
    const int32_t* m = map_w2 + (size_t)6 * c;
    const int32_t* mhc = map_w2h + (size_t)4 * c;
    const int32_t c3 = map_w3_2d[c] - 1;
    if (c3 < 0 || c3 >= undf_w3_2d) return fail(ctx, LFX_INVALID_ARGUMENT, "map_w3_2d out of range");
    const int32_t ew = face_selector_ew[c3], ns = face_selector_ns[c3];
    if (ew < 1 || ew > 2 || ns < 1 || ns > 2)
      return fail(ctx, LFX_INVALID_ARGUMENT, "face selectors must be 1 or 2");
    // W, S, then E (or N when only the N face is selected), then N
    int faces[4] = {0, 1, (ns == 2 && ew == 1) ? 3 : 2, 3};
    const int n = ew + ns;
    int w2b[4] = {0, 0, 0, 0}, whb[4] = {0, 0, 0, 0};
    for (int f = 0; f < n; ++f) {
      w2b[f] = m[faces[f]] - 1;
      whb[f] = mhc[faces[f]] - 1;
      if (w2b[f] < 0 || whb[f] < 0) return fail(ctx, LFX_INVALID_ARGUMENT, "dofmap entries must be >= 1");
      m2 = std::max<int64_t>(m2, (int64_t)w2b[f] + nlayers);
      mh = std::max<int64_t>(mh, (int64_t)whb[f] + nlayers);
    }
    h[2 * c] = make_int4(w2b[0], whb[0], w2b[1], whb[1]);
    h[2 * c + 1] = make_int4(w2b[2], whb[2], w2b[3], whb[3]);
    nh[c] = n;
    const int32_t b = m[4] - 1, vb = map_w2v[(size_t)2 * c] - 1;
    if (b < 0 || vb < 0 || m[5] != m[4] + 1 || map_w2v[(size_t)2 * c + 1] != map_w2v[(size_t)2 * c] + 1)
      return fail(ctx, LFX_INVALID_ARGUMENT,
                  "vertical faces must be one column (top dof = bottom dof + 1)");
    v[c] = make_int2(b, vb);
    m2 = std::max<int64_t>(m2, (int64_t)b + nlayers + 1);
    mv = std::max<int64_t>(mv, (int64_t)vb + nlayers + 1);
  }
  auto* s = new lfx_w2_split();
  s->ctx = ctx;
  s->ncell_2d = ncell_2d;
  s->nlayers = nlayers;
  s->max_w2 = m2;
  s->max_w2h = mh;
  s->max_w2v = mv;
  int rc = dmalloc(ctx, (void**)&s->d_h, h.size() * sizeof(int4));
  if (!rc) rc = dmalloc(ctx, (void**)&s->d_nh, nh.size() * sizeof(int));
  if (!rc) rc = dmalloc(ctx, (void**)&s->d_v, v.size() * sizeof(int2));
  if (!rc && (cudaMemcpy(s->d_h, h.data(), h.size() * sizeof(int4), cudaMemcpyHostToDevice) ||
              cudaMemcpy(s->d_nh, nh.data(), nh.size() * sizeof(int), cudaMemcpyHostToDevice) ||
              cudaMemcpy(s->d_v, v.data(), v.size() * sizeof(int2), cudaMemcpyHostToDevice)))
    rc = fail(ctx, LFX_CUDA_ERROR, "upload of the W2 split tables failed");
  if (rc) {
    lfx_w2_split_destroy(s);
    return rc;
  }
  *out = s;
  return LFX_OK;
}

int lfx_w2_split_field(lfx_w2_split* s, const lfx_vec* uvw, lfx_vec* uv, lfx_vec* w) {
  return run(s, 0, uvw, uv, w);
}

int lfx_w2_combine_field(lfx_w2_split* s, const lfx_vec* uv, const lfx_vec* w, lfx_vec* uvw) {
  return run(s, 1, uvw, uv, w);
}

int lfx_w2_split_destroy(lfx_w2_split* s) {
  if (!s) return LFX_OK;
  dfree(s->ctx, s->d_h, (size_t)s->ncell_2d * 2 * sizeof(int4));
  dfree(s->ctx, s->d_nh, (size_t)s->ncell_2d * sizeof(int));
  dfree(s->ctx, s->d_v, (size_t)s->ncell_2d * sizeof(int2));
  delete s;
  return LFX_OK;
}

}  // extern "C"
