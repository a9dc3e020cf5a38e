// Device field vectors: the abstract_vector_type operations
// (vector_mod.F90:17-189) as implemented by field_vector_type /
// r_solver_field_vector_type (sci_field_vector_mod.x90,
// sci_r_solver_field_vector_mod.x90) through the PSyclone builtins
// setval_c, setval_X, inc_X_plus_bY, inc_aX_plus_Y, aX_plus_bY, inc_a_times_X,
// X_innerproduct_X/Y. Elementwise arithmetic happens in the storage precision
// (FP32 vectors round their scalars to FP32 first, as the r_solver vector
// does, sci_r_solver_field_vector_mod.x90:189); inner products accumulate in
// FP64 in the fixed order of lfx_internal.cuh.
#include <cmath>

#include "lfx_internal.cuh"

using namespace lfx;

namespace lfx {

template <class T>
static int k_set(lfx_ctx* ctx, T* x, T c, int64_t n) {
  return launch_chunks<0>(
      ctx, n, [=] __device__(int64_t) { return V1<T>{c}; },
      [=] __device__(int64_t i, const V1<T>& v, double*) { x[i] = v.a; }, NoFin{});
}
template <class T>
static int k_copy(lfx_ctx* ctx, T* y, const T* x, int64_t n) {
  return launch_chunks<0>(
      ctx, n, [=] __device__(int64_t i) { return V1<T>{x[i]}; },
      [=] __device__(int64_t i, const V1<T>& v, double*) { y[i] = v.a; }, NoFin{});
}
template <class T>
static int k_axpy(lfx_ctx* ctx, T* y, T a, const T* x, int64_t n) {
  return launch_chunks<0>(
      ctx, n, [=] __device__(int64_t i) { return V2<T>{x[i], y[i]}; },
      [=] __device__(int64_t i, const V2<T>& v, double*) { y[i] = fmaT(a, v.a, v.b); }, NoFin{});
}
template <class T>
static int k_aypx(lfx_ctx* ctx, T* y, T a, const T* x, int64_t n) {
  return launch_chunks<0>(
      ctx, n, [=] __device__(int64_t i) { return V2<T>{x[i], y[i]}; },
      [=] __device__(int64_t i, const V2<T>& v, double*) { y[i] = fmaT(a, v.b, v.a); }, NoFin{});
}
template <class T>
static int k_axpby(lfx_ctx* ctx, T* z, T a, const T* x, T b, const T* y, int64_t n) {
  return launch_chunks<0>(
      ctx, n, [=] __device__(int64_t i) { return V2<T>{x[i], y[i]}; },
      [=] __device__(int64_t i, const V2<T>& v, double*) { z[i] = fmaT(a, v.a, b * v.b); },
      NoFin{});
}
template <class T>
static int k_scale(lfx_ctx* ctx, T* x, T a, int64_t n) {
  return launch_chunks<0>(
      ctx, n, [=] __device__(int64_t i) { return V1<T>{x[i]}; },
      [=] __device__(int64_t i, const V1<T>& v, double*) { x[i] = a * v.a; }, NoFin{});
}
template <class T>
static int k_dot(lfx_ctx* ctx, const T* x, const T* y, int64_t n, double* out) {
  return launch_chunks<1>(
      ctx, n, [=] __device__(int64_t i) { return V2<T>{x[i], y[i]}; },
      [=] __device__(int64_t, const V2<T>& v, double* acc) {
        acc[0] = fma((double)v.a, (double)v.b, acc[0]);
      },
      [=] __device__(const double* tot) { *out = tot[0]; });
}
template <class S, class D>
static int k_convert(lfx_ctx* ctx, D* d, const S* s, int64_t n) {
  return launch_chunks<0>(
      ctx, n, [=] __device__(int64_t i) { return V1<S>{s[i]}; },
      [=] __device__(int64_t i, const V1<S>& v, double*) { d[i] = (D)v.a; }, NoFin{});
}

}  // namespace lfx

static bool same_shape(const lfx_vec* a, const lfx_vec* b) {
  return a && b && a->ctx == b->ctx && a->precision == b->precision && a->undf == b->undf;
}

#define VEC_CHECK(v) \
  if (!(v) || !(v)->ctx) return LFX_INVALID_ARGUMENT
#define SHAPE_CHECK(a, b)                                                         \
  if (!same_shape((a), (b)))                                                      \
  return fail((a)->ctx, LFX_TYPE_MISMATCH, "vectors differ in shape or precision")

// result of NF per-field sums combined left to right on the host, as the
// field loops of sci_field_vector_mod.x90:132-182 do
static int read_sums(lfx_ctx* ctx, int nf, double* out_sum) {
  int rc = to_host_small(ctx, ctx->h_scalars_dev, ctx->d_scalars, sizeof(double) * nf);
  if (rc) return rc;
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  double s = 0.0;
  for (int f = 0; f < nf; ++f) s = s + ctx->h_scalars[f];
  *out_sum = s;
  return LFX_OK;
}

extern "C" {

int lfx_vec_create(lfx_ctx* ctx, int32_t nfields, const int64_t* undf, int32_t precision,
                   lfx_vec** out) {
  if (!ctx || !out || nfields < 1 || nfields > 32 || !undf) return LFX_INVALID_ARGUMENT;
  if (precision != LFX_R64 && precision != LFX_R32)
    return fail(ctx, LFX_INVALID_ARGUMENT, "precision must be 64 or 32");
  *out = nullptr;
  lfx_vec* v = new lfx_vec();
  v->ctx = ctx;
  v->precision = precision;
  int64_t maxn = 0;
  for (int f = 0; f < nfields; ++f) {
    if (undf[f] < 0) {
      delete v;
      return fail(ctx, LFX_INVALID_ARGUMENT, "negative field length");
    }
    v->undf.push_back(undf[f]);
    void* p = nullptr;
    int rc = dmalloc(ctx, &p, (size_t)undf[f] * v->elem());
    if (rc) {
      lfx_vec_destroy(v);
      return rc;
    }
    v->data.push_back(p);
    if (undf[f] > maxn) maxn = undf[f];
  }
  int rc = ensure_partials(ctx, maxn, 4);
  if (rc) {
    lfx_vec_destroy(v);
    return rc;
  }
  *out = v;
  return LFX_OK;
}

int lfx_vec_duplicate(const lfx_vec* src, lfx_vec** out) {
  VEC_CHECK(src);
  return lfx_vec_create(src->ctx, (int32_t)src->undf.size(), src->undf.data(), src->precision, out);
}

int lfx_vec_destroy(lfx_vec* v) {
  if (!v) return LFX_OK;
  for (size_t f = 0; f < v->data.size(); ++f) dfree(v->ctx, v->data[f], v->undf[f] * v->elem());
  delete v;
  return LFX_OK;
}

int lfx_vec_set_scalar(lfx_vec* v, double s) {
  VEC_CHECK(v);
  for (size_t f = 0; f < v->data.size(); ++f) {
    int rc = v->precision == LFX_R64 ? k_set(v->ctx, (double*)v->data[f], s, v->undf[f])
                                     : k_set(v->ctx, (float*)v->data[f], (float)s, v->undf[f]);
    if (rc) return rc;
  }
  return LFX_OK;
}

int lfx_vec_axpy(lfx_vec* y, double a, const lfx_vec* x) {
  VEC_CHECK(y);
  SHAPE_CHECK(y, x);
  for (size_t f = 0; f < y->data.size(); ++f) {
    int rc = y->precision == LFX_R64
                 ? k_axpy(y->ctx, (double*)y->data[f], a, (const double*)x->data[f], y->undf[f])
                 : k_axpy(y->ctx, (float*)y->data[f], (float)a, (const float*)x->data[f], y->undf[f]);
    if (rc) return rc;
  }
  return LFX_OK;
}

int lfx_vec_aypx(lfx_vec* y, double a, const lfx_vec* x) {
  VEC_CHECK(y);
  SHAPE_CHECK(y, x);
  for (size_t f = 0; f < y->data.size(); ++f) {
    int rc = y->precision == LFX_R64
                 ? k_aypx(y->ctx, (double*)y->data[f], a, (const double*)x->data[f], y->undf[f])
                 : k_aypx(y->ctx, (float*)y->data[f], (float)a, (const float*)x->data[f], y->undf[f]);
    if (rc) return rc;
  }
  return LFX_OK;
}

int lfx_vec_axpby(lfx_vec* z, double a, const lfx_vec* x, double b, const lfx_vec* y) {
  VEC_CHECK(z);
  SHAPE_CHECK(z, x);
  SHAPE_CHECK(z, y);
  for (size_t f = 0; f < z->data.size(); ++f) {
    int rc = z->precision == LFX_R64
                 ? k_axpby(z->ctx, (double*)z->data[f], a, (const double*)x->data[f], b,
                           (const double*)y->data[f], z->undf[f])
                 : k_axpby(z->ctx, (float*)z->data[f], (float)a, (const float*)x->data[f], (float)b,
                           (const float*)y->data[f], z->undf[f]);
    if (rc) return rc;
  }
  return LFX_OK;
}

int lfx_vec_scale(lfx_vec* v, double s) {
  VEC_CHECK(v);
  for (size_t f = 0; f < v->data.size(); ++f) {
    int rc = v->precision == LFX_R64 ? k_scale(v->ctx, (double*)v->data[f], s, v->undf[f])
                                     : k_scale(v->ctx, (float*)v->data[f], (float)s, v->undf[f]);
    if (rc) return rc;
  }
  return LFX_OK;
}

int lfx_vec_copy(lfx_vec* dst, const lfx_vec* src) {
  VEC_CHECK(dst);
  SHAPE_CHECK(dst, src);
  for (size_t f = 0; f < dst->data.size(); ++f) {
    int rc = dst->precision == LFX_R64
                 ? k_copy(dst->ctx, (double*)dst->data[f], (const double*)src->data[f], dst->undf[f])
                 : k_copy(dst->ctx, (float*)dst->data[f], (const float*)src->data[f], dst->undf[f]);
    if (rc) return rc;
  }
  return LFX_OK;
}

int lfx_vec_dot(const lfx_vec* v, const lfx_vec* x, double* out) {
  VEC_CHECK(v);
  SHAPE_CHECK(v, x);
  if (!out) return LFX_INVALID_ARGUMENT;
  lfx_ctx* ctx = v->ctx;
  int nf = (int)v->data.size();
  for (int f = 0; f < nf; ++f) {
    int rc = v->precision == LFX_R64
                 ? k_dot(ctx, (const double*)v->data[f], (const double*)x->data[f], v->undf[f],
                         ctx->d_scalars + f)
                 : k_dot(ctx, (const float*)v->data[f], (const float*)x->data[f], v->undf[f],
                         ctx->d_scalars + f);
    if (rc) return rc;
  }
  return read_sums(ctx, nf, out);
}

int lfx_vec_norm(const lfx_vec* v, double* out) {
  double s = 0.0;
  int rc = lfx_vec_dot(v, v, &s);
  if (rc) return rc;
  *out = std::sqrt(s);
  return LFX_OK;
}

int lfx_vec_field_norm(const lfx_vec* v, int32_t position, double* out) {
  VEC_CHECK(v);
  if (!out || position < 1 || position > (int32_t)v->data.size())
    return fail(v->ctx, LFX_INVALID_ARGUMENT, "field position out of range");
  lfx_ctx* ctx = v->ctx;
  int f = position - 1;
  int rc = v->precision == LFX_R64
               ? k_dot(ctx, (const double*)v->data[f], (const double*)v->data[f], v->undf[f],
                       ctx->d_scalars)
               : k_dot(ctx, (const float*)v->data[f], (const float*)v->data[f], v->undf[f],
                       ctx->d_scalars);
  if (rc) return rc;
  double s;
  rc = read_sums(ctx, 1, &s);
  if (rc) return rc;
  *out = std::sqrt(s);
  return LFX_OK;
}

int lfx_vec_size(const lfx_vec* v, int32_t* nfields) {
  VEC_CHECK(v);
  if (!nfields) return LFX_INVALID_ARGUMENT;
  *nfields = (int32_t)v->data.size();
  return LFX_OK;
}

int lfx_vec_field_device_ptr(const lfx_vec* v, int32_t position, void** out) {
  VEC_CHECK(v);
  if (!out || position < 1 || position > (int32_t)v->data.size()) return LFX_INVALID_ARGUMENT;
  *out = v->data[position - 1];
  return LFX_OK;
}

int lfx_vec_import_field(lfx_vec* v, int32_t position, const double* host, int64_t n) {
  VEC_CHECK(v);
  lfx_ctx* ctx = v->ctx;
  if (position < 1 || position > (int32_t)v->data.size())
    return fail(ctx, LFX_INVALID_ARGUMENT, "field position bigger than nfields");
  int f = position - 1;
  if (!host || n != v->undf[f]) return fail(ctx, LFX_INVALID_ARGUMENT, "field length mismatch");
  if (v->precision == LFX_R64) {
    LFX_CK(ctx, cudaMemcpyAsync(v->data[f], host, n * 8, cudaMemcpyHostToDevice, ctx->stream));
    LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
    return LFX_OK;
  }
  // FP32 storage: stage the FP64 data and round on the device
  double* tmp = nullptr;
  int rc = dmalloc(ctx, (void**)&tmp, n * 8);
  if (rc) return rc;
  LFX_CK(ctx, cudaMemcpyAsync(tmp, host, n * 8, cudaMemcpyHostToDevice, ctx->stream));
  rc = k_convert(ctx, (float*)v->data[f], (const double*)tmp, n);
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, tmp, n * 8);
  return rc;
}

// Asynchronous transfers of an FP64 field on a caller's stream (null: the
// context's); with pinned host memory they overlap work on other streams.
// The caller orders the stream against the context's stream.
static int field_async(const lfx_vec* v, int32_t position, void* dst, const void* src, int64_t n,
                       void* stream, cudaMemcpyKind kind) {
  lfx_ctx* ctx = v->ctx;
  if (position < 1 || position > (int32_t)v->data.size())
    return fail(ctx, LFX_INVALID_ARGUMENT, "field position bigger than nfields");
  if (!dst || !src || n != v->undf[position - 1])
    return fail(ctx, LFX_INVALID_ARGUMENT, "field length mismatch");
  if (v->precision != LFX_R64)
    return fail(ctx, LFX_NOT_SUPPORTED, "asynchronous transfers take FP64 fields");
  cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
  LFX_CK(ctx, cudaMemcpyAsync(dst, src, n * 8, kind, s));
  return LFX_OK;
}

int lfx_vec_import_field_async(lfx_vec* v, int32_t position, const double* host, int64_t n,
                               void* stream) {
  VEC_CHECK(v);
  if (!host) return LFX_INVALID_ARGUMENT;
  if (position < 1 || position > (int32_t)v->data.size())
    return fail(v->ctx, LFX_INVALID_ARGUMENT, "field position bigger than nfields");
  return field_async(v, position, v->data[position - 1], host, n, stream, cudaMemcpyHostToDevice);
}

int lfx_vec_export_field_async(const lfx_vec* v, int32_t position, double* host, int64_t n,
                               void* stream) {
  VEC_CHECK(v);
  if (!host) return LFX_INVALID_ARGUMENT;
  if (position < 1 || position > (int32_t)v->data.size())
    return fail(v->ctx, LFX_INVALID_ARGUMENT, "field position bigger than nfields");
  return field_async(v, position, host, v->data[position - 1], n, stream, cudaMemcpyDeviceToHost);
}

int lfx_vec_export_field(const lfx_vec* v, int32_t position, double* host, int64_t n) {
  VEC_CHECK(v);
  lfx_ctx* ctx = v->ctx;
  if (position < 1 || position > (int32_t)v->data.size())
    return fail(ctx, LFX_INVALID_ARGUMENT, "field position bigger than nfields");
  int f = position - 1;
  if (!host || n != v->undf[f]) return fail(ctx, LFX_INVALID_ARGUMENT, "field length mismatch");
  if (v->precision == LFX_R64) {
    LFX_CK(ctx, cudaMemcpyAsync(host, v->data[f], n * 8, cudaMemcpyDeviceToHost, ctx->stream));
    LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
    return LFX_OK;
  }
  double* tmp = nullptr;
  int rc = dmalloc(ctx, (void**)&tmp, n * 8);
  if (rc) return rc;
  rc = k_convert(ctx, tmp, (const float*)v->data[f], n);
  LFX_CK(ctx, cudaMemcpyAsync(host, tmp, n * 8, cudaMemcpyDeviceToHost, ctx->stream));
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, tmp, n * 8);
  return rc;
}

}  // extern "C"
