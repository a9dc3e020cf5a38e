// Context: stream, error reporting, device memory accounting, reduction
// scratch and the optional per-apply timing of solves.
#include <cstdio>
#include <cstring>

#include "lfx_internal.cuh"

namespace lfx {

int fail(lfx_ctx* ctx, int status, const std::string& msg) {
  if (ctx) ctx->err = msg;
  return status;
}

int cuda_fail(lfx_ctx* ctx, cudaError_t e, const char* what) {
  if (ctx) ctx->err = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? LFX_OUT_OF_MEMORY : LFX_CUDA_ERROR;
}

int dmalloc(lfx_ctx* ctx, void** p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) return LFX_OK;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(ctx, LFX_OUT_OF_MEMORY,
                "device allocation of " + std::to_string(bytes) + " bytes failed: " +
                    cudaGetErrorString(e));
  }
  ctx->device_bytes += (int64_t)bytes;
  return LFX_OK;
}

void dfree(lfx_ctx* ctx, void* p, size_t bytes) {
  if (!p) return;
  cudaFree(p);
  ctx->device_bytes -= (int64_t)bytes;
}

int ensure_partials(lfx_ctx* ctx, int64_t n, int nsums) {
  int64_t need = nchunks(n) * nsums;
  if (need < 1) need = 1;
  if (need <= ctx->partials_cap) return LFX_OK;
  // never reallocate while a graph capture is recording
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(ctx->stream, &cs);
  if (cs != cudaStreamCaptureStatusNone)
    return fail(ctx, LFX_INVALID_ARGUMENT, "reduction scratch too small inside a capture");
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  dfree(ctx, ctx->d_partials, sizeof(double) * ctx->partials_cap);
  ctx->d_partials = nullptr;
  ctx->partials_cap = 0;
  int64_t cap = need * 2;
  int rc = dmalloc(ctx, (void**)&ctx->d_partials, sizeof(double) * cap);
  if (rc) return rc;
  ctx->partials_cap = cap;
  return LFX_OK;
}

void timing_begin(lfx_ctx* ctx, int32_t precision) {
  if (!ctx->time_applies) return;
  if (ctx->capture_ev) {
    TimedPair p{};
    cudaEventCreate(&p.a);
    cudaEventCreate(&p.b);
    p.prec = precision;
    ctx->capture_ev->push_back(p);
    // inside a capture only an "external" record becomes an event node
    cudaEventRecordWithFlags(p.a, ctx->stream, cudaEventRecordExternal);
    return;
  }
  if (ctx->ev_used + 2 > (int)ctx->ev_pool.size()) {
    for (int i = 0; i < 64; ++i) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ctx->ev_pool.push_back(e);
      ctx->ev_prec.push_back(0);
    }
  }
  ctx->ev_prec[ctx->ev_used] = precision;
  cudaEventRecord(ctx->ev_pool[ctx->ev_used++], ctx->stream);
}

__global__ void small_copy(const unsigned* __restrict__ src, unsigned* dst, int words) {
  for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
}

int host_alloc_mapped(lfx_ctx* ctx, void** host, void** dev, size_t bytes) {
  *host = *dev = nullptr;
  if (cudaHostAlloc(host, bytes, cudaHostAllocMapped) != cudaSuccess) {
    cudaGetLastError();
    *host = nullptr;
    return fail(ctx, LFX_OUT_OF_MEMORY, "pinned host allocation failed");
  }
  if (cudaHostGetDevicePointer(dev, *host, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaFreeHost(*host);
    *host = nullptr;
    return fail(ctx, LFX_CUDA_ERROR, "pinned host memory is not mapped into the device");
  }
  return LFX_OK;
}

// bytes: a multiple of 4, both addresses 4-byte aligned
int to_host_small(lfx_ctx* ctx, void* host_dev, const void* dev, size_t bytes) {
  small_copy<<<1, 64, 0, ctx->stream>>>((const unsigned*)dev, (unsigned*)host_dev,
                                        (int)(bytes / 4));
  ctx->launches++;
  LFX_CK(ctx, cudaGetLastError());
  return LFX_OK;
}

void timing_end(lfx_ctx* ctx) {
  if (!ctx->time_applies) return;
  if (ctx->capture_ev) {
    cudaEventRecordWithFlags(ctx->capture_ev->back().b, ctx->stream, cudaEventRecordExternal);
    return;
  }
  cudaEventRecord(ctx->ev_pool[ctx->ev_used++], ctx->stream);
}

}  // namespace lfx

using namespace lfx;

extern "C" {

int lfx_ctx_create(int device, lfx_ctx** out) {
  if (!out) return LFX_INVALID_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return LFX_CUDA_ERROR;
  }
  if (device < 0 || device >= ndev) return LFX_INVALID_ARGUMENT;
  if (cudaSetDevice(device) != cudaSuccess) return LFX_CUDA_ERROR;
  lfx_ctx* ctx = new lfx_ctx();
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&ctx->l2_bytes, cudaDevAttrL2CacheSize, device);
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return LFX_CUDA_ERROR;
  }
  int rc = dmalloc(ctx, (void**)&ctx->d_ticket, sizeof(unsigned) * 4);
  if (!rc) rc = dmalloc(ctx, (void**)&ctx->d_scalars, sizeof(double) * 64);
  if (!rc) rc = dmalloc(ctx, (void**)&ctx->d_err, sizeof(int) * 4);
  if (!rc && cudaMemset(ctx->d_ticket, 0, sizeof(unsigned) * 4) != cudaSuccess) rc = LFX_CUDA_ERROR;
  if (!rc && cudaMemset(ctx->d_err, 0, sizeof(int) * 4) != cudaSuccess) rc = LFX_CUDA_ERROR;
  if (!rc)
    rc = host_alloc_mapped(ctx, (void**)&ctx->h_scalars, (void**)&ctx->h_scalars_dev,
                           sizeof(double) * 64);
  if (!rc) rc = ensure_partials(ctx, (int64_t)RCHUNK * 4096, 1);
  if (rc) {
    lfx_ctx_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return LFX_OK;
}

int lfx_ctx_destroy(lfx_ctx* ctx) {
  if (!ctx) return LFX_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto e : ctx->ev_pool) cudaEventDestroy(e);
  dfree(ctx, ctx->d_partials, sizeof(double) * ctx->partials_cap);
  dfree(ctx, ctx->d_ticket, sizeof(unsigned) * 4);
  dfree(ctx, ctx->d_scalars, sizeof(double) * 64);
  dfree(ctx, ctx->d_err, sizeof(int) * 4);
  if (ctx->h_scalars) cudaFreeHost(ctx->h_scalars);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return LFX_OK;
}

const char* lfx_last_error(const lfx_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int lfx_ctx_synchronize(lfx_ctx* ctx) {
  if (!ctx) return LFX_INVALID_ARGUMENT;
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  return LFX_OK;
}

void* lfx_ctx_stream(lfx_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int64_t lfx_ctx_device_bytes(const lfx_ctx* ctx) { return ctx ? ctx->device_bytes : 0; }

int lfx_ctx_enable_apply_timing(lfx_ctx* ctx, int32_t enable) {
  if (!ctx) return LFX_INVALID_ARGUMENT;
  ctx->time_applies = enable != 0;
  return LFX_OK;
}

// Folds the recorded event pairs into the running totals (the stream must be
// idle, which lfx_solver_apply guarantees on return).
static int collect_timing(lfx_ctx* ctx) {
  for (int i = 0; i + 1 < ctx->ev_used; i += 2) {
    float ms = 0.f;
    cudaError_t e = cudaEventElapsedTime(&ms, ctx->ev_pool[i], ctx->ev_pool[i + 1]);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaEventElapsedTime");
    const int k = ctx->ev_prec[i] == LFX_R32 ? 1 : 0;
    ctx->timed_ms[k] += ms;
    ctx->timed_launches[k] += 1;
  }
  ctx->ev_used = 0;
  return LFX_OK;
}

int lfx_ctx_apply_timing(lfx_ctx* ctx, int32_t precision, int64_t* launches, double* total_ms,
                         int32_t reset) {
  if (!ctx) return LFX_INVALID_ARGUMENT;
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  int rc = collect_timing(ctx);
  if (rc) return rc;
  const bool all = precision == 0;
  const int k = precision == LFX_R32 ? 1 : 0;
  if (launches) *launches = all ? ctx->timed_launches[0] + ctx->timed_launches[1] : ctx->timed_launches[k];
  if (total_ms) *total_ms = all ? ctx->timed_ms[0] + ctx->timed_ms[1] : ctx->timed_ms[k];
  if (reset) {
    for (int j = 0; j < 2; ++j) {
      ctx->timed_launches[j] = 0;
      ctx->timed_ms[j] = 0.0;
    }
  }
  return LFX_OK;
}

int64_t lfx_ctx_launch_count(const lfx_ctx* ctx) { return ctx ? ctx->launches : 0; }

int lfx_ctx_set_apply_kernel(lfx_ctx* ctx, int32_t which) {
  if (!ctx || which < -1 || which > 6 || which == 2) return LFX_INVALID_ARGUMENT;
  ctx->lma_kernel = which;
  return LFX_OK;
}

int lfx_ctx_check_device_error(lfx_ctx* ctx) {
  if (!ctx) return LFX_INVALID_ARGUMENT;
  int h = 0;
  LFX_CK(ctx, cudaStreamSynchronize(ctx->stream));
  LFX_CK(ctx, cudaMemcpy(&h, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    // the flag, and the grid barrier words of a persistent apply that left early
    LFX_CK(ctx, cudaMemset(ctx->d_err, 0, sizeof(int) * 4));
    return fail(ctx, LFX_TIMEOUT, "a device-side bounded wait ran out (pipeline stage never filled)");
  }
  return LFX_OK;
}

}  // extern "C"

namespace lfx {
// exported for the solver translation unit: drain events between solves so the
// pool does not grow without bound
int drain_timing(lfx_ctx* ctx) { return collect_timing(ctx); }
}  // namespace lfx
