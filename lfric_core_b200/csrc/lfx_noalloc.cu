// Allocation-free FP64 inner product.
//
// Some callers cannot allocate device memory at the point where they need an
// inner product: a host model whose device memory belongs to another
// allocator (a Fortran runtime's OpenMP/OpenACC pool, say, which must stay
// the only owner of the device's memory), or a latency-critical loop that must
// not take the implicit synchronisation of cudaMalloc/cudaFree. lfx_dot_noalloc
// serves them:
// the caller passes the inputs and the (device) output, and the only scratch
// the reduction needs -- one partial sum per 2048-element chunk plus a
// completion ticket -- lives in the file-scope array below, which every GPU
// that loads this library holds until the process exits.
//
// The sum is computed in the same fixed order as lfx_vec_dot, so the two give
// bit-identical results.
//
// The array's device address is looked up once per device and kept for the
// life of the process. A cudaDeviceReset (or any reset of the device's primary
// context) unloads the module, which may come back at another address: after
// one, this entry point must not be called again in the same process.
#include <mutex>
#include <string>

#include "lfx_internal.cuh"

using namespace lfx;

namespace {

// Largest input: kMaxChunks chunks of RCHUNK elements (16 Mi elements).
constexpr int64_t kMaxChunks = 8192;
// partials [0, kMaxChunks); the completion ticket in the next slot
static __device__ __align__(256) double g_noalloc_scratch[kMaxChunks + 32];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
int g_num_sms[kMaxDevices] = {0};
thread_local std::string g_err;

int noalloc_fail(int status, const std::string& msg) {
  g_err = msg;
  return status;
}

}  // namespace

extern "C" {

int64_t lfx_dot_noalloc_max_n(void) { return kMaxChunks * RCHUNK; }

const char* lfx_noalloc_last_error(void) { return g_err.c_str(); }

int lfx_dot_noalloc(const double* x, const double* y, int64_t n, double* result, void* stream) {
  if (!result || n < 0 || (n > 0 && (!x || !y)))
    return noalloc_fail(LFX_INVALID_ARGUMENT, "lfx_dot_noalloc: null pointer or negative length");
  if (n > kMaxChunks * RCHUNK)
    return noalloc_fail(LFX_INVALID_ARGUMENT,
                        "lfx_dot_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " +
                            std::to_string(kMaxChunks * RCHUNK) +
                            " elements (use lfx_vec_dot for larger vectors)");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(LFX_CUDA_ERROR, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(LFX_NOT_SUPPORTED, "device id too large");
  double* scratch = nullptr;
  int sms = 0;
  {
    // one-time set-up per device, with that device current: the host cannot
    // use the symbol itself as a device address, so ask the runtime for it
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return noalloc_fail(LFX_CUDA_ERROR,
                            std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      int s = 0;
      e = cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return noalloc_fail(LFX_CUDA_ERROR, cudaGetErrorString(e));
      g_scratch_ptr[dev] = (double*)p;
      g_num_sms[dev] = s;
    }
    scratch = g_scratch_ptr[dev];
    sms = g_num_sms[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  unsigned* ticket = (unsigned*)(scratch + kMaxChunks);
  // the ticket must start at zero; the partials are overwritten before use
  e = cudaMemsetAsync(ticket, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return noalloc_fail(LFX_CUDA_ERROR, cudaGetErrorString(e));
  const int64_t nch = nchunks(n);
  int64_t grid = nch < (int64_t)sms * 32 ? nch : (int64_t)sms * 32;
  if (grid < 1) grid = 1;
  chunk_kernel<1><<<(int)grid, RT, 0, st>>>(
      n, [=] __device__(int64_t i) { return V2<double>{x[i], y[i]}; },
      [=] __device__(int64_t, const V2<double>& v, double* a) { a[0] = fma(v.a, v.b, a[0]); },
      [=] __device__(const double* t) { *result = t[0]; }, scratch, ticket, (const int*)nullptr);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(LFX_CUDA_ERROR, cudaGetErrorString(e));
  return LFX_OK;
}

}  // extern "C"
