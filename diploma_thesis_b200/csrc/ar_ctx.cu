// Context, error reporting and the scratch arena.
#include <cstdarg>
#include <cstring>
#include <string>

#include "ar_internal.cuh"
#include "ar_sort.cuh"

#include <atomic>

namespace {
thread_local char g_last_error[512] = "";
// Allocation fault injection (ar_test_fail_allocations): -1 = off, else the number of
// allocations that still succeed before every later one fails.
std::atomic<long> g_alloc_budget{-1};

bool injected_failure() {
  long b = g_alloc_budget.load();
  while (b >= 0) {
    if (b == 0) return true;
    if (g_alloc_budget.compare_exchange_weak(b, b - 1)) return false;
  }
  return false;
}
}  // namespace

namespace arh {

cudaError_t dev_malloc(void** p, size_t bytes) {
  if (injected_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

cudaError_t dev_malloc_async(void** p, size_t bytes, cudaStream_t st) {
  if (injected_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocAsync(p, bytes, st);
}

cudaError_t host_malloc(void** p, size_t bytes) {
  if (injected_failure()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocHost(p, bytes);
}

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

ar_status check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return AR_ERR_CUDA;
  }
  return AR_OK;
}

void* scratch(ar_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->scratch_bytes) return ctx->scratch;
  // Growing: the old arena may still be read by queued work, so drain the device first.
  // Callers that capture graphs reserve up front (ar_ctx_reserve) so this never runs then.
  if (cudaDeviceSynchronize() != cudaSuccess) return nullptr;
  if (ctx->scratch) cudaFree(ctx->scratch);
  ctx->scratch = nullptr;
  ctx->scratch_bytes = 0;
  size_t grow = bytes + bytes / 4 + (1u << 20);
  if (dev_malloc(&ctx->scratch, grow) != cudaSuccess) {
    cudaGetLastError();
    set_error("scratch arena: cudaMalloc(%zu) failed", grow);
    return nullptr;
  }
  ctx->scratch_bytes = grow;
  return ctx->scratch;
}

}  // namespace arh

extern "C" {

const char* ar_last_error(void) { return g_last_error; }
const char* ar_version(void) { return "arsim-b200 0.1 (sm_100a)"; }

ar_status ar_ctx_create(int device, ar_ctx** out) {
  if (!out) return AR_ERR_INVALID_ARG;
  *out = nullptr;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    arh::set_error("cudaSetDevice(%d) failed", device);
    return AR_ERR_CUDA;
  }
  ar_ctx* c = new ar_ctx();
  c->device = device;
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  auto release = [c]() {  // everything created so far, on any failure below
    if (c->d_err) cudaFree(c->d_err);
    if (c->h_err) cudaFreeHost(c->h_err);
    delete c;
  };
  if (arh::dev_malloc((void**)&c->d_err, sizeof(int)) != cudaSuccess ||
      arh::host_malloc((void**)&c->h_err, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    arh::set_error("ar_ctx_create: allocation failed");
    release();
    return AR_ERR_OOM;
  }
  cudaMemset(c->d_err, 0, sizeof(int));
  *c->h_err = 0;
  // scenes come from the device's stream-ordered pool: keep freed memory in the pool instead
  // of returning it to the driver at every synchronisation
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  ar_sort::init();
  if (cudaDeviceSynchronize() != cudaSuccess) {
    arh::set_error("ar_ctx_create: device error (%s)", cudaGetErrorString(cudaGetLastError()));
    release();
    return AR_ERR_CUDA;
  }
  *out = c;
  return AR_OK;
}

ar_status ar_test_fail_allocations(long after) {
  g_alloc_budget.store(after < 0 ? -1 : after);
  return AR_OK;
}

ar_status ar_ctx_destroy(ar_ctx* ctx) {
  if (!ctx) return AR_ERR_INVALID_ARG;
  cudaDeviceSynchronize();
  if (ctx->scratch) cudaFree(ctx->scratch);
  if (ctx->d_err) cudaFree(ctx->d_err);
  if (ctx->h_err) cudaFreeHost(ctx->h_err);
  delete ctx;
  return AR_OK;
}

ar_status ar_ctx_reserve(ar_ctx* ctx, size_t bytes) {
  if (!ctx) return AR_ERR_INVALID_ARG;
  return arh::scratch(ctx, bytes) ? AR_OK : AR_ERR_OOM;
}

ar_status ar_ctx_status(ar_ctx* ctx, ar_stream_t stream) {
  if (!ctx) return AR_ERR_INVALID_ARG;
  cudaStream_t s = arh::stream(stream);
  if (cudaMemcpyAsync(ctx->h_err, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    arh::set_error("ar_ctx_status: %s", cudaGetErrorString(cudaGetLastError()));
    return AR_ERR_CUDA;
  }
  int bits = *ctx->h_err;
  if (bits) {
    cudaMemsetAsync(ctx->d_err, 0, sizeof(int), s);
    cudaStreamSynchronize(s);
  }
  if (bits & ar::kErrTimeout) {
    arh::set_error("device: a bounded wait timed out");
    return AR_ERR_TIMEOUT;
  }
  if (bits & ar::kErrNaN) {
    arh::set_error("device: non-finite body state");
    return AR_ERR_NAN;
  }
  if (bits & ar::kErrOverflow) {
    arh::set_error("device: output capacity exceeded");
    return AR_ERR_OVERFLOW;
  }
  return AR_OK;
}

}  // extern "C"
