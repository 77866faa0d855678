// Context management and error reporting of the C ABI (include/mcb200.h).
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "internal.h"

namespace mcb {

mcb_status set_error(mcb_ctx *ctx, mcb_status st, const char *fmt, ...) {
  if (!ctx) return st;
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  ctx->err = buf;
  return st;
}

mcb_status pool_get(mcb_ctx *ctx, int slot, size_t bytes, void **out) {
  if ((int)ctx->pool.size() <= slot) ctx->pool.resize(slot + 1);
  DevBuf &b = ctx->pool[slot];
  if (b.bytes < bytes) {
    if (b.ptr) {
      cudaStreamSynchronize(ctx->stream);
      cudaFree(b.ptr);
      b.ptr = nullptr;
      b.bytes = 0;
    }
    const size_t want = bytes + bytes / 8;
    cudaError_t e = cudaMalloc(&b.ptr, want);
    if (e != cudaSuccess) {
      cudaGetLastError();
      b.ptr = nullptr;
      return set_error(ctx, MCB_ENOMEM, "device allocation of %zu bytes failed: %s", want, cudaGetErrorString(e));
    }
    b.bytes = want;
  }
  *out = b.ptr;
  return MCB_OK;
}

}  // namespace mcb

extern "C" mcb_status mcb_ctx_create(int device, mcb_ctx **out) {
  if (!out) return MCB_EINVAL;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return MCB_ECUDA;
  }
  if (device < 0 || device >= n) return MCB_EINVAL;
  mcb_ctx *ctx = new mcb_ctx();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess) {
    cudaGetLastError();
    delete ctx;
    return MCB_ECUDA;
  }
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  int *h = nullptr;
  if (cudaHostAlloc((void **)&h, sizeof(int) * 4, cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer((void **)&ctx->cancel_dev, h, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return MCB_ECUDA;
  }
  h[0] = 0;
  ctx->cancel_host = h;
  *out = ctx;
  return MCB_OK;
}

extern "C" mcb_status mcb_ctx_destroy(mcb_ctx *ctx) {
  if (!ctx) return MCB_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto &b : ctx->pool)
    if (b.ptr) cudaFree(b.ptr);
  if (ctx->heat) mcb_heat_state_destroy(ctx->heat);
  if (ctx->cancel_host) cudaFreeHost((void *)ctx->cancel_host);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return MCB_OK;
}

extern "C" const char *mcb_last_error(const mcb_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

extern "C" volatile int *mcb_cancel_flag(mcb_ctx *ctx) { return ctx ? ctx->cancel_host : nullptr; }
