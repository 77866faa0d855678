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
  {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) ctx->gpuName = prop.name;
    mcb::tune_file_load(ctx);
  }
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

namespace {

// Scattered FP64 atomicAdd throughput: every thread adds to pseudo-random slots of a buffer
// (xorshift64 sequence per thread, multiplicative hash to a slot).
__global__ void atomic_probe_kernel(double *buf, unsigned long long slots, int perThread) {
  unsigned long long x = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x + 1) * 0x9E3779B97F4A7C15ull;
  for (int k = 0; k < perThread; k++) {
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    atomicAdd(buf + (x * 0x2545F4914F6CDD1Dull) % slots, 1.0);
  }
}

}  // namespace

extern "C" mcb_status mcb_probe_atomics(mcb_ctx *ctx, int64_t slots, double *atomicsPerSecond) {
  using namespace mcb;
  if (!ctx) return MCB_EINVAL;
  if (slots < 1 || !atomicsPerSecond) return set_error(ctx, MCB_EINVAL, "slots must be >= 1");
  MCB_CUDA(ctx, cudaSetDevice(ctx->device));
  void *buf = nullptr;
  MCB_TRY(pool_get(ctx, SLOT_PROBE, 8 * (size_t)slots, &buf));
  const int grid = ctx->num_sms * 8, threads = 256, perThread = 256;
  MCB_CUDA(ctx, cudaMemsetAsync(buf, 0, 8 * (size_t)slots, ctx->stream));
  atomic_probe_kernel<<<grid, threads, 0, ctx->stream>>>((double *)buf, (unsigned long long)slots, perThread);
  MCB_CUDA(ctx, cudaEventRecord(ctx->ev0, ctx->stream));
  atomic_probe_kernel<<<grid, threads, 0, ctx->stream>>>((double *)buf, (unsigned long long)slots, perThread);
  MCB_CUDA(ctx, cudaEventRecord(ctx->ev1, ctx->stream));
  MCB_CUDA(ctx, cudaGetLastError());
  MCB_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
  float ms = 0.f;
  MCB_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  *atomicsPerSecond = (double)grid * threads * perThread / (ms * 1e-3);
  return MCB_OK;
}
