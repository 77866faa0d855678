// Sub-media binning of fluence-rate / temperature / damage dependent optical properties on the
// device: the greedy farthest-point downsampling of getDownsampledParamVals.c:54-202, with the
// same single-precision normalisation (value times the reciprocal of the row's range, as the
// reference's -Ofast build evaluates its loop-invariant division), the same float-accumulated
// squared distances (each term a double square added in double and rounded to float), and the
// same index choices, so bins and representatives match the reference build bit for bit.
//
// The reference scans the points serially. Its running "farthest point" index is carried over
// from one new centre to the next and compared against values that may not have been updated
// yet in the current scan; that choice is reproduced exactly in parallel:
//   m0 = the carried index, d0 = its distance before the scan, d' = the distances after it;
//   k1 = the first k < m0 with d'[k] > d0 (if any); start = k1 if it exists, else m0;
//   m = the first index of the maximum of d' over [start, n); the next centre is m when
//   d'[m] > d'[0], else point 0; m is carried to the next centre.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "internal.h"

namespace mcb {
namespace {

constexpr unsigned long long kNoIndex = ~0ull;

struct DsState {
  float center[3];      // normalised coordinates of the current centre
  long long m0;         // carried running index of the serial scan
  float d0;             // its distance before the current scan
  unsigned long long k1;   // first k < m0 whose updated distance exceeds d0 (atomicMin)
  unsigned long long key;  // (distance bits << 32) | ~index, maximised (first index of the maximum)
  long long pick;       // index of the point that becomes the next centre
};

struct DsArgs {
  const float *par;  // input [3 x n], column-major (mua, mus, g per point)
  float *nv[3];      // normalised coordinates of the varying rows
  float *d;          // squared distance to the nearest centre so far
  uint8_t *bin;      // 1-based nearest centre
  float *centers;    // [3 x n2] normalised centres
  DsState *s;
  long long n;
  int rows;
  int vary[3];       // mua, mus, g take more than one value
  float range[3];
  float inv[3];      // 1 / range
  float meanTerm[3];
};

// float accumulation of a double square, as `acc += pow(a - b, 2)` does with a float acc
__device__ __forceinline__ float add_sq(float acc, float diff) {
  const double t = (double)diff;
  return __double2float_rn(__dadd_rn((double)acc, __dmul_rn(t, t)));
}

__device__ __forceinline__ unsigned long long dist_key(float d, long long k) {
  return ((unsigned long long)__float_as_uint(d) << 32) | (0xFFFFFFFFull - (unsigned long long)k);
}

__device__ __forceinline__ void block_max_key(unsigned long long v, unsigned long long *dst) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_down_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0 && v) atomicMax(dst, v);
}

// normalisation and the distance to the mean; the first centre is the farthest point from it
__global__ void ds_init_kernel(DsArgs a) {
  unsigned long long best = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < a.n; k += (long long)gridDim.x * blockDim.x) {
    float acc = 0.f;
    int r = 0;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (!a.vary[c]) continue;
      const float nvk = a.par[3 * k + c] * a.inv[c];
      a.nv[r][k] = nvk;
      acc = add_sq(acc, nvk - a.meanTerm[c]);
      r++;
    }
    best = max(best, dist_key(acc, k));
  }
  block_max_key(best, &a.s->key);
}

// the distance to the first centre; every point starts in bin 1
__global__ void ds_first_kernel(DsArgs a) {
  const long long c0 = a.s->pick;
  unsigned long long best = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < a.n; k += (long long)gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int r = 0; r < a.rows; r++) acc = add_sq(acc, a.nv[r][k] - a.nv[r][c0]);
    a.d[k] = acc;
    a.bin[k] = 1;
    best = max(best, dist_key(acc, k));
  }
  block_max_key(best, &a.s->key);
}

// one new centre j (0-based): nearest-centre update and the first-exceeding index below m0
__global__ void ds_update_kernel(DsArgs a, int j) {
  const long long m0 = a.s->m0;
  const float d0 = a.s->d0;
  float c[3];
  for (int r = 0; r < a.rows; r++) c[r] = a.s->center[r];
  unsigned long long first = kNoIndex;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < a.n; k += (long long)gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int r = 0; r < a.rows; r++) acc = add_sq(acc, a.nv[r][k] - c[r]);
    float dk = a.d[k];
    if (acc < dk) {
      dk = acc;
      a.d[k] = acc;
      a.bin[k] = (uint8_t)(j + 1);
    }
    if (k < m0 && dk > d0) first = min(first, (unsigned long long)k);
  }
  for (int o = 16; o > 0; o >>= 1) first = min(first, __shfl_down_sync(0xffffffffu, first, o));
  if ((threadIdx.x & 31) == 0 && first != kNoIndex) atomicMin(&a.s->k1, first);
}

// first index of the maximum of the updated distances over [start, n)
__global__ void ds_argmax_kernel(DsArgs a) {
  const long long start = a.s->k1 != kNoIndex ? (long long)a.s->k1 : a.s->m0;
  unsigned long long best = 0;
  for (long long k = start + blockIdx.x * (long long)blockDim.x + threadIdx.x; k < a.n; k += (long long)gridDim.x * blockDim.x)
    best = max(best, dist_key(a.d[k], k));
  block_max_key(best, &a.s->key);
}

// after the first-centre pass (stage 0) or a centre's update (stage 1): record the next centre
__global__ void ds_pick_kernel(DsArgs a, int j, int stage) {
  DsState &s = *a.s;
  const long long m = (long long)(0xFFFFFFFFull - (s.key & 0xFFFFFFFFull));
  long long next;
  if (stage == 0) {
    next = m;     // serial maxDistIdx after the first-centre pass
    s.m0 = 0;     // the carried index starts at 0
  } else {
    next = a.d[m] > a.d[0] ? m : 0;
    s.m0 = m;
  }
  s.d0 = a.d[s.m0];
  s.pick = next;
  for (int r = 0; r < a.rows; r++) {
    s.center[r] = a.nv[r][next];
    a.centers[3 * (j + 1) + r] = s.center[r];
  }
  s.key = 0;
  s.k1 = kNoIndex;
}

__global__ void ds_first_center_kernel(DsArgs a) {
  DsState &s = *a.s;
  const long long m = (long long)(0xFFFFFFFFull - (s.key & 0xFFFFFFFFull));
  s.pick = m;
  for (int r = 0; r < a.rows; r++) a.centers[r] = a.nv[r][m];
  s.key = 0;
  s.k1 = kNoIndex;
}

}  // namespace
}  // namespace mcb

extern "C" mcb_status mcb_downsample_params(mcb_ctx *ctx, const float *paramVals, int64_t n, int32_t nBins,
                                            float *downsampled, uint8_t *binidx) {
  using namespace mcb;
  if (!ctx) return MCB_EINVAL;
  if (!paramVals || !downsampled || !binidx) return set_error(ctx, MCB_EINVAL, "NULL argument");
  if (n < 1 || n > 0x7FFFFFFFll) return set_error(ctx, MCB_EINVAL, "the number of points must be in 1..2^31-1");
  if (nBins < 1 || nBins > 255) return set_error(ctx, MCB_EINVAL, "nBins must be in 1..255 (bins are uint8, 1-based)");
  // per-row extremes and sums in float, in point order, as the reference accumulates them
  float mx[3], mn[3], sm[3];
  for (int c = 0; c < 3; c++) mx[c] = mn[c] = sm[c] = paramVals[c];
  for (long long i = 1; i < n; i++)
    for (int c = 0; c < 3; c++) {
      const float v = paramVals[3 * i + c];
      mx[c] = v > mx[c] ? v : mx[c];
      mn[c] = v < mn[c] ? v : mn[c];
      sm[c] += v;
    }
  DsArgs a{};
  a.n = n;
  a.rows = 0;
  for (int c = 0; c < 3; c++) {
    const bool varying = mx[c] != mn[c];
    a.vary[c] = varying;
    a.range[c] = varying ? mx[c] - mn[c] : 0.f;
    a.inv[c] = varying ? 1.0f / a.range[c] : 0.f;
    const volatile float q = varying ? sm[c] / a.range[c] : 0.f;  // float division, then by the count as a float
    a.meanTerm[c] = varying ? q / (float)n : 0.f;
    a.rows += varying;
  }
  MCB_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t bytes = al(12 * (size_t)n) + 3 * al(4 * (size_t)n) + al(4 * (size_t)n) + al((size_t)n) +
                       al(12 * (size_t)nBins) + al(sizeof(DsState));
  void *block = nullptr;
  MCB_TRY(pool_get(ctx, SLOT_DOWNSAMPLE, bytes, &block));
  char *cur = (char *)block;
  auto take = [&](size_t b) {
    char *q = cur;
    cur += al(b);
    return (void *)q;
  };
  float *dPar = (float *)take(12 * (size_t)n);
  for (int r = 0; r < 3; r++) a.nv[r] = (float *)take(4 * (size_t)n);
  a.d = (float *)take(4 * (size_t)n);
  a.bin = (uint8_t *)take((size_t)n);
  a.centers = (float *)take(12 * (size_t)nBins);
  a.s = (DsState *)take(sizeof(DsState));
  a.par = dPar;
  MCB_CUDA(ctx, cudaMemcpyAsync(dPar, paramVals, 12 * (size_t)n, cudaMemcpyHostToDevice, st));
  DsState s0{};
  s0.k1 = kNoIndex;
  MCB_CUDA(ctx, cudaMemcpyAsync(a.s, &s0, sizeof(DsState), cudaMemcpyHostToDevice, st));
  const int grid = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, (long long)ctx->num_sms * 8));
  if (a.rows > 0) {
    ds_init_kernel<<<grid, 256, 0, st>>>(a);
    ds_first_center_kernel<<<1, 1, 0, st>>>(a);
    ds_first_kernel<<<grid, 256, 0, st>>>(a);
    if (nBins > 1) ds_pick_kernel<<<1, 1, 0, st>>>(a, 0, 0);  // writes the second representative
    for (int j = 1; j < nBins; j++) {
      ds_update_kernel<<<grid, 256, 0, st>>>(a, j);
      if (j + 1 == nBins) break;  // the last centre needs no successor
      ds_argmax_kernel<<<grid, 256, 0, st>>>(a);
      ds_pick_kernel<<<1, 1, 0, st>>>(a, j, 1);
    }
    MCB_CUDA(ctx, cudaGetLastError());
  } else {
    MCB_CUDA(ctx, cudaMemsetAsync(a.bin, 1, (size_t)n, st));  // nothing varies: every point in bin 1
  }
  std::vector<float> cen(3 * (size_t)nBins, 0.f);
  if (a.rows > 0) MCB_CUDA(ctx, cudaMemcpyAsync(cen.data(), a.centers, 12 * (size_t)nBins, cudaMemcpyDeviceToHost, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(binidx, a.bin, (size_t)n, cudaMemcpyDeviceToHost, st));
  MCB_CUDA(ctx, cudaStreamSynchronize(st));
  // rescale the centres; rows that do not vary take the first point's value
  for (int i = 0; i < nBins; i++) {
    int r = 0;
    for (int c = 0; c < 3; c++) {
      const bool varying = mx[c] != mn[c];
      downsampled[3 * i + c] = varying ? cen[3 * (size_t)i + r] * a.range[c] : paramVals[c];
      r += varying;
    }
  }
  return MCB_OK;
}
