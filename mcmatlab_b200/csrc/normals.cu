// Interface normals on the device, behind mcb_interface_normals. The reference computes them
// in its MATLAB host before the MEX call (+MCmatlab/@model/private/getOpticalMediaProperties.m
// :222-244): per class of voxels sharing a refractive index, the 3D Sobel gradient of the
// class indicator (imgradientxyz.m:38-59) divided by the voxel size, optionally smoothed by
// smoothn with a fixed smoothness s = max(1, round(smoothingLengthScale / max d)) (:230-231),
// written into the class's voxels; then (theta, phi) of the gradient (cart2sph, theta =
// pi/2 - elevation).
//
// Sobel: d/dx = D_x (x) K_yz with D = [-1 0 1] and the 3x3 cross kernel
// K = [1 3 1; 3 6 3; 1 3 1] over the two other axes, replicate boundaries.
// Smoothing (smoothn without weights or robust steps): z = IDCT(Gamma DCT(y)) with the
// orthonormal DCT-II along each axis, Gamma = 1 / (1 + s Lambda^2) and
// Lambda = sum_i (2 - 2 cos(pi k_i / n_i)) / h_i^2, h = spacing / max(spacing). Each axis
// transform is a dense n x n matrix applied to every line along that axis (FP32).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "internal.h"

namespace mcb {
namespace {

constexpr int kNrmMaxLine = 1024;  // longest axis the line transforms stage in shared memory

// Sobel gradient of the indicator (riClass[M1 - 1] == cls) along `axis`, divided by h.
__global__ void sobel_kernel(const uint8_t *M1, const int *riClass, int cls, int nx, int ny, int nz, int axis,
                             float invh, float *out) {
  const long long L = (long long)nx * ny * nz;
  const int n[3] = {nx, ny, nz};
  const long long st[3] = {1, nx, (long long)nx * ny};
  const int o1 = axis == 0 ? 1 : 0, o2 = axis == 2 ? 1 : 2;
  const float K[3][3] = {{1.f, 3.f, 1.f}, {3.f, 6.f, 3.f}, {1.f, 3.f, 1.f}};
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < L; v += (long long)gridDim.x * blockDim.x) {
    const int c[3] = {(int)(v % nx), (int)((v / nx) % ny), (int)(v / ((long long)nx * ny))};
    float acc = 0.f;
    for (int a = -1; a <= 1; a++) {
      const int p1 = min(max(c[o1] + a, 0), n[o1] - 1);
      for (int b = -1; b <= 1; b++) {
        const int p2 = min(max(c[o2] + b, 0), n[o2] - 1);
        const long long base = v + (p1 - c[o1]) * st[o1] + (p2 - c[o2]) * st[o2];
        const int lo = max(c[axis] - 1, 0), hi = min(c[axis] + 1, n[axis] - 1);
        const float fl = riClass[M1[base + (lo - c[axis]) * st[axis]] - 1] == cls ? 1.f : 0.f;
        const float fh = riClass[M1[base + (hi - c[axis]) * st[axis]] - 1] == cls ? 1.f : 0.f;
        acc += K[a + 1][b + 1] * (fh - fl);
      }
    }
    out[v] = acc * invh;
  }
}

// out[k] = sum_j CT[j][k] in[j] along `axis`, for every line along that axis (CT: n x n,
// row-major; dct_matrix_t gives it for the forward and the inverse transform). A block stages
// 32 lines (32 consecutive positions of the fastest other axis) in shared memory and computes
// all their outputs.
__global__ void __launch_bounds__(256) axis_transform_kernel(const float *in, float *out, const float *CT, int nx, int ny,
                                                             int nz, int axis) {
  extern __shared__ float tile[];  // [n][33]
  const int n = axis == 0 ? nx : (axis == 1 ? ny : nz);
  const long long sx = 1, sy = nx, sz = (long long)nx * ny;
  // lines: for axis 0 the other coordinates are (y, z) and the 32 lines of a tile are 32
  // consecutive y; for axes 1 and 2 they are 32 consecutive x
  const int wa = axis == 0 ? ny : nx;            // extent of the tiled coordinate
  const int wb = axis == 2 ? ny : nz;            // the remaining coordinate
  const long long stA = axis == 0 ? sy : sx;     // stride of the tiled coordinate
  const long long stB = axis == 2 ? sy : sz;     // stride of the remaining coordinate
  const long long stL = axis == 0 ? sx : (axis == 1 ? sy : sz);
  const int tilesA = (wa + 31) / 32;
  for (long long t = blockIdx.x; t < (long long)tilesA * wb; t += gridDim.x) {
    const int a0 = (int)(t % tilesA) * 32, b = (int)(t / tilesA);
    const int cnt = min(32, wa - a0);
    const long long base = (long long)a0 * stA + (long long)b * stB;
    for (int e = threadIdx.x; e < 32 * n; e += blockDim.x) {
      // axis 0: lines are contiguous, so read along the line; otherwise across the 32 lines
      int l, j;
      if (axis == 0) { l = e / n; j = e - l * n; } else { j = e / 32; l = e - j * 32; }
      if (l < cnt) tile[j * 33 + l] = in[base + l * stA + j * stL];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 32 * n; e += blockDim.x) {
      int l, k;
      if (axis == 0) { l = e / n; k = e - l * n; } else { k = e / 32; l = e - k * 32; }
      if (l < cnt) {
        float acc = 0.f;
        for (int j = 0; j < n; j++) acc = fmaf(__ldg(CT + (size_t)j * n + k), tile[j * 33 + l], acc);
        out[base + l * stA + k * stL] = acc;
      }
    }
    __syncthreads();
  }
}

// y *= 1 / (1 + s Lambda^2) in the DCT basis.
__global__ void gamma_kernel(float *y, int nx, int ny, int nz, float s, float hx2, float hy2, float hz2) {
  const long long L = (long long)nx * ny * nz;
  const float pi = 3.14159265358979f;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < L; v += (long long)gridDim.x * blockDim.x) {
    const int kx = (int)(v % nx), ky = (int)((v / nx) % ny), kz = (int)(v / ((long long)nx * ny));
    const float lam = (2.f - 2.f * cosf(pi * kx / nx)) / hx2 + (2.f - 2.f * cosf(pi * ky / ny)) / hy2 +
                      (2.f - 2.f * cosf(pi * kz / nz)) / hz2;
    y[v] = y[v] / (1.f + s * lam * lam);
  }
}

__global__ void scatter_class_kernel(const uint8_t *M1, const int *riClass, int cls, const float *g, float *G, long long L) {
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < L; v += (long long)gridDim.x * blockDim.x)
    if (riClass[M1[v] - 1] == cls) G[v] = g[v];
}

__global__ void angles_kernel(const float *Gx, const float *Gy, const float *Gz, float *out, long long L) {
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < L; v += (long long)gridDim.x * blockDim.x) {
    const float x = Gx[v], y = Gy[v], z = Gz[v];
    out[2 * v] = 1.57079632679490f - atan2f(z, hypotf(x, y));
    out[2 * v + 1] = atan2f(y, x);
  }
}

// Orthonormal DCT-II matrix of size n, transposed: CT[j][k] = alpha_k cos(pi (2j + 1) k / 2n).
std::vector<float> dct_matrix_t(int n, bool inverse) {
  std::vector<float> m((size_t)n * n);
  for (int k = 0; k < n; k++)
    for (int j = 0; j < n; j++) {
      const double a = k == 0 ? std::sqrt(1.0 / n) : std::sqrt(2.0 / n);
      const double c = a * std::cos(M_PI * (2.0 * j + 1.0) * k / (2.0 * n));
      // forward: out[k] = sum_j C[k][j] in[j], stored as CT[j][k] = C[k][j];
      // inverse: out[j] = sum_k C[k][j] in[k], stored as CT[k][j] = C[k][j]
      if (inverse) m[(size_t)k * n + j] = (float)c;
      else m[(size_t)j * n + k] = (float)c;
    }
  return m;
}

}  // namespace
}  // namespace mcb

extern "C" mcb_status mcb_interface_normals(mcb_ctx *ctx, int32_t nx, int32_t ny, int32_t nz, const uint8_t *M1, int32_t nM,
                                            const int32_t *riClass, int32_t nClass, double dx, double dy, double dz,
                                            double smoothingLengthScale, float *thetaPhi) {
  using namespace mcb;
  if (!ctx) return MCB_EINVAL;
  if (!M1 || !riClass || !thetaPhi) return set_error(ctx, MCB_EINVAL, "NULL argument");
  if (nx < 1 || ny < 1 || nz < 1 || nM < 1 || nM > 256 || nClass < 1)
    return set_error(ctx, MCB_EINVAL, "invalid grid, media or class counts");
  if (!(dx > 0 && dy > 0 && dz > 0)) return set_error(ctx, MCB_EINVAL, "voxel sizes must be positive");
  for (int m = 0; m < nM; m++)
    if (riClass[m] < 0 || riClass[m] >= nClass) return set_error(ctx, MCB_EINVAL, "riClass[%d] out of range", m);
  const bool smooth = smoothingLengthScale > 0;
  if (smooth && std::max(nx, std::max(ny, nz)) > kNrmMaxLine)
    return set_error(ctx, MCB_EINVAL, "smoothing supports axes of at most %d voxels", kNrmMaxLine);
  const long long L = (long long)nx * ny * nz;
  for (long long v = 0; v < L; v++)
    if (M1[v] < 1 || M1[v] > nM) return set_error(ctx, MCB_EINVAL, "M1[%lld] = %d is not a medium in 1..%d", v, (int)M1[v], nM);
  MCB_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const size_t fbytes = 4 * (size_t)L;
  const int dims[3] = {nx, ny, nz};
  size_t matBytes = 0;
  for (int a = 0; a < 3 && smooth; a++) matBytes += 2 * 4 * (size_t)dims[a] * dims[a];
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t bytes = al(L) + al(4 * (size_t)nM) + 6 * al(fbytes) + al(8 * (size_t)L) + al(matBytes) + 4096;
  void *block = nullptr;
  MCB_TRY(pool_get(ctx, SLOT_NORMALS, bytes, &block));
  char *cur = (char *)block;
  auto take = [&](size_t b) {
    char *q = cur;
    cur += al(b);
    return (void *)q;
  };
  uint8_t *dM = (uint8_t *)take(L);
  int *dCls = (int *)take(4 * (size_t)nM);
  float *G[3], *g[3];
  for (int c = 0; c < 3; c++) G[c] = (float *)take(fbytes);
  for (int c = 0; c < 3; c++) g[c] = (float *)take(fbytes);
  float *dOut = (float *)take(8 * (size_t)L);
  float *mats[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // fwd x, inv x, fwd y, ...
  for (int a = 0; a < 3 && smooth; a++) {
    for (int inv = 0; inv < 2; inv++) {
      std::vector<float> m = dct_matrix_t(dims[a], inv == 1);
      mats[2 * a + inv] = (float *)take(4 * m.size());
      MCB_CUDA(ctx, cudaMemcpyAsync(mats[2 * a + inv], m.data(), 4 * m.size(), cudaMemcpyHostToDevice, st));
      MCB_CUDA(ctx, cudaStreamSynchronize(st));  // m is released at the end of the scope
    }
  }
  MCB_CUDA(ctx, cudaMemcpyAsync(dM, M1, L, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(dCls, riClass, 4 * (size_t)nM, cudaMemcpyHostToDevice, st));
  const int grid = ctx->num_sms * 8;
  for (int c = 0; c < 3; c++) MCB_CUDA(ctx, cudaMemsetAsync(G[c], 0xFF, fbytes, st));  // NaN where no class writes
  const double h[3] = {dx, dy, dz};
  const double hmax = std::max(dx, std::max(dy, dz));
  const int s = smooth ? std::max(1, (int)std::lround(smoothingLengthScale / hmax)) : 0;
  size_t maxSmem = 0;
  for (int a = 0; a < 3; a++) maxSmem = std::max(maxSmem, (size_t)dims[a] * 33 * 4);
  if (smooth)
    MCB_CUDA(ctx, cudaFuncSetAttribute(axis_transform_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)maxSmem));
  for (int cls = 0; cls < nClass; cls++) {
    for (int c = 0; c < 3; c++) sobel_kernel<<<grid, 256, 0, st>>>(dM, dCls, cls, nx, ny, nz, c, (float)(1.0 / h[c]), g[c]);
    if (smooth) {
      float *tmp = dOut;  // the angle buffer doubles as scratch until the end
      for (int c = 0; c < 3; c++) {
        float *a = g[c], *b = tmp;
        for (int ax = 0; ax < 3; ax++) {
          const int tiles = ((ax == 0 ? ny : nx) + 31) / 32 * (ax == 2 ? ny : nz);
          axis_transform_kernel<<<std::min(tiles, grid * 4), 256, (size_t)dims[ax] * 33 * 4, st>>>(a, b, mats[2 * ax], nx,
                                                                                                 ny, nz, ax);
          std::swap(a, b);
        }
        gamma_kernel<<<grid, 256, 0, st>>>(a, nx, ny, nz, (float)s, (float)std::pow(dx / hmax, 2), (float)std::pow(dy / hmax, 2),
                                           (float)std::pow(dz / hmax, 2));
        for (int ax = 2; ax >= 0; ax--) {
          const int tiles = ((ax == 0 ? ny : nx) + 31) / 32 * (ax == 2 ? ny : nz);
          axis_transform_kernel<<<std::min(tiles, grid * 4), 256, (size_t)dims[ax] * 33 * 4, st>>>(a, b, mats[2 * ax + 1],
                                                                                                 nx, ny, nz, ax);
          std::swap(a, b);
        }
        // after six transforms the result is back in g[c]
      }
    }
    for (int c = 0; c < 3; c++) scatter_class_kernel<<<grid, 256, 0, st>>>(dM, dCls, cls, g[c], G[c], L);
  }
  angles_kernel<<<grid, 256, 0, st>>>(G[0], G[1], G[2], dOut, L);
  MCB_CUDA(ctx, cudaGetLastError());
  MCB_CUDA(ctx, cudaMemcpyAsync(thetaPhi, dOut, 8 * (size_t)L, cudaMemcpyDeviceToHost, st));
  MCB_CUDA(ctx, cudaStreamSynchronize(st));
  return MCB_OK;
}
