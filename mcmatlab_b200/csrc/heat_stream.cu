// Streamed DG-ADI stepper for sm_100a: the forward heat path of mcb_heat_forward and
// mcb_heat_state_* (replacing +MCmatlab/src/finiteElementHeatPropagator.c:688-821) for grids
// whose axes are at most 512 voxels long.
//
// One time step of the reference is six grid passes (substep1a..3b, :249-647). Here it is three
// streaming passes, one per direction, and nothing per voxel is stored besides the state:
//   X pass: explicit stencil of the whole step on T^n (1a, and the half-corrections 2a, 3a),
//           solve along x (1b); writes A1 - S_y with S_y = dt/2 D_y T^n.
//   Y pass: solve along y (2b) on A1 - S_y; writes A2.
//   Z pass: forms S_z = dt/2 D_z T^n from the T^n tile (3a), solves along z on A2 - S_z (3b),
//           adds the Arrhenius damage with the mid-step temperature and the per-medium running
//           maxima, and writes T^{n+1} in place.
// Per voxel and step the passes move 38 bytes of DRAM traffic (X: T, Q, medium, neighbourhood
// code in, A out; Y: A and medium in, A out; Z: A, T and medium in, T out) plus the damage
// increment where damage accumulates.
//
// Tiles are staged in shared memory with TMA (cp.async.bulk.tensor, a two-stage mbarrier
// pipeline in persistent blocks; X tiles are 8 x-lines with their y halo rows and the z
// neighbour rows, Y and Z tiles 16 columns of whole lines, 64-byte swizzled), and the Y and Z
// results leave through TMA stores. f32 grids are described to TMA as pairs (8-byte elements) and
// byte grids as quads, so one box spans a whole x row of up to 512 voxels.
//
// Line coefficients are formed on the fly from the media and the per-call table
// H(d, mi, mj) = dt/2 c(mi, mj, d) (substep1b builds its diagonal the same way, :326-349), and so
// are the LU pivots b'_i = b_i - a_i c_{i-1} / b'_{i-1} of each line: a lane that owns the chunk
// [s, e) of a line starts the pivot recurrence W rows before s from b'_{s-W} := b_{s-W}. The map
// b -> b_i - a_i c_{i-1} / b is increasing, so the started value stays above the true pivot, and its
// relative error shrinks by at most rho = max a c / (1 + a + c) per row (a = H(q, p), c = H(p, q)
// over medium pairs; this uses b'_j >= 1 + c_j, which holds for these diagonally dominant rows).
// The host picks W with rho^W <= 2^-26, below FP32 rounding; where rho >= 1 no bound holds and
// every lane starts at row 0, which is the serial recurrence itself. Each line is then solved by
// a warp (X) or a 16-lane group (Y, Z) as two chunked affine scans (forward elimination, back
// substitution) in registers.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "heat_host.h"
#include "tma.cuh"

namespace mcb {

namespace {

// x-lines per X tile: 8 warps, each solving 32 / G lines (G lanes per line: 16 for x lines up to
// 128 voxels, 32 beyond)
__host__ __device__ constexpr int x_lanes(int nx) { return nx <= 128 ? 16 : 32; }
__host__ __device__ constexpr int x_tile_lines(int nx) { return 8 * (32 / x_lanes(nx)); }
constexpr int kTW = 16;  // columns per Y/Z tile
constexpr int kCodeSink = 64;

// Shared-memory layout of one X-tile stage of kXL lines (byte offsets): T rows y0-1..y0+kXL of
// plane z, T rows y0..y0+kXL-1 of planes z-1 and z+1, Q rows, medium rows y0-1..y0+kXL, code rows.
struct XLayout {
  int offTm, offTp, offQ, offM, offC, stage;
  uint32_t tx;
};

__host__ __device__ inline int up128(int b) { return (b + 127) & ~127; }

__host__ __device__ inline XLayout x_layout(int px, bool q, int kXL) {
  XLayout L;
  const int rowF = 4 * px;
  L.offTm = up128((kXL + 2) * rowF);
  L.offTp = L.offTm + up128(kXL * rowF);
  L.offQ = L.offTp + up128(kXL * rowF);
  L.offM = L.offQ + (q ? up128(kXL * rowF) : 0);
  L.offC = L.offM + up128((kXL + 2) * px);
  const int end = L.offC + up128(kXL * px);
  L.stage = (end + 1023) & ~1023;
  L.tx = (uint32_t)((kXL + 2) * rowF + 2 * kXL * rowF + (q ? kXL * rowF : 0) + (kXL + 2) * px + kXL * px);
  return L;
}

// One Y/Z tile: nb boxes of BN rows (BN a multiple of 16, <= 256) of 16 columns; f32 tiles are
// 64-byte swizzled rows, the medium tile plain 16-byte rows.
struct YZLayout {
  int nb, BN, offM, offT, stage;
  uint32_t tx;
};

__host__ __device__ inline YZLayout yz_layout(int n, bool zpass) {
  YZLayout L;
  L.nb = n > 256 ? 2 : 1;
  L.BN = (((n + L.nb - 1) / L.nb) + 15) & ~15;
  const int rows = L.nb * L.BN;
  L.offM = rows * 64;
  L.offT = L.offM + ((rows * 16 + 1023) & ~1023);
  L.stage = L.offT + (zpass ? rows * 64 : 0);
  L.tx = (uint32_t)(rows * (64 + 16 + (zpass ? 64 : 0)));
  return L;
}

// Byte offset of element (row i, column j) of a 64-byte-swizzled f32 tile (TMA SWIZZLE_64B:
// address bits 4-5 are XORed with bits 7-8).
__device__ __forceinline__ int swz(int i, int j) { return i * 64 + ((((j >> 2) ^ (i >> 1)) & 3) << 4) + ((j & 3) << 2); }

}  // namespace

struct StreamDev {
  int nx, ny, nz, nM, px, W;
  long long sxy;  // px * ny
  float *T, *A;
  const uint8_t *M, *code;
  const float *Q;     // or nullptr (light off)
  float *dOmega;      // or nullptr
  const float *H;     // [3][nM][nM]: H[d*nM*nM + mj*nM + mi] = dt/2 c(mi, mj, d)
  const float4 *Hd;   // [nM] diagonal {H(m,m,0), H(m,m,1), H(m,m,2), 0}
  const float4 *Hs;   // [nM] 1 / b*(m, d): inverse fixed-point pivot of a line of medium m along d
  const float2 *dmg;  // [nM] Arrhenius exponent about the base temperature
  float T0, dt;
  unsigned int *maxEnc;
  int hs;
  double base;
  int nS;
  const double *sIdx, *sW;
  double *sens;
  int *stepCounter;
  int *err;
  // per-call tables of the homogeneous lane chunks (medium + 1, or 0): X pass [nz][ny][lanes],
  // column-layout Y and Z passes [nOther][chunks][px] (stream_setup)
  const uint8_t *uniX, *uniY, *uniZ;
};

namespace {

// First 1024-byte boundary at or after p in shared memory (the swizzle pattern of the Y/Z tiles
// is a function of the address bits, so tiles start on such a boundary; the dynamic allocation
// carries 1 KB of slack for it).
__device__ __forceinline__ unsigned char *align1024(unsigned char *p) {
  const uint32_t a = smem_addr(p);
  return p + (((a + 1023u) & ~1023u) - a);
}

// Reciprocal of a pivot (>= 1): the approximate reciprocal refined by one Newton step, within
// about half an ulp; the pivots' rounding enters every step of long runs, so the bare 1-ulp
// approximation is not used.
__device__ __forceinline__ float frcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return fmaf(r, fmaf(-x, r, 1.f), r);
}

__device__ __forceinline__ float hcoef(const StreamDev &h, int d, int mi, int mj) {
  return __ldg(h.H + (d * h.nM + mj) * h.nM + mi);
}

// Sensor interpolation (recordTempSensors, finiteElementHeatPropagator.c:652-664) on the pitched
// state; sensor corner indices are dense 0-based linear indices.
__device__ void record_sensors_p(const StreamDev &h, int col) {
  for (int j = threadIdx.x; j < h.nS; j += blockDim.x) {
    const long long li = (long long)h.sIdx[j];
    const long long nxy = (long long)h.nx * h.ny;
    const long long iz = li / nxy, r = li - iz * nxy, iy = r / h.nx, ix = r - iy * h.nx;
    const long long i = ix + iy * h.px + iz * h.sxy, sx = 1, sy = h.px, sz = h.sxy;
    const double wx = h.sW[j], wy = h.sW[j + h.nS], wz = h.sW[j + 2 * h.nS];
    auto T = [&](long long k) { return (double)h.T[k] + h.base; };
    h.sens[j + (long long)col * h.nS] =
        (1 - wx) * (1 - wy) * (1 - wz) * T(i) + (1 - wx) * (1 - wy) * wz * T(i + sz) + (1 - wx) * wy * (1 - wz) * T(i + sy) +
        (1 - wx) * wy * wz * T(i + sy + sz) + wx * (1 - wy) * (1 - wz) * T(i + sx) + wx * (1 - wy) * wz * T(i + sx + sz) +
        wx * wy * (1 - wz) * T(i + sx + sy) + wx * wy * wz * T(i + sx + sy + sz);
  }
}

// Pivots of a lane's `count` rows from their coefficients a[k], c[k] (rows s+k), given the
// started pivot of row s-1 (bp, its coupling cprev; bp = 0 for s = 0); the remaining slots become
// identity maps (chunk_solve).
template <int K>
__device__ __forceinline__ void lane_pivots(const float (&a)[K], const float (&c)[K], float bp, float cprev, int count,
                                            float (&fm)[K], float (&bm)[K], float (&ib)[K]) {
  float ibp = bp > 0.f ? frcp(bp) : 0.f;
#pragma unroll
  for (int k = 0; k < K; k++) {
    if (k < count) {
      const float b = fmaf(-a[k] * cprev, ibp, 1.f + a[k] + c[k]);
      ib[k] = frcp(b);
      fm[k] = a[k] * ibp;
      bm[k] = c[k] * ib[k];
      ibp = ib[k];
      cprev = c[k];
    } else {
      fm[k] = bm[k] = 1.f;
      ib[k] = 0.f;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// X pass
// ---------------------------------------------------------------------------------------------

// One x-line (tile row l, grid row y of plane z) solved by the G lanes of an aligned group; an
// invalid line (past the grid's last row) only takes part in the group's shuffles.
template <int K, int G>
__device__ __forceinline__ void x_line(const StreamDev &h, unsigned char *b, const XLayout &lay, int l, int y, int z, int lane,
                                       bool valid) {
  const int nx = h.nx, px = h.px;
  const float *Tc = reinterpret_cast<const float *>(b) + (l + 1) * px;
  float *rowA = reinterpret_cast<float *>(b + lay.offTm) + l * px;  // z-1 row, then the line's a_i
  float *rowC = reinterpret_cast<float *>(b + lay.offTp) + l * px;  // z+1 row, then the line's c_i
  const float *Qr = h.Q ? reinterpret_cast<const float *>(b + lay.offQ) + l * px : nullptr;
  const uint8_t *Mc = b + lay.offM + (l + 1) * px;
  const uint8_t *Cr = b + lay.offC + l * px;
  const int s = valid ? lane * K : nx;  // an invalid line holds no rows
  const long long rowBase = (long long)y * px + (long long)z * h.sxy;
  const bool yLo = y > 0, yHi = y < h.ny - 1, zLo = z > 0, zHi = z < h.nz - 1;
  float r[K], sy[K], ca[K], cc[K];
#pragma unroll
  for (int k = 0; k < K; k++) r[k] = sy[k] = ca[k] = cc[k] = 0.f;
  const bool act = s < nx;
  if (act) {
    float tprev = s > 0 ? Tc[s - 1] : 0.f;
#pragma unroll
    for (int k4 = 0; k4 < K / 4; k4++) {
      const int x4 = s + 4 * k4;
      const float4 t4 = *reinterpret_cast<const float4 *>(Tc + x4);
      const float4 ym4 = *reinterpret_cast<const float4 *>(Tc - px + x4);
      const float4 yp4 = *reinterpret_cast<const float4 *>(Tc + px + x4);
      const float4 zm4 = *reinterpret_cast<const float4 *>(rowA + x4);
      const float4 zp4 = *reinterpret_cast<const float4 *>(rowC + x4);
      const float4 q4 = Qr ? *reinterpret_cast<const float4 *>(Qr + x4) : make_float4(0.f, 0.f, 0.f, 0.f);
      const float tnext = x4 + 4 < nx ? Tc[x4 + 4] : 0.f;
      const uint32_t m4 = *reinterpret_cast<const uint32_t *>(Mc + x4);
      const uint32_t c4 = *reinterpret_cast<const uint32_t *>(Cr + x4);
      const float tv[4] = {t4.x, t4.y, t4.z, t4.w}, ymv[4] = {ym4.x, ym4.y, ym4.z, ym4.w},
                  ypv[4] = {yp4.x, yp4.y, yp4.z, yp4.w}, zmv[4] = {zm4.x, zm4.y, zm4.z, zm4.w},
                  zpv[4] = {zp4.x, zp4.y, zp4.z, zp4.w}, qv[4] = {q4.x, q4.y, q4.z, q4.w};
      float av[4], cv[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int k = 4 * k4 + u, x = x4 + u;
        const float t = tv[u];
        const float tL = u ? tv[u - 1] : tprev;
        const float tR = u < 3 ? tv[u + 1] : tnext;
        const int m = (m4 >> (8 * u)) & 255, code = (c4 >> (8 * u)) & 255;
        float a = 0.f, c = 0.f, dy = 0.f, dz = 0.f, rr = 0.f;
        if (x < nx) {
          rr = t;
          if (!(code & kCodeSink)) {
            // faces to missing neighbours carry no coefficient; faces to another medium look the
            // pair up (rare: interfaces), the others take the medium's diagonal
            const float4 H = __ldg(h.Hd + m);
            a = x > 0 ? H.x : 0.f;
            c = x < nx - 1 ? H.x : 0.f;
            float aym = yLo ? H.y : 0.f, ayp = yHi ? H.y : 0.f, azm = zLo ? H.z : 0.f, azp = zHi ? H.z : 0.f;
            if (code & 63) {
              const long long p = rowBase + x;
              if (code & 1) a = hcoef(h, 0, m, Mc[x - 1]);
              if (code & 2) c = hcoef(h, 0, m, Mc[x + 1]);
              if (code & 4) aym = hcoef(h, 1, m, Mc[x - px]);
              if (code & 8) ayp = hcoef(h, 1, m, Mc[x + px]);
              if (code & 16) azm = hcoef(h, 2, m, h.M[p - h.sxy]);
              if (code & 32) azp = hcoef(h, 2, m, h.M[p + h.sxy]);
            }
            dy = aym * (ymv[u] - t) + ayp * (ypv[u] - t);
            dz = azm * (zmv[u] - t) + azp * (zpv[u] - t);
            // rhs of 1a: T + dt (Q + D_y T + D_z T) + dt/2 D_x T, with dt D_y T = 2 S_y
            rr = t + h.dt * qv[u] + 2.f * (dy + dz) + (a * (tL - t) + c * (tR - t));
          }
        }
        r[k] = rr;
        sy[k] = dy;
        ca[k] = a;
        cc[k] = c;
        av[u] = a;
        cv[u] = c;
      }
      // the z-1 / z+1 values of these rows have been used: the rows now hold the coefficients
      *reinterpret_cast<float4 *>(rowA + x4) = make_float4(av[0], av[1], av[2], av[3]);
      *reinterpret_cast<float4 *>(rowC + x4) = make_float4(cv[0], cv[1], cv[2], cv[3]);
      tprev = tv[3];
    }
  }
  __syncwarp();
  float fm[K], bm[K], ib[K];
  // homogeneous lanes: rows s - W - 1 .. e of the line all of one medium (code bit 1 clear on rows
  // s - W - 1 .. e - 1), none heat-sinked, none a line end. Their exact pivots lie within rho^(W+1)
  // of the medium's fixed point b*, so every row takes a = c = h and 1 / b' = 1 / b*.
  const int e = min(s + K, nx);
  const int um = act ? h.uniX[((long long)z * h.ny + y) * G + lane] : 0;  // uni_x_kernel
  const bool uni = um != 0;
  if (uni) {
    const int m0 = um - 1;
    const float ibs = __ldg(&h.Hs[m0].x), f = __ldg(&h.Hd[m0].x) * ibs;
#pragma unroll
    for (int k = 0; k < K; k++) {
      const bool in = k < e - s;
      fm[k] = in ? f : 1.f;
      bm[k] = in ? f : 1.f;
      ib[k] = in ? ibs : 0.f;
    }
  } else {
    // started pivot of row s-1 (W rows of the recurrence before the lane's chunk)
    float bp = 0.f, cprev = 0.f;
    if (act && s > 0) {
      const int i0 = max(0, s - max(h.W, 1));
      bp = 1.f + rowA[i0] + rowC[i0];
      for (int i = i0 + 1; i < s; i++) {
        const float a = rowA[i];
        bp = fmaf(-a * rowC[i - 1], frcp(bp), 1.f + a + rowC[i]);
      }
      cprev = rowC[s - 1];
    }
    lane_pivots<K>(ca, cc, bp, cprev, min(max(nx - s, 0), K), fm, bm, ib);
  }
  chunk_solve<K, G>(r, fm, bm, ib, lane);
  if (act) {
#pragma unroll
    for (int k4 = 0; k4 < K / 4; k4++) {
      const int x4 = s + 4 * k4;
      *reinterpret_cast<float4 *>(h.A + rowBase + x4) =
          make_float4(r[4 * k4] - sy[4 * k4], r[4 * k4 + 1] - sy[4 * k4 + 1], r[4 * k4 + 2] - sy[4 * k4 + 2],
                      r[4 * k4 + 3] - sy[4 * k4 + 3]);
    }
  }
}

template <int K, int G>
__global__ void __launch_bounds__(256, G == 16 ? 3 : 2)
    sx_kernel(const __grid_constant__ CUtensorMap mTh, const __grid_constant__ CUtensorMap mTr,
              const __grid_constant__ CUtensorMap mQr, const __grid_constant__ CUtensorMap mMh,
              const __grid_constant__ CUtensorMap mCr, const StreamDev h) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem = align1024(smem_raw);
  constexpr int kXL = 8 * (32 / G);
  const XLayout lay = x_layout(h.px, h.Q != nullptr, kXL);
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * lay.stage);
  const int yTiles = (h.ny + kXL - 1) / kXL;
  const int nTiles = yTiles * h.nz;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (blockIdx.x == 0 && h.nS > 0) record_sensors_p(h, *h.stepCounter);
  auto issue = [&](int tile, int st) {
    unsigned char *b = smem + st * lay.stage;
    const int y0 = (tile % yTiles) * kXL, z = tile / yTiles;
    mbar_expect_tx(&bar[st], lay.tx);
    tma_load_3d(b, &mTh, 0, y0 - 1, z, &bar[st]);
    tma_load_3d(b + lay.offTm, &mTr, 0, y0, z - 1, &bar[st]);
    tma_load_3d(b + lay.offTp, &mTr, 0, y0, z + 1, &bar[st]);
    if (h.Q) tma_load_3d(b + lay.offQ, &mQr, 0, y0, z, &bar[st]);
    tma_load_3d(b + lay.offM, &mMh, 0, y0 - 1, z, &bar[st]);
    tma_load_3d(b + lay.offC, &mCr, 0, y0, z, &bar[st]);
  };
  if (threadIdx.x == 0) {
    for (int k = 0; k < 2; k++) {
      const int t = blockIdx.x + k * gridDim.x;
      if (t < nTiles) issue(t, k);
    }
  }
  const int lane = threadIdx.x & (G - 1), l = (threadIdx.x >> 5) * (32 / G) + ((threadIdx.x & 31) / G);
  int it = 0;
  for (int tile = blockIdx.x; tile < nTiles; tile += gridDim.x, ++it) {
    const int st = it & 1;
    if (!mbar_wait_bounded(&bar[st], (it >> 1) & 1)) {
      if (threadIdx.x == 0) atomicExch(h.err, 1);
      return;
    }
    unsigned char *b = smem + st * lay.stage;
    const int y0 = (tile % yTiles) * kXL, z = tile / yTiles;
    // lines past the grid's last row still take part in the group's shuffles (an empty line)
    x_line<K, G>(h, b, lay, l, min(y0 + l, h.ny - 1), z, lane, y0 + l < h.ny);
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      const int nt = tile + 2 * gridDim.x;
      if (nt < nTiles) issue(nt, st);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Y and Z passes
// ---------------------------------------------------------------------------------------------

template <int K, int G, bool ZP>
__global__ void __launch_bounds__(16 * G, 2)
    syz_kernel(const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mM,
               const __grid_constant__ CUtensorMap mT, const StreamDev h) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem = align1024(smem_raw);
  __shared__ unsigned int mloc[256];
  const int nx = h.nx;
  const int n = ZP ? h.nz : h.ny;
  const int d = ZP ? 2 : 1;
  const YZLayout lay = yz_layout(n, ZP);
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + 2 * lay.stage);
  const int xTiles = (nx + kTW - 1) / kTW;
  const int nOther = ZP ? h.ny : h.nz;
  const int nTiles = xTiles * nOther;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (ZP)
    for (int k = threadIdx.x; k < h.nM; k += blockDim.x) mloc[k] = 0u;
  __syncthreads();
  auto issue = [&](int tile, int st) {
    unsigned char *b = smem + st * lay.stage;
    const int x0 = (tile % xTiles) * kTW, o = tile / xTiles;
    mbar_expect_tx(&bar[st], lay.tx);
    for (int k = 0; k < lay.nb; k++) {
      const int r0 = k * lay.BN;
      if (ZP) {
        tma_load_3d(b + r0 * 64, &mA, x0 / 2, o, r0, &bar[st]);
        tma_load_3d(b + lay.offM + r0 * 16, &mM, x0 / 4, o, r0, &bar[st]);
        tma_load_3d(b + lay.offT + r0 * 64, &mT, x0 / 2, o, r0, &bar[st]);
      } else {
        tma_load_3d(b + r0 * 64, &mA, x0 / 2, r0, o, &bar[st]);
        tma_load_3d(b + lay.offM + r0 * 16, &mM, x0 / 4, r0, o, &bar[st]);
      }
    }
  };
  if (threadIdx.x == 0) {
    for (int k = 0; k < 2; k++) {
      const int t = blockIdx.x + k * gridDim.x;
      if (t < nTiles) issue(t, k);
    }
  }
  const int j = threadIdx.x / G, g = threadIdx.x % G;
  const int kk = (n + G - 1) / G;
  const int s = g * kk, e = min(s + kk, n);
  const int dn = d * h.nM * h.nM;
  int curM = -1;
  unsigned int curMax = 0u;
  int it = 0;
  for (int tile = blockIdx.x; tile < nTiles; tile += gridDim.x, ++it) {
    const int st = it & 1;
    if (!mbar_wait_bounded(&bar[st], (it >> 1) & 1)) {
      if (threadIdx.x == 0) atomicExch(h.err, 2);
      break;
    }
    unsigned char *b = smem + st * lay.stage;
    float *At = reinterpret_cast<float *>(b);
    const uint8_t *Mt = b + lay.offM;
    const float *Tt = reinterpret_cast<const float *>(b + lay.offT);
    const int x0 = (tile % xTiles) * kTW, o = tile / xTiles;
    const int x = x0 + j;
    const bool colValid = x < nx;
    // the whole line is heat-sinked when it lies on a boundary face of the other two axes
    const bool lineSink = h.hs && (x == 0 || x == nx - 1 || o == 0 || o == nOther - 1);
    auto at = [&](const float *tile_, int i) { return *reinterpret_cast<const float *>(reinterpret_cast<const unsigned char *>(tile_) + swz(i, j)); };
    auto med = [&](int i) { return (int)Mt[i * kTW + j]; };
    auto coef = [&](int i, int mi, int mprev, int mnext, float &a, float &c) {
      a = c = 0.f;
      if (lineSink || (h.hs && (i == 0 || i == n - 1))) return;
      const float hm = __ldg(h.H + dn + mi * h.nM + mi);
      if (i > 0) a = mprev == mi ? hm : __ldg(h.H + dn + mprev * h.nM + mi);
      if (i < n - 1) c = mnext == mi ? hm : __ldg(h.H + dn + mnext * h.nM + mi);
    };
    float r[K], ca[K], cc[K];
    {
      int mprev = s > 0 ? med(s - 1) : 0, mcur = med(min(s, n - 1));
      float tprev = 0.f, tcur = 0.f;
      if (ZP) {
        tprev = s > 0 ? at(Tt, s - 1) : 0.f;
        tcur = at(Tt, min(s, n - 1));
      }
#pragma unroll
      for (int k = 0; k < K; k++) {
        const int i = s + k;
        r[k] = ca[k] = cc[k] = 0.f;
        if (k < kk && i < e) {
          const int mnext = i + 1 < n ? med(i + 1) : 0;
          float a, c;
          coef(i, mcur, mprev, mnext, a, c);
          float rhs = at(At, i);
          if (ZP) {
            const float tnext = i + 1 < n ? at(Tt, i + 1) : 0.f;
            rhs -= a * (tprev - tcur) + c * (tnext - tcur);  // A2 - S_z (3a)
            tprev = tcur;
            tcur = tnext;
          }
          r[k] = colValid ? rhs : 0.f;
          ca[k] = a;
          cc[k] = c;
          mprev = mcur;
          mcur = mnext;
        }
      }
    }
    float bp = 0.f, cprev = 0.f;
    if (s > 0 && s < n) {
      const int i0 = max(0, s - max(h.W, 1));
      int mp = i0 > 0 ? med(i0 - 1) : 0, mc = med(i0);
      float a, c;
      int mn = med(i0 + 1);
      coef(i0, mc, mp, mn, a, c);
      bp = 1.f + a + c;
      for (int i = i0 + 1; i < s; i++) {
        mp = mc;
        mc = mn;
        mn = i + 1 < n ? med(i + 1) : 0;
        const float cpre = c;
        coef(i, mc, mp, mn, a, c);
        bp = fmaf(-a * cpre, frcp(bp), 1.f + a + c);
      }
      cprev = c;
    }
    float fm[K], bm[K], ib[K];
    lane_pivots<K>(ca, cc, bp, cprev, max(e - s, 0), fm, bm, ib);
    chunk_solve<K, G>(r, fm, bm, ib, g);
#pragma unroll
    for (int k = 0; k < K; k++) {
      const int i = s + k;
      if (k < kk && i < e) *reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(At) + swz(i, j)) = colValid ? r[k] : 0.f;
    }
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int k = 0; k < lay.nb; k++) {
        const int r0 = k * lay.BN;
        if (ZP) tma_store_3d(&mT, x0 / 2, o, r0, b + r0 * 64);
        else tma_store_3d(&mA, x0 / 2, r0, o, b + r0 * 64);
      }
      tma_store_commit();
    }
    if (ZP) {
      // damage with the mid-step temperature (finiteElementHeatPropagator.c:600-602) and the
      // running per-medium maxima, over the tile in x-contiguous order
      for (int q = threadIdx.x; q < kTW * n; q += blockDim.x) {
        const int i = q >> 4, jj = q & 15, xx = x0 + jj;
        if (xx >= nx) continue;
        const int off = i * 64 + ((((jj >> 2) ^ (i >> 1)) & 3) << 4) + ((jj & 3) << 2);
        const float tnew = *reinterpret_cast<const float *>(b + off);
        const int m = Mt[i * kTW + jj];
        const float2 dg = h.dmg[m];
        if (h.dOmega && dg.y > 0.f) {
          // log A - E / (R (T0 + d)) = x0 + (E/R) d / (T0 (T0 + d)), x0 formed in FP64 per call
          const float told = *reinterpret_cast<const float *>(b + lay.offT + off);
          const float dm = 0.5f * (tnew + told);
          h.dOmega[xx + (long long)o * h.px + (long long)i * h.sxy] += h.dt * expf(dg.x + dg.y * dm / (h.T0 * (h.T0 + dm)));
        }
        const unsigned int enc = enc_max((float)((double)tnew + h.base));
        if (m != curM) {
          if (curM >= 0) atomicMax(&mloc[curM], curMax);
          curM = m;
          curMax = enc;
        } else if (enc > curMax) {
          curMax = enc;
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int nt = tile + 2 * gridDim.x;
      tma_store_wait_read();
      if (nt < nTiles) {
        fence_proxy_async();
        issue(nt, st);
      }
    }
  }
  if (threadIdx.x == 0) tma_store_wait_all();
  if (ZP) {
    if (curM >= 0) atomicMax(&mloc[curM], curMax);
    __syncthreads();
    for (int k = threadIdx.x; k < h.nM; k += blockDim.x)
      if (mloc[k]) atomicMax(&h.maxEnc[k], mloc[k]);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(h.stepCounter, 1);
  }
}

// ---------------------------------------------------------------------------------------------
// Y and Z passes, column layout (lines up to 320 rows)
// ---------------------------------------------------------------------------------------------

// A block of G warps owns 32 consecutive x columns of whole lines (Y: one z, Z: one y); lane l
// is column x0 + l in every warp, and warp w holds rows [w*kk, w*kk + kk) of its column in
// registers (kk = ceil(n / G) <= K). The tiles (A, media, and for Z the T^n rows) are
// prefetched with TMA into a two-stage shared-memory pipeline of plain 128-byte rows (lane l reads
// bank l), so the next tile streams in while this one is solved. The chunk maps of both scans are
// combined across the warps through shared memory (G - 1 fused multiply-adds per carry). The Z
// pass forms S_z from the T^n rows it holds and adds the damage and the running maxima of its
// rows before writing T^{n+1}; results leave with coalesced row stores.
struct ColLayout {
  int nb, BN, offM, offT, stage, sums;
  uint32_t tx;
};

__host__ __device__ inline ColLayout col_layout(int n, bool zpass, int G) {
  ColLayout L;
  L.nb = n > 256 ? 2 : 1;
  L.BN = (((n + L.nb - 1) / L.nb) + 3) & ~3;  // multiple of 4: every box starts 128-byte aligned
  const int rows = L.nb * L.BN;
  L.offM = (rows * 128 + 127) & ~127;
  L.offT = L.offM + ((rows * 32 + 127) & ~127);
  L.stage = (L.offT + (zpass ? rows * 128 : 0) + 1023) & ~1023;
  L.sums = 2 * L.stage;
  L.tx = (uint32_t)(rows * (128 + 32 + (zpass ? 128 : 0)));
  (void)G;
  return L;
}

template <int K, bool ZP, int MAXT>
__global__ void __launch_bounds__(MAXT, MAXT <= 256 ? 3 : MAXT <= 512 ? 2 : 1)
    scol_kernel(const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mM,
                const __grid_constant__ CUtensorMap mT, const StreamDev h, int G) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem = align1024(smem_raw);
  __shared__ unsigned int mloc[256];
  __shared__ float2 sdmg[256];  // Arrhenius exponent terms per medium (y = 0: no damage)
  __shared__ float hd[256];   // H(m, m) of this direction
  __shared__ float hsv[256];  // 1 / b*(m) of this direction
  const int n = ZP ? h.nz : h.ny;
  const ColLayout lay = col_layout(n, ZP, G);
  float2 *sums = reinterpret_cast<float2 *>(smem + lay.sums);  // [2 tiles][2 scans][G][32] chunk maps (A, B)
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + lay.sums + 4 * G * 32 * sizeof(float2));
  const long long st = ZP ? h.sxy : (long long)h.px;
  const int nOther = ZP ? h.ny : h.nz;
  const int nx = h.nx, nM = h.nM;
  const int xTiles = (nx + 31) >> 5;
  const int nTiles = xTiles * nOther;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int kk = (n + G - 1) / G;
  const int s = min(w * kk, n), e = min(s + kk, n), cnt = e - s;
  const float *Hl = h.H + (ZP ? 2 : 1) * nM * nM;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  for (int k = threadIdx.x; k < nM; k += blockDim.x) {
    hd[k] = Hl[k * nM + k];
    const float4 f4 = h.Hs[k];
    hsv[k] = ZP ? f4.z : f4.y;
    if (ZP) {
      mloc[k] = 0u;
      sdmg[k] = h.dOmega ? h.dmg[k] : make_float2(0.f, 0.f);
    }
  }
  __syncthreads();
  auto issue = [&](int tile, int stg) {
    unsigned char *b = smem + stg * lay.stage;
    const int x0 = (tile % xTiles) << 5, o = tile / xTiles;
    mbar_expect_tx(&bar[stg], lay.tx);
    for (int k = 0; k < lay.nb; k++) {
      const int r0 = k * lay.BN;
      if (ZP) {
        tma_load_3d(b + r0 * 128, &mA, x0 / 2, o, r0, &bar[stg]);
        tma_load_3d(b + lay.offM + r0 * 32, &mM, x0 / 4, o, r0, &bar[stg]);
        tma_load_3d(b + lay.offT + r0 * 128, &mT, x0 / 2, o, r0, &bar[stg]);
      } else {
        tma_load_3d(b + r0 * 128, &mA, x0 / 2, r0, o, &bar[stg]);
        tma_load_3d(b + lay.offM + r0 * 32, &mM, x0 / 4, r0, o, &bar[stg]);
      }
    }
  };
  if (threadIdx.x == 0) {
    for (int k = 0; k < 2; k++) {
      const int t = blockIdx.x + k * gridDim.x;
      if (t < nTiles) issue(t, k);
    }
  }
  int curM = -1;
  float curMax = 0.f;  // running maximum of the deviation in medium curM
  int it = 0;
  for (int tile = blockIdx.x; tile < nTiles; tile += gridDim.x, ++it) {
    const int stg = it & 1;
    if (!mbar_wait_bounded(&bar[stg], (it >> 1) & 1)) {
      if (threadIdx.x == 0) atomicExch(h.err, 3);
      break;
    }
    const unsigned char *b = smem + stg * lay.stage;
    const float *At = reinterpret_cast<const float *>(b);
    const uint8_t *Mt = b + lay.offM;
    const float *Tt = reinterpret_cast<const float *>(b + lay.offT);
    float2 *sF = sums + (stg * 2 * G) * 32, *sB = sF + G * 32;
    const int x = ((tile % xTiles) << 5) + l, o = tile / xTiles;
    const bool colValid = x < nx;
    const long long base = x + (ZP ? (long long)o * h.px : (long long)o * h.sxy);
    const bool lineSink = h.hs && (x == 0 || x == nx - 1 || o == 0 || o == nOther - 1);
    const int nv = colValid ? cnt : 0;  // rows of this lane
    auto med = [&](int i) { return (int)Mt[i * 32 + l]; };
    // coupling of row i (medium mi) to a neighbour of medium mj: the diagonal from shared memory,
    // the pair table only across an interface
    auto hc = [&](int mi, int mj) { return mi == mj ? hd[mi] : __ldg(Hl + mj * nM + mi); };
    auto rowSink = [&](int i) { return lineSink || (h.hs && (i == 0 || i == n - 1)); };
    float r[K], fm[K], bm[K], ib[K];
    float A = 0.f, B = 1.f;
    // homogeneous lanes: rows s - W - 1 .. e all of one medium, none heat-sinked, none a line end.
    // Their exact pivots lie within rho^(W+1) of the medium's fixed point b* (the recurrence
    // contracts towards it from any start), so every row takes a = c = h, 1 / b' = 1 / b*.
    // (uni_col_kernel forms the answer once per call)
    const int um = nv > 0 ? (ZP ? h.uniZ : h.uniY)[((long long)o * G + w) * h.px + x] : 0;
    const bool uni = um != 0;
    const int m0 = um - 1;
    if (uni) {
      const float h0 = hd[m0], ibs = hsv[m0], f = h0 * ibs;
      float tPrev = ZP ? Tt[(s - 1) * 32 + l] : 0.f, tCur = ZP ? Tt[s * 32 + l] : 0.f;
#pragma unroll
      for (int k = 0; k < K; k++) {
        fm[k] = bm[k] = 1.f;
        ib[k] = r[k] = 0.f;
        if (k < nv) {
          const int i = s + k;
          float rhs = At[i * 32 + l];
          if (ZP) {
            const float tNext = Tt[(i + 1) * 32 + l];  // i + 1 <= e <= n - 1
            rhs -= h0 * ((tPrev - tCur) + (tNext - tCur));  // A2 - S_z (3a)
            tPrev = tCur;
            tCur = tNext;
          }
          fm[k] = bm[k] = f;
          ib[k] = ibs;
          r[k] = rhs;
          A = fmaf(f, A, rhs);
          B *= f;
        }
      }
    } else {
    // started pivot of row s-1 from W rows of the recurrence before the chunk
    float bp = 0.f, cprev = 0.f;
    if (nv > 0 && s > 0) {
      const int i0 = max(0, s - max(h.W, 1));
      int mp = i0 > 0 ? med(i0 - 1) : 0, mc = med(i0), mn = med(i0 + 1);
      const bool rs0 = rowSink(i0);
      float a = (rs0 || i0 == 0) ? 0.f : hc(mc, mp), c = rs0 ? 0.f : hc(mc, mn);
      bp = 1.f + a + c;
      for (int i = i0 + 1; i < s; i++) {
        mp = mc;
        mc = mn;
        mn = med(i + 1);
        const float cpre = c;
        const bool rs = rowSink(i);
        a = rs ? 0.f : hc(mc, mp);
        c = rs ? 0.f : hc(mc, mn);
        bp = fmaf(-a * cpre, frcp(bp), 1.f + a + c);
      }
      cprev = c;
    }
    // one pass over the lane's rows: coefficients, (Z) A2 - S_z, pivots, forward chunk map
    float ibp = bp > 0.f ? frcp(bp) : 0.f;
    int mPrev = (nv > 0 && s > 0) ? med(s - 1) : 0, mCur = nv > 0 ? med(s) : 0;
    float tPrev = (ZP && nv > 0 && s > 0) ? Tt[(s - 1) * 32 + l] : 0.f, tCur = (ZP && nv > 0) ? Tt[s * 32 + l] : 0.f;
#pragma unroll
    for (int k = 0; k < K; k++) {
      fm[k] = bm[k] = 1.f;
      ib[k] = r[k] = 0.f;
      if (k < nv) {
        const int i = s + k;
        const int mNext = i + 1 < n ? med(i + 1) : 0;
        const bool rs = rowSink(i);
        const float a = (rs || i == 0) ? 0.f : hc(mCur, mPrev);
        const float c = (rs || i == n - 1) ? 0.f : hc(mCur, mNext);
        float rhs = At[i * 32 + l];
        if (ZP) {
          const float tNext = i + 1 < n ? Tt[(i + 1) * 32 + l] : 0.f;
          rhs -= a * (tPrev - tCur) + c * (tNext - tCur);  // A2 - S_z (3a)
          tPrev = tCur;
          tCur = tNext;
        }
        const float bk = fmaf(-a * cprev, ibp, 1.f + a + c);
        ib[k] = frcp(bk);
        fm[k] = a * ibp;
        bm[k] = c * ib[k];
        ibp = ib[k];
        cprev = c;
        r[k] = rhs;
        A = fmaf(fm[k], A, rhs);
        B *= fm[k];
        mPrev = mCur;
        mCur = mNext;
      }
    }
    }
    sF[w * 32 + l] = make_float2(A, B);
    __syncthreads();
    float dcar = 0.f;
    for (int q = 0; q < w; q++) {
      const float2 m2 = sF[q * 32 + l];
      dcar = fmaf(m2.y, dcar, m2.x);
    }
    A = 0.f;
    B = 1.f;
#pragma unroll
    for (int k = 0; k < K; k++) {
      dcar = fmaf(fm[k], dcar, r[k]);
      r[k] = dcar * ib[k];
    }
    // back substitution: chunk map x_in = A + B x_out, combined from the last warp down
#pragma unroll
    for (int k = K - 1; k >= 0; k--) {
      A = fmaf(bm[k], A, r[k]);
      B *= bm[k];
    }
    sB[w * 32 + l] = make_float2(A, B);
    __syncthreads();
    float tcar = 0.f;
    for (int q = G - 1; q > w; q--) {
      const float2 m2 = sB[q * 32 + l];
      tcar = fmaf(m2.y, tcar, m2.x);
    }
#pragma unroll
    for (int k = K - 1; k >= 0; k--) {
      tcar = fmaf(bm[k], tcar, r[k]);
      r[k] = tcar;
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      if (k < nv) {
        const long long v = base + (long long)(s + k) * st;
        if (ZP) {
          const float tnew = r[k];
          const int m = med(s + k);  // the stage still holds this tile (reissued below)
          {
            const float2 dg = sdmg[m];
            if (dg.y > 0.f) {
              // Arrhenius integral with the mid-step temperature (finiteElementHeatPropagator.c:600-602):
              // log A - E / (R (T0 + d)) = x0 + (E/R) d / (T0 (T0 + d)), x0 formed in FP64 per call
              const float dm = 0.5f * (tnew + Tt[(s + k) * 32 + l]);
              h.dOmega[v] += h.dt * expf(dg.x + dg.y * dm / (h.T0 * (h.T0 + dm)));
            }
          }
          h.T[v] = tnew;
        } else {
          h.A[v] = r[k];
        }
      }
      if (ZP && k < nv) {
        // running maxima per lane, flushed to shared memory when the lane's medium changes
        const int mk = med(s + k);
        if (mk != curM) {
          if (curM >= 0) atomicMax(&mloc[curM], enc_max((float)((double)curMax + h.base)));
          curM = mk;
          curMax = r[k];
        } else {
          curMax = fmaxf(curMax, r[k]);
        }
      }
    }
    // every warp is done with this stage: prefetch the tile after next into it. (The chunk maps
    // alternate between two buffers by tile parity, so the next tile's map writes cannot meet a
    // warp still reading this tile's: it passes this barrier first.)
    __syncthreads();
    if (threadIdx.x == 0) {
      const int nt = tile + 2 * gridDim.x;
      if (nt < nTiles) {
        fence_proxy_async();
        issue(nt, stg);
      }
    }
  }
  if (ZP) {
    if (curM >= 0) atomicMax(&mloc[curM], enc_max((float)((double)curMax + h.base)));
    __syncthreads();
    for (int k = threadIdx.x; k < nM; k += blockDim.x)
      if (mloc[k]) atomicMax(&h.maxEnc[k], mloc[k]);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(h.stepCounter, 1);
  }
}

// ---------------------------------------------------------------------------------------------
// Homogeneous-chunk tables (once per call: they depend on the media, the boundary type and the
// pivot warm-up length only)
// ---------------------------------------------------------------------------------------------

// X pass: lane g of the line (y, z) owns rows [g K, g K + K); its chunk is homogeneous when rows
// s - W - 1 .. e of the line are one medium (code bit 1 clear on rows s - W - 1 .. e - 1), none
// heat-sinked, none a line end. Entry: medium + 1, or 0.
__global__ void uni_x_kernel(const StreamDev h, int K, int G, uint8_t *out) {
  const long long n = (long long)h.ny * h.nz * G;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(t % G);
    const long long line = t / G;
    const int y = (int)(line % h.ny), z = (int)(line / h.ny);
    const long long row = (long long)y * h.px + (long long)z * h.sxy;
    const int s = g * K, e = min(s + K, h.nx);
    bool uni = s < h.nx && s >= h.W + 1 && e <= h.nx - 1;
    for (int i = s - h.W - 1; uni && i <= e; i++) {
      const int cd = h.code[row + i];
      uni = !(cd & kCodeSink) && (i == e || !(cd & 2));
    }
    const int m0 = uni ? h.M[row + s] : 255;
    out[t] = (uint8_t)(m0 < 255 ? m0 + 1 : 0);
  }
}

// Column-layout Y (ZP false) and Z passes: chunk w of G (kk = ceil(n / G) rows) of the line at
// column x, other index o. Homogeneous: rows s - W - 1 .. e one medium, the line not heat-sinked,
// none a line end. Entry [o][w][x]: medium + 1, or 0.
__global__ void uni_col_kernel(const StreamDev h, bool ZP, int G, uint8_t *out) {
  const int n = ZP ? h.nz : h.ny, nOther = ZP ? h.ny : h.nz;
  const int kk = (n + G - 1) / G;
  const long long st = ZP ? h.sxy : (long long)h.px;
  const long long cnt = (long long)nOther * G * h.px;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < cnt; t += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(t % h.px);
    const long long ow = t / h.px;
    const int w = (int)(ow % G), o = (int)(ow / G);
    const int s = min(w * kk, n), e = min(s + kk, n);
    const bool lineSink = h.hs && (x == 0 || x == h.nx - 1 || o == 0 || o == nOther - 1);
    const long long base = x + (ZP ? (long long)o * h.px : (long long)o * h.sxy);
    bool uni = x < h.nx && e > s && !lineSink && s >= h.W + 1 && e <= n - 1;
    const int m0 = uni ? h.M[base + s * st] : 255;
    for (int i = s - h.W - 1; uni && i <= e; i++) uni = h.M[base + i * st] == m0;
    out[t] = (uint8_t)(uni && m0 < 255 ? m0 + 1 : 0);
  }
}

// ---------------------------------------------------------------------------------------------
// Layout conversions and per-call set-up kernels
// ---------------------------------------------------------------------------------------------

// Pitched layout of a dense grid (x rows padded to px elements). The dense <-> pitched
// conversions walk one (y, z) row per warp (dense row r starts at r nx, pitched row r at r px),
// so no element index is divided.
struct Pitch {
  int nx, ny, nz, px;
  __device__ __forceinline__ long long p(long long v) const {
    const long long nxy = (long long)nx * ny;
    const long long iz = v / nxy, r = v - iz * nxy, iy = r / nx, ix = r - iy * nx;
    return ix + (iy + iz * ny) * px;
  }
};

template <typename S, typename D, typename F>
__device__ __forceinline__ void row_walk(const Pitch &P, bool toPitched, const S *src, D *dst, F f) {
  const long long rows = (long long)P.ny * P.nz;
  const int lane = threadIdx.x & 31;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < rows; r += nw) {
    const long long d = r * P.nx, q = r * P.px;
    for (int x = lane; x < P.nx; x += 32) {
      if (toPitched) dst[q + x] = f(src[d + x]);
      else dst[d + x] = f(src[q + x]);
    }
  }
}

// f32 rows of a grid whose nx is a multiple of 4, between 16-byte aligned buffers (every dense
// and pitched row then starts on a 16-byte boundary): 16-byte accesses.
template <typename F>
__device__ __forceinline__ void row_walk4(const Pitch &P, bool toPitched, const float *src, float *dst, F f) {
  const long long rows = (long long)P.ny * P.nz;
  const int lane = threadIdx.x & 31, n4 = P.nx >> 2;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < rows; r += nw) {
    const long long d = r * P.nx, q = r * P.px;
    const float4 *s4 = reinterpret_cast<const float4 *>(src + (toPitched ? d : q));
    float4 *d4 = reinterpret_cast<float4 *>(dst + (toPitched ? q : d));
    for (int x = lane; x < n4; x += 32) {
      float4 v = s4[x];
      v.x = f(v.x);
      v.y = f(v.y);
      v.z = f(v.z);
      v.w = f(v.w);
      d4[x] = v;
    }
  }
}

__global__ void to_pitched_dev_kernel(const float *dense, float *out, double base, Pitch P) {
  auto f = [base](float v) { return (float)((double)v - base); };
  if ((P.nx & 3) == 0 && ((reinterpret_cast<uintptr_t>(dense) | reinterpret_cast<uintptr_t>(out)) & 15) == 0)
    row_walk4(P, true, dense, out, f);
  else row_walk(P, true, dense, out, f);
}

__global__ void from_pitched_dev_kernel(const float *pitched, float *dense, double base, Pitch P) {
  auto f = [base](float v) { return (float)((double)v + base); };
  if ((P.nx & 3) == 0 && ((reinterpret_cast<uintptr_t>(pitched) | reinterpret_cast<uintptr_t>(dense)) & 15) == 0)
    row_walk4(P, false, pitched, dense, f);
  else row_walk(P, false, pitched, dense, f);
}

__global__ void to_pitched_f32_kernel(const float *dense, float *out, Pitch P) {
  row_walk(P, true, dense, out, [](float v) { return v; });
}

__global__ void to_pitched_u8_kernel(const uint8_t *dense, uint8_t *out, Pitch P) {
  row_walk(P, true, dense, out, [](uint8_t v) { return v; });
}

// Neighbourhood code (once per call): bit 2d (2d+1) set when the lower (upper) neighbour along d
// exists and is of another medium (its face coefficient needs the pair table); kCodeSink marks
// heat-sinked voxels (held fixed). Missing neighbours are masked by position in the passes.
__global__ void code_kernel(const uint8_t *M, uint8_t *code, Pitch P, int hs, long long L) {
  const long long px = P.px, sxy = px * P.ny;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < L; v += (long long)gridDim.x * blockDim.x) {
    const long long nxy = (long long)P.nx * P.ny;
    const int iz = (int)(v / nxy);
    const long long r = v - iz * nxy;
    const int iy = (int)(r / P.nx), ix = (int)(r - (long long)iy * P.nx);
    const long long p = ix + iy * px + iz * sxy;
    const int m = M[p];
    int c = 0;
    if (hs && (ix == 0 || ix == P.nx - 1 || iy == 0 || iy == P.ny - 1 || iz == 0 || iz == P.nz - 1)) c = kCodeSink;
    if (ix > 0 && M[p - 1] != m) c |= 1;
    if (ix < P.nx - 1 && M[p + 1] != m) c |= 2;
    if (iy > 0 && M[p - px] != m) c |= 4;
    if (iy < P.ny - 1 && M[p + px] != m) c |= 8;
    if (iz > 0 && M[p - sxy] != m) c |= 16;
    if (iz < P.nz - 1 && M[p + sxy] != m) c |= 32;
    code[p] = (uint8_t)c;
  }
}

__global__ void merge_omega_p_kernel(float *Omega, const float *dOmega, Pitch P, long long L) {
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < L; v += (long long)gridDim.x * blockDim.x)
    Omega[v] = (float)((double)Omega[v] + (double)dOmega[P.p(v)]);
}

__global__ void final_sensors_p_kernel(StreamDev h) { record_sensors_p(h, *h.stepCounter); }

// H <- hdt * c in place (FP32 products, as the stepper forms its coefficients), the diagonal table
// Hd[m] = {H(m, m, 0), H(m, m, 1), H(m, m, 2), 0}, and Hs[m] = 1 / b* per direction, b* the fixed
// point of the pivot recurrence b -> 1 + 2h - h^2 / b of a line of one medium (h = H(m, m, d)):
// b* = (1 + 2h + sqrt(1 + 4h)) / 2, in FP64. One block writes Hd and Hs after its grid-stride pass,
// from the products it forms itself.
__global__ void h_table_kernel(float *H, float4 *Hd, float hdt, int nM) {
  const int n = 3 * nM * nM;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int mi = k % nM, mj = (k / nM) % nM;
    if (mi != mj) H[k] *= hdt;
  }
  if (blockIdx.x == 0) {
    for (int m = threadIdx.x; m < nM; m += blockDim.x) {
      float v[3], ibs[3];
      for (int d = 0; d < 3; d++) {
        const int k = (d * nM + m) * nM + m;
        v[d] = hdt * H[k];
        H[k] = v[d];
        const double hh = v[d];
        ibs[d] = (float)(2.0 / (1.0 + 2.0 * hh + sqrt(1.0 + 4.0 * hh)));
      }
      Hd[m] = make_float4(v[0], v[1], v[2], 0.f);
      Hd[nM + m] = make_float4(ibs[0], ibs[1], ibs[2], 0.f);
    }
  }
}

__global__ void decode_max_p_kernel(const unsigned int *enc, float *out, int nM) {
  for (int k = threadIdx.x; k < nM; k += blockDim.x) {
    const unsigned int e = enc[k];
    if (e == 0u) out[k] = -__int_as_float(0x7f800000);
    else out[k] = __uint_as_float((e & 0x80000000u) ? (e & 0x7fffffffu) : ~e);
  }
}

// ---------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------

// voxels per lane of an x-line: 16 lanes x 8 up to 128 voxels, then 32 lanes x 8, 12 or 16
int x_chunk(int nx) { return nx <= 256 ? 8 : nx <= 384 ? 12 : 16; }

// x pitch: a multiple of 16 that also holds every lane's whole chunk of K voxels
int pitch_of(int nx) {
  const int K = x_chunk(nx);
  const int w = (nx + K - 1) / K * K;
  return (w + 15) / 16 * 16;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 3D map over a pitched grid. f32 grids are addressed as 8-byte pairs, byte grids as 4-byte quads.
mcb_status make_map(mcb_ctx *ctx, CUtensorMap *map, void *base, bool f32, const StreamShape &S, int b0, int b1, int b2,
                    bool swz64) {
  PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
  if (!fn) return set_error(ctx, MCB_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const int es = f32 ? 8 : 4;
  const int per = f32 ? 2 : 4;
  const int rowBytes = f32 ? 4 * S.px : S.px;
  cuuint64_t dims[3] = {(cuuint64_t)(S.px / per), (cuuint64_t)S.ny, (cuuint64_t)S.nz};
  cuuint64_t strides[2] = {(cuuint64_t)rowBytes, (cuuint64_t)rowBytes * S.ny};
  cuuint32_t box[3] = {(cuuint32_t)b0, (cuuint32_t)b1, (cuuint32_t)b2};
  cuuint32_t estr[3] = {1, 1, 1};
  (void)es;
  const CUresult r = fn(map, f32 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, base, dims, strides,
                        box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(ctx, MCB_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return MCB_OK;
}

// dynamic shared memory: two stages, the two mbarriers, and 1 KB of alignment slack
size_t x_smem(int px, bool q, int nx) { return 2 * (size_t)x_layout(px, q, x_tile_lines(nx)).stage + 64 + 1024; }
size_t yz_smem(int n, bool z) { return 2 * (size_t)yz_layout(n, z).stage + 64 + 1024; }

template <int K, int G>
mcb_status x_attr(mcb_ctx *ctx, size_t bytes) {
  MCB_CUDA(ctx, cudaFuncSetAttribute(sx_kernel<K, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return MCB_OK;
}

template <int K, int G, bool Z>
mcb_status yz_attr(mcb_ctx *ctx, size_t bytes, int *blocksPerSm) {
  MCB_CUDA(ctx, cudaFuncSetAttribute(syz_kernel<K, G, Z>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  MCB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocksPerSm, syz_kernel<K, G, Z>, 16 * G, bytes));
  return MCB_OK;
}

// Line-length class of the Y/Z passes: K rows per lane, G lanes per line.
int yz_class(int n) { return n <= 64 ? 0 : n <= 128 ? 1 : n <= 192 ? 2 : n <= 256 ? 3 : n <= 384 ? 4 : 5; }

// Column-layout Y/Z pass (lines up to 320 rows): 8 rows per lane for lines up to 256 rows, 16
// beyond; G = ceil(n / rows) warps.
constexpr int kColMaxN = 320;
int col_rows(int n) { return n <= 256 ? 8 : 16; }
int col_warps(int n) { return (n + col_rows(n) - 1) / col_rows(n); }
size_t col_smem(int n, bool z) {
  const int G = col_warps(n);
  return (size_t)col_layout(n, z, G).sums + 4 * G * 32 * sizeof(float2) + 64 + 1024;
}

template <int K, bool Z, int MAXT>
mcb_status col_attr(mcb_ctx *ctx, int n, int *bps) {
  const size_t sm = col_smem(n, Z);
  MCB_CUDA(ctx, cudaFuncSetAttribute(scol_kernel<K, Z, MAXT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  MCB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, scol_kernel<K, Z, MAXT>, 32 * col_warps(n), sm));
  return MCB_OK;
}

// block-size classes: up to 256 threads (3 blocks per SM), 512 (2), 1024 (1; 16-row lanes: 640)
template <bool Z>
mcb_status col_occupancy(mcb_ctx *ctx, int n, int *bps) {
  const int G = col_warps(n);
  if (col_rows(n) == 16) return col_attr<16, Z, 640>(ctx, n, bps);
  if (G <= 8) return col_attr<8, Z, 256>(ctx, n, bps);
  if (G <= 16) return col_attr<8, Z, 512>(ctx, n, bps);
  return col_attr<8, Z, 1024>(ctx, n, bps);
}

template <bool Z>
void col_launch(int n, int grid, cudaStream_t st, const CUtensorMap &a, const CUtensorMap &m, const CUtensorMap &t,
                const StreamDev &h) {
  const int G = col_warps(n);
  const size_t sm = col_smem(n, Z);
  if (col_rows(n) == 16) scol_kernel<16, Z, 640><<<grid, 32 * G, sm, st>>>(a, m, t, h, G);
  else if (G <= 8) scol_kernel<8, Z, 256><<<grid, 32 * G, sm, st>>>(a, m, t, h, G);
  else if (G <= 16) scol_kernel<8, Z, 512><<<grid, 32 * G, sm, st>>>(a, m, t, h, G);
  else scol_kernel<8, Z, 1024><<<grid, 32 * G, sm, st>>>(a, m, t, h, G);
}

template <bool Z>
mcb_status yz_setup(mcb_ctx *ctx, int n, int *bps) {
  const size_t b = yz_smem(n, Z);
  switch (yz_class(n)) {
    case 0: return yz_attr<4, 16, Z>(ctx, b, bps);
    case 1: return yz_attr<8, 16, Z>(ctx, b, bps);
    case 2: return yz_attr<12, 16, Z>(ctx, b, bps);
    case 3: return yz_attr<16, 16, Z>(ctx, b, bps);
    case 4: return yz_attr<12, 32, Z>(ctx, b, bps);
    default: return yz_attr<16, 32, Z>(ctx, b, bps);
  }
}

template <bool Z>
void yz_launch(int n, int grid, cudaStream_t st, const CUtensorMap &a, const CUtensorMap &m, const CUtensorMap &t,
               const StreamDev &h) {
  const size_t b = yz_smem(n, Z);
  switch (yz_class(n)) {
    case 0: syz_kernel<4, 16, Z><<<grid, 256, b, st>>>(a, m, t, h); break;
    case 1: syz_kernel<8, 16, Z><<<grid, 256, b, st>>>(a, m, t, h); break;
    case 2: syz_kernel<12, 16, Z><<<grid, 256, b, st>>>(a, m, t, h); break;
    case 3: syz_kernel<16, 16, Z><<<grid, 256, b, st>>>(a, m, t, h); break;
    case 4: syz_kernel<12, 32, Z><<<grid, 512, b, st>>>(a, m, t, h); break;
    default: syz_kernel<16, 32, Z><<<grid, 512, b, st>>>(a, m, t, h); break;
  }
}

}  // namespace

bool stream_supported(int nx, int ny, int nz) {
  if (nx < 2 || ny < 2 || nz < 2 || nx > 512 || ny > 512 || nz > 512) return false;
  const int px = pitch_of(nx);
  // 227 KB per block, less the Y/Z kernels' 1 KB of static maxima
  return x_smem(px, true, nx) <= 226 * 1024 && yz_smem(ny, false) <= 226 * 1024 && yz_smem(nz, true) <= 226 * 1024 &&
         (ny > kColMaxN || col_smem(ny, false) <= 226 * 1024) && (nz > kColMaxN || col_smem(nz, true) <= 226 * 1024);
}

StreamShape stream_shape(int nx, int ny, int nz) {
  StreamShape S;
  S.nx = nx;
  S.ny = ny;
  S.nz = nz;
  S.px = pitch_of(nx);
  S.Lp = (long long)S.px * ny * nz;
  return S;
}

// Pivot warm-up length for H = hdt c (see the file comment): rho^W <= 2^-26 with
// rho = max over medium pairs of a c / (1 + a + c); 1 << 30 (every lane from row 0) when rho >= 1.
int stream_warmup(const float *c, float hdt, int nM) {
  double rho = 0.0;
  for (int d = 0; d < 3; d++)
    for (int p = 0; p < nM; p++)
      for (int q = 0; q < nM; q++) {
        const double a = hdt * c[(size_t)(d * nM + p) * nM + q];  // row q's coupling to its predecessor p
        const double cc = hdt * c[(size_t)(d * nM + q) * nM + p];  // row p's coupling to its successor q
        rho = std::max(rho, a * cc / (1.0 + a + cc));
      }
  if (!(rho < 1.0)) return 1 << 30;
  const double target = std::ldexp(1.0, -26);
  if (rho <= target) return 1;
  return std::max(1, (int)std::ceil(std::log(target) / std::log(rho)));
}

mcb_status stream_maps(mcb_ctx *ctx, mcb_heat_state *s) {
  const StreamShape &S = s->shape;
  StreamMaps &m = *s->maps;
  const int xf = S.px / 2, xq = S.px / 4;
  const YZLayout ly = yz_layout(S.ny, false), lz = yz_layout(S.nz, true);
  const int kXL = x_tile_lines(S.nx);
  MCB_TRY(make_map(ctx, &m.xTh, s->T, true, S, xf, kXL + 2, 1, false));
  MCB_TRY(make_map(ctx, &m.xTr, s->T, true, S, xf, kXL, 1, false));
  // without a source buffer (light never on) the Q map points at T; it is then never loaded
  MCB_TRY(make_map(ctx, &m.xQr, s->Q ? s->Q : s->T, true, S, xf, kXL, 1, false));
  MCB_TRY(make_map(ctx, &m.xMh, s->M, false, S, xq, kXL + 2, 1, false));
  MCB_TRY(make_map(ctx, &m.xCr, s->code, false, S, xq, kXL, 1, false));
  MCB_TRY(make_map(ctx, &m.yA, s->A, true, S, kTW / 2, ly.BN, 1, true));
  MCB_TRY(make_map(ctx, &m.yM, s->M, false, S, kTW / 4, ly.BN, 1, false));
  MCB_TRY(make_map(ctx, &m.zA, s->A, true, S, kTW / 2, 1, lz.BN, true));
  MCB_TRY(make_map(ctx, &m.zM, s->M, false, S, kTW / 4, 1, lz.BN, false));
  MCB_TRY(make_map(ctx, &m.zT, s->T, true, S, kTW / 2, 1, lz.BN, true));
  // column-layout Y/Z tiles: 32 columns (16 pairs, 8 quads) of whole lines, plain rows
  if (S.ny <= kColMaxN) {
    const ColLayout cy = col_layout(S.ny, false, col_warps(S.ny));
    MCB_TRY(make_map(ctx, &m.cyA, s->A, true, S, 16, cy.BN, 1, false));
    MCB_TRY(make_map(ctx, &m.cyM, s->M, false, S, 8, cy.BN, 1, false));
  }
  if (S.nz <= kColMaxN) {
    const ColLayout cz = col_layout(S.nz, true, col_warps(S.nz));
    MCB_TRY(make_map(ctx, &m.czA, s->A, true, S, 16, 1, cz.BN, false));
    MCB_TRY(make_map(ctx, &m.czM, s->M, false, S, 8, 1, cz.BN, false));
    MCB_TRY(make_map(ctx, &m.czT, s->T, true, S, 16, 1, cz.BN, false));
  }
  return MCB_OK;
}

// Buffers of the streamed state, carved by `take` (256-byte aligned pieces).
void stream_carve(const std::function<void *(size_t)> &take, mcb_heat_state *s, const mcb_heat_params *p, bool damage,
                  bool withQ) {
  const StreamShape S = stream_shape(p->nx, p->ny, p->nz);
  const long long L = (long long)p->nx * p->ny * p->nz, Lp = S.Lp;
  const int nM = p->nM, nS = p->nSensors;
  s->shape = S;
  s->T = (float *)take(4 * Lp);
  s->A = (float *)take(4 * Lp);
  s->Q = withQ ? (float *)take(4 * Lp) : nullptr;
  s->M = (uint8_t *)take(Lp);
  s->code = (uint8_t *)take(Lp);
  s->dOm = damage ? (float *)take(4 * Lp) : nullptr;
  s->Om = damage ? (float *)take(4 * L) : nullptr;
  s->stage = (float *)take(4 * (size_t)std::max<long long>(L, nM));
  s->H = (float *)take(12 * (size_t)nM * nM);
  s->Hd = (float4 *)take(32 * (size_t)nM);  // Hd, then the fixed-point table Hs
  s->dmg = (float2 *)take(8 * (size_t)nM);
  s->maxEnc = (unsigned int *)take(4 * (size_t)nM);
  s->step = (int *)take(16);
  // homogeneous-chunk tables of the X pass and of the column-layout Y and Z passes
  s->uniX = (uint8_t *)take((size_t)S.ny * S.nz * x_lanes(S.nx));
  s->uniY = S.ny <= kColMaxN ? (uint8_t *)take((size_t)S.px * S.nz * col_warps(S.ny)) : nullptr;
  s->uniZ = S.nz <= kColMaxN ? (uint8_t *)take((size_t)S.px * S.ny * col_warps(S.nz)) : nullptr;
  (void)nS;
}

// Uploads M (pitched), the neighbourhood code, T (pitched deviations from the mean input
// temperature) and Omega; clears the padding of every pitched grid.
mcb_status stream_upload(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, const float *T, const float *Omega) {
  cudaStream_t st = ctx->stream;
  const StreamShape &S = s->shape;
  const long long L = (long long)S.nx * S.ny * S.nz;
  const Pitch P{S.nx, S.ny, S.nz, S.px};
  const int grid = ctx->num_sms * 8;
  double sum = 0.0;
  for (long long k = 0; k < L; k++) sum += T[k];
  s->base = sum / (double)L;
  MCB_CUDA(ctx, cudaMemsetAsync(s->T, 0, 4 * S.Lp, st));
  MCB_CUDA(ctx, cudaMemsetAsync(s->A, 0, 4 * S.Lp, st));
  if (s->Q) MCB_CUDA(ctx, cudaMemsetAsync(s->Q, 0, 4 * S.Lp, st));
  MCB_CUDA(ctx, cudaMemsetAsync(s->M, 0, S.Lp, st));
  MCB_CUDA(ctx, cudaMemsetAsync(s->code, 0, S.Lp, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(s->stage, p->M, L, cudaMemcpyHostToDevice, st));
  to_pitched_u8_kernel<<<grid, 256, 0, st>>>((const uint8_t *)s->stage, s->M, P);
  code_kernel<<<grid, 256, 0, st>>>(s->M, s->code, P, p->heatBoundaryType != 0, L);
  MCB_CUDA(ctx, cudaMemcpyAsync(s->stage, T, 4 * L, cudaMemcpyHostToDevice, st));
  to_pitched_dev_kernel<<<grid, 256, 0, st>>>(s->stage, s->T, s->base, P);
  if (s->Om && Omega) MCB_CUDA(ctx, cudaMemcpyAsync(s->Om, Omega, 4 * L, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaGetLastError());
  s->codeHs = (int)(p->heatBoundaryType != 0);
  s->qValid = false;
  return MCB_OK;
}

mcb_status stream_upload_q(mcb_ctx *ctx, mcb_heat_state *s, const float *Q) {
  cudaStream_t st = ctx->stream;
  const StreamShape &S = s->shape;
  const long long L = (long long)S.nx * S.ny * S.nz;
  MCB_CUDA(ctx, cudaMemcpyAsync(s->stage, Q, 4 * L, cudaMemcpyHostToDevice, st));
  to_pitched_f32_kernel<<<ctx->num_sms * 8, 256, 0, st>>>(s->stage, s->Q, Pitch{S.nx, S.ny, S.nz, S.px});
  MCB_CUDA(ctx, cudaGetLastError());
  s->qValid = true;
  return MCB_OK;
}

// Launch configuration of one streamed step on a state.
struct StreamStepper {
  StreamDev h;
  StreamShape S;
  const StreamMaps *maps = nullptr;
  int K = 8, XG = 16, gX = 1, gY = 1, gZ = 1;
  size_t xs = 0;
  bool colY = true, colZ = true;
};

// Per-call set-up of the streamed stepper on a state: the per-call tables (H = dt/2 c in FP32, as
// the stepper multiplies them, and its diagonal and fixed points, formed on the device; the
// damage exponents about the base temperature; the pivot warm-up length), cleared maxima, step
// counter and damage increments, kernel attributes and grids. `sens` is the device buffer of the
// sensor history ([nS x (steps + 1)] doubles) or nullptr.
mcb_status stream_setup(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, double *sens, StreamStepper *out) {
  cudaStream_t st = ctx->stream;
  const StreamShape &S = s->shape;
  const long long L = (long long)S.nx * S.ny * S.nz;
  const int nM = p->nM, nS = p->nSensors;
  if (p->lightsOn && !s->qValid) return set_error(ctx, MCB_EINVAL, "dTdt_abs missing while lightsOn");
  if (s->codeHs != (int)(p->heatBoundaryType != 0)) {
    code_kernel<<<ctx->num_sms * 8, 256, 0, st>>>(s->M, s->code, Pitch{S.nx, S.ny, S.nz, S.px}, p->heatBoundaryType != 0, L);
    s->codeHs = (int)(p->heatBoundaryType != 0);
  }
  const float hdt = (float)(p->dt / 2);
  MCB_CUDA(ctx, cudaMemcpyAsync(s->H, p->dTdtperdeltaT, 12 * (size_t)nM * nM, cudaMemcpyHostToDevice, st));
  h_table_kernel<<<std::max(1, std::min(1024, (3 * nM * nM + 255) / 256)), 256, 0, st>>>(s->H, s->Hd, hdt, nM);
  float2 dmg[256];
  heat_damage_table(p, s->base, dmg);
  const int W = stream_warmup(p->dTdtperdeltaT, hdt, nM);
  MCB_CUDA(ctx, cudaMemcpyAsync(s->dmg, dmg, 8 * (size_t)nM, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemsetAsync(s->maxEnc, 0, 4 * (size_t)nM, st));
  MCB_CUDA(ctx, cudaMemsetAsync(s->step, 0, 16, st));
  if (s->dOm) MCB_CUDA(ctx, cudaMemsetAsync(s->dOm, 0, 4 * (size_t)S.Lp, st));

  StreamStepper &k = *out;
  StreamDev &h = k.h;
  h = StreamDev{};
  h.nx = S.nx; h.ny = S.ny; h.nz = S.nz; h.nM = nM; h.px = S.px; h.W = std::min(W, std::max({S.nx, S.ny, S.nz}));
  h.sxy = (long long)S.px * S.ny;
  h.T = s->T; h.A = s->A; h.M = s->M; h.code = s->code;
  h.Q = p->lightsOn ? s->Q : nullptr;
  h.dOmega = s->dOm; h.H = s->H; h.Hd = s->Hd; h.Hs = s->Hd + nM; h.dmg = s->dmg;
  h.T0 = (float)(s->base + kCelsiusZero); h.dt = (float)p->dt;
  h.maxEnc = s->maxEnc; h.hs = p->heatBoundaryType != 0; h.base = s->base;
  h.nS = nS; h.sIdx = s->sIdx; h.sW = s->sW; h.sens = sens; h.stepCounter = s->step; h.err = s->step + 1;
  s->lastW = h.W;

  h.uniX = s->uniX;
  h.uniY = s->uniY;
  h.uniZ = s->uniZ;
  k.S = S;
  k.maps = s->maps;
  k.K = x_chunk(S.nx);
  k.XG = x_lanes(S.nx);
  uni_x_kernel<<<ctx->num_sms * 4, 256, 0, st>>>(h, k.K, k.XG, s->uniX);
  if (s->uniY) uni_col_kernel<<<ctx->num_sms * 4, 256, 0, st>>>(h, false, col_warps(S.ny), s->uniY);
  if (s->uniZ) uni_col_kernel<<<ctx->num_sms * 4, 256, 0, st>>>(h, true, col_warps(S.nz), s->uniZ);
  MCB_CUDA(ctx, cudaGetLastError());
  const int XL = x_tile_lines(S.nx);
  k.xs = x_smem(S.px, h.Q != nullptr, S.nx);
  if (k.XG == 16) MCB_TRY((x_attr<8, 16>(ctx, k.xs)));
  else if (k.K == 8) MCB_TRY((x_attr<8, 32>(ctx, k.xs)));
  else if (k.K == 12) MCB_TRY((x_attr<12, 32>(ctx, k.xs)));
  else MCB_TRY((x_attr<16, 32>(ctx, k.xs)));
  int bpsY = 1, bpsZ = 1;
  k.colY = S.ny <= kColMaxN;
  k.colZ = S.nz <= kColMaxN;
  if (k.colY) MCB_TRY(col_occupancy<false>(ctx, S.ny, &bpsY));
  else MCB_TRY(yz_setup<false>(ctx, S.ny, &bpsY));
  if (k.colZ) MCB_TRY(col_occupancy<true>(ctx, S.nz, &bpsZ));
  else MCB_TRY(yz_setup<true>(ctx, S.nz, &bpsZ));
  const int xbps = std::max(1, std::min(k.XG == 16 ? 3 : 2, (int)((227u * 1024u) / (unsigned)(k.xs + 1024))));
  const long long tilesX = (long long)((S.ny + XL - 1) / XL) * S.nz;
  const long long tilesY = (long long)((S.nx + (k.colY ? 31 : kTW - 1)) / (k.colY ? 32 : kTW)) * S.nz;
  const long long tilesZ = (long long)((S.nx + (k.colZ ? 31 : kTW - 1)) / (k.colZ ? 32 : kTW)) * S.ny;
  k.gX = (int)std::min<long long>(tilesX, (long long)ctx->num_sms * xbps);
  k.gY = (int)std::min<long long>(tilesY, (long long)ctx->num_sms * std::max(1, bpsY));
  k.gZ = (int)std::min<long long>(tilesZ, (long long)ctx->num_sms * std::max(1, bpsZ));
  return MCB_OK;
}

// Enqueues one DG-ADI step (X, Y and Z passes).
void stream_step_launch(const StreamStepper &k, cudaStream_t q) {
  const StreamMaps &mp = *k.maps;
  const StreamDev &h = k.h;
  const StreamShape &S = k.S;
  if (k.XG == 16) sx_kernel<8, 16><<<k.gX, 256, k.xs, q>>>(mp.xTh, mp.xTr, mp.xQr, mp.xMh, mp.xCr, h);
  else if (k.K == 8) sx_kernel<8, 32><<<k.gX, 256, k.xs, q>>>(mp.xTh, mp.xTr, mp.xQr, mp.xMh, mp.xCr, h);
  else if (k.K == 12) sx_kernel<12, 32><<<k.gX, 256, k.xs, q>>>(mp.xTh, mp.xTr, mp.xQr, mp.xMh, mp.xCr, h);
  else sx_kernel<16, 32><<<k.gX, 256, k.xs, q>>>(mp.xTh, mp.xTr, mp.xQr, mp.xMh, mp.xCr, h);
  if (k.colY) col_launch<false>(S.ny, k.gY, q, mp.cyA, mp.cyM, mp.cyA, h);
  else yz_launch<false>(S.ny, k.gY, q, mp.yA, mp.yM, mp.yA, h);
  if (k.colZ) col_launch<true>(S.nz, k.gZ, q, mp.czA, mp.czM, mp.czT, h);
  else yz_launch<true>(S.nz, k.gZ, q, mp.zA, mp.zM, mp.zT, h);
}

mcb_status stream_stepper_new(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, StreamStepper **out) {
  StreamStepper *k = new StreamStepper();
  const mcb_status rc = stream_setup(ctx, s, p, nullptr, k);
  if (rc != MCB_OK) {
    delete k;
    return rc;
  }
  *out = k;
  return MCB_OK;
}

void stream_stepper_free(StreamStepper *k) { delete k; }

void stream_stepper_launch(const StreamStepper *k, cudaStream_t st) { stream_step_launch(*k, st); }

void stream_dense_copy(mcb_ctx *ctx, const mcb_heat_state *s, float *dense, cudaStream_t st) {
  const StreamShape &S = s->shape;
  from_pitched_dev_kernel<<<ctx->num_sms * 8, 256, 0, st>>>(s->T, dense, 0.0, Pitch{S.nx, S.ny, S.nz, S.px});
}

void stream_dense_set(mcb_ctx *ctx, mcb_heat_state *s, const float *dense, cudaStream_t st) {
  const StreamShape &S = s->shape;
  to_pitched_dev_kernel<<<ctx->num_sms * 8, 256, 0, st>>>(dense, s->T, 0.0, Pitch{S.nx, S.ny, S.nz, S.px});
}

long long stream_pitched_index(const mcb_heat_state *s, long long v) {
  const StreamShape &S = s->shape;
  const long long nxy = (long long)S.nx * S.ny;
  const long long iz = v / nxy, r = v - iz * nxy, iy = r / S.nx, ix = r - iy * S.nx;
  return ix + (iy + iz * S.ny) * S.px;
}

// Runs p->steps steps on the device-resident streamed state. Sensor and maximum outputs go to
// host memory; `sens` is the device buffer of the sensor history ([nS x (steps + 1)] doubles).
mcb_status stream_step(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, double *sens, double *sensorTemps,
                       float *maxMediaTemps, bool graphs) {
  cudaStream_t st = ctx->stream;
  const StreamShape &S = s->shape;
  const long long L = (long long)S.nx * S.ny * S.nz, nt = p->steps;
  const int nM = p->nM, nS = p->nSensors;
  StreamStepper ks;
  MCB_TRY(stream_setup(ctx, s, p, sens, &ks));
  const StreamDev &h = ks.h;
  auto step = [&](cudaStream_t q) { stream_step_launch(ks, q); };
  MCB_CUDA(ctx, cudaEventRecord(ctx->ev0, st));
  const int chunk = 16;
  long long done = 0;
  if (graphs && nt >= chunk) {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    MCB_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < chunk; k++) step(st);
    MCB_CUDA(ctx, cudaStreamEndCapture(st, &graph));
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    if (ie != cudaSuccess) {
      cudaGraphDestroy(graph);
      MCB_CUDA(ctx, ie);
    }
    for (; done + chunk <= nt; done += chunk) {
      const cudaError_t le = cudaGraphLaunch(exec, st);
      if (le != cudaSuccess) {
        cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        MCB_CUDA(ctx, le);
      }
    }
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
  }
  for (; done < nt; done++) step(st);
  if (nS) final_sensors_p_kernel<<<1, 128, 0, st>>>(h);
  if (s->dOm) merge_omega_p_kernel<<<ctx->num_sms * 8, 256, 0, st>>>(s->Om, s->dOm, Pitch{S.nx, S.ny, S.nz, S.px}, L);
  MCB_CUDA(ctx, cudaGetLastError());
  MCB_CUDA(ctx, cudaEventRecord(ctx->ev1, st));
  decode_max_p_kernel<<<1, 256, 0, st>>>(s->maxEnc, s->stage, nM);
  if (maxMediaTemps) MCB_CUDA(ctx, cudaMemcpyAsync(maxMediaTemps, s->stage, 4 * (size_t)nM, cudaMemcpyDeviceToHost, st));
  if (nS && sensorTemps)
    MCB_CUDA(ctx, cudaMemcpyAsync(sensorTemps, sens, 8 * (size_t)nS * (nt + 1), cudaMemcpyDeviceToHost, st));
  int flags[4] = {0, 0, 0, 0};
  MCB_CUDA(ctx, cudaMemcpyAsync(flags, s->step, 16, cudaMemcpyDeviceToHost, st));
  MCB_CUDA(ctx, cudaStreamSynchronize(st));
  if (flags[1]) return set_error(ctx, MCB_ETIMEOUT, "heat stepper: a TMA tile wait timed out (pass %d)", flags[1]);
  float ms = 0.f;
  MCB_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->lastKernelMs = ms;
  return MCB_OK;
}

mcb_status stream_download(mcb_ctx *ctx, mcb_heat_state *s, float *T, float *Omega) {
  cudaStream_t st = ctx->stream;
  const StreamShape &S = s->shape;
  const long long L = (long long)S.nx * S.ny * S.nz;
  from_pitched_dev_kernel<<<ctx->num_sms * 8, 256, 0, st>>>(s->T, s->stage, s->base, Pitch{S.nx, S.ny, S.nz, S.px});
  MCB_CUDA(ctx, cudaGetLastError());
  if (T) MCB_CUDA(ctx, cudaMemcpyAsync(T, s->stage, 4 * L, cudaMemcpyDeviceToHost, st));
  if (Omega && s->Om) MCB_CUDA(ctx, cudaMemcpyAsync(Omega, s->Om, 4 * L, cudaMemcpyDeviceToHost, st));
  MCB_CUDA(ctx, cudaStreamSynchronize(st));
  return MCB_OK;
}

}  // namespace mcb
