// Douglas-Gunn ADI heat stepper with Arrhenius damage for sm_100a, behind mcb_heat_forward
// (replacing +MCmatlab/src/finiteElementHeatPropagator.c:688-821).
//
// One time step of the reference is six grid passes (substep1a..3b, :249-647). Here it is
// three, one per direction. All explicit work happens in the first, which reads T^n once:
//   X pass: rhs = T + dt(Q + x/2 + y + z) on T^n (1a), solve along x (1b); it also forms the
//           half-corrections S_y = dt/2 y(T^n), S_z = dt/2 z(T^n) of 2a and 3a  -> A1 - S_y, S_z
//   Y pass: solve along y (2b) on A1 - S_y                                       -> A2
//   Z pass: solve along z (3b) on A2 - S_z, Arrhenius damage with the mid-step
//           temperature and per-medium running maxima                             -> T
// The tridiagonal matrices depend only on (M, c, dt, boundary type), so each voxel's inverse
// pivot and scan multipliers are factored once per call; each pass then solves its lines with
// a warp-parallel chunked scan of the two first-order recurrences of the Thomas algorithm
// instead of one serial thread per line.
//
// Temperatures are stored as deviations from a per-call base temperature (the mean input
// temperature). The scheme is linear and shift-invariant in T, so this is exact algebra; it
// keeps FP32 rounding relative to the temperature rise rather than to ~37 degC, which is
// what lets the FP32 stepper track an FP64 run to ~1e-6 where the reference's FP32 stepper
// drifts by about 4e-7 relative per step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "heat_host.h"

namespace mcb {

// Sensor interpolation (recordTempSensors, finiteElementHeatPropagator.c:652-664) on the
// current state, written to column `col`.
__device__ void record_sensors(const HeatDev &h, int col) {
  const long long sxy = (long long)h.nx * h.ny;
  for (int j = threadIdx.x; j < h.nS; j += blockDim.x) {
    const long long i = (long long)h.sIdx[j];
    const double wx = h.sW[j], wy = h.sW[j + h.nS], wz = h.sW[j + 2 * h.nS];
    auto T = [&](long long k) { return (double)h.T[k] + h.base; };
    h.sens[j + (long long)col * h.nS] =
        (1 - wx) * (1 - wy) * (1 - wz) * T(i) + (1 - wx) * (1 - wy) * wz * T(i + sxy) + (1 - wx) * wy * (1 - wz) * T(i + h.nx) +
        (1 - wx) * wy * wz * T(i + h.nx + sxy) + wx * (1 - wy) * (1 - wz) * T(i + 1) + wx * (1 - wy) * wz * T(i + 1 + sxy) +
        wx * wy * (1 - wz) * T(i + 1 + h.nx) + wx * wy * wz * T(i + 1 + h.nx + sxy);
  }
}


// Line factorisation, once per call and dt: inverse pivots 1/b'_i and the two scan multipliers
// {fm_i, bm_i} = {a_i / b'_{i-1}, cc_i / b'_i} of every voxel's row, one thread per line.
__global__ void factor_kernel(HeatDev h, int dir, float *ibOut, float2 *fbOut) {
  const int nx = h.nx, ny = h.ny, nz = h.nz;
  const long long nLines = dir == 0 ? (long long)ny * nz : (dir == 1 ? (long long)nx * nz : (long long)nx * ny);
  const int n = dir == 0 ? nx : (dir == 1 ? ny : nz);
  const long long st = dir == 0 ? 1 : (dir == 1 ? nx : (long long)nx * ny);
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < nLines; l += (long long)gridDim.x * blockDim.x) {
    int ix0, iy0, iz0;
    if (dir == 0) { ix0 = 0; iy0 = (int)(l % ny); iz0 = (int)(l / ny); }
    else if (dir == 1) { ix0 = (int)(l % nx); iy0 = 0; iz0 = (int)(l / nx); }
    else { ix0 = (int)(l % nx); iy0 = (int)(l / nx); iz0 = 0; }
    const long long base = ix0 + (long long)iy0 * nx + (long long)iz0 * nx * ny;
    const bool lineSinked = h.hs && (dir == 0 ? (iy0 == 0 || iy0 == ny - 1 || iz0 == 0 || iz0 == nz - 1)
                                     : dir == 1 ? (ix0 == 0 || ix0 == nx - 1 || iz0 == 0 || iz0 == nz - 1)
                                                : (ix0 == 0 || ix0 == nx - 1 || iy0 == 0 || iy0 == ny - 1));
    float bprev = 1.f, ccprev = 0.f, ibprev = 1.f;
    for (int i = 0; i < n; i++) {
      const long long v = base + i * st;
      float a = 0.f, cc = 0.f;
      if (!row_sinked(h, lineSinked, i, n)) {
        const int mi = h.M[v];
        if (i > 0) a = h.hdt * cf(h, mi, h.M[v - st], dir);
        if (i < n - 1) cc = h.hdt * cf(h, mi, h.M[v + st], dir);
      }
      float b = 1.f + a + cc;
      if (i > 0) b -= a * ccprev / bprev;
      const float ib = 1.f / b;
      ibOut[v] = ib;
      fbOut[v] = make_float2(i > 0 ? a * ibprev : 0.f, cc * ib);
      bprev = b;
      ccprev = cc;
      ibprev = ib;
    }
  }
}

// Neighbourhood code of every voxel (once per call): bit 2d (2d+1) is set when the lower
// (upper) neighbour along d is missing or of another medium; kNbSink marks heat-sinked voxels.
__global__ void neighbour_code_kernel(HeatDev h, uint8_t *out) {
  const long long sxy = (long long)h.nx * h.ny, L = sxy * h.nz;
  for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < L; v += (long long)gridDim.x * blockDim.x) {
    const int iz = (int)(v / sxy);
    const long long r = v - iz * sxy;
    const int iy = (int)(r / h.nx), ix = (int)(r - (long long)iy * h.nx);
    const int m = h.M[v];
    int code = sinked(h, ix, iy, iz) ? kNbSink : 0;
    if (ix == 0 || h.M[v - 1] != m) code |= 1;
    if (ix == h.nx - 1 || h.M[v + 1] != m) code |= 2;
    if (iy == 0 || h.M[v - h.nx] != m) code |= 4;
    if (iy == h.ny - 1 || h.M[v + h.nx] != m) code |= 8;
    if (iz == 0 || h.M[v - sxy] != m) code |= 16;
    if (iz == h.nz - 1 || h.M[v + sxy] != m) code |= 32;
    out[v] = (uint8_t)code;
  }
}

// Loads of one voxel's explicit stencil (T^n and its six neighbours, code, medium, source) and
// the stencil itself: rhs1 = T + dt (Q + D_y T + D_z T) + dt/2 D_x T, with the half-corrections
// S_y = dt/2 D_y T and S_z = dt/2 D_z T that the Y and Z solves subtract. Voxels whose six
// neighbours exist and share their medium (neighbourhood code 0) take the diagonal coefficients
// c(m, m, d); the others look every face up. Heat-sinked voxels keep T (identity rows).
struct VoxIn {
  float t, n[6], q;
  int code, m;
};

__device__ __forceinline__ void voxel_load(const HeatDev &h, int v, int x, int iy, int iz, VoxIn &o) {
  const int nx = h.nx, ny = h.ny, nz = h.nz, sxy = nx * ny;
  const float *__restrict__ T = h.T;
  o.code = h.nb[v];
  o.t = T[v];
  o.m = h.M[v];
  o.q = h.Q ? h.Q[v] : 0.f;
  o.n[0] = x > 0 ? T[v - 1] : 0.f;
  o.n[1] = x < nx - 1 ? T[v + 1] : 0.f;
  o.n[2] = iy > 0 ? T[v - nx] : 0.f;
  o.n[3] = iy < ny - 1 ? T[v + nx] : 0.f;
  o.n[4] = iz > 0 ? T[v - sxy] : 0.f;
  o.n[5] = iz < nz - 1 ? T[v + sxy] : 0.f;
}

__device__ __forceinline__ void voxel_explicit(const HeatDev &h, int v, int x, int iy, int iz, const VoxIn &a, float &r,
                                               float &hy, float &hz) {
  const int nx = h.nx, ny = h.ny, nz = h.nz, sxy = nx * ny;
  const float t = a.t;
  r = t;
  hy = hz = 0.f;
  if (a.code & kNbSink) return;
  const int mi = a.m;
  float dx, dy, dz;
  if ((a.code & 63) == 0) {
    dx = cf(h, mi, mi, 0) * (a.n[0] + a.n[1] - 2.f * t);
    dy = cf(h, mi, mi, 1) * (a.n[2] + a.n[3] - 2.f * t);
    dz = cf(h, mi, mi, 2) * (a.n[4] + a.n[5] - 2.f * t);
  } else {
    dx = dy = dz = 0.f;
    if (x > 0) dx += cf(h, mi, h.M[v - 1], 0) * (a.n[0] - t);
    if (x < nx - 1) dx += cf(h, mi, h.M[v + 1], 0) * (a.n[1] - t);
    if (iy > 0) dy += cf(h, mi, h.M[v - nx], 1) * (a.n[2] - t);
    if (iy < ny - 1) dy += cf(h, mi, h.M[v + nx], 1) * (a.n[3] - t);
    if (iz > 0) dz += cf(h, mi, h.M[v - sxy], 2) * (a.n[4] - t);
    if (iz < nz - 1) dz += cf(h, mi, h.M[v + sxy], 2) * (a.n[5] - t);
  }
  r = t + h.dt * (a.q + dy + dz) + h.hdt * dx;
  hy = h.hdt * dy;
  hz = h.hdt * dz;
}

// X pass: the whole explicit stencil of the step (1a, 2a, 3a) and the solve along x (1b).
// A block owns h.xl consecutive x-lines (consecutive y at one z); U elements per thread are
// loaded at a time (all their global loads issued before use). S_y is subtracted from the x
// solution here, which gives the Y pass its right-hand side A1 - S_y; S_z is stored for the
// Z pass.
__global__ void __launch_bounds__(256, 3) pass_x_kernel(HeatDev h) {
  extern __shared__ unsigned char smem[];
  const int nx = h.nx, ny = h.ny, nz = h.nz;
  const int sxy = nx * ny;
  const int P = nx + 1;  // line pitch
  const int XL = h.xl;
  float *rhs = (float *)smem;
  float *fm = rhs + XL * P;
  float *bm = fm + XL * P;
  float *ib = bm + XL * P;
  float *sy = ib + XL * P;
  if (blockIdx.x == 0 && h.nS > 0) record_sensors(h, *h.stepCounter);
  const float *ibx = h.ib;
  const float2 *fbx = h.fb;
  const int yTiles = (ny + XL - 1) / XL;
  // e / nx as a multiply-high by ceil(2^32 / nx): exact while e * nx < 2^32 (e < XL * nx here)
  const unsigned mag = 0xFFFFFFFFu / (unsigned)nx + 1u;
  for (int tile = blockIdx.x; tile < yTiles * nz; tile += gridDim.x) {
    const int y0 = (tile % yTiles) * XL, iz = tile / yTiles;
    const int cnt = min(XL, ny - y0);
    const int total = cnt * nx;
    constexpr int U = 2;  // elements in flight per thread (4 measured slower: register spills)
    for (int e0 = threadIdx.x; e0 < total; e0 += blockDim.x * U) {
      VoxIn in[U];
      float vi[U];
      float2 vf[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int e = e0 + u * blockDim.x;
        if (e < total) {
          const int l = (int)__umulhi((unsigned)e, mag), x = e - l * nx;
          const int v = x + (y0 + l) * nx + iz * sxy;
          voxel_load(h, v, x, y0 + l, iz, in[u]);
          vi[u] = ibx[v];
          vf[u] = fbx[v];
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int e = e0 + u * blockDim.x;
        if (e < total) {
          const int l = (int)__umulhi((unsigned)e, mag), x = e - l * nx;
          const int v = x + (y0 + l) * nx + iz * sxy;
          float r, hy, hz;
          voxel_explicit(h, v, x, y0 + l, iz, in[u], r, hy, hz);
          h.Sz[v] = hz;
          rhs[l * P + x] = r;
          fm[l * P + x] = vf[u].x;
          bm[l * P + x] = vf[u].y;
          ib[l * P + x] = vi[u];
          sy[l * P + x] = hy;
        }
      }
    }
    __syncthreads();
    solve_lines(rhs, fm, bm, ib, nx, 1, P, cnt);
    __syncthreads();
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int l = (int)__umulhi((unsigned)e, mag), x = e - l * nx;
      h.A[x + (y0 + l) * nx + iz * sxy] = rhs[l * P + x] - sy[l * P + x];
    }
    __syncthreads();
  }
}

template <int TW>
__host__ __device__ constexpr size_t yz_tile_bytes(int n) {
  return (size_t)n * (5 * (TW + 1) * 4 + TW);
}

// Y and Z passes: a block owns TW consecutive x positions and one line per x along `dir`
// (dir 1: fixed iz; dir 2: fixed iy). Right-hand sides come from the previous pass (Y: A1 - S_y
// as the X pass wrote it; Z: A2 - S_z). The tile's rows (TW values each, coalesced) of rhs,
// pivots, multiplier pairs (and S_z) are staged with asynchronous copies, all in flight at
// once, then the TW lines are solved together from shared memory. The Z pass adds the
// Arrhenius damage with the mid-step temperature and the per-medium running maxima, and writes
// T^{n+1}.
template <int TW, bool ZPASS>
__global__ void __launch_bounds__(256, 3) pass_yz_kernel(HeatDev h) {
  extern __shared__ unsigned char smem[];
  constexpr int P = TW + 1;  // padded pitch
  const int nx = h.nx, ny = h.ny, nz = h.nz;
  const int sxy = nx * ny;
  const int n = ZPASS ? nz : ny;
  const int st = ZPASS ? sxy : nx;
  const int dir = ZPASS ? 2 : 1;
  float *rhs = (float *)smem;
  float *ib = rhs + n * P;
  float2 *fb = (float2 *)(ib + n * P);
  float *sz = (float *)(fb + n * P);
  uint8_t *Ms = (uint8_t *)(sz + n * P);
  __shared__ unsigned int mloc[256];
  const int xTiles = (nx + TW - 1) / TW;
  const int nOther = ZPASS ? ny : nz;
  const float *ibd = h.ib + (size_t)dir * sxy * nz;
  const float2 *fbd = h.fb + (size_t)dir * sxy * nz;
  if (ZPASS) {
    for (int k = threadIdx.x; k < h.nM; k += blockDim.x) mloc[k] = 0u;
  }
  int curM = -1;
  unsigned int curMax = 0u;
  constexpr int RPI = 256 / TW;  // rows covered by one pass of the block
  constexpr int U = 4;
  const int cx = threadIdx.x % TW, r0 = threadIdx.x / TW;
  for (int tile = blockIdx.x; tile < xTiles * nOther; tile += gridDim.x) {
    const int x0 = (tile % xTiles) * TW;
    const int other = tile / xTiles;
    const int base = ZPASS ? other * nx : other * sxy;
    const int x = x0 + cx;
    if (x < nx) {
      for (int r = r0; r < n; r += RPI) {
        const int v = base + x + r * st;
        cp_async4(&rhs[r * P + cx], &h.A[v]);
        cp_async4(&ib[r * P + cx], &ibd[v]);
        cp_async8(&fb[r * P + cx], &fbd[v]);
        if (ZPASS) cp_async4(&sz[r * P + cx], &h.Sz[v]);
      }
      if (ZPASS) {
        // media (bytes) for the damage and maxima, U rows in flight per thread
        for (int rb = r0; rb < n; rb += RPI * U) {
          uint8_t vM[U];
#pragma unroll
          for (int u = 0; u < U; u++) {
            const int r = rb + u * RPI;
            if (r < n) vM[u] = h.M[base + x + r * st];
          }
#pragma unroll
          for (int u = 0; u < U; u++) {
            const int r = rb + u * RPI;
            if (r < n) Ms[r * TW + cx] = vM[u];
          }
        }
      }
    }
    cp_async_wait_all();
    if (ZPASS && x < nx) {
      for (int r = r0; r < n; r += RPI) rhs[r * P + cx] -= sz[r * P + cx];
    }
    __syncthreads();
    solve_lines(rhs, (const float *)fb, (const float *)fb + 1, ib, n, P, 1, min(TW, nx - x0), 2);
    __syncthreads();
    if (x < nx) {
      for (int r = r0; r < n; r += RPI) {
        const int v = base + x + r * st;
        const float tnew = rhs[r * P + cx];
        if (ZPASS) {
          const int m = Ms[r * TW + cx];
          const float2 dg = h.dmg[m];
          if (h.dOmega && dg.y > 0.f) {
            // Arrhenius integral with the mid-step temperature (finiteElementHeatPropagator.c:600-602):
            // log A - E / (R (T0 + d)) = x0 + (E/R) d / (T0 (T0 + d)) with x0 = log A - E / (R T0)
            // formed in FP64 per call, so the large cancelling terms (log A ~ 154) never meet in FP32
            const float d = 0.5f * (tnew + h.T[v]);
            h.dOmega[v] += h.dt * expf(dg.x + dg.y * d / (h.T0 * (h.T0 + d)));
          }
          // running per-medium maximum, flushed when this thread's medium changes
          const unsigned int enc = enc_max((float)((double)tnew + h.base));
          if (m != curM) {
            if (curM >= 0) atomicMax(&mloc[curM], curMax);
            curM = m;
            curMax = enc;
          } else if (enc > curMax) {
            curMax = enc;
          }
          h.T[v] = tnew;
        } else {
          h.A[v] = tnew;
        }
      }
    }
    __syncthreads();
  }
  if (ZPASS) {
    if (curM >= 0) atomicMax(&mloc[curM], curMax);
    __syncthreads();
    for (int k = threadIdx.x; k < h.nM; k += blockDim.x)
      if (mloc[k]) atomicMax(&h.maxEnc[k], mloc[k]);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(h.stepCounter, 1);
  }
}

// Omega += the damage accumulated over the call (kept apart so the per-step increments are
// not rounded against Omega's magnitude).
__global__ void merge_omega_kernel(float *Omega, const float *dOmega, long long L) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < L; k += (long long)gridDim.x * blockDim.x)
    Omega[k] = (float)((double)Omega[k] + (double)dOmega[k]);
}

__global__ void final_sensors_kernel(HeatDev h) { record_sensors(h, *h.stepCounter); }

__global__ void to_dev_kernel(const float *T, float *out, double base, long long L) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < L; k += (long long)gridDim.x * blockDim.x)
    out[k] = (float)((double)T[k] - base);
}

__global__ void from_dev_kernel(const float *d, float *out, double base, long long L) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < L; k += (long long)gridDim.x * blockDim.x)
    out[k] = (float)((double)d[k] + base);
}

__global__ void decode_max_kernel(const unsigned int *enc, float *out, int nM) {
  for (int k = threadIdx.x; k < nM; k += blockDim.x) {
    const unsigned int e = enc[k];
    if (e == 0u) out[k] = -__int_as_float(0x7f800000);
    else out[k] = __uint_as_float((e & 0x80000000u) ? (e & 0x7fffffffu) : ~e);
  }
}

}  // namespace mcb

namespace {
using namespace mcb;

// Widest tile that keeps two blocks per SM (<= 100 KB each), else one block (<= 200 KB).
// (16-wide tiles measured faster than 32-wide ones on the 100^3 grid: twice the blocks)
int yz_tile_width(int n) {
  if (yz_tile_bytes<16>(n) <= 100000) return 16;
  if (yz_tile_bytes<8>(n) <= 200000) return 8;
  return 0;
}

size_t yz_smem(int TW, int n) {
  return (TW == 32 ? yz_tile_bytes<32>(n) : TW == 16 ? yz_tile_bytes<16>(n) : yz_tile_bytes<8>(n)) + 64;
}

size_t x_smem_lines(int nx, int xl) { return (size_t)xl * 5 * 4 * (nx + 1) + 64; }

// x-lines per X-pass block: at most 8 (more, smaller blocks measured faster on 300-long lines),
// fewer if the block's shared memory would exceed 100 KB
int x_lines(int nx) {
  for (int xl = 8; xl >= 2; xl >>= 1)
    if (x_smem_lines(nx, xl) <= 100000) return xl;
  return x_smem_lines(nx, 1) <= 200000 ? 1 : 0;
}

size_t x_smem(int nx) { return x_smem_lines(nx, x_lines(nx)); }


template <int TW>
mcb_status setup_yz(mcb_ctx *ctx, int ny, int nz) {
  MCB_CUDA(ctx, cudaFuncSetAttribute(pass_yz_kernel<TW, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)yz_smem(TW, ny)));
  MCB_CUDA(ctx, cudaFuncSetAttribute(pass_yz_kernel<TW, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)yz_smem(TW, nz)));
  return MCB_OK;
}

template <int TW>
void launch_yz(const HeatDev &h, int grid, cudaStream_t st) {
  pass_yz_kernel<TW, false><<<grid, 256, yz_smem(TW, h.ny), st>>>(h);
  pass_yz_kernel<TW, true><<<grid, 256, yz_smem(TW, h.nz), st>>>(h);
}

mcb_status check_params(mcb_ctx *ctx, const mcb_heat_params *p) {
  if (!p) return set_error(ctx, MCB_EINVAL, "NULL parameters");
  if (p->nx < 2 || p->ny < 2 || p->nz < 2) return set_error(ctx, MCB_EINVAL, "grid dimensions must be > 1");
  if (p->nM < 1 || p->nM > 256) return set_error(ctx, MCB_EINVAL, "nM must be in [1, 256]");
  if (!p->M || !p->dTdtperdeltaT || !p->A || !p->E) return set_error(ctx, MCB_EINVAL, "missing heat parameters");
  if (p->lightsOn && !p->dTdt_abs) return set_error(ctx, MCB_EINVAL, "dTdt_abs missing while lightsOn");
  if (p->steps < 0) return set_error(ctx, MCB_EINVAL, "steps must be >= 0");
  if (!(p->dt > 0) && p->steps > 0) return set_error(ctx, MCB_EINVAL, "dt must be positive");
  if (p->nSensors < 0) return set_error(ctx, MCB_EINVAL, "nSensors must be >= 0");
  if (p->nSensors > 0 && (!p->tempSensorCornerIdxs || !p->tempSensorInterpWeights))
    return set_error(ctx, MCB_EINVAL, "sensor arrays missing");
  const long long nx = p->nx, ny = p->ny, nz = p->nz, L = nx * ny * nz;
  if (L > 2147483647ll) return set_error(ctx, MCB_EINVAL, "grid too large");
  for (int s = 0; s < p->nSensors; s++) {
    const double li = p->tempSensorCornerIdxs[s];
    if (!(li >= 0) || li + 1 + nx + nx * ny > (double)(L - 1))
      return set_error(ctx, MCB_EINVAL, "sensor %d corner index out of range", s);
  }
  for (int m = 0; m < p->nM; m++)
    if (!(p->A[m] >= 0) || !(p->E[m] >= 0)) return set_error(ctx, MCB_EINVAL, "A and E must be non-negative");
  // every kernel indexes the media tables with M: reject indices beyond them
  for (long long k = 0; k < L; k++)
    if (p->M[k] >= p->nM) return set_error(ctx, MCB_EINVAL, "M holds a medium index outside 0..nM-1 (voxel %lld)", k);
  if (std::min(yz_tile_width((int)ny), yz_tile_width((int)nz)) == 0)
    return set_error(ctx, MCB_EINVAL, "y or z lines longer than the shared-memory tile limit");
  if (x_lines((int)nx) == 0) return set_error(ctx, MCB_EINVAL, "x lines longer than the shared-memory limit");
  return MCB_OK;
}

}  // namespace


namespace {

void free_state_buffers(mcb_heat_state *s) {
  if (s->block) cudaFree(s->block);
  if (s->sens) cudaFree(s->sens);
  if (s->sIdx) cudaFree(s->sIdx);
  delete s->maps;
  s->maps = nullptr;
  s->block = nullptr;
  s->sens = s->sIdx = nullptr;
  s->sensCap = 0;
  s->sCap = 0;
  s->streamed = false;
}

// Streamed state (heat_stream.cu) for p's grid in one allocation, with its TMA descriptors.
mcb_status stream_alloc(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, bool damage) {
  free_state_buffers(s);
  size_t need = 0;
  mcb_heat_state probe{};
  stream_carve([&](size_t b) { need += (b + 255) & ~(size_t)255; return (void *)nullptr; }, &probe, p, damage, true);
  MCB_CUDA(ctx, cudaMalloc(&s->block, need));
  char *cur = (char *)s->block;
  stream_carve([&](size_t b) { char *q = cur; cur += (b + 255) & ~(size_t)255; return (void *)q; }, s, p, damage, true);
  s->streamed = true;
  s->nx = p->nx;
  s->ny = p->ny;
  s->nz = p->nz;
  s->nM = p->nM;
  s->L = (long long)p->nx * p->ny * p->nz;
  s->damage = damage;
  s->maps = new StreamMaps();
  return stream_maps(ctx, s);
}

// Grow-only device buffers of the sensor inputs and history; uploads the sensor inputs.
mcb_status sensor_buffers(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p) {
  const int nS = p->nSensors;
  const long long nt = p->steps;
  if (nS <= 0) return MCB_OK;
  if (s->sCap < nS) {
    if (s->sIdx) cudaFree(s->sIdx);
    s->sIdx = nullptr;
    s->sCap = 0;
    MCB_CUDA(ctx, cudaMalloc(&s->sIdx, 32 * (size_t)nS));
    s->sW = s->sIdx + nS;
    s->sCap = nS;
  }
  if (s->sensCap < (long long)nS * (nt + 1)) {
    if (s->sens) cudaFree(s->sens);
    s->sens = nullptr;
    s->sensCap = 0;
    MCB_CUDA(ctx, cudaMalloc(&s->sens, 8 * (size_t)nS * (nt + 1)));
    s->sensCap = (long long)nS * (nt + 1);
  }
  MCB_CUDA(ctx, cudaMemcpyAsync(s->sIdx, p->tempSensorCornerIdxs, 8 * (size_t)nS, cudaMemcpyHostToDevice, ctx->stream));
  MCB_CUDA(ctx, cudaMemcpyAsync(s->sW, p->tempSensorInterpWeights, 24 * (size_t)nS, cudaMemcpyHostToDevice, ctx->stream));
  return MCB_OK;
}

// Whether a state of the right kind and shape for p exists.
bool state_fits(const mcb_heat_state *s, const mcb_heat_params *p, bool damage, bool streamed) {
  return s->block && s->streamed == streamed && s->nx == p->nx && s->ny == p->ny && s->nz == p->nz && s->nM == p->nM &&
         s->damage == damage;
}

mcb_status state_alloc(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, bool damage) {
  const long long L = (long long)p->nx * p->ny * p->nz;
  const int nM = p->nM;
  const size_t need = 4 * L * 3 /*T A Q*/ + 4 * (size_t)std::max<long long>(L, nM) /*stage*/ + 12 * L /*ib*/ +
                      24 * L /*fb*/ + L /*nb*/ + 4 * L /*Sz*/ + (damage ? 8 * L : 0) + L + 12 * (size_t)nM * nM +
                      24 * (size_t)nM /*logA E dmg*/ + 4 * (size_t)nM + 64 + 25 * 256;
  free_state_buffers(s);
  MCB_CUDA(ctx, cudaMalloc(&s->block, need));
  char *cur = (char *)s->block;
  auto take = [&](size_t bytes) {
    char *q = cur;
    cur += (bytes + 255) & ~(size_t)255;
    return (void *)q;
  };
  s->T = (float *)take(4 * L);
  s->A = (float *)take(4 * L);
  s->Q = (float *)take(4 * L);
  s->stage = (float *)take(4 * (size_t)std::max<long long>(L, nM));
  s->ib = (float *)take(12 * L);
  s->fb = (float2 *)take(24 * L);
  s->nb = (uint8_t *)take(L);
  s->Sz = (float *)take(4 * L);
  s->Om = damage ? (float *)take(4 * L) : nullptr;
  s->dOm = damage ? (float *)take(4 * L) : nullptr;
  s->M = (uint8_t *)take(L);
  s->c = (float *)take(12 * (size_t)nM * nM);
  s->logA = (double *)take(8 * (size_t)nM);
  s->E = (double *)take(8 * (size_t)nM);
  s->dmg = (float2 *)take(8 * (size_t)nM);
  s->maxEnc = (unsigned int *)take(4 * (size_t)nM);
  s->step = (int *)take(16);
  s->nx = p->nx;
  s->ny = p->ny;
  s->nz = p->nz;
  s->nM = nM;
  s->L = L;
  s->damage = damage;
  s->tw = std::min(yz_tile_width(p->ny), yz_tile_width(p->nz));
  return MCB_OK;
}

void damage_table(const mcb_heat_params *p, double base, float2 *out) { heat_damage_table(p, base, out); }

// Uploads the media/coefficients/source of p and the state T, Omega (host pointers).
mcb_status state_upload(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, const float *T, const float *Omega) {
  cudaStream_t st = ctx->stream;
  const long long L = s->L;
  const int nM = s->nM;
  double sum = 0.0;
  for (long long k = 0; k < L; k++) sum += T[k];
  s->base = sum / (double)L;
  std::vector<double> logA(nM);
  for (int m = 0; m < nM; m++) logA[m] = std::log(p->A[m]);
  std::vector<float2> dmg(nM);
  damage_table(p, s->base, dmg.data());
  MCB_CUDA(ctx, cudaMemcpyAsync(s->stage, T, 4 * L, cudaMemcpyHostToDevice, st));
  to_dev_kernel<<<ctx->num_sms * 8, 256, 0, st>>>(s->stage, s->T, s->base, L);
  MCB_CUDA(ctx, cudaMemcpyAsync(s->M, p->M, L, cudaMemcpyHostToDevice, st));
  if (p->dTdt_abs) MCB_CUDA(ctx, cudaMemcpyAsync(s->Q, p->dTdt_abs, 4 * L, cudaMemcpyHostToDevice, st));
  if (s->Om && Omega) MCB_CUDA(ctx, cudaMemcpyAsync(s->Om, Omega, 4 * L, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(s->c, p->dTdtperdeltaT, 12 * (size_t)nM * nM, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(s->logA, logA.data(), 8 * nM, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(s->E, p->E, 8 * nM, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(s->dmg, dmg.data(), 8 * nM, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaStreamSynchronize(st));  // host buffers (logA, dmg) go out of scope
  s->factoredDt = -1.0;
  return MCB_OK;
}

HeatDev make_dev(const mcb_heat_state *s, const mcb_heat_params *p) {
  HeatDev h{};
  h.nx = s->nx; h.ny = s->ny; h.nz = s->nz; h.nM = s->nM;
  h.T = s->T; h.A = s->A; h.M = s->M; h.c = s->c;
  h.Q = p->lightsOn ? s->Q : nullptr;
  h.ib = s->ib; h.fb = s->fb; h.nb = s->nb; h.Sz = s->Sz; h.Omega = s->Om; h.dOmega = s->dOm; h.logA = s->logA; h.E = s->E;
  h.dmg = s->dmg; h.T0 = (float)(s->base + kCelsiusZero);
  h.maxEnc = s->maxEnc; h.hs = p->heatBoundaryType != 0;
  h.dt = (float)p->dt; h.hdt = (float)(p->dt / 2); h.dtd = p->dt; h.base = s->base;
  h.nS = p->nSensors; h.sIdx = s->sIdx; h.sW = s->sW; h.sens = s->sens; h.stepCounter = s->step;
  h.xl = x_lines(s->nx);
  return h;
}

// Runs p->steps DG-ADI steps on the device-resident state; sensor and maximum outputs to host.
mcb_status state_step(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, double *sensorTemps, float *maxMediaTemps) {
  cudaStream_t st = ctx->stream;
  const long long nt = p->steps;
  const int nS = p->nSensors;
  MCB_TRY(sensor_buffers(ctx, s, p));
  if (p->lightsOn && p->dTdt_abs == nullptr) return set_error(ctx, MCB_EINVAL, "dTdt_abs missing while lightsOn");
  HeatStepper ks;
  MCB_TRY(heat_stepper(ctx, s, p, &ks));
  const HeatDev &h = ks.h;
  const int grid = ctx->num_sms * 8;
  const long long L = s->L;
  auto step = [&](cudaStream_t q) { heat_step_launch(ks, q); };
  MCB_CUDA(ctx, cudaEventRecord(ctx->ev0, st));
  const int chunk = 16;
  if (nt >= chunk) {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    MCB_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < chunk; k++) step(st);
    MCB_CUDA(ctx, cudaStreamEndCapture(st, &graph));
    MCB_CUDA(ctx, cudaGraphInstantiate(&exec, graph, 0));
    for (long long k = 0; k + chunk <= nt; k += chunk) MCB_CUDA(ctx, cudaGraphLaunch(exec, st));
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
  }
  for (long long k = (nt / chunk) * chunk; k < nt; k++) step(st);
  if (nS) final_sensors_kernel<<<1, 128, 0, st>>>(h);
  if (s->dOm) merge_omega_kernel<<<grid, 256, 0, st>>>(s->Om, s->dOm, L);
  MCB_CUDA(ctx, cudaGetLastError());
  MCB_CUDA(ctx, cudaEventRecord(ctx->ev1, st));
  decode_max_kernel<<<1, 256, 0, st>>>(s->maxEnc, s->stage, s->nM);
  if (maxMediaTemps) MCB_CUDA(ctx, cudaMemcpyAsync(maxMediaTemps, s->stage, 4 * (size_t)s->nM, cudaMemcpyDeviceToHost, st));
  if (nS && sensorTemps)
    MCB_CUDA(ctx, cudaMemcpyAsync(sensorTemps, s->sens, 8 * (size_t)nS * (nt + 1), cudaMemcpyDeviceToHost, st));
  MCB_CUDA(ctx, cudaStreamSynchronize(st));
  float ms = 0.f;
  MCB_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->lastKernelMs = ms;
  return MCB_OK;
}

mcb_status state_download(mcb_ctx *ctx, mcb_heat_state *s, float *T, float *Omega) {
  cudaStream_t st = ctx->stream;
  const long long L = s->L;
  from_dev_kernel<<<ctx->num_sms * 8, 256, 0, st>>>(s->T, s->stage, s->base, L);
  if (T) MCB_CUDA(ctx, cudaMemcpyAsync(T, s->stage, 4 * L, cudaMemcpyDeviceToHost, st));
  if (Omega && s->Om) MCB_CUDA(ctx, cudaMemcpyAsync(Omega, s->Om, 4 * L, cudaMemcpyDeviceToHost, st));
  MCB_CUDA(ctx, cudaStreamSynchronize(st));
  return MCB_OK;
}

}  // namespace

namespace mcb {

// Per medium {x0, E/R} with x0 = log A - E / (R T0), T0 = base temperature in kelvin (FP64 on the
// host); E/R = 0 marks media without damage.
void heat_damage_table(const mcb_heat_params *p, double base, float2 *out) {
  const double T0 = base + kCelsiusZero;
  for (int m = 0; m < p->nM; m++) {
    const double c1 = p->E[m] / kGasR;
    out[m] = p->E[m] != 0.0 ? make_float2((float)(std::log(p->A[m]) - c1 / T0), (float)c1) : make_float2(0.f, 0.f);
  }
}

mcb_status heat_check_params(mcb_ctx *ctx, const mcb_heat_params *p) { return check_params(ctx, p); }

mcb_status heat_state_init(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, const float *T,
                           const float *Omega) {
  const bool damage = Omega != nullptr;
  if (!state_fits(s, p, damage, false)) MCB_TRY(state_alloc(ctx, s, p, damage));
  return state_upload(ctx, s, p, T, Omega);
}

void heat_state_release(mcb_heat_state *s) { free_state_buffers(s); }

mcb_status heat_stepper(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, HeatStepper *out) {
  cudaStream_t st = ctx->stream;
  HeatStepper &k = *out;
  k.h = make_dev(s, p);
  const HeatDev &h = k.h;
  const int grid = ctx->num_sms * 8;
  const long long L = s->L, nx = s->nx, ny = s->ny, nz = s->nz;
  if (s->factoredDt != p->dt || s->factoredHs != (int)(p->heatBoundaryType != 0)) {
    for (int dir = 0; dir < 3; dir++)
      factor_kernel<<<grid, 128, 0, st>>>(h, dir, s->ib + (size_t)dir * L, s->fb + (size_t)dir * L);
    neighbour_code_kernel<<<grid, 256, 0, st>>>(h, s->nb);
    MCB_CUDA(ctx, cudaGetLastError());
    s->factoredDt = p->dt;
    s->factoredHs = (int)(p->heatBoundaryType != 0);
  }
  MCB_CUDA(ctx, cudaMemsetAsync(s->maxEnc, 0, 4 * (size_t)s->nM, st));
  MCB_CUDA(ctx, cudaMemsetAsync(s->step, 0, 16, st));
  if (s->dOm) MCB_CUDA(ctx, cudaMemsetAsync(s->dOm, 0, 4 * (size_t)L, st));
  k.smemX = x_smem((int)nx);
  MCB_CUDA(ctx, cudaFuncSetAttribute(pass_x_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smemX));
  k.tw = s->tw;
  if (k.tw == 32) MCB_TRY(setup_yz<32>(ctx, (int)ny, (int)nz));
  else if (k.tw == 16) MCB_TRY(setup_yz<16>(ctx, (int)ny, (int)nz));
  else MCB_TRY(setup_yz<8>(ctx, (int)ny, (int)nz));
  const long long tilesX = ((ny + h.xl - 1) / h.xl) * nz;
  k.gridX = (int)std::min<long long>(tilesX, (long long)ctx->num_sms * 64);
  const long long tiles = ((nx + k.tw - 1) / k.tw) * std::max(ny, nz);
  k.gridYZ = (int)std::min<long long>(tiles, (long long)ctx->num_sms * 64);
  return MCB_OK;
}

void heat_step_launch(const HeatStepper &k, cudaStream_t q) {
  pass_x_kernel<<<k.gridX, 256, k.smemX, q>>>(k.h);
  if (k.tw == 32) launch_yz<32>(k.h, k.gridYZ, q);
  else if (k.tw == 16) launch_yz<16>(k.h, k.gridYZ, q);
  else launch_yz<8>(k.h, k.gridYZ, q);
}

}  // namespace mcb

extern "C" mcb_status mcb_heat_forward(mcb_ctx *ctx, const mcb_heat_params *p, float *T, float *Omega, double *sensorTemps,
                                       float *maxMediaTemps) {
  using namespace mcb;
  if (!ctx) return MCB_EINVAL;
  MCB_TRY(check_params(ctx, p));
  if (!T || !maxMediaTemps) return set_error(ctx, MCB_EINVAL, "NULL T or maxMediaTemps");
  if (p->nSensors > 0 && !sensorTemps) return set_error(ctx, MCB_EINVAL, "sensorTemps is NULL");
  MCB_CUDA(ctx, cudaSetDevice(ctx->device));
  // the context keeps one state; it is reallocated when the grid, its kind or the damage setting changes
  mcb_heat_state *s = ctx->heat;
  const bool damage = Omega != nullptr;
  if (!s) {
    s = new mcb_heat_state();
    s->ctx = ctx;
    ctx->heat = s;
  }
  if (stream_supported(p->nx, p->ny, p->nz)) {
    if (!state_fits(s, p, damage, true)) MCB_TRY(stream_alloc(ctx, s, p, damage));
    MCB_TRY(stream_upload(ctx, s, p, T, Omega));
    if (p->lightsOn) MCB_TRY(stream_upload_q(ctx, s, p->dTdt_abs));
    MCB_TRY(sensor_buffers(ctx, s, p));
    MCB_TRY(stream_step(ctx, s, p, s->sens, sensorTemps, maxMediaTemps, true));
    return stream_download(ctx, s, T, Omega);
  }
  if (!state_fits(s, p, damage, false)) MCB_TRY(state_alloc(ctx, s, p, damage));
  MCB_TRY(state_upload(ctx, s, p, T, Omega));
  MCB_TRY(state_step(ctx, s, p, sensorTemps, maxMediaTemps));
  return state_download(ctx, s, T, Omega);
}

extern "C" mcb_status mcb_heat_state_create(mcb_ctx *ctx, const mcb_heat_params *p, const float *T, const float *Omega,
                                            mcb_heat_state **out) {
  using namespace mcb;
  if (!ctx) return MCB_EINVAL;
  if (!out || !T) return set_error(ctx, MCB_EINVAL, "NULL argument");
  MCB_TRY(check_params(ctx, p));
  MCB_CUDA(ctx, cudaSetDevice(ctx->device));
  mcb_heat_state *s = new mcb_heat_state();
  s->ctx = ctx;
  mcb_status st;
  if (stream_supported(p->nx, p->ny, p->nz)) {
    st = stream_alloc(ctx, s, p, Omega != nullptr);
    if (st == MCB_OK) st = stream_upload(ctx, s, p, T, Omega);
    if (st == MCB_OK && p->lightsOn) st = stream_upload_q(ctx, s, p->dTdt_abs);
  } else {
    st = state_alloc(ctx, s, p, Omega != nullptr);
    if (st == MCB_OK) st = state_upload(ctx, s, p, T, Omega);
  }
  if (st != MCB_OK) {
    free_state_buffers(s);
    delete s;
    return st;
  }
  *out = s;
  return MCB_OK;
}

extern "C" mcb_status mcb_heat_state_step(mcb_heat_state *s, const mcb_heat_params *p, double *sensorTemps,
                                          float *maxMediaTemps) {
  using namespace mcb;
  if (!s) return MCB_EINVAL;
  mcb_ctx *ctx = s->ctx;
  MCB_TRY(check_params(ctx, p));
  if (p->nx != s->nx || p->ny != s->ny || p->nz != s->nz || p->nM != s->nM)
    return set_error(ctx, MCB_EINVAL, "parameters do not match the state's grid");
  if (p->nSensors > 0 && !sensorTemps) return set_error(ctx, MCB_EINVAL, "sensorTemps is NULL");
  MCB_CUDA(ctx, cudaSetDevice(ctx->device));
  if (s->streamed) {
    if (p->lightsOn && p->dTdt_abs) MCB_TRY(stream_upload_q(ctx, s, p->dTdt_abs));
    MCB_TRY(sensor_buffers(ctx, s, p));
    return stream_step(ctx, s, p, s->sens, sensorTemps, maxMediaTemps, true);
  }
  if (p->lightsOn && p->dTdt_abs)
    MCB_CUDA(ctx, cudaMemcpyAsync(s->Q, p->dTdt_abs, 4 * s->L, cudaMemcpyHostToDevice, ctx->stream));
  return state_step(ctx, s, p, sensorTemps, maxMediaTemps);
}

extern "C" mcb_status mcb_heat_state_read(mcb_heat_state *s, float *T, float *Omega) {
  using namespace mcb;
  if (!s) return MCB_EINVAL;
  MCB_CUDA(s->ctx, cudaSetDevice(s->ctx->device));
  if (s->streamed) return stream_download(s->ctx, s, T, Omega);
  return state_download(s->ctx, s, T, Omega);
}

extern "C" mcb_status mcb_heat_state_destroy(mcb_heat_state *s) {
  if (!s) return MCB_OK;
  cudaSetDevice(s->ctx->device);
  cudaStreamSynchronize(s->ctx->stream);
  free_state_buffers(s);
  delete s;
  return MCB_OK;
}

extern "C" double mcb_last_kernel_ms(const mcb_ctx *ctx) { return ctx ? ctx->lastKernelMs : 0.0; }

// ---------------------------------------------------------------------------------------------
// mcb_heat_forward_static: mcb_heat_forward with no device (or host heap) allocation.
//
// Who cannot allocate: a host that shares the GPU with an allocator that has already reserved
// most of HBM (MATLAB's gpuArray pool, a PyTorch caching allocator) sees cudaMalloc fail at call
// time; and a caller whose other streams keep working on the same device is stalled by the
// device-wide synchronisation of cudaFree, which the grow-only buffers of mcb_heat_forward
// perform when the grid changes. This entry instead carves every buffer it needs out of one
// file-scope __device__ array of kHeatScratchBytes (32 MiB, reserved when the module loads);
// requests that do not fit are rejected with MCB_EINVAL and a message naming the limit.
//
// Zero-initialised state: the per-medium maxima, the step counter and the damage increments
// must start at zero for every call; the call clears them itself (cudaMemsetAsync) before its
// first step, and writes every other buffer before reading it, so nothing carries over from a
// previous call.
//
// There is one scratch per device. Calls that overlap in time on the same device (two host
// threads, or two contexts on one device) share it and race; callers serialise them.
// The first call on a device performs the set-up: it looks up the scratch's device address
// with cudaGetSymbolAddress (which may load this file's module) and caches it.
// The call is synchronous: it sums T on the host, then waits for ctx->stream and reads its
// events before returning, so it must not be made while ctx->stream is being captured.
// ---------------------------------------------------------------------------------------------
namespace {
constexpr size_t kHeatScratchBytes = (size_t)32 << 20;
constexpr int kScratchDevices = 64;
}  // namespace

static __device__ __align__(256) unsigned char g_heat_scratch[kHeatScratchBytes];

namespace {

std::mutex g_scratch_mu;
void *g_scratch_ptr[kScratchDevices];

// Device address of g_heat_scratch on the context's device (current device already set).
mcb_status heat_scratch(mcb_ctx *ctx, void **out) {
  using namespace mcb;
  if (ctx->device < 0 || ctx->device >= kScratchDevices)
    return set_error(ctx, MCB_EINVAL, "mcb_heat_forward_static: device %d out of range", ctx->device);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[ctx->device]) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_heat_scratch);
    if (e != cudaSuccess || !ptr)
      return set_error(ctx, MCB_ECUDA, "mcb_heat_forward_static: cudaGetSymbolAddress of the scratch failed: %s",
                       cudaGetErrorString(e));
    g_scratch_ptr[ctx->device] = ptr;
  }
  *out = g_scratch_ptr[ctx->device];
  return MCB_OK;
}

// Bump carving of the scratch (256-byte aligned pieces); base == nullptr only measures.
struct ScratchCarve {
  char *base;
  size_t used;
  void *take(size_t bytes) {
    void *q = base ? base + used : nullptr;
    used += (bytes + 255) & ~(size_t)255;
    return q;
  }
};

// Lays the streamed stepper's buffers and the sensor arrays out in the scratch (or measures
// them when c.base is null).
void carve_static_stream(ScratchCarve &c, mcb_heat_state *s, const mcb_heat_params *p, bool damage) {
  const int nS = p->nSensors;
  stream_carve([&](size_t b) { return c.take(b); }, s, p, damage, p->lightsOn != 0);
  s->sIdx = nS ? (double *)c.take(8 * (size_t)nS) : nullptr;
  s->sW = nS ? (double *)c.take(24 * (size_t)nS) : nullptr;
  s->sens = nS ? (double *)c.take(8 * (size_t)nS * (size_t)(p->steps + 1)) : nullptr;
}

// Lays the factored stepper's buffers out in the scratch (or measures them when c.base is null).
void carve_static_state(ScratchCarve &c, mcb_heat_state *s, const mcb_heat_params *p, bool damage) {
  const long long L = (long long)p->nx * p->ny * p->nz;
  const int nM = p->nM, nS = p->nSensors;
  s->T = (float *)c.take(4 * L);
  s->A = (float *)c.take(4 * L);
  s->Q = p->lightsOn ? (float *)c.take(4 * L) : nullptr;
  s->stage = (float *)c.take(4 * (size_t)std::max<long long>(L, nM));
  s->ib = (float *)c.take(12 * L);
  s->fb = (float2 *)c.take(24 * L);
  s->nb = (uint8_t *)c.take(L);
  s->Sz = (float *)c.take(4 * L);
  s->Om = damage ? (float *)c.take(4 * L) : nullptr;
  s->dOm = damage ? (float *)c.take(4 * L) : nullptr;
  s->M = (uint8_t *)c.take(L);
  s->c = (float *)c.take(12 * (size_t)nM * nM);
  s->logA = (double *)c.take(8 * (size_t)nM);
  s->dmg = (float2 *)c.take(8 * (size_t)nM);
  s->E = (double *)c.take(8 * (size_t)nM);
  s->maxEnc = (unsigned int *)c.take(4 * (size_t)nM);
  s->step = (int *)c.take(16);
  s->sIdx = nS ? (double *)c.take(8 * (size_t)nS) : nullptr;
  s->sW = nS ? (double *)c.take(24 * (size_t)nS) : nullptr;
  s->sens = nS ? (double *)c.take(8 * (size_t)nS * (size_t)(p->steps + 1)) : nullptr;
}

}  // namespace

extern "C" mcb_status mcb_heat_forward_static(mcb_ctx *ctx, const mcb_heat_params *p, float *T, float *Omega,
                                              double *sensorTemps, float *maxMediaTemps) {
  using namespace mcb;
  if (!ctx) return MCB_EINVAL;
  MCB_TRY(check_params(ctx, p));
  if (!T || !maxMediaTemps) return set_error(ctx, MCB_EINVAL, "NULL T or maxMediaTemps");
  if (p->nSensors > 0 && !sensorTemps) return set_error(ctx, MCB_EINVAL, "sensorTemps is NULL");
  const bool damage = Omega != nullptr;
  // the sensor history alone must fit before it is measured: 8 * nS * (steps + 1) could wrap
  if (p->nSensors > 0 && (unsigned long long)p->steps + 1 > kHeatScratchBytes / (8 * (size_t)p->nSensors))
    return set_error(ctx, MCB_EINVAL,
                     "mcb_heat_forward_static: %d sensors over %d steps need more device scratch than its static "
                     "limit of %zu bytes (8 bytes per sensor and step); use mcb_heat_forward",
                     p->nSensors, p->steps, kHeatScratchBytes);
  mcb_heat_state s{};  // a view of the scratch; nothing in it is freed
  const bool streamed = stream_supported(p->nx, p->ny, p->nz);
  ScratchCarve measure{nullptr, 0};
  if (streamed) carve_static_stream(measure, &s, p, damage);
  else carve_static_state(measure, &s, p, damage);
  if (measure.used > kHeatScratchBytes)
    return set_error(ctx, MCB_EINVAL,
                     "mcb_heat_forward_static: this grid needs %zu bytes of device scratch, more than its static "
                     "limit of %zu bytes (about 22 bytes per voxel, 30 with damage, of the x-padded grid, plus 8 per "
                     "sensor and step); use mcb_heat_forward",
                     measure.used, kHeatScratchBytes);
  MCB_CUDA(ctx, cudaSetDevice(ctx->device));
  void *base = nullptr;
  MCB_TRY(heat_scratch(ctx, &base));
  ScratchCarve carve{(char *)base, 0};
  if (streamed) {
    carve_static_stream(carve, &s, p, damage);
    StreamMaps maps;  // on the stack: the descriptors only live for this call
    s.maps = &maps;
    s.ctx = ctx;
    s.streamed = true;
    mcb_status rc = stream_maps(ctx, &s);
    if (rc == MCB_OK) rc = stream_upload(ctx, &s, p, T, Omega);
    if (rc == MCB_OK && p->lightsOn) rc = stream_upload_q(ctx, &s, p->dTdt_abs);
    if (rc == MCB_OK && p->nSensors) {
      const cudaError_t e1 = cudaMemcpyAsync(s.sIdx, p->tempSensorCornerIdxs, 8 * (size_t)p->nSensors,
                                             cudaMemcpyHostToDevice, ctx->stream);
      const cudaError_t e2 = cudaMemcpyAsync(s.sW, p->tempSensorInterpWeights, 24 * (size_t)p->nSensors,
                                             cudaMemcpyHostToDevice, ctx->stream);
      if (e1 != cudaSuccess || e2 != cudaSuccess)
        rc = set_error(ctx, MCB_ECUDA, "mcb_heat_forward_static: sensor upload failed");
    }
    // plain launches per step: instantiating a CUDA graph may allocate
    if (rc == MCB_OK) rc = stream_step(ctx, &s, p, s.sens, sensorTemps, maxMediaTemps, false);
    if (rc == MCB_OK) rc = stream_download(ctx, &s, T, Omega);
    s.maps = nullptr;
    return rc;
  }
  carve_static_state(carve, &s, p, damage);
  s.ctx = ctx;
  s.nx = p->nx;
  s.ny = p->ny;
  s.nz = p->nz;
  s.nM = p->nM;
  s.L = (long long)p->nx * p->ny * p->nz;
  s.damage = damage;
  s.tw = std::min(yz_tile_width(p->ny), yz_tile_width(p->nz));

  cudaStream_t st = ctx->stream;
  const long long L = s.L, nt = p->steps;
  const int nM = s.nM, nS = p->nSensors;
  // upload (the same steps as the allocating path; logA is staged on the stack: nM <= 256)
  double sum = 0.0;
  for (long long k = 0; k < L; k++) sum += T[k];
  s.base = sum / (double)L;
  double logA[256];
  for (int m = 0; m < nM; m++) logA[m] = std::log(p->A[m]);
  float2 dmg[256];
  damage_table(p, s.base, dmg);
  MCB_CUDA(ctx, cudaMemcpyAsync(s.stage, T, 4 * L, cudaMemcpyHostToDevice, st));
  to_dev_kernel<<<ctx->num_sms * 8, 256, 0, st>>>(s.stage, s.T, s.base, L);
  MCB_CUDA(ctx, cudaMemcpyAsync(s.M, p->M, L, cudaMemcpyHostToDevice, st));
  if (s.Q) MCB_CUDA(ctx, cudaMemcpyAsync(s.Q, p->dTdt_abs, 4 * L, cudaMemcpyHostToDevice, st));
  if (s.Om) MCB_CUDA(ctx, cudaMemcpyAsync(s.Om, Omega, 4 * L, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(s.c, p->dTdtperdeltaT, 12 * (size_t)nM * nM, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(s.logA, logA, 8 * (size_t)nM, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(s.E, p->E, 8 * (size_t)nM, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(s.dmg, dmg, 8 * (size_t)nM, cudaMemcpyHostToDevice, st));
  if (nS) {
    MCB_CUDA(ctx, cudaMemcpyAsync(s.sIdx, p->tempSensorCornerIdxs, 8 * (size_t)nS, cudaMemcpyHostToDevice, st));
    MCB_CUDA(ctx, cudaMemcpyAsync(s.sW, p->tempSensorInterpWeights, 24 * (size_t)nS, cudaMemcpyHostToDevice, st));
  }
  // step: factor the line matrices, clear the zero-start state, then plain launches per step
  HeatStepper ks;
  MCB_TRY(heat_stepper(ctx, &s, p, &ks));
  const HeatDev &h = ks.h;
  const int grid = ctx->num_sms * 8;
  MCB_CUDA(ctx, cudaEventRecord(ctx->ev0, st));
  for (long long k = 0; k < nt; k++) heat_step_launch(ks, st);
  if (nS) final_sensors_kernel<<<1, 128, 0, st>>>(h);
  if (s.dOm) merge_omega_kernel<<<grid, 256, 0, st>>>(s.Om, s.dOm, L);
  MCB_CUDA(ctx, cudaGetLastError());
  MCB_CUDA(ctx, cudaEventRecord(ctx->ev1, st));
  decode_max_kernel<<<1, 256, 0, st>>>(s.maxEnc, s.stage, nM);
  MCB_CUDA(ctx, cudaMemcpyAsync(maxMediaTemps, s.stage, 4 * (size_t)nM, cudaMemcpyDeviceToHost, st));
  if (nS) MCB_CUDA(ctx, cudaMemcpyAsync(sensorTemps, s.sens, 8 * (size_t)nS * (nt + 1), cudaMemcpyDeviceToHost, st));
  // download (after the maxima have left the stage buffer: same-stream order)
  from_dev_kernel<<<ctx->num_sms * 8, 256, 0, st>>>(s.T, s.stage, s.base, L);
  MCB_CUDA(ctx, cudaMemcpyAsync(T, s.stage, 4 * L, cudaMemcpyDeviceToHost, st));
  if (s.Om) MCB_CUDA(ctx, cudaMemcpyAsync(Omega, s.Om, 4 * L, cudaMemcpyDeviceToHost, st));
  MCB_CUDA(ctx, cudaGetLastError());
  MCB_CUDA(ctx, cudaStreamSynchronize(st));
  float ms = 0.f;
  MCB_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->lastKernelMs = ms;
  return MCB_OK;
}

namespace mcb {
mcb_status stream_state_create(mcb_ctx *ctx, mcb_heat_state *s, const mcb_heat_params *p, const float *T) {
  s->ctx = ctx;
  MCB_TRY(stream_alloc(ctx, s, p, false));
  MCB_TRY(stream_upload(ctx, s, p, T, nullptr));
  if (p->lightsOn) MCB_TRY(stream_upload_q(ctx, s, p->dTdt_abs));
  return MCB_OK;
}
}  // namespace mcb
