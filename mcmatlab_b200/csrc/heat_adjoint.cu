// Reverse-time adjoint of the DG-ADI heat stepper with sqrt(N) checkpointing, behind
// mcb_heat_adjoint. No counterpart in the reference (finiteElementHeatPropagator.c has no
// derivative code); the forward it differentiates is the stepper of heat_adi.cu, i.e. the
// scheme of finiteElementHeatPropagator.c:249-647.
//
// One forward step, as linear algebra on the grid (D_d: the conduction operator along d, rows of
// heat-sinked voxels zero; X, Y, Z = I - dt/2 D_x, D_y, D_z):
//   A1 = X^-1 (T + dt (Q + D_x T / 2 + D_y T + D_z T))
//   A2 = Y^-1 (A1 - dt/2 D_y T)
//   T' = Z^-1 (A2 - dt/2 D_z T)
// The reverse step takes lambda' = dJ/dT' (plus the objective's terms at T') to
//   rho3 = Z^-T lambda',  rho2 = Y^-T rho3,  rho1 = X^-T rho2
//   lambda = rho1 + D_x^T (dt/2 rho1) + D_y^T (dt rho1 - dt/2 rho2) + D_z^T (dt rho1 - dt/2 rho3)
// and accumulates dJ/dQ += dt rho1 and dJ/dc over the medium pairs of every voxel face.
//
// The transposed line solves reuse the forward's inverse pivots: with X = L U (Thomas), the
// system X^T y = r is the same two first-order recurrences with the multipliers shifted by one
// row (forward multiplier of row i = cc_{i-1} / b'_{i-1}, backward multiplier = a_{i+1} / b'_i),
// so the warp-scan solvers of the forward run unchanged. A1 and A2 are not stored by the
// forward: they follow from T and T' by explicit stencils, A2 = T' - dt/2 D_z (T' - T) and
// A1 = A2 - dt/2 D_y (A2 - T), which the assembly forms in shared memory from its staged planes.
//
// Memory: nCheckpoints states of T from the forward sweep and its final state, a ring of the
// K - 1 inner states of a segment recomputed during the reverse sweep (K = ceil(steps /
// nCheckpoints); a segment's end states are checkpoints), and six grid-sized work arrays. With
// nCheckpoints = steps every state is stored and nothing is recomputed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "heat_host.h"

namespace mcb {
namespace {

constexpr int kAdjMaxMedia = 32;

struct AdjDev {
  HeatDev h;             // grid, media, coefficients, pivots, boundary type, dt
  const float *Tn, *Tp;  // T^n, T^{n+1} (deviations from the state's base temperature)
  float *lam;            // lambda^{n+1}; the objective's terms at T^{n+1} are added in place
  float *r1, *r2, *r3;   // adjoints of the three solves' right-hand sides
  float *lamOut;         // lambda^n
  float *dQ;             // dJ/dQ accumulator, or nullptr (light off or not requested)
  int dQinX;             // dQ accumulated by the X^T x-line solve (adj_xline_kernel) instead of the assembly
  double *dc;            // [nM x nM x 3] dJ/dc accumulator
  // objective terms as sparse lists
  int nD;
  const int *dIdx;
  const float *dW;
  float *gbuf;  // per damage-list entry: d(damage increment)/dT (same for T^n and T^{n+1})
  double *Jd;
  int nP;
  const int *pIdx;
  const float *pW;
  const int *pStep;  // step (1..steps) at which each peak-list voxel reached its maximum
  int step;          // n + 1 of the step being reversed
};

// Objective terms at T^{n+1}: damage (weight w, increment dt A exp(-E / R Tmid)) contributes
// w dOmega/dT to lambda' (and, kept in gbuf, the same to lambda^n); a peak-list voxel whose
// maximum was reached at this step contributes its weight.
__global__ void adj_seed_kernel(AdjDev a) {
  const HeatDev &h = a.h;
  double jd = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.nD; k += gridDim.x * blockDim.x) {
    const int v = a.dIdx[k];
    const int m = h.M[v];
    float g = 0.f;
    if (h.E[m] != 0.0) {
      const double tk = 0.5 * ((double)a.Tn[v] + (double)a.Tp[v]) + h.base + kCelsiusZero;
      const double rate = exp(h.logA[m] - h.E[m] / (kGasR * tk));
      const double w = a.dW[k];
      jd += w * h.dtd * rate;
      g = (float)(0.5 * w * h.dtd * rate * h.E[m] / (kGasR * tk * tk));
      atomicAdd(&a.lam[v], g);
    }
    a.gbuf[k] = g;
  }
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.nP; k += gridDim.x * blockDim.x)
    if (a.pStep[k] == a.step) atomicAdd(&a.lam[a.pIdx[k]], a.pW[k]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) jd += __shfl_down_sync(0xffffffffu, jd, off);
  if ((threadIdx.x & 31) == 0 && jd != 0.0) atomicAdd(a.Jd, jd);
}

__global__ void adj_damage_tail_kernel(AdjDev a) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.nD; k += gridDim.x * blockDim.x)
    a.lamOut[a.dIdx[k]] += a.gbuf[k];
}

// X^T solve: rho1 = X^-T rho2, for x lines longer than adj_xline_kernel takes (512 voxels; the
// assembly then adds dJ/dQ). Same tiling as the factored forward X pass (h.xl lines per block),
// lines staged in shared memory and solved by solve_lines.
__global__ void __launch_bounds__(256, 3) adj_solve_x_kernel(AdjDev a) {
  extern __shared__ unsigned char smem[];
  const HeatDev &h = a.h;
  const int nx = h.nx, ny = h.ny, nz = h.nz;
  const int sxy = nx * ny;
  const int P = nx + 1;
  const int XL = h.xl;
  float *rhs = (float *)smem;
  float *fm = rhs + XL * P;
  float *bm = fm + XL * P;
  float *ib = bm + XL * P;
  const float *ibx = h.ib;
  const int yTiles = (ny + XL - 1) / XL;
  for (int tile = blockIdx.x; tile < yTiles * nz; tile += gridDim.x) {
    const int y0 = (tile % yTiles) * XL, iz = tile / yTiles;
    const int cnt = min(XL, ny - y0);
    const int total = cnt * nx;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int l = e / nx, x = e - l * nx;
      const int iy = y0 + l;
      const int v = x + iy * nx + iz * sxy;
      const bool lineSinked = h.hs && (iy == 0 || iy == ny - 1 || iz == 0 || iz == nz - 1);
      const int mi = h.M[v];
      const float ibv = ibx[v];
      float f = 0.f, b = 0.f;
      if (x > 0 && !row_sinked(h, lineSinked, x - 1, nx)) f = h.hdt * cf(h, h.M[v - 1], mi, 0) * ibx[v - 1];
      if (x < nx - 1 && !row_sinked(h, lineSinked, x + 1, nx)) b = h.hdt * cf(h, h.M[v + 1], mi, 0) * ibv;
      rhs[l * P + x] = a.r2[v];
      fm[l * P + x] = f;
      bm[l * P + x] = b;
      ib[l * P + x] = ibv;
    }
    __syncthreads();
    solve_lines(rhs, fm, bm, ib, nx, 1, P, cnt);
    __syncthreads();
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int l = e / nx, x = e - l * nx;
      a.r1[x + (y0 + l) * nx + iz * sxy] = rhs[l * P + x];
    }
    __syncthreads();
  }
}

template <int TW>
__host__ __device__ constexpr size_t adj_yz_tile_bytes(int n) {
  return (size_t)n * (4 * (TW + 1) * 4 + TW);
}

// Y^T / Z^T solves: rho2 = Y^-T rho3 (ZPASS false), rho3 = Z^-T lambda' (ZPASS true), for lines
// longer than adj_col_kernel takes (320 rows). Same tiling as the factored forward Y/Z passes:
// TW consecutive x positions, one line per x.
template <int TW, bool ZPASS>
__global__ void __launch_bounds__(256, 3) adj_solve_yz_kernel(AdjDev a) {
  extern __shared__ unsigned char smem[];
  constexpr int P = TW + 1;
  const HeatDev &h = a.h;
  const int nx = h.nx, ny = h.ny, nz = h.nz;
  const int sxy = nx * ny;
  const int n = ZPASS ? nz : ny;
  const int st = ZPASS ? sxy : nx;
  const int dir = ZPASS ? 2 : 1;
  float *rhs = (float *)smem;
  float *ib = rhs + n * P;
  float *fm = ib + n * P;
  float *bm = fm + n * P;
  uint8_t *Ms = (uint8_t *)(bm + n * P);
  const float *in = ZPASS ? a.lam : a.r3;
  float *out = ZPASS ? a.r3 : a.r2;
  const int xTiles = (nx + TW - 1) / TW;
  const int nOther = ZPASS ? ny : nz;
  const float *ibd = h.ib + (size_t)dir * sxy * nz;
  constexpr int RPI = 256 / TW;
  const int cx = threadIdx.x % TW, r0 = threadIdx.x / TW;
  for (int tile = blockIdx.x; tile < xTiles * nOther; tile += gridDim.x) {
    const int x0 = (tile % xTiles) * TW;
    const int other = tile / xTiles;
    const int base = ZPASS ? other * nx : other * sxy;
    const bool otherSinked = h.hs && (other == 0 || other == nOther - 1);
    const int x = x0 + cx;
    if (x < nx) {
      for (int r = r0; r < n; r += RPI) {
        const int v = base + x + r * st;
        rhs[r * P + cx] = in[v];
        ib[r * P + cx] = ibd[v];
        Ms[r * TW + cx] = h.M[v];
      }
    }
    __syncthreads();
    if (x < nx) {
      const bool lineSinked = otherSinked || (h.hs && (x == 0 || x == nx - 1));
      for (int r = r0; r < n; r += RPI) {
        const int mi = Ms[r * TW + cx];
        float f = 0.f, b = 0.f;
        if (r > 0 && !row_sinked(h, lineSinked, r - 1, n))
          f = h.hdt * cf(h, Ms[(r - 1) * TW + cx], mi, dir) * ib[(r - 1) * P + cx];
        if (r < n - 1 && !row_sinked(h, lineSinked, r + 1, n))
          b = h.hdt * cf(h, Ms[(r + 1) * TW + cx], mi, dir) * ib[r * P + cx];
        fm[r * P + cx] = f;
        bm[r * P + cx] = b;
      }
    }
    __syncthreads();
    solve_lines(rhs, fm, bm, ib, n, P, 1, min(TW, nx - x0));
    __syncthreads();
    if (x < nx) {
      for (int r = r0; r < n; r += RPI) out[base + x + r * st] = rhs[r * P + cx];
    }
    __syncthreads();
  }
}


// The assembly marching along z: a block owns a 32 x 8 tile of (x, y) columns, one thread per
// column, and walks the planes of its z chunk. r1, T^n, T^{n+1} and the media are staged in
// shared memory per plane with a one-voxel halo, on a ring of four planes that also serves their
// z neighbours; r3 on a ring of four centre tiles, r2 with its y halo on two planes. Each array
// is read from memory once (plus the tile halos) instead of once per neighbour, and loads run a
// plane ahead of the staging. The step's intermediates are formed per plane from the staged
// tiles, one plane ahead of the assembly (two barriers per plane): A2 = T' - dt/2 D_z (T' - T) on
// the halo tile, then A1 = A2 - dt/2 D_y (A2 - T) on the x-halo rows.
constexpr int kZX = 32, kZY = 8, kZHX = kZX + 2, kZHY = kZY + 2;
constexpr int kZHN = kZHX * kZHY;  // halo tile (340)
constexpr int kZCN = kZX * kZY;    // centre tile, one thread per column (256)
constexpr int kZA1 = kZY * kZHX;   // x-halo tile (272)
constexpr int kZR2 = kZHY * kZX;   // y-halo tile (320)
constexpr int kZChunk = 25;        // planes per block
static_assert(kZHN <= 2 * kZCN && kZR2 <= 2 * kZCN && kZA1 <= 2 * kZCN, "two staging slots per thread cover every tile");

// out = U - dt/2 D_d (U - T^n) at one voxel along the line direction d, from its value u, T^n
// value t and medium m and those of its two line neighbours (l, r; has*: the neighbour exists).
// Both neighbours present in the voxel's own medium take one coefficient; a heat-sinked voxel
// keeps U.
// C: the conduction table of direction d in shared memory (C[mi + nM mj] = c(mi, mj, d)).
__device__ __forceinline__ float recon_point(const float *C, int nM, float hdt, bool sink, int m, float u, float t,
                                             bool hasl, int ml, float ul, float tl, bool hasr, int mr, float ur, float tr) {
  if (sink) return u;
  const float w = u - t;
  float dd;
  if (hasl && hasr && ml == m && mr == m) {
    dd = C[m + nM * m] * ((ul - tl) + (ur - tr) - 2.f * w);
  } else {
    dd = 0.f;
    if (hasl) dd += C[m + nM * ml] * ((ul - tl) - w);
    if (hasr) dd += C[m + nM * mr] * ((ur - tr) - w);
  }
  return u - hdt * dd;
}

__global__ void __launch_bounds__(kZCN, 1024 / kZCN) adj_assemble_z_kernel(AdjDev a) {
  const HeatDev &h = a.h;
  // dynamic: the dJ/dc block sums [3 nM^2] (double) and the conduction table c [3 nM^2]
  extern __shared__ double sdc[];
  __shared__ float sR1[4][kZHN], sTN[4][kZHN], sTP[4][kZHN], sR3[4][kZCN];
  __shared__ float sR2[2][kZR2], sA2[2][kZHN], sA1[2][kZA1];
  __shared__ uint8_t sM[4][kZHN + 4];
  const int nM = h.nM, nM2 = nM * nM;
  float *sC = reinterpret_cast<float *>(sdc + 3 * nM2);
  for (int k = threadIdx.x; k < 3 * nM2; k += blockDim.x) {
    sdc[k] = 0.0;
    sC[k] = h.c[k];
  }
  auto cfs = [&](int mi, int mj, int d) { return sC[mi + nM * mj + d * nM2]; };
  const int nx = h.nx, ny = h.ny, nz = h.nz;
  const long long sxy = (long long)nx * ny;
  const int x0 = blockIdx.x * kZX, y0 = blockIdx.y * kZY;
  const int t = threadIdx.x, tx = t % kZX, ty = t / kZX;
  // this thread's staging slots: halo elements t and t + kZCN (< kZHN), centre element t, y-halo
  // elements t and t + kZCN (< kZR2)
  auto hoff = [&](int e, int &x, int &y) { x = x0 - 1 + e % kZHX; y = y0 - 1 + e / kZHX; };
  auto inside = [&](int x, int y) { return x >= 0 && x < nx && y >= 0 && y < ny; };
  // prefetch registers of one plane
  float pR1[2], pTN[2], pTP[2], pR3, pR2[2];
  int pM[2];
  auto load_ring = [&](int iz) {
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int e = t + kZCN * q;
      pR1[q] = pTN[q] = pTP[q] = 0.f;
      pM[q] = 0;
      if (e < kZHN) {
        int x, y;
        hoff(e, x, y);
        if (inside(x, y)) {
          const long long v = x + (long long)y * nx + iz * sxy;
          pR1[q] = a.r1[v];
          pTN[q] = a.Tn[v];
          pTP[q] = a.Tp[v];
          pM[q] = h.M[v];
        }
      }
    }
    pR3 = 0.f;
    const int x = x0 + tx, y = y0 + ty;
    if (x < nx && y < ny) pR3 = a.r3[x + (long long)y * nx + iz * sxy];
  };
  auto store_ring = [&](int slot) {
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int e = t + kZCN * q;
      if (e < kZHN) {
        sR1[slot][e] = pR1[q];
        sTN[slot][e] = pTN[q];
        sTP[slot][e] = pTP[q];
        sM[slot][e] = (uint8_t)pM[q];
      }
    }
    sR3[slot][t] = pR3;
  };
  auto load_single = [&](int iz) {
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int e = t + kZCN * q;
      pR2[q] = 0.f;
      if (e < kZR2) {
        const int x = x0 + e % kZX, y = y0 - 1 + e / kZX;
        if (inside(x, y)) pR2[q] = a.r2[x + (long long)y * nx + iz * sxy];
      }
    }
  };
  auto store_single = [&](int slot) {
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int e = t + kZCN * q;
      if (e < kZR2) sR2[slot][e] = pR2[q];
    }
  };
  // this block's planes [z0, z1) (blockIdx.z: z chunks of kZChunk planes, for more blocks in flight)
  const int z0 = blockIdx.z * kZChunk, z1 = min(nz, z0 + kZChunk);
  const float dt = h.dt, hdt = h.hdt;
  // A2 of plane p on the halo tile, into sA2[p & 1] (z neighbours from the ring)
  auto form_a2 = [&](int p) {
    const int sc = p & 3, sp = (p + 1) & 3, sm = (p + 3) & 3;
    float *dst = sA2[p & 1];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int e = t + kZCN * q;
      if (e < kZHN) {
        int x, y;
        hoff(e, x, y);
        float v = 0.f;
        if (inside(x, y))
          v = recon_point(sC + 2 * nM2, nM, hdt, sinked(h, x, y, p), sM[sc][e], sTP[sc][e], sTN[sc][e], p > 0,
                          sM[sm][e], sTP[sm][e], sTN[sm][e], p < nz - 1, sM[sp][e], sTP[sp][e], sTN[sp][e]);
        dst[e] = v;
      }
    }
  };
  // A1 of plane p on the x-halo rows, into sA1[p & 1] (y neighbours from the A2 tile)
  auto form_a1 = [&](int p) {
    const int sc = p & 3;
    const float *A2 = sA2[p & 1];
    float *dst = sA1[p & 1];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int e = t + kZCN * q;
      if (e < kZA1) {
        const int x = x0 - 1 + e % kZHX, y = y0 + e / kZHX;
        const int hh = e + kZHX;  // the same voxel in the halo tile
        float v = 0.f;
        if (inside(x, y))
          v = recon_point(sC + nM2, nM, hdt, sinked(h, x, y, p), sM[sc][hh], A2[hh], sTN[sc][hh], y > 0,
                          sM[sc][hh - kZHX], A2[hh - kZHX], sTN[sc][hh - kZHX], y < ny - 1, sM[sc][hh + kZHX],
                          A2[hh + kZHX], sTN[sc][hh + kZHX]);
        dst[e] = v;
      }
    }
  };
  // prologue: ring planes z0 - 1 .. z0 + 2 and r2 of plane z0 staged, A2 and A1 of plane z0
  // formed; ring plane z0 + 3 and r2 of plane z0 + 1 in flight
  for (int p = max(z0 - 1, 0); p <= min(z0 + 2, min(z1, nz - 1)); p++) {
    load_ring(p);
    store_ring(p & 3);
  }
  load_single(z0);
  store_single(z0 & 1);
  __syncthreads();
  form_a2(z0);
  if (z0 + 3 < nz && z0 + 3 <= z1) load_ring(z0 + 3);
  if (z0 + 1 < z1) load_single(z0 + 1);
  __syncthreads();
  form_a1(z0);
  __syncthreads();
  int curM = -1;
  float same[3] = {0.f, 0.f, 0.f};
  const int ix = x0 + tx, iy = y0 + ty;
  const bool col = ix < nx && iy < ny;
  const int hc = (ty + 1) * kZHX + tx + 1;  // centre in the halo tile
  // per plane, two phases: (1) assemble plane iz and form A2 of plane iz + 1; (2) form A1 of
  // plane iz + 1, stage the prefetched ring plane iz + 3 (into the slot of iz - 1) and r2 of plane
  // iz + 1, and start the loads of ring plane iz + 4 and r2 of plane iz + 2
  for (int iz = z0; iz < z1; iz++) {
    const int sc = iz & 3, sp = (iz + 1) & 3, sm = (iz + 3) & 3, q1 = iz & 1;
    const float *A2c = sA2[q1], *A1c = sA1[q1];
    if (iz + 1 < z1) form_a2(iz + 1);
    if (col) {
      const long long v = ix + (long long)iy * nx + iz * sxy;
      const int mv = sM[sc][hc];
      const bool nsv = !sinked(h, ix, iy, iz);
      const float r1v = sR1[sc][hc], r2v = sR2[q1][(ty + 1) * kZX + tx], r3v = sR3[sc][t];
      const float tv = sTN[sc][hc];
      const float a1v = A1c[ty * kZHX + tx + 1], a2v = A2c[hc], tpv = sTP[sc][hc];
      if (nsv && mv != curM) {
        if (curM >= 0)
          for (int d = 0; d < 3; d++) atomicAdd(&sdc[curM + curM * nM + d * nM2], (double)same[d]);
        curM = mv;
        same[0] = same[1] = same[2] = 0.f;
      }
      float lam = r1v;
      // all six neighbours present, of the voxel's medium, and none of them (nor the voxel)
      // heat-sinked
      const int lo = h.hs ? 2 : 1;
      const bool interior = ix >= lo && ix < nx - lo && iy >= lo && iy < ny - lo && iz >= lo && iz < nz - lo &&
                            sM[sc][hc - 1] == mv && sM[sc][hc + 1] == mv && sM[sc][hc - kZHX] == mv &&
                            sM[sc][hc + kZHX] == mv && sM[sm][hc] == mv && sM[sp][hc] == mv;
      if (interior) {
        const float cx = cfs(mv, mv, 0), cy = cfs(mv, mv, 1), cz = cfs(mv, mv, 2);
        const float r1xl = sR1[sc][hc - 1], r1xr = sR1[sc][hc + 1], r1yl = sR1[sc][hc - kZHX],
                    r1yr = sR1[sc][hc + kZHX];
        const float r1zl = sR1[sm][hc], r1zr = sR1[sp][hc];
        const float r2yl = sR2[q1][ty * kZX + tx], r2yr = sR2[q1][(ty + 2) * kZX + tx];
        const float r3zl = sR3[sm][t], r3zr = sR3[sp][t];
        const float txl = sTN[sc][hc - 1], txr = sTN[sc][hc + 1], tyl = sTN[sc][hc - kZHX], tyr = sTN[sc][hc + kZHX];
        const float tzl = sTN[sm][hc], tzr = sTN[sp][hc];
        const float a1l = A1c[ty * kZHX + tx], a1r = A1c[ty * kZHX + tx + 2];
        const float a2l = A2c[hc - kZHX], a2r = A2c[hc + kZHX];
        const float tpl = sTP[sm][hc], tpr = sTP[sp][hc];
        const float qy = dt * r1v - hdt * r2v, qz = dt * r1v - hdt * r3v;
        lam += cx * hdt * (r1xl + r1xr - 2.f * r1v) +
               cy * ((dt * r1yl - hdt * r2yl) + (dt * r1yr - hdt * r2yr) - 2.f * qy) +
               cz * ((dt * r1zl - hdt * r3zl) + (dt * r1zr - hdt * r3zr) - 2.f * qz);
        same[0] += hdt * r1v * ((txl + a1l) + (txr + a1r) - 2.f * (tv + a1v));
        same[1] += dt * r1v * (tyl + tyr - 2.f * tv) + hdt * r2v * ((a2l - tyl) + (a2r - tyr) - 2.f * (a2v - tv));
        same[2] += dt * r1v * (tzl + tzr - 2.f * tv) + hdt * r3v * ((tpl - tzl) + (tpr - tzr) - 2.f * (tpv - tv));
        a.lamOut[v] = lam;
        if (a.dQ && !a.dQinX) a.dQ[v] += dt * r1v;
      } else {
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const int pos = d == 0 ? ix : (d == 1 ? iy : iz);
          const int n = d == 0 ? nx : (d == 1 ? ny : nz);
          const float qv = d == 0 ? hdt * r1v : (d == 1 ? dt * r1v - hdt * r2v : dt * r1v - hdt * r3v);
          const float pv = d == 0 ? tv + a1v : (d == 1 ? a2v - tv : tpv - tv);
#pragma unroll
          for (int side = -1; side <= 1; side += 2) {
            if ((side < 0 && pos == 0) || (side > 0 && pos == n - 1)) continue;
            // the neighbour u in the staged tiles
            const int hu = d == 0 ? hc + side : (d == 1 ? hc + side * kZHX : hc);
            const int rs = d == 2 ? (side < 0 ? sm : sp) : sc;
            const int mu = sM[rs][hu];
            const float r1u = sR1[rs][hu], tu = sTN[rs][hu];
            const int ux = d == 0 ? ix + side : ix, uy = d == 1 ? iy + side : iy, uz = d == 2 ? iz + side : iz;
            if (!sinked(h, ux, uy, uz)) {
              const float qu = d == 0   ? hdt * r1u
                               : d == 1 ? dt * r1u - hdt * sR2[q1][(ty + 1 + side) * kZX + tx]
                                        : dt * r1u - hdt * sR3[rs][t];
              lam += cfs(mu, mv, d) * qu;
            }
            if (nsv) {
              lam -= cfs(mv, mu, d) * qv;
              float contrib;
              if (d == 0) contrib = hdt * r1v * ((tu + A1c[ty * kZHX + tx + 1 + side]) - pv);
              else if (d == 1) contrib = dt * r1v * (tu - tv) + hdt * r2v * ((A2c[hu] - tu) - pv);
              else contrib = dt * r1v * (tu - tv) + hdt * r3v * ((sTP[rs][hc] - tu) - pv);
              if (mu == mv) same[d] += contrib;
              else atomicAdd(&sdc[mv + mu * nM + d * nM2], (double)contrib);
            }
          }
        }
        a.lamOut[v] = lam;
        if (a.dQ && !a.dQinX && nsv) a.dQ[v] += dt * r1v;
      }
    }
    __syncthreads();
    if (iz + 1 < z1) form_a1(iz + 1);
    if (iz + 3 < nz && iz + 3 <= z1) store_ring((iz + 3) & 3);
    if (iz + 1 < z1) store_single((iz + 1) & 1);
    if (iz + 4 < nz && iz + 4 <= z1) load_ring(iz + 4);
    if (iz + 2 < z1) load_single(iz + 2);
    __syncthreads();
  }
  if (curM >= 0)
    for (int d = 0; d < 3; d++) atomicAdd(&sdc[curM + curM * nM + d * nM2], (double)same[d]);
  __syncthreads();
  for (int k = threadIdx.x; k < 3 * nM2; k += blockDim.x)
    if (sdc[k] != 0.0) atomicAdd(&a.dc[k], sdc[k]);
}

// Running per-voxel maximum over the peak list after forward step `step`.
__global__ void peak_track_kernel(const float *T, int nP, const int *idx, float *val, int *at, int step) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nP; k += gridDim.x * blockDim.x) {
    const float t = T[idx[k]];
    if (t > val[k]) {
      val[k] = t;
      at[k] = step;
    }
  }
}

__global__ void fill_kernel(float *p, float v, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    p[k] = v;
}

// X^T solve, one warp per x-line (lines up to 512 voxels): the line's right-hand side, inverse
// pivots and media are read coalesced into the warp's slice of shared memory (element i at
// i + i / 32, so the lanes' chunk reads fall in distinct banks), lane g solves rows [g K, g K + K)
// in registers (chunk_solve over the 32 lanes, transposed multipliers as in adj_solve_x_kernel),
// and the solution leaves through the same slice with coalesced stores.
constexpr int kAdjXWarps = 4;
int adj_xline_rows(int nx) { return nx <= 128 ? 4 : nx <= 256 ? 8 : nx <= 384 ? 12 : 16; }

template <int K>
__global__ void __launch_bounds__(32 * kAdjXWarps, K <= 8 ? 8 : 4) adj_xline_kernel(AdjDev a) {
  constexpr int NS = 32 * K + K;  // skewed slice length
  const HeatDev &h = a.h;
  __shared__ float sH[kAdjMaxMedia * kAdjMaxMedia];  // dt/2 c(mi, mj, x)
  __shared__ float sR[kAdjXWarps][NS], sI[kAdjXWarps][NS];
  __shared__ int sM[kAdjXWarps][NS];
  const int nx = h.nx, ny = h.ny, nz = h.nz, nM = h.nM;
  for (int k = threadIdx.x; k < nM * nM; k += blockDim.x) sH[k] = h.hdt * h.c[k];
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float *R = sR[w], *I = sI[w];
  int *Mw = sM[w];
  auto sk = [](int i) { return i + (i >> 5); };
  const int s = lane * K, nv = max(min(s + K, nx) - s, 0);
  const long long lines = (long long)ny * nz;
  const long long nw = (long long)gridDim.x * kAdjXWarps;
  for (long long line = (long long)blockIdx.x * kAdjXWarps + w; line < lines; line += nw) {
    const int iy = (int)(line % ny), iz = (int)(line / ny);
    const long long row = line * nx;
    for (int i = lane; i < nx; i += 32) {
      R[sk(i)] = a.r2[row + i];
      I[sk(i)] = h.ib[row + i];
      Mw[sk(i)] = h.M[row + i];
    }
    __syncwarp();
    const bool lineSinked = h.hs && (iy == 0 || iy == ny - 1 || iz == 0 || iz == nz - 1);
    auto rowSink = [&](int i) { return lineSinked || (h.hs && (i == 0 || i == nx - 1)); };
    float r[K], fm[K], bm[K], ib[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      fm[k] = bm[k] = 1.f;
      ib[k] = r[k] = 0.f;
      if (k < nv) {
        const int i = s + k, mi = Mw[sk(i)];
        ib[k] = I[sk(i)];
        r[k] = R[sk(i)];
        fm[k] = (i > 0 && !rowSink(i - 1)) ? sH[Mw[sk(i - 1)] + nM * mi] * I[sk(i - 1)] : 0.f;
        bm[k] = (i < nx - 1 && !rowSink(i + 1)) ? sH[Mw[sk(i + 1)] + nM * mi] * ib[k] : 0.f;
      }
    }
    chunk_solve<K, 32>(r, fm, bm, ib, lane);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < K; k++)
      if (k < nv) R[sk(s + k)] = r[k];
    __syncwarp();
    for (int i = lane; i < nx; i += 32) {
      const float v = R[sk(i)];
      a.r1[row + i] = v;
      if (a.dQ && !rowSink(i)) a.dQ[row + i] += h.dt * v;  // dJ/dQ += dt rho1 (heat-sinked voxels: none)
    }
    __syncwarp();
  }
}

void adj_xline_launch(const AdjDev &a, int grid, cudaStream_t st) {
  const int K = adj_xline_rows(a.h.nx);
  if (K == 4) adj_xline_kernel<4><<<grid, 32 * kAdjXWarps, 0, st>>>(a);
  else if (K == 8) adj_xline_kernel<8><<<grid, 32 * kAdjXWarps, 0, st>>>(a);
  else if (K == 12) adj_xline_kernel<12><<<grid, 32 * kAdjXWarps, 0, st>>>(a);
  else adj_xline_kernel<16><<<grid, 32 * kAdjXWarps, 0, st>>>(a);
}

mcb_status adj_xline_setup(mcb_ctx *ctx, int nx, int *grid) {
  const int K = adj_xline_rows(nx);
  int bps = 0;
  if (K == 4) MCB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, adj_xline_kernel<4>, 32 * kAdjXWarps, 0));
  else if (K == 8) MCB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, adj_xline_kernel<8>, 32 * kAdjXWarps, 0));
  else if (K == 12) MCB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, adj_xline_kernel<12>, 32 * kAdjXWarps, 0));
  else MCB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, adj_xline_kernel<16>, 32 * kAdjXWarps, 0));
  if (bps < 1) return set_error(ctx, MCB_ECUDA, "adjoint x-line solve: no block fits on an SM");
  *grid = ctx->num_sms * bps;
  return MCB_OK;
}

// Y^T / Z^T solves in the column layout, for lines up to 320 rows: a block of G warps owns 32
// consecutive x columns of whole lines (Y^T: one z, Z^T: one y); lane l is column x0 + l in every
// warp and warp w holds rows [w kk, w kk + kk) of its column in registers (kk = ceil(n / G) <= K).
// A warp reads 128 contiguous bytes per row and array, all its rows' loads in flight at once; the
// chunk maps of the two scans combine across the warps through shared memory (buffers alternate
// by tile parity, so two barriers per tile suffice), and the solution leaves with coalesced row
// stores. Multipliers of the transposed system from the factored state's inverse pivots:
// forward c_{i-1} / b'_{i-1}, backward a_{i+1} / b'_i (same products as adj_solve_yz_kernel).
constexpr int kAdjColMaxN = 320;
int adj_col_rows(int n) { return n <= 256 ? 8 : 16; }
int adj_col_warps(int n) { return (n + adj_col_rows(n) - 1) / adj_col_rows(n); }

template <int K, bool ZP, int MAXT>
__global__ void __launch_bounds__(MAXT, MAXT <= 256 ? 3 : MAXT <= 512 ? 2 : 1) adj_col_kernel(AdjDev a, int G) {
  const HeatDev &h = a.h;
  __shared__ float sH[kAdjMaxMedia * kAdjMaxMedia];  // dt/2 c(mi, mj, d) of this direction
  __shared__ float2 sums[2][2][32 * 32];              // [tile parity][scan][warp * 32 + lane]
  const int nx = h.nx, nM = h.nM;
  const long long sxy = (long long)nx * h.ny;
  const int n = ZP ? h.nz : h.ny, nOther = ZP ? h.ny : h.nz, d = ZP ? 2 : 1;
  const long long st = ZP ? sxy : nx;
  const float *__restrict__ in = ZP ? a.lam : a.r3;
  float *__restrict__ out = ZP ? a.r3 : a.r2;
  const float *__restrict__ ibd = h.ib + (size_t)d * sxy * h.nz;
  for (int k = threadIdx.x; k < nM * nM; k += blockDim.x) sH[k] = h.hdt * h.c[k + d * nM * nM];
  __syncthreads();
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int kk = (n + G - 1) / G;
  const int s = min(w * kk, n), e = min(s + kk, n), cnt = e - s;
  const int xTiles = (nx + 31) >> 5, nTiles = xTiles * nOther;
  int it = 0;
  for (int tile = blockIdx.x; tile < nTiles; tile += gridDim.x, ++it) {
    const int x = ((tile % xTiles) << 5) + l, o = tile / xTiles;
    const long long base = x + (ZP ? (long long)o * nx : (long long)o * sxy);
    const bool lineSink = h.hs && (x == 0 || x == nx - 1 || o == 0 || o == nOther - 1);
    const int nv = x < nx ? cnt : 0;  // rows of this lane
    auto rowSink = [&](int i) { return lineSink || (h.hs && (i == 0 || i == n - 1)); };
    float r[K], fm[K], bm[K], ib[K];
    int mk[K];
    float ibPrev = 0.f;
    int mPrev = 0, mNext = 0;
    if (nv > 0 && s > 0) {
      ibPrev = ibd[base + (s - 1) * st];
      mPrev = h.M[base + (s - 1) * st];
    }
    if (nv > 0 && e < n) mNext = h.M[base + e * st];
#pragma unroll
    for (int k = 0; k < K; k++) {
      r[k] = ib[k] = 0.f;
      mk[k] = 0;
      if (k < nv) {
        const long long v = base + (s + k) * st;
        r[k] = in[v];
        ib[k] = ibd[v];
        mk[k] = h.M[v];
      }
    }
    // multipliers (slots past the lane's rows: identity maps, fm = bm = 1 with r = ib = 0) and the
    // forward chunk map
    float A = 0.f, B = 1.f;
#pragma unroll
    for (int k = 0; k < K; k++) {
      fm[k] = bm[k] = 1.f;
      if (k < nv) {
        const int i = s + k, mi = mk[k];
        const int mp = k == 0 ? mPrev : mk[k > 0 ? k - 1 : 0];
        const float ibp = k == 0 ? ibPrev : ib[k > 0 ? k - 1 : 0];
        const int mn = k + 1 < nv ? mk[k + 1 < K ? k + 1 : K - 1] : mNext;
        fm[k] = (i > 0 && !rowSink(i - 1)) ? sH[mp + nM * mi] * ibp : 0.f;
        bm[k] = (i < n - 1 && !rowSink(i + 1)) ? sH[mn + nM * mi] * ib[k] : 0.f;
      }
      A = fmaf(fm[k], A, r[k]);
      B *= fm[k];
    }
    float2 *sF = sums[it & 1][0], *sB = sums[it & 1][1];
    sF[w * 32 + l] = make_float2(A, B);
    __syncthreads();
    float dcar = 0.f;
    for (int q = 0; q < w; q++) {
      const float2 m2 = sF[q * 32 + l];
      dcar = fmaf(m2.y, dcar, m2.x);
    }
#pragma unroll
    for (int k = 0; k < K; k++) {
      dcar = fmaf(fm[k], dcar, r[k]);
      r[k] = dcar * ib[k];
    }
    // back substitution: chunk map y_in = A + B y_out, combined from the last warp down
    A = 0.f;
    B = 1.f;
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
    for (int k = 0; k < K; k++)
      if (k < nv) out[base + (s + k) * st] = r[k];
  }
}

// Column-layout configurations: 8 rows per lane for lines up to 256 rows (block-size classes
// 256, 512, 1024 threads), 16 beyond (640).
template <bool ZP>
mcb_status adj_col_setup(mcb_ctx *ctx, int n, int *grid) {
  const int G = adj_col_warps(n);
  int bps = 0;
  if (adj_col_rows(n) == 16)
    MCB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, adj_col_kernel<16, ZP, 640>, 32 * G, 0));
  else if (G <= 8)
    MCB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, adj_col_kernel<8, ZP, 256>, 32 * G, 0));
  else if (G <= 16)
    MCB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, adj_col_kernel<8, ZP, 512>, 32 * G, 0));
  else
    MCB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, adj_col_kernel<8, ZP, 1024>, 32 * G, 0));
  if (bps < 1) return set_error(ctx, MCB_ECUDA, "adjoint column solve: no block fits on an SM");
  *grid = ctx->num_sms * bps;
  return MCB_OK;
}

template <bool ZP>
void adj_col_launch(const AdjDev &a, int n, int grid, cudaStream_t st) {
  const int G = adj_col_warps(n);
  if (adj_col_rows(n) == 16) adj_col_kernel<16, ZP, 640><<<grid, 32 * G, 0, st>>>(a, G);
  else if (G <= 8) adj_col_kernel<8, ZP, 256><<<grid, 32 * G, 0, st>>>(a, G);
  else if (G <= 16) adj_col_kernel<8, ZP, 512><<<grid, 32 * G, 0, st>>>(a, G);
  else adj_col_kernel<8, ZP, 1024><<<grid, 32 * G, 0, st>>>(a, G);
}

template <int TW>
mcb_status adj_setup_yz(mcb_ctx *ctx, int ny, int nz) {
  MCB_CUDA(ctx, cudaFuncSetAttribute(adj_solve_yz_kernel<TW, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(adj_yz_tile_bytes<TW>(ny) + 64)));
  MCB_CUDA(ctx, cudaFuncSetAttribute(adj_solve_yz_kernel<TW, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)(adj_yz_tile_bytes<TW>(nz) + 64)));
  return MCB_OK;
}

template <int TW>
void adj_launch_yz(const AdjDev &a, bool zpass, int grid, cudaStream_t st) {
  if (zpass) adj_solve_yz_kernel<TW, true><<<grid, 256, adj_yz_tile_bytes<TW>(a.h.nz) + 64, st>>>(a);
  else adj_solve_yz_kernel<TW, false><<<grid, 256, adj_yz_tile_bytes<TW>(a.h.ny) + 64, st>>>(a);
}

// Compressed (index, weight) list of the nonzero entries of a per-voxel weight array.
void weight_list(const float *w, long long L, std::vector<int> &idx, std::vector<float> &val) {
  idx.clear();
  val.clear();
  if (!w) return;
  for (long long v = 0; v < L; v++)
    if (w[v] != 0.f) {
      idx.push_back((int)v);
      val.push_back(w[v]);
    }
}

}  // namespace
}  // namespace mcb

extern "C" mcb_status mcb_heat_adjoint(mcb_ctx *ctx, const mcb_heat_params *pin, const float *T0,
                                       const mcb_heat_objective *obj, int32_t nCheckpoints, mcb_heat_grad *out) {
  using namespace mcb;
  if (!ctx) return MCB_EINVAL;
  MCB_TRY(heat_check_params(ctx, pin));
  if (!T0 || !obj || !out) return set_error(ctx, MCB_EINVAL, "NULL argument");
  if (pin->steps < 1) return set_error(ctx, MCB_EINVAL, "the adjoint needs steps >= 1");
  if (pin->nM > kAdjMaxMedia) return set_error(ctx, MCB_EINVAL, "the adjoint supports at most %d media", kAdjMaxMedia);
  if (pin->lightsOn && !pin->dTdt_abs) return set_error(ctx, MCB_EINVAL, "dTdt_abs missing while lightsOn");
  mcb_heat_params p = *pin;
  p.nSensors = 0;  // sensors are not part of the objective
  p.tempSensorCornerIdxs = p.tempSensorInterpWeights = nullptr;
  const long long nt = p.steps, L = (long long)p.nx * p.ny * p.nz;
  const int nM = p.nM;
  const long long nC = nCheckpoints > 0 ? std::min<long long>(nCheckpoints, nt)
                                        : (long long)std::ceil(std::sqrt((double)nt));
  const long long K = (nt + nC - 1) / nC;
  const long long nSeg = (nt + K - 1) / K;
  std::vector<int> dIdx, pIdx;
  std::vector<float> dW, pW;
  weight_list(obj->damageWeight, L, dIdx, dW);
  weight_list(obj->peakWeight, L, pIdx, pW);
  const int nD = (int)dIdx.size(), nP = (int)pIdx.size();

  MCB_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  mcb_heat_state s;
  s.ctx = ctx;
  mcb_status rc = heat_state_init(ctx, &s, &p, T0, nullptr);
  if (rc != MCB_OK) {
    heat_state_release(&s);
    return rc;
  }
  // work memory: checkpoints, the segment ring, six grid arrays, the lists and accumulators
  const size_t grid4 = 4 * (size_t)L;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t bytes = al(grid4) * (size_t)(nSeg + 1 + std::max<long long>(K - 1, 1) + 6) + al(8 * (size_t)nM * nM * 3) + al(16) +
                       al(12 * (size_t)std::max(nD, 1)) + al(12 * (size_t)std::max(nP, 1)) + al(8 * (size_t)std::max(nP, 1)) +
                       4096;
  void *block = nullptr;
  rc = pool_get(ctx, SLOT_HEAT_ADJ, bytes, &block);
  if (rc != MCB_OK) {
    heat_state_release(&s);
    return rc;
  }
  char *cur = (char *)block;
  auto take = [&](size_t b) {
    char *q = cur;
    cur += al(b);
    return (void *)q;
  };
  float *ckpt = (float *)take(grid4 * (size_t)(nSeg + 1));  // slot nSeg: the final state
  float *ring = (float *)take(grid4 * (size_t)std::max<long long>(K - 1, 1));
  AdjDev a{};
  a.r1 = (float *)take(grid4);
  a.r2 = (float *)take(grid4);
  a.r3 = (float *)take(grid4);
  float *lamA = (float *)take(grid4);
  float *lamB = (float *)take(grid4);
  float *dQ = (float *)take(grid4);
  a.dc = (double *)take(8 * (size_t)nM * nM * 3);
  a.Jd = (double *)take(16);
  int *dIdxD = (int *)take(4 * (size_t)std::max(nD, 1));
  float *dWD = (float *)take(4 * (size_t)std::max(nD, 1));
  a.gbuf = (float *)take(4 * (size_t)std::max(nD, 1));
  int *pIdxD = (int *)take(4 * (size_t)std::max(nP, 1));
  float *pWD = (float *)take(4 * (size_t)std::max(nP, 1));
  float *pVal = (float *)take(4 * (size_t)std::max(nP, 1));
  int *pStepD = (int *)take(4 * (size_t)std::max(nP, 1));
  mcb_heat_state ss;  // streamed state of the forward sweeps (below)
  StreamStepper *sk = nullptr;
  auto fail = [&](mcb_status r) {
    if (sk) {
      stream_stepper_free(sk);
      heat_state_release(&ss);
    }
    heat_state_release(&s);
    return r;
  };
#define ADJ_CUDA(call)                                                                                          \
  do {                                                                                                          \
    cudaError_t _e = (call);                                                                                    \
    if (_e != cudaSuccess)                                                                                      \
      return fail(set_error(ctx, MCB_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(_e), __FILE__, \
                            __LINE__));                                                                         \
  } while (0)
  if (nD) {
    ADJ_CUDA(cudaMemcpyAsync(dIdxD, dIdx.data(), 4 * (size_t)nD, cudaMemcpyHostToDevice, st));
    ADJ_CUDA(cudaMemcpyAsync(dWD, dW.data(), 4 * (size_t)nD, cudaMemcpyHostToDevice, st));
  }
  if (nP) {
    ADJ_CUDA(cudaMemcpyAsync(pIdxD, pIdx.data(), 4 * (size_t)nP, cudaMemcpyHostToDevice, st));
    ADJ_CUDA(cudaMemcpyAsync(pWD, pW.data(), 4 * (size_t)nP, cudaMemcpyHostToDevice, st));
    fill_kernel<<<64, 256, 0, st>>>(pVal, -__builtin_huge_valf(), nP);
    ADJ_CUDA(cudaMemsetAsync(pStepD, 0, 4 * (size_t)nP, st));
  }
  ADJ_CUDA(cudaMemsetAsync(a.dc, 0, 8 * (size_t)nM * nM * 3, st));
  ADJ_CUDA(cudaMemsetAsync(a.Jd, 0, 16, st));
  ADJ_CUDA(cudaMemsetAsync(dQ, 0, grid4, st));
  ADJ_CUDA(cudaMemsetAsync(lamA, 0, grid4, st));

  HeatStepper ks;
  rc = heat_stepper(ctx, &s, &p, &ks);
  if (rc != MCB_OK) return fail(rc);
  a.h = ks.h;
  a.dQ = p.lightsOn ? dQ : nullptr;
  a.nD = nD;
  a.dIdx = dIdxD;
  a.dW = dWD;
  a.nP = nP;
  a.pIdx = pIdxD;
  a.pW = pWD;
  a.pStep = pStepD;
  const int tw = s.tw;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const size_t smemX = (size_t)a.h.xl * 16 * (nx + 1) + 64;
  ADJ_CUDA(cudaFuncSetAttribute(adj_solve_x_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemX));
  if (tw == 32) rc = adj_setup_yz<32>(ctx, ny, nz);
  else if (tw == 16) rc = adj_setup_yz<16>(ctx, ny, nz);
  else rc = adj_setup_yz<8>(ctx, ny, nz);
  if (rc != MCB_OK) return fail(rc);
  const int gridX = ks.gridX, gridYZ = ks.gridYZ;
  // Y^T and Z^T in the column layout where the lines are short enough (grid 0: the tiled kernel)
  int gridColY = 0, gridColZ = 0;
  if (ny <= kAdjColMaxN) rc = adj_col_setup<false>(ctx, ny, &gridColY);
  if (rc == MCB_OK && nz <= kAdjColMaxN) rc = adj_col_setup<true>(ctx, nz, &gridColZ);
  int gridXL = 0;  // X^T one warp per line (grid 0: the tiled kernel)
  if (rc == MCB_OK && nx <= 512) rc = adj_xline_setup(ctx, nx, &gridXL);
  if (rc != MCB_OK) return fail(rc);
  const int gridL = std::max(1, std::min(ctx->num_sms * 4, (std::max(nD, nP) + 255) / 256));
  const dim3 gridZ((nx + kZX - 1) / kZX, (ny + kZY - 1) / kZY, (nz + kZChunk - 1) / kZChunk);
  const size_t smemZ = (size_t)3 * nM * nM * (8 + 4);
  ADJ_CUDA(cudaFuncSetAttribute(adj_assemble_z_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smemZ));
  a.dQinX = gridXL != 0;

  // The forward sweeps (checkpoints, segment recomputation) step a streamed state where the grid
  // allows: the same steps up to FP32 rounding at the streamed stepper's speed. The reverse
  // sweep keeps the factored state's LU pivots for its transposed solves.
  int *pIdxS = pIdxD;
  if (stream_supported(p.nx, p.ny, p.nz)) {
    rc = stream_state_create(ctx, &ss, &p, T0);
    if (rc == MCB_OK) rc = stream_stepper_new(ctx, &ss, &p, &sk);
    if (rc != MCB_OK) {
      if (sk) stream_stepper_free(sk);
      sk = nullptr;
      heat_state_release(&ss);
      return fail(rc);
    }
    if (nP) {
      // the peak list's voxels in the streamed state's pitched grid
      std::vector<int> pIdxP(nP);
      for (int k = 0; k < nP; k++) pIdxP[k] = (int)stream_pitched_index(&ss, pIdx[k]);
      pIdxS = (int *)take(4 * (size_t)nP);
      ADJ_CUDA(cudaMemcpyAsync(pIdxS, pIdxP.data(), 4 * (size_t)nP, cudaMemcpyHostToDevice, st));
      ADJ_CUDA(cudaStreamSynchronize(st));
    }
  }
  // forward sweep: checkpoints every K steps, running maxima of the peak list
  ADJ_CUDA(cudaEventRecord(ctx->ev0, st));
  for (long long n = 0; n < nt; n++) {
    float *ck = ckpt + (size_t)(n / K) * L;
    if (sk) {
      if (n % K == 0) stream_dense_copy(ctx, &ss, ck, st);
      stream_stepper_launch(sk, st);
      if (nP) peak_track_kernel<<<gridL, 256, 0, st>>>(ss.T, nP, pIdxS, pVal, pStepD, (int)(n + 1));
    } else {
      if (n % K == 0) ADJ_CUDA(cudaMemcpyAsync(ck, s.T, grid4, cudaMemcpyDeviceToDevice, st));
      heat_step_launch(ks, st);
      if (nP) peak_track_kernel<<<gridL, 256, 0, st>>>(s.T, nP, pIdxD, pVal, pStepD, (int)(n + 1));
    }
  }
  if (sk) stream_dense_copy(ctx, &ss, ckpt + (size_t)nSeg * L, st);
  else ADJ_CUDA(cudaMemcpyAsync(ckpt + (size_t)nSeg * L, s.T, grid4, cudaMemcpyDeviceToDevice, st));
  ADJ_CUDA(cudaGetLastError());
  ADJ_CUDA(cudaEventRecord(ctx->ev1, st));
  ADJ_CUDA(cudaEventSynchronize(ctx->ev1));
  float msF = 0.f;
  ADJ_CUDA(cudaEventElapsedTime(&msF, ctx->ev0, ctx->ev1));

  // reverse sweep, one segment at a time: its end states are checkpoints seg and seg + 1, its
  // inner states are recomputed from the first into the ring (the stepper is deterministic, so
  // they equal the forward sweep's)
  ADJ_CUDA(cudaEventRecord(ctx->ev0, st));
  float *lam = lamA, *lamNext = lamB;
  for (long long seg = nSeg - 1; seg >= 0; seg--) {
    const long long n0 = seg * K, n1 = std::min(n0 + K, nt);
    const float *first = ckpt + (size_t)seg * L, *last = ckpt + (size_t)(seg + 1) * L;
    if (n1 - n0 > 1) {
      if (sk) {
        stream_dense_set(ctx, &ss, first, st);
        for (long long j = 1; j < n1 - n0; j++) {
          stream_stepper_launch(sk, st);
          stream_dense_copy(ctx, &ss, ring + (size_t)(j - 1) * L, st);
        }
      } else {
        ADJ_CUDA(cudaMemcpyAsync(s.T, first, grid4, cudaMemcpyDeviceToDevice, st));
        for (long long j = 1; j < n1 - n0; j++) {
          heat_step_launch(ks, st);
          ADJ_CUDA(cudaMemcpyAsync(ring + (size_t)(j - 1) * L, s.T, grid4, cudaMemcpyDeviceToDevice, st));
        }
      }
    }
    // state n0 + j of the segment
    auto state = [&](long long j) { return j == 0 ? first : (j == n1 - n0 ? last : ring + (size_t)(j - 1) * L); };
    for (long long n = n1 - 1; n >= n0; n--) {
      a.Tn = state(n - n0);
      a.Tp = state(n - n0 + 1);
      a.lam = lam;
      a.lamOut = lamNext;
      a.step = (int)(n + 1);
      if (nD || nP) adj_seed_kernel<<<gridL, 256, 0, st>>>(a);
      if (gridColZ) adj_col_launch<true>(a, nz, gridColZ, st);
      else if (tw == 32) adj_launch_yz<32>(a, true, gridYZ, st);
      else if (tw == 16) adj_launch_yz<16>(a, true, gridYZ, st);
      else adj_launch_yz<8>(a, true, gridYZ, st);
      if (gridColY) adj_col_launch<false>(a, ny, gridColY, st);
      else if (tw == 32) adj_launch_yz<32>(a, false, gridYZ, st);
      else if (tw == 16) adj_launch_yz<16>(a, false, gridYZ, st);
      else adj_launch_yz<8>(a, false, gridYZ, st);
      if (gridXL) adj_xline_launch(a, gridXL, st);
      else adj_solve_x_kernel<<<gridX, 256, smemX, st>>>(a);
      adj_assemble_z_kernel<<<gridZ, kZCN, smemZ, st>>>(a);
      if (nD) adj_damage_tail_kernel<<<gridL, 256, 0, st>>>(a);
      std::swap(lam, lamNext);
    }
  }
  ADJ_CUDA(cudaGetLastError());
  ADJ_CUDA(cudaEventRecord(ctx->ev1, st));
  // outputs
  std::vector<float> pv(std::max(nP, 1));
  double Jd = 0.0;
  if (nP) ADJ_CUDA(cudaMemcpyAsync(pv.data(), pVal, 4 * (size_t)nP, cudaMemcpyDeviceToHost, st));
  ADJ_CUDA(cudaMemcpyAsync(&Jd, a.Jd, 8, cudaMemcpyDeviceToHost, st));
  if (out->dJ_dc) ADJ_CUDA(cudaMemcpyAsync(out->dJ_dc, a.dc, 8 * (size_t)nM * nM * 3, cudaMemcpyDeviceToHost, st));
  if (out->dJ_dQ) ADJ_CUDA(cudaMemcpyAsync(out->dJ_dQ, dQ, grid4, cudaMemcpyDeviceToHost, st));
  if (out->dJ_dT0) ADJ_CUDA(cudaMemcpyAsync(out->dJ_dT0, lam, grid4, cudaMemcpyDeviceToHost, st));
  ADJ_CUDA(cudaStreamSynchronize(st));
  float msR = 0.f;
  ADJ_CUDA(cudaEventElapsedTime(&msR, ctx->ev0, ctx->ev1));
#undef ADJ_CUDA
  double Jp = 0.0;
  for (int k = 0; k < nP; k++) Jp += (double)pW[k] * ((double)pv[k] + s.base);
  out->J_damage = Jd;
  out->J_peak = Jp;
  out->J = Jd + Jp;
  out->forwardMs = msF;
  out->adjointMs = msR;
  ctx->lastKernelMs = msF + msR;
  if (sk) {
    stream_stepper_free(sk);
    heat_state_release(&ss);
  }
  heat_state_release(&s);
  return MCB_OK;
}
