// Device-side pieces shared by the heat stepper (heat_adi.cu) and its adjoint
// (heat_adjoint.cu): the kernel argument block, coefficient lookups and the tridiagonal line
// solvers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace mcb {

constexpr double kGasR = 8.3144598;      // finiteElementHeatPropagator.c:86
constexpr double kCelsiusZero = 273.15;  // finiteElementHeatPropagator.c:87

struct HeatDev {
  int nx, ny, nz, nM;
  float *T;        // deviations, in/out
  float *A;        // intermediate (T1, then T2)
  const uint8_t *M;
  const float *c;  // [nM x nM x 3]
  const float *Q;  // dTdt_abs or nullptr when the light is off
  const float *ib; // [3][L] inverse pivots
  const float2 *fb;  // [3][L] scan multipliers {fm, bm} of every voxel's row
  const uint8_t *nb; // [L] neighbourhood code (pass_x_kernel)
  float *Sz;       // [L] z half-correction carried from the X pass to the Y pass
  float *Omega;    // or nullptr
  float *dOmega;   // damage accumulated during the current call, or nullptr
  const double *logA, *E;  // [nM]
  const float2 *dmg;       // [nM] Arrhenius exponent about the base temperature (damage_table)
  float T0;                // base temperature in kelvin
  unsigned int *maxEnc;    // [nM] order-preserving encoded running maxima
  int hs;          // heat-sinked faces
  float dt, hdt;
  double dtd, base;
  // sensors
  int nS;
  const double *sIdx, *sW;  // [nS], [nS x 3]
  double *sens;             // [nS x (nt+1)]
  int *stepCounter;
  int xl;  // x-lines per block in the X pass
};

constexpr int kNbSink = 64;  // neighbourhood-code bit of heat-sinked voxels (neighbour_code_kernel)

__device__ __forceinline__ unsigned int enc_max(float f) {
  const unsigned int b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ bool sinked(const HeatDev &h, int ix, int iy, int iz) {
  return h.hs && (ix == 0 || ix == h.nx - 1 || iy == 0 || iy == h.ny - 1 || iz == 0 || iz == h.nz - 1);
}

__device__ __forceinline__ float cf(const HeatDev &h, int mi, int mj, int dir) {
  return __ldg(h.c + mi + h.nM * mj + dir * h.nM * h.nM);
}

// Tridiagonal line coefficients: a = dt/2 c(M_i, M_prev) couples a row to its predecessor,
// cc = dt/2 c(M_i, M_next) to its successor; both vanish at the line ends and on heat-sinked
// rows (identity rows), which reproduces the reference's heat-sink exceptions (:334-349).
__device__ __forceinline__ bool row_sinked(const HeatDev &h, bool lineSinked, int i, int n) {
  return lineSinked || (h.hs && (i == 0 || i == n - 1));
}

// Chunked two-scan solve of one line whose lanes hold K consecutive rows each (G lanes per line,
// an aligned sub-warp group): r (right-hand side in, solution out), fm = a_i / b'_{i-1},
// bm = c_i / b'_i, ib = 1 / b'_i. Register slots past a lane's rows (a lane may hold fewer than K
// rows, also in the middle of a line) are identity maps of both scans: fm = bm = 1, ib = r = 0.
template <int K, int G>
__device__ __forceinline__ void chunk_solve(float (&r)[K], const float (&fm)[K], const float (&bm)[K], const float (&ib)[K],
                                            int g) {
  float A = 0.f, B = 1.f;
#pragma unroll
  for (int k = 0; k < K; k++) {
    A = fmaf(fm[k], A, r[k]);
    B *= fm[k];
  }
#pragma unroll
  for (int off = 1; off < G; off <<= 1) {
    const float Au = __shfl_up_sync(0xffffffffu, A, off, G);
    const float Bu = __shfl_up_sync(0xffffffffu, B, off, G);
    if (g >= off) {
      A = fmaf(B, Au, A);
      B *= Bu;
    }
  }
  float d = __shfl_up_sync(0xffffffffu, A, 1, G);
  if (g == 0) d = 0.f;
#pragma unroll
  for (int k = 0; k < K; k++) {
    d = fmaf(fm[k], d, r[k]);
    r[k] = d * ib[k];
  }
  A = 0.f;
  B = 1.f;
#pragma unroll
  for (int k = K - 1; k >= 0; k--) {
    A = fmaf(bm[k], A, r[k]);
    B *= bm[k];
  }
#pragma unroll
  for (int off = 1; off < G; off <<= 1) {
    const float Ad = __shfl_down_sync(0xffffffffu, A, off, G);
    const float Bd = __shfl_down_sync(0xffffffffu, B, off, G);
    if (g + off < G) {
      A = fmaf(B, Ad, A);
      B *= Bd;
    }
  }
  float t = __shfl_down_sync(0xffffffffu, A, 1, G);
  if (g == G - 1) t = 0.f;
#pragma unroll
  for (int k = K - 1; k >= 0; k--) {
    t = fmaf(bm[k], t, r[k]);
    r[k] = t;
  }
}

// Solves one tridiagonal line with one warp. Shared-memory inputs (element stride st):
//   rhs  right-hand side, replaced by the solution
//   fm   forward multipliers  a_i / b'_{i-1}      (Thomas elimination d'_i = rhs_i + fm_i d'_{i-1})
//   bm   backward multipliers cc_i / b'_i         (back substitution T_i = d'_i / b'_i + bm_i T_{i+1})
//   ib   inverse pivots 1 / b'_i
// fm and bm may be interleaved ({fm, bm} pairs): their element stride is fs * st.
// Each recurrence is evaluated as a chunked warp scan of affine maps: every lane composes the
// map of its contiguous chunk, a 5-step shuffle scan combines the lanes, and each lane then
// replays its chunk from the carried-in value.
static __device__ void warp_solve(float *rhs, const float *fm, const float *bm, const float *ib, int n, int st,
                                  int fs = 1) {
  const int sm = fs * st;
  const int lane = threadIdx.x & 31;
  const int k = (n + 31) >> 5;
  const int s = min(lane * k, n), e = min(s + k, n);
  float A = 0.f, B = 1.f;
  for (int i = s; i < e; i++) {
    const float m = fm[i * sm];
    A = fmaf(m, A, rhs[i * st]);
    B *= m;
  }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const float Au = __shfl_up_sync(0xffffffffu, A, off);
    const float Bu = __shfl_up_sync(0xffffffffu, B, off);
    if (lane >= off) {
      A = fmaf(B, Au, A);
      B *= Bu;
    }
  }
  float d = __shfl_up_sync(0xffffffffu, A, 1);
  if (lane == 0) d = 0.f;
  for (int i = s; i < e; i++) {
    d = fmaf(fm[i * sm], d, rhs[i * st]);
    rhs[i * st] = d;
  }
  A = 0.f;
  B = 1.f;
  for (int i = e - 1; i >= s; i--) {
    const float f = bm[i * sm];
    A = fmaf(f, A, rhs[i * st] * ib[i * st]);
    B *= f;
  }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const float Ad = __shfl_down_sync(0xffffffffu, A, off);
    const float Bd = __shfl_down_sync(0xffffffffu, B, off);
    if (lane + off < 32) {
      A = fmaf(B, Ad, A);
      B *= Bd;
    }
  }
  float t = __shfl_down_sync(0xffffffffu, A, 1);
  if (lane == 31) t = 0.f;
  for (int i = e - 1; i >= s; i--) {
    t = fmaf(bm[i * sm], t, rhs[i * st] * ib[i * st]);
    rhs[i * st] = t;
  }
  __syncwarp();
}

// Grouped variant for short lines: G lanes (an aligned sub-warp group) share one line, each
// holding K consecutive elements with fully unrolled chunk loops; 32/G lines are solved by a
// warp at once. Requires n <= G*K.
template <int K, int G>
__device__ __forceinline__ void group_solve(float *rhs, const float *fm, const float *bm, const float *ib, int n, int st,
                                            int fs = 1) {
  const int sm = fs * st;
  const int g = threadIdx.x & (G - 1);
  const int kk = (n + G - 1) / G;  // chunk length (<= K); odd lengths spread the lanes over banks
  const int s = g * kk;
  const int e = min(s + kk, n);
  float A = 0.f, B = 1.f;
#pragma unroll
  for (int j = 0; j < K; j++) {
    const int i = s + j;
    if (i < e) {
      const float m = fm[i * sm];
      A = fmaf(m, A, rhs[i * st]);
      B *= m;
    }
  }
#pragma unroll
  for (int off = 1; off < G; off <<= 1) {
    const float Au = __shfl_up_sync(0xffffffffu, A, off, G);
    const float Bu = __shfl_up_sync(0xffffffffu, B, off, G);
    if (g >= off) {
      A = fmaf(B, Au, A);
      B *= Bu;
    }
  }
  float d = __shfl_up_sync(0xffffffffu, A, 1, G);
  if (g == 0) d = 0.f;
#pragma unroll
  for (int j = 0; j < K; j++) {
    const int i = s + j;
    if (i < e) {
      d = fmaf(fm[i * sm], d, rhs[i * st]);
      rhs[i * st] = d;
    }
  }
  A = 0.f;
  B = 1.f;
#pragma unroll
  for (int j = K - 1; j >= 0; j--) {
    const int i = s + j;
    if (i < e) {
      const float f = bm[i * sm];
      A = fmaf(f, A, rhs[i * st] * ib[i * st]);
      B *= f;
    }
  }
#pragma unroll
  for (int off = 1; off < G; off <<= 1) {
    const float Ad = __shfl_down_sync(0xffffffffu, A, off, G);
    const float Bd = __shfl_down_sync(0xffffffffu, B, off, G);
    if (g + off < G) {
      A = fmaf(B, Ad, A);
      B *= Bd;
    }
  }
  float t = __shfl_down_sync(0xffffffffu, A, 1, G);
  if (g == G - 1) t = 0.f;
#pragma unroll
  for (int j = K - 1; j >= 0; j--) {
    const int i = s + j;
    if (i < e) {
      t = fmaf(bm[i * sm], t, rhs[i * st] * ib[i * st]);
      rhs[i * st] = t;
    }
  }
  __syncwarp();
}


// Solves `count` lines of one tile; line l starts at base + l*lstride (elements), element
// stride st. Dispatches on the line length.
template <int K, int G>
__device__ __forceinline__ void solve_lines_g(float *rhs, const float *fm, const float *bm, const float *ib, int n, int st,
                                              int lstride, int count, int fs) {
  constexpr int LPW = 32 / G;  // lines per warp at once
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int sub = (threadIdx.x & 31) / G;
  for (int l0 = warp * LPW; l0 < count; l0 += nw * LPW) {
    const int l = l0 + sub;
    // groups without a line run the same shuffles on an empty line so the warp stays converged
    if (l < count)
      group_solve<K, G>(rhs + l * lstride, fm + fs * l * lstride, bm + fs * l * lstride, ib + l * lstride, n, st, fs);
    else group_solve<K, G>(rhs, fm, bm, ib, 0, st, fs);
  }
}

// Solves `count` lines; line l starts at element l * lstride, element stride st (fm and bm:
// fs times both strides, fs = 2 for interleaved {fm, bm} pairs). Lines up to 128 use groups of
// 16 lanes holding 8 elements each, up to 256 16 lanes of 16, up to 512 32 lanes of 16, longer
// lines one warp each (16-lane groups measured faster than 8- and 32-lane groups on 100-long
// lines).
__device__ __forceinline__ void solve_lines(float *rhs, const float *fm, const float *bm, const float *ib, int n, int st,
                                            int lstride, int count, int fs = 1) {
  if (n <= 128) solve_lines_g<8, 16>(rhs, fm, bm, ib, n, st, lstride, count, fs);
  else if (n <= 256) solve_lines_g<16, 16>(rhs, fm, bm, ib, n, st, lstride, count, fs);
  else if (n <= 512) solve_lines_g<16, 32>(rhs, fm, bm, ib, n, st, lstride, count, fs);
  else {
    for (int l = threadIdx.x >> 5; l < count; l += blockDim.x >> 5)
      warp_solve(rhs + l * lstride, fm + fs * l * lstride, bm + fs * l * lstride, ib + l * lstride, n, st, fs);
  }
}

// Asynchronous global -> shared copies (cp.async, no registers held while in flight).
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

}  // namespace mcb
