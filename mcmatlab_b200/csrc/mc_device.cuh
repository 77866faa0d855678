// Device-side photon-packet transport for sm_100a.
//
// One packet per lane; FP32 transport state in registers; FP64 tallies in global memory.
// The physics restates the reference packet loop (+MCmatlab/src/MCmatlab.c:245-265) and
// its helpers in +MCmatlab/src/MCmatlablib.c — launchPhoton :519-732, propagatePhoton
// :1019-1119, getInterpolatedNormal :920-1014, checkEscape :821-889, formImage :737-788,
// formFarField :793-797, formEdgeFluxes :802-816, checkRoulette :1124-1133,
// scatterPhoton :1138-1184, depositionCriteriaMet :126-136 — with the single-precision
// constants the reference uses on its GPU path (FLT_EPSILON nudges, MCmatlab.c:91-108).
// Random numbers come from a per-packet Philox stream (philox.cuh), so a packet's path
// depends only on (seed, instance, wavelength, packet id).
#pragma once
#include <cstdint>

#include "philox.cuh"

namespace mcb {

constexpr float kC = 29979245800.0f;  // speed of light [cm/s] (MCmatlab.c:158)
constexpr float kThreshold = 0.01f;   // roulette threshold (MCmatlab.c:159)
constexpr float kChance = 0.1f;       // roulette survival chance (MCmatlab.c:160)
constexpr int kKillRange = 5;         // MCmatlab.c:164
constexpr int kCdfSize = 201;         // MCmatlab.c:171
constexpr float kPi = 3.14159265358979323846f;
constexpr float kFltEps = 1.1920928955078125e-07f;

// Per-instance (model x wavelength) description, resident in device memory.
struct Inst {
  int n[3];
  float d[3];
  float invd[3];  // 1 / d
  int bt;   // boundaryType
  int ffr;  // farFieldRes
  const uint8_t *M0;    // 0-based medium per voxel
  const float4 *nrm;    // unit interface normal per voxel, or nullptr (matched interfaces)
  int nM;
  const float4 *med;    // per medium: mua, mus, g, RI
  const int *cdfidx;    // per medium
  const float *CDFs;    // [201 x nCDF]
  // source
  int beamType;
  float emitterLength;
  const float *FP1, *FP2, *AI1, *AI2;  // beam CDFs (or a single negative code)
  int LFP1, LFP2, LAI1, LAI2;
  float FPw1, FPw2, AIw1, AIw2;
  const double *S;  // distributed source CDF [L+1] or nullptr
  float focus[3], u[3], v[3], w[3];
  // light collector
  int useLC;
  int lcFinite;
  float LCr[3], LCth, LCph, LCf, LCdiam, LCfs;
  int LCres0, LCres1;
  float tStart, tEnd;
  // deposition criteria (counters saturate at UINT32_MAX = "infinity")
  uint32_t minS, maxS, minRefr, maxRefr, minRefl, maxRefl, minI, maxI, minIdx, maxIdx;
  int onlyCollected, eol;
  int crit;  // a deposition criterion is set (criteria_met is true otherwise)
  // FP64 tallies
  double *NFR, *image, *FF, *NIxp, *NIxn, *NIyp, *NIyn, *NIzp, *NIzn;
  unsigned long long *ctr;  // [0] launched, [1] collected, [2] unused, [3] failed launches,
                            // [4] free-step cuts, [5] their weight (a double)
  // RNG stream
  uint32_t key0, key1, ctr2hi, stream;
  // packet range of this instance in the global packet index space
  unsigned long long first, count;
  // packet k of this instance runs the stream of packet index pOff + k * pStride (sharding)
  unsigned long long pOff, pStride;
  // perturbation-MC objectives (gradient runs only)
  int nR;            // radial reflectance bins on the z < 0 face
  float rbin;        // bin width [cm]
  int box[6];        // target box [x0, x1) x [y0, y1) x [z0, z1) for the mean fluence rate
  double *gR;        // [nR][1 + 2 nM]: value, d/dmua_m, d/dmus_m
  double *gF;        // [1 + 2 nM]
};

constexpr int kGradMedia = 10;  // media supported by gradient runs

// A packet ends (as killed) after this many propagation sub-steps without a scattering event.
// The reference has no such limit: a packet that totally reflects into air voxels keeps the
// tissue's refractive index there, meets an index mismatch at every further voxel boundary and
// can reflect indefinitely without scattering or losing weight (seen with smoothed interface
// normals: ~1 us per sub-step, 10 s for one packet). Between two scattering events an ordinary
// packet crosses at most a few grid diagonals (about 3e3 voxel boundaries per diagonal of a
// 1000^3 grid).
constexpr uint32_t kMaxFreeSteps = 20000u;

// d/dmua of c(mua) = w (1 - exp(-mua s)) / mua is w s^2 phi(mua s) with
// phi(x) = (exp(-x) - (1 - exp(-x)) / x) / x; its Taylor series -1/2 + x/3 - x^2/8 + x^3/30
// replaces the cancelling direct form for small x (air has mua = 1e-8 /cm)
__device__ __forceinline__ float self_phi(float x) {
  if (x < 0.05f) return -0.5f + x * (1.f / 3.f - x * (0.125f - x * (1.f / 30.f)));
  return (expf(-x) + expm1f(-x) / x) / x;
}

struct Photon {
  float i[3], u[3], D[3];
  float dOverU[3];  // d_k / |u_k| (voxel-crossing length along the ray), recomputed when u changes
  int j;
  float mua, mus, RI;
  float stepLeft, weight, time;
  bool inside, alive, sameVoxel;
  int med;   // medium of the current voxel
  int jn, mn;  // voxel and medium entered by the last boundary-crossing sub-step (propagate)
  bool inbox;  // current voxel inside the gradient target box
  uint32_t scat, refr, refl, itr;
  uint32_t nsteps;  // propagation sub-steps since launch or the last scattering event
  int kec;  // 0 killed, 1 escaped, 2 collected
  // RNG
  uint32_t pidlo, pidhi;
  uint32_t draw;
  uint32_t r0, r1, r2, r3;
};

__device__ __forceinline__ float rnd(Photon &P, const Inst &I) {
  const uint32_t k = P.draw & 3u;
  if (k == 0) {
    Philox4 o = philox_block(P.draw >> 2, P.pidlo, (P.pidhi & 0xFFFFu) | I.ctr2hi, I.stream, I.key0, I.key1);
    P.r0 = o.x;
    P.r1 = o.y;
    P.r2 = o.z;
    P.r3 = o.w;
  }
  const uint32_t w = k == 0 ? P.r0 : (k == 1 ? P.r1 : (k == 2 ? P.r2 : P.r3));
  P.draw++;
  return u01_from_word(w);
}

__device__ __forceinline__ float sqrf(float x) { return x * x; }

__device__ __forceinline__ void axis_rotate(const float *r, const float *u, float th, float *o) {
  float st, ct;
  sincosf(th, &st, &ct);
  o[0] = (u[0] * u[0] * (1 - ct) + ct) * r[0] + (u[0] * u[1] * (1 - ct) - u[2] * st) * r[1] + (u[0] * u[2] * (1 - ct) + u[1] * st) * r[2];
  o[1] = (u[1] * u[0] * (1 - ct) + u[2] * st) * r[0] + (u[1] * u[1] * (1 - ct) + ct) * r[1] + (u[1] * u[2] * (1 - ct) - u[0] * st) * r[2];
  o[2] = (u[2] * u[0] * (1 - ct) - u[1] * st) * r[0] + (u[2] * u[1] * (1 - ct) + u[0] * st) * r[1] + (u[2] * u[2] * (1 - ct) + ct) * r[2];
}

__device__ __forceinline__ void to_lc_frame(const float *r, float th, float ph, float *o) {
  float st, ct, sp, cp;
  sincosf(th, &st, &ct);
  sincosf(ph, &sp, &cp);
  o[0] = sp * r[0] - cp * r[1];
  o[1] = ct * cp * r[0] + ct * sp * r[1] - st * r[2];
  o[2] = st * cp * r[0] + st * sp * r[1] + ct * r[2];
}

// j in [0, N-1] with D[j] < r <= D[j+1] for nondecreasing D[0..N] (MCmatlablib.c:263-276)
template <typename T>
__device__ __forceinline__ int cdf_search(float r, int N, const T *D) {
  int lo = 0, hi = N;
  while (lo + 1 < hi) {
    const int mid = (lo + hi) >> 1;
    if ((float)D[mid] >= r) hi = mid; else lo = mid;
  }
  return lo;
}

__device__ __forceinline__ long long cdf_search_d(double r, long long N, const double *D) {
  long long lo = 0, hi = N;
  while (lo + 1 < hi) {
    const long long mid = (lo + hi) >> 1;
    if (__ldg(D + mid) >= r) hi = mid; else lo = mid;
  }
  return lo;
}

// Lambert W, branch -1, on [-1/e, 0): Corless et al. (1996) initial guesses and Halley steps.
__device__ double lambert_wm1(double x) {
  if (x >= 0.0) return 0.0;
  const double em1 = 0.36787944117144233;
  if (x < -em1) return -1.0;
  double w;
  if (x < -0.25) {
    const double p = -sqrt(2.0 * (2.718281828459045 * x + 1.0));
    w = -1.0 + p - p * p / 3.0 + 11.0 / 72.0 * p * p * p;
  } else {
    const double L1 = log(-x), L2 = log(-L1);
    w = L1 - L2 + L2 / L1;
  }
  for (int it = 0; it < 40; it++) {
    const double ew = exp(w);
    const double f = w * ew - x;
    const double wp1 = w + 1.0;
    if (wp1 == 0.0) break;
    const double dw = f / (ew * wp1 - (w + 2.0) * f / (2.0 * wp1));
    w -= dw;
    if (fabs(dw) <= 8.9e-16 * fmax(1.0, fabs(w))) break;
  }
  return w;
}

__device__ __forceinline__ bool criteria_met(const Photon &P, const Inst &I) {
  if (!I.crit) return true;
  const bool killed = !P.alive && P.kec == 0;
  return P.scat >= I.minS && (killed ? 0xFFFFFFFFu : P.scat) <= I.maxS && P.refr >= I.minRefr &&
         (killed ? 0xFFFFFFFFu : P.refr) <= I.maxRefr && P.refl >= I.minRefl &&
         (killed ? 0xFFFFFFFFu : P.refl) <= I.maxRefl && P.itr >= I.minI && (killed ? 0xFFFFFFFFu : P.itr) <= I.maxI &&
         (I.onlyCollected ? P.kec == 2 : true);
}

__device__ __forceinline__ bool in_cuboid(const Inst &I, const float *i) {
  return i[0] < I.n[0] && i[0] >= 0 && i[1] < I.n[1] && i[1] >= 0 && i[2] < I.n[2] && i[2] >= 0;
}

// Voxel index clamped to the cuboid (getNewj, MCmatlablib.c:281-285); NaN coordinates map to 0.
__device__ __forceinline__ int clamp_coord(float v, int n) {
  return v >= 0.f ? (v < (float)n ? (int)floorf(v) : n - 1) : 0;
}

__device__ __forceinline__ int voxel_index(const Inst &I, const float *i) {
  return (clamp_coord(i[2], I.n[2]) * I.n[1] + clamp_coord(i[1], I.n[1])) * I.n[0] + clamp_coord(i[0], I.n[0]);
}

// Voxel of position i inside the gradient target box.
__device__ __forceinline__ bool in_box(const Inst &I, const float *i) {
  const int cx = clamp_coord(i[0], I.n[0]), cy = clamp_coord(i[1], I.n[1]), cz = clamp_coord(i[2], I.n[2]);
  return cx >= I.box[0] && cx < I.box[1] && cy >= I.box[2] && cy < I.box[3] && cz >= I.box[4] && cz < I.box[5];
}

__device__ __forceinline__ void direction_changed(Photon &P, const Inst &I) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    P.D[k] = P.u[k] != 0.f ? (floorf(P.i[k]) + (P.u[k] > 0) - P.i[k]) * I.d[k] / P.u[k] : __int_as_float(0x7f800000);
    P.dOverU[k] = I.d[k] / fabsf(P.u[k]);
  }
}

__device__ __forceinline__ void medium_props(Photon &P, const Inst &I, int m) {
  P.med = m;
  const float4 mp = I.med[m];
  P.mua = mp.x;
  P.mus = mp.y;
}

__device__ __forceinline__ void voxel_props(Photon &P, const Inst &I) {
  P.j = voxel_index(I, P.i);
  medium_props(P, I, __ldg(I.M0 + P.j));
}

// After a boundary-crossing sub-step and check_escape: the voxel and medium propagate already
// looked up, unless the packet was wrapped to the opposite face (then looked up again).
__device__ __forceinline__ void voxel_props_crossed(Photon &P, const Inst &I, bool teleported) {
  if (teleported) {
    voxel_props(P, I);
  } else {
    P.j = P.jn;
    medium_props(P, I, P.mn);
  }
}

__device__ __forceinline__ float launch_time(const Photon &P, const Inst &I, const float *t) {
  return -P.RI / kC *
         sqrtf(sqrf((P.i[0] - I.n[0] / 2.0f) * I.d[0] - t[0]) + sqrf((P.i[1] - I.n[1] / 2.0f) * I.d[1] - t[1]) +
               sqrf(P.i[2] * I.d[2] - t[2]));
}

// launchPhoton (MCmatlablib.c:519-732). Returns false when 1e6 attempts all land outside.
__device__ __forceinline__ bool launch_packet(Photon &P, const Inst &I) {
  P.sameVoxel = false;
  P.weight = 1.f;
  P.kec = 0;
  P.nsteps = 0;
  int attempts = 0;
  float tgt[3] = {0.f, 0.f, 0.f}, w0[3];
  const float hk = kKillRange / 2.0f;
  do {
    if (I.S) {
      const long long L = (long long)I.n[0] * I.n[1] * I.n[2];
      const long long jj = cdf_search_d((double)rnd(P, I), L, I.S);
      P.i[0] = (float)(jj % I.n[0]) + 1 - rnd(P, I);
      P.i[1] = (float)(jj / I.n[0] % I.n[1]) + 1 - rnd(P, I);
      P.i[2] = (float)(jj / I.n[0] / I.n[1]) + 1 - rnd(P, I);
      const float ct = 1 - 2 * rnd(P, I);
      const float st = sqrtf(1 - ct * ct);
      const float ph = 2 * kPi * rnd(P, I);
      float sp, cp;
      sincosf(ph, &sp, &cp);
      P.u[0] = st * cp;
      P.u[1] = st * sp;
      P.u[2] = ct;
      P.j = voxel_index(I, P.i);
      P.RI = I.med[__ldg(I.M0 + P.j)].w;
      P.time = 0;
    } else {
      switch (I.beamType) {
        case 0:
          P.i[0] = (I.focus[0] - I.focus[2] * I.u[0] / I.u[2]) / I.d[0] + I.n[0] / 2.0f;
          P.i[1] = (I.focus[1] - I.focus[2] * I.u[1] / I.u[2]) / I.d[1] + I.n[1] / 2.0f;
          P.i[2] = 0;
          for (int k = 0; k < 3; k++) P.u[k] = I.u[k];
          P.j = voxel_index(I, P.i);
          P.RI = I.med[__ldg(I.M0 + P.j)].w;
          P.time = launch_time(P, I, I.focus);
          break;
        case 1: {
          const float r = rnd(P, I);
          P.i[0] = (I.focus[0] + I.u[0] * (r - 0.5f) * I.emitterLength) / I.d[0] + I.n[0] / 2.0f;
          P.i[1] = (I.focus[1] + I.u[1] * (r - 0.5f) * I.emitterLength) / I.d[1] + I.n[1] / 2.0f;
          P.i[2] = (I.focus[2] + I.u[2] * (r - 0.5f) * I.emitterLength) / I.d[2];
          const float ct = 1 - 2 * rnd(P, I);
          const float st = sqrtf(1 - ct * ct);
          const float ph = 2 * kPi * rnd(P, I);
          float sp, cp;
          sincosf(ph, &sp, &cp);
          P.u[0] = st * cp;
          P.u[1] = st * sp;
          P.u[2] = ct;
          P.j = voxel_index(I, P.i);
          P.RI = I.med[__ldg(I.M0 + P.j)].w;
          P.time = 0;
          break;
        }
        case 2: {
          const float span = (I.bt == 1 || I.bt == 3) ? 1.f : (float)kKillRange;
          P.i[0] = span * I.n[0] * (rnd(P, I) - 0.5f) + I.n[0] / 2.0f;
          P.i[1] = span * I.n[1] * (rnd(P, I) - 0.5f) + I.n[1] / 2.0f;
          P.i[2] = 0;
          for (int k = 0; k < 3; k++) P.u[k] = I.u[k];
          P.j = voxel_index(I, P.i);
          P.RI = I.med[__ldg(I.M0 + P.j)].w;
          P.time = P.RI / kC *
                   ((P.i[0] - I.n[0] / 2.0f) * I.d[0] * I.u[0] + (P.i[1] - I.n[1] / 2.0f) * I.d[1] * I.u[1] + P.i[2] * I.d[2] * I.u[2]);
          break;
        }
        case 3: {
          const float ph = rnd(P, I) * 2 * kPi;
          axis_rotate(I.v, I.u, ph, w0);
          const float r = I.FPw1 * sqrtf(((float)lambert_wm1(-(double)rnd(P, I) * 0.36787944117144233) + 1) / (-2)) / 1.50087f;
          for (int k = 0; k < 3; k++) tgt[k] = I.focus[k] + r * w0[k];
          const float ph2 = I.AIw1 * sqrtf(((float)lambert_wm1(-(double)rnd(P, I) * 0.36787944117144233) + 1) / (-2)) / 1.50087f;
          axis_rotate(I.u, w0, ph2, P.u);
          P.i[0] = (tgt[0] - tgt[2] * P.u[0] / P.u[2]) / I.d[0] + I.n[0] / 2.0f;
          P.i[1] = (tgt[1] - tgt[2] * P.u[1] / P.u[2]) / I.d[1] + I.n[1] / 2.0f;
          P.i[2] = 0;
          P.j = voxel_index(I, P.i);
          P.RI = I.med[__ldg(I.M0 + P.j)].w;
          P.time = launch_time(P, I, tgt);
          break;
        }
        case 4: {
          axis_rotate(I.v, I.u, rnd(P, I) * 2 * kPi, w0);
          float r;
          if (I.FP1[0] == -1.f) r = I.FPw1 * sqrtf(rnd(P, I));
          else if (I.FP1[0] == -2.f) r = I.FPw1 * sqrtf(-0.5f * logf(rnd(P, I)));
          else {
            const float a = rnd(P, I);
            const int jj = cdf_search(a, I.LFP1 - 1, I.FP1);
            r = I.FPw1 * (jj + rnd(P, I)) / (I.LFP1 - 1);
          }
          for (int k = 0; k < 3; k++) tgt[k] = I.focus[k] + r * w0[k];
          axis_rotate(I.v, I.u, rnd(P, I) * 2 * kPi, w0);
          float ph;
          if (I.AI1[0] == -1.f) ph = atanf(tanf(I.AIw1) * sqrtf(rnd(P, I)));
          else if (I.AI1[0] == -2.f) ph = atanf(tanf(I.AIw1) * sqrtf(-0.5f * logf(rnd(P, I))));
          else if (I.AI1[0] == -3.f) ph = asinf(sqrtf(rnd(P, I)));
          else {
            const float a = rnd(P, I);
            const int jj = cdf_search(a, I.LAI1 - 1, I.AI1);
            ph = atanf(tanf(I.AIw1) * (jj + rnd(P, I)) / (I.LAI1 - 1));
          }
          axis_rotate(I.u, w0, ph, P.u);
          P.i[0] = (tgt[0] - tgt[2] * P.u[0] / P.u[2]) / I.d[0] + I.n[0] / 2.0f;
          P.i[1] = (tgt[1] - tgt[2] * P.u[1] / P.u[2]) / I.d[1] + I.n[1] / 2.0f;
          P.i[2] = 0;
          P.j = voxel_index(I, P.i);
          P.RI = I.med[__ldg(I.M0 + P.j)].w;
          P.time = launch_time(P, I, tgt);
          break;
        }
        default: {  // 5: X/Y factorizable
          float X, Y;
          if (I.FP1[0] == -1.f) X = I.FPw1 * (rnd(P, I) * 2 - 1);
          else if (I.FP1[0] == -2.f) {
            const float a = rnd(P, I);
            X = I.FPw1 * sqrtf(-0.5f * logf(a)) * cosf(2 * kPi * rnd(P, I));
          } else {
            const float a = rnd(P, I);
            const int jj = cdf_search(a, I.LFP1 - 1, I.FP1);
            X = I.FPw1 * ((jj + rnd(P, I)) / (I.LFP1 - 1) * 2 - 1);
          }
          if (I.FP2[0] == -1.f) Y = I.FPw2 * (rnd(P, I) * 2 - 1);
          else if (I.FP2[0] == -2.f) {
            const float a = rnd(P, I);
            Y = I.FPw2 * sqrtf(-0.5f * logf(a)) * cosf(2 * kPi * rnd(P, I));
          } else {
            const float a = rnd(P, I);
            const int jj = cdf_search(a, I.LFP2 - 1, I.FP2);
            Y = I.FPw2 * ((jj + rnd(P, I)) / (I.LFP2 - 1) * 2 - 1);
          }
          for (int k = 0; k < 3; k++) tgt[k] = I.focus[k] + X * I.v[k] + Y * I.w[k];
          if (I.AI1[0] == -3.f) {
            axis_rotate(I.v, I.u, rnd(P, I) * 2 * kPi, w0);
            axis_rotate(I.u, w0, asinf(sqrtf(rnd(P, I))), P.u);
          } else {
            float tx, ty;
            // custom angular X/Y distributions are scaled by L, not L-1 (MCmatlablib.c:678-688)
            if (I.AI1[0] == -1.f) tx = tanf(I.AIw1) * (rnd(P, I) * 2 - 1);
            else if (I.AI1[0] == -2.f) {
              const float a = rnd(P, I);
              tx = tanf(I.AIw1) * sqrtf(-0.5f * logf(a)) * cosf(2 * kPi * rnd(P, I));
            } else {
              const float a = rnd(P, I);
              const int jj = cdf_search(a, I.LAI1 - 1, I.AI1);
              tx = tanf(I.AIw1) * ((jj + rnd(P, I)) / I.LAI1 * 2 - 1);
            }
            if (I.AI2[0] == -1.f) ty = tanf(I.AIw2) * (rnd(P, I) * 2 - 1);
            else if (I.AI2[0] == -2.f) {
              const float a = rnd(P, I);
              ty = tanf(I.AIw2) * sqrtf(-0.5f * logf(a)) * cosf(2 * kPi * rnd(P, I));
            } else {
              const float a = rnd(P, I);
              const int jj = cdf_search(a, I.LAI2 - 1, I.AI2);
              ty = tanf(I.AIw2) * ((jj + rnd(P, I)) / I.LAI2 * 2 - 1);
            }
            axis_rotate(I.v, I.u, atan2f(tx, ty), w0);
            axis_rotate(I.u, w0, atanf(sqrtf(tx * tx + ty * ty)), P.u);
          }
          P.i[0] = (tgt[0] - tgt[2] * P.u[0] / P.u[2]) / I.d[0] + I.n[0] / 2.0f;
          P.i[1] = (tgt[1] - tgt[2] * P.u[1] / P.u[2]) / I.d[1] + I.n[1] / 2.0f;
          P.i[2] = 0;
          P.j = voxel_index(I, P.i);
          P.RI = I.med[__ldg(I.M0 + P.j)].w;
          P.time = launch_time(P, I, tgt);
          break;
        }
      }
    }
    if (I.bt == 0) {
      P.alive = fabsf(P.i[0] / I.n[0] - 0.5f) < hk && fabsf(P.i[1] / I.n[1] - 0.5f) < hk && fabsf(P.i[2] / I.n[2] - 0.5f) < hk;
    } else if (I.bt == 2) {
      P.alive = fabsf(P.i[0] / I.n[0] - 0.5f) < hk && fabsf(P.i[1] / I.n[1] - 0.5f) < hk && P.i[2] / I.n[2] - 0.5f < hk && P.i[2] >= 0;
    } else {
      P.alive = in_cuboid(I, P.i);
    }
  } while (!P.alive && ++attempts < 1000000);
  direction_changed(P, I);
  P.inside = in_cuboid(I, P.i);
  P.stepLeft = -logf(rnd(P, I));
  P.scat = P.refr = P.refl = P.itr = 0;
  return P.alive;
}

// getInterpolatedNormal (MCmatlablib.c:920-1014): the reference truncates the coerced position
// to an integer before subtracting 0.5, so all eight weights are 0.5; the normal is the
// normalised sum over the 2x2x2 block {k-1, k}^3 of voxels whose RI equals the new voxel's.
__device__ __forceinline__ void interface_normal(const Photon &P, const Inst &I, int jn, float *nv) {
  int i0[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    i0[k] = clamp_coord(P.i[k], I.n[k]) - 1;
  }
  const float ri = I.med[__ldg(I.M0 + jn)].w;
  float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const int cx = c & 1, cy = (c >> 1) & 1, cz = c >> 2;
    const int jx = i0[0] + cx, jy = i0[1] + cy, jz = i0[2] + cz;
    const bool ok = (cx ? i0[0] < I.n[0] - 1 : jx >= 0) && (cy ? i0[1] < I.n[1] - 1 : jy >= 0) &&
                    (cz ? i0[2] < I.n[2] - 1 : jz >= 0);
    if (!ok) continue;
    const int jc = (jz * I.n[1] + jy) * I.n[0] + jx;
    if (I.med[__ldg(I.M0 + jc)].w != ri) continue;
    const float4 nn = __ldg(I.nrm + jc);
    sx += nn.x;
    sy += nn.y;
    sz += nn.z;
  }
  const float inv = rsqrtf(sx * sx + sy * sy + sz * sz);
  nv[0] = sx * inv;
  nv[1] = sy * inv;
  nv[2] = sz * inv;
}

// propagatePhoton without the deposit (MCmatlablib.c:1019-1091); returns the step length s.
__device__ __forceinline__ float propagate(Photon &P, const Inst &I) {
  P.sameVoxel = true;
  // fast division (two-ulp, a reciprocal and a multiply): q only decides the sub-step length,
  // and the comparison s == q below uses this same q
  const float q = __fdividef(P.stepLeft, P.mus);
  const float s = fminf(q, fminf(P.D[0], fminf(P.D[1], P.D[2])));
  P.stepLeft = s == q ? 0.f : P.stepLeft - s * P.mus;
  P.time += s * P.RI * (1.0f / kC);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float io = floorf(P.i[k]);
    if (s == P.D[k]) {
      P.i[k] = P.u[k] > 0 ? io + 1 : io - kFltEps * (fabsf(io) + 1);
      P.D[k] = P.dOverU[k];
      P.sameVoxel = false;
    } else {
      P.i[k] += s * (P.u[k] * I.invd[k]);
      if (floorf(P.i[k]) != io) P.i[k] = P.u[k] > 0 ? io + 1 - kFltEps * (fabsf(io) + 1) : io;
      P.D[k] -= s;
    }
  }
  if (!P.sameVoxel) {
    const int jn = voxel_index(I, P.i);
    const int mn = __ldg(I.M0 + jn);
    P.jn = jn;
    P.mn = mn;
    const float rin = I.med[mn].w;
    const float mu = P.RI / rin;
    if (mu != 1.f) {
      float nv[3];
      interface_normal(P, I, jn, nv);
      const float cin = nv[0] * P.u[0] + nv[1] * P.u[1] + nv[2] * P.u[2];
      if (cin > 0) {
        const float cos2 = 1 - mu * mu * (1 - cin * cin);
        bool refl;
        if (cos2 > 0) {
          const float co = sqrtf(cos2);
          const float Rf = sqrf((mu * cin - co) / (mu * cin + co)) / 2 + sqrf((mu * co - cin) / (mu * co + cin)) / 2;
          refl = rnd(P, I) <= Rf;
        } else {
          refl = true;
        }
        if (refl) {
          for (int k = 0; k < 3; k++) P.u[k] -= 2 * nv[k] * cin;
          direction_changed(P, I);
          if ((uint32_t)mn >= I.minIdx && (uint32_t)mn <= I.maxIdx) P.refl++;
        } else {
          const float nc = sqrtf(cos2) - mu * cin;
          for (int k = 0; k < 3; k++) P.u[k] = nc * nv[k] + mu * P.u[k];
          direction_changed(P, I);
          P.RI = rin;
          if ((uint32_t)mn >= I.minIdx && (uint32_t)mn <= I.maxIdx) {
            P.refr++;
            P.itr++;
          }
        }
      }
    } else {
      const int mo = P.med;  // medium of the voxel left (voxel_props)
      if (mn != mo && I.med[mo].w == P.RI && (uint32_t)mn >= I.minIdx && (uint32_t)mn <= I.maxIdx) P.itr++;
    }
  }
  return s;
}

__device__ __forceinline__ void atomic_add_f64(double *p, double v) { atomicAdd(p, v); }

// Absorbed fraction 1 - exp(-x), x = mua s >= 0 (MCmatlablib.c evaluates -expm1(-mua s)):
// the Taylor series below x = 1/16 (truncation below 2e-9 relative), 1 - expf(-x) above, where
// the subtraction loses at most a factor 16 of expf's relative error
__device__ __forceinline__ float one_minus_exp_neg(float x) {
  if (x < 0.0625f)
    return x * (1.f - x * (0.5f - x * (1.f / 6.f - x * (1.f / 24.f - x * (1.f / 120.f - x * (1.f / 720.f))))));
  return 1.f - expf(-x);
}

// formImage (MCmatlablib.c:737-788)
// With tally == false only the classification (P.kec) is updated.
__device__ __forceinline__ void form_image(Photon &P, const Inst &I, bool tally) {
  float U[3];
  to_lc_frame(P.u, I.LCth, I.LCph, U);
  if (!(U[2] < 0)) return;
  const float resc[3] = {(P.i[0] - I.n[0] / 2.0f) * I.d[0] - I.LCr[0], (P.i[1] - I.n[1] / 2.0f) * I.d[1] - I.LCr[1],
                         P.i[2] * I.d[2] - I.LCr[2]};
  float Re[3];
  to_lc_frame(resc, I.LCth, I.LCph, Re);
  if (!(Re[2] > 0)) return;
  const float RL0 = Re[0] - Re[2] * U[0] / U[2], RL1 = Re[1] - Re[2] * U[1] / U[2];
  if (!(sqrtf(RL0 * RL0 + RL1 * RL1) < I.LCdiam / 2)) return;
  if (I.lcFinite) {
    const float RI0 = RL0 + I.LCf * U[0] / U[2], RI1 = RL1 + I.LCf * U[1] / U[2];
    if (!(sqrtf(RI0 * RI0 + RI1 * RI1) < I.LCfs / 2)) return;
    // pixel indices; the clamp only acts when float rounding lands exactly on the far edge
    const int Xi = min(max((int)(I.LCres0 * (RI0 / I.LCfs + 0.5f)), 0), I.LCres0 - 1);
    const int Yi = min(max((int)(I.LCres0 * (RI1 / I.LCfs + 0.5f)), 0), I.LCres0 - 1);
    int ti = 0;
    if (I.LCres1 > 1) {
      const float v = 1 + (I.LCres1 - 2) * (P.time - (Re[2] - I.LCf) / U[2] * P.RI / kC - I.tStart) / (I.tEnd - I.tStart);
      const long long vl = (long long)v;
      ti = (int)(vl < 0 ? 0 : (vl > I.LCres1 - 1 ? I.LCres1 - 1 : vl));
    }
    P.kec = 2;
    if (tally && criteria_met(P, I)) {
      atomic_add_f64(&I.image[Xi + Yi * I.LCres0 + ti * I.LCres0 * I.LCres0], (double)P.weight);
      atomicAdd(&I.ctr[1], 1ull);
    }
  } else {
    const float thFF = atanf(-sqrtf(U[0] * U[0] + U[1] * U[1]) / U[2]);
    if (!(thFF < asinf(fminf(1.0f, I.LCfs)))) return;
    int ti = 0;
    if (I.LCres1 > 1) {
      const float v = 1 + (I.LCres1 - 2) * (P.time - Re[2] / U[2] * P.RI / kC - I.tStart) / (I.tEnd - I.tStart);
      const long long vl = (long long)v;
      ti = (int)(vl < 0 ? 0 : (vl > I.LCres1 - 1 ? I.LCres1 - 1 : vl));
    }
    P.kec = 2;
    if (tally && criteria_met(P, I)) {
      atomic_add_f64(&I.image[ti], (double)P.weight);
      atomicAdd(&I.ctr[1], 1ull);
    }
  }
}

// formEdgeFluxes (MCmatlablib.c:802-816)
// Face pixel of a coordinate: truncation as in the reference, clamped to the face so that a
// packet leaving exactly through an edge (two boundaries crossed in one sub-step) stays in bounds.
__device__ __forceinline__ int face_px(float v, int n) {
  const int k = v >= 0.f ? (v < (float)n ? (int)v : n - 1) : 0;
  return k;
}

__device__ __forceinline__ void edge_fluxes(const Photon &P, const Inst &I) {
  const double w = P.weight;
  const int n0 = I.n[0], n1 = I.n[1], n2 = I.n[2];
  if (I.bt == 1) {
    if (P.i[2] < 0) atomic_add_f64(&I.NIzn[face_px(P.i[0], n0) + n0 * face_px(P.i[1], n1)], w);
    else if (P.i[2] >= n2) atomic_add_f64(&I.NIzp[face_px(P.i[0], n0) + n0 * face_px(P.i[1], n1)], w);
    else if (P.i[1] < 0) atomic_add_f64(&I.NIyn[face_px(P.i[0], n0) + n0 * face_px(P.i[2], n2)], w);
    else if (P.i[1] >= n1) atomic_add_f64(&I.NIyp[face_px(P.i[0], n0) + n0 * face_px(P.i[2], n2)], w);
    else if (P.i[0] < 0) atomic_add_f64(&I.NIxn[face_px(P.i[1], n1) + n1 * face_px(P.i[2], n2)], w);
    else if (P.i[0] >= n0) atomic_add_f64(&I.NIxp[face_px(P.i[1], n1) + n1 * face_px(P.i[2], n2)], w);
  } else if (I.bt == 2) {
    if (P.i[2] < 0)
      atomic_add_f64(&I.NIzn[face_px(P.i[0] + n0 * (kKillRange - 1) / 2.0f, kKillRange * n0) +
                             (kKillRange * n0) * face_px(P.i[1] + n1 * (kKillRange - 1) / 2.0f, kKillRange * n1)],
                     w);
  } else {
    if (P.i[2] < 0) atomic_add_f64(&I.NIzn[face_px(P.i[0], n0) + n0 * face_px(P.i[1], n1)], w);
    else if (P.i[2] >= n2) atomic_add_f64(&I.NIzp[face_px(P.i[0], n0) + n0 * face_px(P.i[1], n1)], w);
  }
}

// checkEscape (MCmatlablib.c:821-889). `tally` is false while replaying a packet.
// Returns true when a cyclic wrap teleported the packet.
__device__ __forceinline__ bool check_escape(Photon &P, const Inst &I, bool tally) {
  bool esc = false, teleported = false;
  const float hk = kKillRange / 2.0f;
  switch (I.bt) {
    case 0:
      P.alive = fabsf(P.i[0] / I.n[0] - 0.5f) < hk && fabsf(P.i[1] / I.n[1] - 0.5f) < hk && fabsf(P.i[2] / I.n[2] - 0.5f) < hk;
      break;
    case 1:
      P.alive = in_cuboid(I, P.i);
      esc = !P.alive && P.RI == 1.f;
      break;
    case 2:
      P.alive = fabsf(P.i[0] / I.n[0] - 0.5f) < hk && fabsf(P.i[1] / I.n[1] - 0.5f) < hk && P.i[2] / I.n[2] - 0.5f < hk && P.i[2] >= 0;
      esc = P.i[2] < 0 && P.RI == 1.f;
      break;
    default: {
      const bool tooOld = P.time > 1000 / kC * sqrtf(sqrf(I.d[0] * I.n[0]) + sqrf(I.d[1] * I.n[1]));
      P.alive = P.i[2] < I.n[2] && P.i[2] >= 0 && !tooOld;
      esc = !P.alive && P.RI == 1.f && !tooOld;
      if (P.i[0] >= I.n[0]) { P.i[0] = 0; teleported = true; }
      if (P.i[0] < 0) { P.i[0] = I.n[0] * (1 - kFltEps); teleported = true; }
      if (P.i[1] >= I.n[1]) { P.i[1] = 0; teleported = true; }
      if (P.i[1] < 0) { P.i[1] = I.n[1] * (1 - kFltEps); teleported = true; }
      break;
    }
  }
  P.inside = in_cuboid(I, P.i);
  if (esc) {
    P.kec = 1;
    if (I.image) form_image(P, I, tally);
    if (tally && I.FF && criteria_met(P, I)) {
      const float th = (1 - kFltEps) * acosf(fminf(fmaxf(P.u[2], -1.f), 1.f));
      const float ph = (1 - kFltEps) * (kPi + atan2f(P.u[1], P.u[0]));
      const int bt = min(max((int)floorf(th / kPi * I.ffr), 0), I.ffr - 1);
      const int bp = min(max((int)floorf(ph / (2 * kPi) * I.ffr), 0), I.ffr - 1);
      atomic_add_f64(&I.FF[bt + I.ffr * bp], (double)P.weight);
    }
  }
  if (tally && !P.alive && I.bt && criteria_met(P, I)) edge_fluxes(P, I);
  return teleported;
}

// scatterPhoton (MCmatlablib.c:1138-1184)
__device__ __forceinline__ void scatter(Photon &P, const Inst &I) {
  P.nsteps = 0;
  float ct;
  const float g = I.med[P.med].z;  // the medium's anisotropy (NaN: custom phase function)
  if (isnan(g)) {
    const float a = rnd(P, I);
    const int jt = cdf_search(a, kCdfSize - 1, I.CDFs + I.cdfidx[P.med] * kCdfSize);
    ct = cosf((jt + rnd(P, I)) * kPi / (kCdfSize - 1));
  } else {
    if (fabsf(g) == 1.0f) ct = g;
    else if (fabsf(g) <= 3.4526698e-4f) ct = 2 * rnd(P, I) - 1;  // sqrt(FLT_EPSILON)
    else ct = (1 + g * g - sqrf((1 - g * g) / (1 - g + 2 * g * rnd(P, I)))) / (2 * g);
  }
  const float st = sqrtf(1 - ct * ct);
  const float ph = 2 * kPi * rnd(P, I);
  float sp, cp;
  sincosf(ph, &sp, &cp);
  if (fabsf(P.u[2]) < 1) {
    const float qq = sqrtf(P.u[0] * P.u[0] + P.u[1] * P.u[1]);
    const float ux = st * (P.u[0] * P.u[2] * cp - P.u[1] * sp) / qq + P.u[0] * ct;
    const float uy = st * (P.u[1] * P.u[2] * cp + P.u[0] * sp) / qq + P.u[1] * ct;
    P.u[2] = -st * cp * qq + P.u[2] * ct;
    P.u[1] = uy;
    P.u[0] = ux;
  } else {
    P.u[0] = st * cp;
    P.u[1] = st * sp;
    P.u[2] = ct * (P.u[2] >= 0 ? 1.f : -1.f);
  }
  direction_changed(P, I);
  P.stepLeft = -logf(rnd(P, I));
  const int m = __ldg(I.M0 + P.j);
  if ((uint32_t)m >= I.minIdx && (uint32_t)m <= I.maxIdx) P.scat++;
}

}  // namespace mcb
