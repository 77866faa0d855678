// Persistent photon-packet transport kernel, its helpers, and the host driver behind
// mcb_mc_run / mcb_mc_run_batch (replacing +MCmatlab/src/MCmatlab.c:317-791).
//
// Work decomposition: every (model, wavelength) pair is an "instance" owning a contiguous
// range of a global packet index space. One persistent grid (SM count x resident blocks)
// runs until the space is exhausted; a lane whose packet dies takes the next index from a
// warp-aggregated atomic counter, so lanes stay busy regardless of packet lifetimes and
// instances of very different cost share one launch.
//
// Deposition: absorbed weight goes into FP64 tallies with native double atomics; consecutive
// sub-steps inside one voxel are summed in a register first (one atomic per voxel visit
// instead of one per sub-step).
//
// End-of-life deposition criteria (MCmatlab.c:262-264): instead of per-packet growable
// records, a packet that meets the criteria at death is replayed from its counter-based RNG
// stream, bit-identically, depositing w_final * absorb at every in-cuboid sub-step.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.h"
#include "mc_device.cuh"

namespace cg = cooperative_groups;

namespace mcb {

struct KernelArgs {
  const Inst *insts;
  const unsigned long long *instFirst;  // [nInst + 1]
  int nInst;
  unsigned long long *nextPacket;
  unsigned long long totalPackets;
  int openEnded;                   // single instance without a fixed packet count
  unsigned long long collectTarget;  // open-ended: stop once this many were collected (0: unused)
  unsigned long long deadlineNs;     // open-ended: stop fetching after this %globaltimer value (0: unused)
  const volatile int *cancel;        // host-mapped cancel flag
  int *status;                       // bit 0: cancelled, bit 1: a launch failed 1e6 times
  unsigned long long *steps;
  // Refill threshold: a warp re-launches free lanes only when at least this many are free (or
  // none is alive), so the divergent launch code runs once for a group of lanes.
  int refillMin;   // free lanes a warp waits for before launching new packets
  int scatterMin;  // waiting lanes before roulette + scattering run
};

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int find_instance(const KernelArgs &a, unsigned long long g) {
  int lo = 0, hi = a.nInst;  // instFirst[lo] <= g < instFirst[hi]
  while (lo + 1 < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(a.instFirst + mid) <= g) lo = mid; else hi = mid;
  }
  return lo;
}

// Next global packet index for the calling lane, or ~0ull when the run is over.
__device__ __forceinline__ unsigned long long fetch_packet(const KernelArgs &a) {
  cg::coalesced_group grp = cg::coalesced_threads();
  unsigned long long base = 0;
  int stop = 0;
  if (grp.thread_rank() == 0) {
    volatile int *st = a.status;
    stop = *st;
    if (!stop) {
      base = atomicAdd(a.nextPacket, (unsigned long long)grp.size());
      if ((base & 0x3FFFull) < grp.size() && *a.cancel) {
        atomicOr(a.status, 1);
        stop = 1;
      }
      if (a.openEnded) {
        if (a.collectTarget) {
          volatile unsigned long long *col = a.insts[0].ctr + 1;
          if (*col >= a.collectTarget) stop = 1;
        }
        if (a.deadlineNs && global_ns() >= a.deadlineNs) stop = 1;
      }
    }
  }
  stop = grp.shfl(stop, 0);
  base = grp.shfl(base, 0);
  if (stop) return ~0ull;
  const unsigned long long g = base + grp.thread_rank();
  if (!a.openEnded && g >= a.totalPackets) return ~0ull;
  return g;
}


// Launch bounds: the plain kernel runs 4 blocks of 256 per SM at 64 registers (about 100 bytes
// of spill stores; measured 3-9% more packets/s than 3 blocks at 80 registers without spills);
// the gradient variant runs 3 blocks without spills (at 64 registers it ran slower). The gradient
// variant keeps its per-packet state (path length L_m and scattering count k_m per medium) and
// its per-thread box partial sums in dynamic shared memory, one column per thread
// (grad_smem_bytes), so that it holds 3 blocks per SM; the medium index selects the row directly.
template <bool GRAD>
__global__ void __launch_bounds__(256, GRAD ? 3 : 4) transport_kernel(KernelArgs a) {
  // single-instance runs read the instance and its medium table from shared memory
  __shared__ Inst sInst;
  __shared__ float4 sMed[256];
  __shared__ int sCdf[256];
  __shared__ float sInvMus[kGradMedia];
  extern __shared__ double gradSmem[];
  const bool single = a.nInst == 1;
  if (single) {
    const Inst *g0 = a.insts;
    if (threadIdx.x == 0) sInst = *g0;
    for (int k = threadIdx.x; k < g0->nM; k += blockDim.x) {
      sMed[k] = g0->med[k];
      sCdf[k] = g0->cdfidx[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      sInst.med = sMed;
      sInst.cdfidx = sCdf;
    }
    __syncthreads();
  }
  int nGM = 0, nGR = 0;
  // gradient state (GRAD only): radial-bin and box sums of the block, and per-thread columns
  // (stride blockDim.x) of the packet's L_m, k_m, A_m, E_m and the thread's box partial sums
  // [value, d/dmua, d/dmus]. The box derivatives are summed per packet in deferred form: with
  // C the packet's box tally so far, A_m = sum over its sub-steps in m of s C (C after the
  // sub-step) and E_m = sum over its interactions in m of C, the per-sub-step terms
  // sum_t L_m(t) c(t) and sum_t k_m(t) c(t) equal L_m C - A_m and k_m C - E_m at the packet's
  // end, so a box sub-step costs O(1) instead of a loop over the media.
  double *sR = gradSmem, *sF = gradSmem;
  float *sGL = nullptr, *sGK = nullptr, *sGA = nullptr, *sGE = nullptr, *sBox = nullptr;
  float boxC = 0.f;
  const int tid = threadIdx.x, bd = blockDim.x;
  if (GRAD) {
    // gradient runs are single-instance (enforced by the host)
    nGM = sInst.nM;
    nGR = sInst.nR;
    sF = sR + nGR * (1 + 2 * nGM);
    sGL = (float *)(sF + 1 + 2 * nGM);
    sGK = sGL + nGM * bd;
    sGA = sGK + nGM * bd;
    sGE = sGA + nGM * bd;
    sBox = sGE + nGM * bd;
    for (int k = threadIdx.x; k < nGR * (1 + 2 * nGM); k += blockDim.x) sR[k] = 0.0;
    for (int k = threadIdx.x; k < 1 + 2 * nGM; k += blockDim.x) sF[k] = 0.0;
    for (int k = threadIdx.x; k < nGM; k += blockDim.x) sInvMus[k] = 1.0f / sMed[k].y;
    for (int q = 0; q < 1 + 2 * nGM; q++) sBox[q * bd + tid] = 0.f;
    __syncthreads();
  }
  Photon P;
  P.alive = false;
  P.inbox = false;
  const Inst *I = single ? &sInst : a.insts;
  bool replay = false;
  bool started = false;
  bool retired = false;
  float wfinal = 0.f;
  float acc = 0.f;  // deposit run in one voxel (a few sub-steps)
  int accj = -1;
  unsigned int steps = 0;  // this thread's sub-steps (a 32-bit count: about 1e7 per thread at 1e10 packets)
  unsigned long long pid = 0;
  for (;;) {
    // 1. a finished packet: flush its deposit run, then either queue its end-of-life replay
    //    (MCmatlab.c:262-264) or mark the lane free
    bool relaunch = false;
    if (!P.alive && started) {
      if (accj >= 0) {
        atomic_add_f64(&I->NFR[accj], (double)acc);
        accj = -1;
        acc = 0.f;
      }
      if (GRAD && boxC > 0.f) {
        for (int m = 0; m < nGM; m++) {
          const float lc = sGL[m * bd + tid] * boxC - sGA[m * bd + tid];
          const float kc = sGK[m * bd + tid] * boxC - sGE[m * bd + tid];
          sBox[(1 + m) * bd + tid] -= lc;
          sBox[(1 + nGM + m) * bd + tid] += kc * sInvMus[m] - lc;
        }
        boxC = 0.f;
      }
      if (I->eol && !replay && I->NFR && criteria_met(P, *I)) {
        replay = true;
        wfinal = P.weight;
        relaunch = true;
      } else {
        replay = false;
        started = false;
      }
    }
    // 2. refill free lanes in groups
    const bool idle = !P.alive && !retired && !relaunch;
    const unsigned freeLanes = __ballot_sync(0xffffffffu, idle);
    const unsigned liveLanes = __ballot_sync(0xffffffffu, P.alive || relaunch);
    bool fresh = false;
    if (freeLanes && (__popc(freeLanes) >= a.refillMin || liveLanes == 0)) {
      if (idle) {
        const unsigned long long g = fetch_packet(a);
        if (g == ~0ull) {
          retired = true;
        } else {
          const int ii = single ? 0 : find_instance(a, g);
          if (!single) I = a.insts + ii;
          pid = g - (single ? 0ull : __ldg(a.instFirst + ii));
          pid = I->pOff + I->pStride * pid;
          fresh = true;
        }
      }
    }
    // one call site launches new packets and replays (launchPhoton is the largest routine; two
    // inlined copies cost instruction-cache misses)
    if (fresh || relaunch) {
      P.pidlo = (uint32_t)pid;
      P.pidhi = (uint32_t)(pid >> 32);
      P.draw = 0;
      const bool ok = launch_packet(P, *I);
      if (ok || relaunch) voxel_props(P, *I);
      if (fresh) {
        if (ok) {
          atomicAdd(&I->ctr[0], 1ull);
          started = true;
          if (GRAD) {
            for (int m = 0; m < nGM; m++) {
              sGL[m * bd + tid] = 0.f;
              sGK[m * bd + tid] = 0.f;
              sGA[m * bd + tid] = 0.f;
              sGE[m * bd + tid] = 0.f;
            }
            P.inbox = in_box(*I, P.i);
          }
        } else {
          atomicAdd(&I->ctr[3], 1ull);
          atomicOr(a.status, 2);
        }
      }
    }
    if (__all_sync(0xffffffffu, retired && !P.alive)) break;
    // 3. one propagation sub-step for every packet with free path left
    if (P.alive) {
      if (P.stepLeft > 0) {
        const int mj = GRAD ? P.med : 0;
        const float wpre = GRAD ? P.weight : 0.f;
        const float s = propagate(P, *I);
        steps++;
        const float absorb = P.weight * one_minus_exp_neg(P.mua * s);
        P.weight -= absorb;
        if (GRAD) {
          // perturbation MC: the box tally c = absorb / mua_j (fluence-rate estimator) depends on
          // mua through the weight (-L_m c) and through the sub-step itself; on mus through the
          // score of the sampled path up to the end of this sub-step: k_m / mus_m - L_m, where
          // k counts the interaction that ends the sub-step when the free path ran out here.
          // This sub-step's own terms are added now; the terms of the earlier path (L_m, k_m
          // before this sub-step) are added at the packet's end in the deferred form above.
          if (P.inside && P.inbox) {
            const float mua = P.mua;
            const float c = absorb / mua;
            const float dself = wpre * s * s * self_phi(mua * s);
            const float kself = P.stepLeft > 0 ? 0.f : 1.f;
            boxC += c;
            sBox[tid] += c;
            sBox[(1 + mj) * bd + tid] += dself;
            sBox[(1 + nGM + mj) * bd + tid] += (kself * sInvMus[mj] - s) * c;
          }
          sGL[mj * bd + tid] += s;
          if (boxC > 0.f) sGA[mj * bd + tid] += s * boxC;
        }
        if (P.inside && I->NFR) {
          float c = 0.f;
          bool dep = false;
          if (replay) {
            c = wfinal * absorb;
            dep = true;
          } else if (!I->eol && criteria_met(P, *I)) {
            c = absorb;
            dep = true;
          }
          if (dep) {
            if (P.j == accj) {
              acc += c;
            } else {
              if (accj >= 0) atomic_add_f64(&I->NFR[accj], (double)acc);
              accj = P.j;
              acc = c;
            }
          }
        }
        if (!P.sameVoxel) {
          const bool tele = check_escape(P, *I, !replay);
          if (GRAD && !P.alive && P.kec != 0 && P.i[2] < 0 && nGR > 0) {
            // reflectance: escaping weight W on the top face, d/dmua_m = -L_m W,
            // d/dmus_m = (k_m / mus_m - L_m) W
            const float x = (P.i[0] - I->n[0] / 2.0f) * I->d[0], y = (P.i[1] - I->n[1] / 2.0f) * I->d[1];
            const int b = (int)(sqrtf(x * x + y * y) / I->rbin);
            if (b < nGR) {
              const float W = P.weight;
              double *row = sR + b * (1 + 2 * nGM);
              atomicAdd(row, (double)W);
              for (int m = 0; m < nGM; m++) {
                const float Lm = sGL[m * bd + tid];
                atomicAdd(row + 1 + m, (double)(-Lm * W));
                atomicAdd(row + 1 + nGM + m, (double)((sGK[m * bd + tid] * sInvMus[m] - Lm) * W));
              }
            }
          }
          if (P.alive) {
            voxel_props_crossed(P, *I, tele);
            if (GRAD) P.inbox = in_box(*I, P.i);
          }
        }
        if (++P.nsteps >= kMaxFreeSteps) {
          P.alive = false;
          if (!replay) {
            atomicAdd(&I->ctr[4], 1ull);
            atomicAdd(reinterpret_cast<double *>(&I->ctr[5]), (double)P.weight);
          }
        }
      }
    }
    // 4. scattering events in groups: a packet whose free path is used up waits (no sub-step)
    //    until enough lanes of its warp are waiting too, or no lane can take a sub-step, so the
    //    long scattering code runs with most lanes active. A packet's events and random draws do
    //    not change, only when its warp performs them. The group size (a.scatterMin) is a launch
    //    parameter of the autotuner; against single-lane scattering, groups of 8 gave the plain
    //    kernel 9.5% more packets/s on the 100^3 cube.
    {
      const bool want = P.alive && !(P.stepLeft > 0);
      const unsigned waiting = __ballot_sync(0xffffffffu, want);
      const unsigned stepping = __ballot_sync(0xffffffffu, P.alive && P.stepLeft > 0);
      if (want && (__popc(waiting) >= a.scatterMin || stepping == 0)) {
        if (P.weight < kThreshold) {
          if (rnd(P, *I) <= kChance) P.weight /= kChance;
          else P.alive = false;
        }
        if (P.alive) {
          if (GRAD) {
            sGK[P.med * bd + tid] += 1.f;
            if (boxC > 0.f) sGE[P.med * bd + tid] += boxC;
          }
          scatter(P, *I);
        }
      }
    }
  }
  // lanes leave the loop at different times, so each adds its own count
  atomicAdd(a.steps, (unsigned long long)steps);
  if (GRAD) {
    if (nGM > 0 && (I->box[1] > I->box[0]))
      for (int q = 0; q < 1 + 2 * nGM; q++) atomicAdd(&sF[q], (double)sBox[q * bd + tid]);
    __syncthreads();
    for (int k = threadIdx.x; k < nGR * (1 + 2 * nGM); k += blockDim.x)
      if (sR[k] != 0.0) atomicAdd(&sInst.gR[k], sR[k]);
    for (int k = threadIdx.x; k < 1 + 2 * nGM; k += blockDim.x)
      if (sF[k] != 0.0) atomicAdd(&sInst.gF[k], sF[k]);
  }
}

// (theta, phi) pairs -> unit vectors, as getNormal computes them (MCmatlablib.c:909-918).
__global__ void normals_kernel(const float2 *tp, float4 *out, long long L) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < L; k += (long long)gridDim.x * blockDim.x) {
    const float2 v = tp[k];
    float st, ct, sp, cp;
    sincosf(v.x, &st, &ct);
    sincosf(v.y, &sp, &cp);
    out[k] = make_float4(st * cp, st * sp, ct, 0.f);
  }
}

__global__ void to_zero_based_kernel(const uint8_t *M1, uint8_t *M0, long long L) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < L; k += (long long)gridDim.x * blockDim.x)
    M0[k] = (uint8_t)(M1[k] - 1);
}

// NFR = deposit / (V * normfactor * mua(M)) (MCmatlablib.c:1199-1203), written as float.
__global__ void normalize_nfr_kernel(const double *acc, const uint8_t *M0, const float4 *med, double scale, float *out,
                                     long long L) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < L; k += (long long)gridDim.x * blockDim.x)
    out[k] = (float)(acc[k] / (scale * (double)med[M0[k]].x));
}

__global__ void scale_kernel(const double *acc, double inv, float *out, long long n) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    out[k] = (float)(acc[k] * inv);
}

// Example paths (MCmatlablib.c:465-514, updatePaths calls in launchPhoton/propagatePhoton/
// scatterPhoton/checkEscape): packets 0, 1, 2, ... of the first instance are replayed serially
// by one thread and their vertices recorded, NaN-separated, until nPaths paths are finished.
struct PathWriter {
  double *data;
  long long cap, n;
  bool started;
};

__device__ void path_add(PathWriter &W, const Photon &P, const Inst &I, int nanCols) {
  if (W.n + nanCols + 1 > W.cap) {
    W.n = W.cap + 1;  // overflow marker
    return;
  }
  for (int c = 0; c < nanCols; c++) {
    for (int r = 0; r < 4; r++) W.data[4 * W.n + r] = __longlong_as_double(0x7ff8000000000000ll);
    W.n++;
  }
  W.data[4 * W.n + 0] = (P.i[0] - I.n[0] / 2.0f) * I.d[0];
  W.data[4 * W.n + 1] = (P.i[1] - I.n[1] / 2.0f) * I.d[1];
  W.data[4 * W.n + 2] = P.i[2] * I.d[2];
  W.data[4 * W.n + 3] = P.weight;
  W.n++;
  W.started = true;
}

__device__ void path_update(PathWriter &W, const Photon &P, const Inst &I, bool teleported) {
  if (W.n > W.cap) return;
  if (I.eol || criteria_met(P, I)) path_add(W, P, I, W.started ? (teleported ? 1 : 0) : 2);
}

__global__ void example_paths_kernel(const Inst *inst, int nPaths, unsigned long long maxPackets, double *data,
                                     long long cap, long long *outN) {
  if (threadIdx.x || blockIdx.x) return;
  const Inst &I = *inst;
  PathWriter W{data, cap, 0, false};
  int finished = 0;
  Photon P;
  for (unsigned long long pid = 0; pid < maxPackets && finished < nPaths && W.n <= cap; pid++) {
    const long long startN = W.n;
    P.pidlo = (uint32_t)pid;
    P.pidhi = (uint32_t)(pid >> 32);
    P.draw = 0;
    W.started = false;
    if (!launch_packet(P, I)) continue;
    path_update(W, P, I, false);
    voxel_props(P, I);
    while (P.alive) {
      while (P.alive && P.stepLeft > 0) {
        const float s = propagate(P, I);
        const float absorb = P.weight * one_minus_exp_neg(P.mua * s);
        P.weight -= absorb;
        path_update(W, P, I, false);
        if (!P.sameVoxel) {
          const bool tele = check_escape(P, I, false);
          if (tele && (I.eol || criteria_met(P, I))) path_update(W, P, I, true);
          if (P.alive) voxel_props_crossed(P, I, tele);
        }
        if (++P.nsteps >= kMaxFreeSteps) P.alive = false;
      }
      if (P.alive && P.weight < kThreshold) {
        if (rnd(P, I) <= kChance) P.weight /= kChance;
        else P.alive = false;
      }
      if (P.alive) {
        scatter(P, I);
        path_update(W, P, I, false);
      }
    }
    if (W.started) {
      if (I.eol && !criteria_met(P, I)) W.n = startN;  // deletePhotonPath
      else finished++;
    }
  }
  *outN = W.n > cap ? cap : W.n;
}

__global__ void read_globaltimer(unsigned long long *out) { *out = global_ns(); }

}  // namespace mcb

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------
namespace {

using namespace mcb;

struct Arena {
  char *base = nullptr;
  size_t cap = 0, used = 0;
  bool overflow = false;
  template <typename T>
  T *take(size_t n) {
    used = (used + 255) & ~(size_t)255;
    if (used + n * sizeof(T) > cap) {
      overflow = true;
      return (T *)base;  // callers check `overflow` before any device work uses the pointer
    }
    T *p = (T *)(base + used);
    used += n * sizeof(T);
    return p;
  }
};

uint32_t inf_cast(double x) {
  if (std::isinf(x)) return 0xFFFFFFFFu;
  if (x >= 4294967295.0) return 0xFFFFFFFFu;
  return (uint32_t)x;
}

void unit_cross(const double *a, const double *b, double *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
  const double nrm = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
  for (int k = 0; k < 3; k++) c[k] /= nrm;
}

void axis_rotate_h(const double *r, const double *u, double th, double *o) {
  const double st = std::sin(th), ct = std::cos(th);
  o[0] = (u[0] * u[0] * (1 - ct) + ct) * r[0] + (u[0] * u[1] * (1 - ct) - u[2] * st) * r[1] + (u[0] * u[2] * (1 - ct) + u[1] * st) * r[2];
  o[1] = (u[1] * u[0] * (1 - ct) + u[2] * st) * r[0] + (u[1] * u[1] * (1 - ct) + ct) * r[1] + (u[1] * u[2] * (1 - ct) - u[0] * st) * r[2];
  o[2] = (u[2] * u[0] * (1 - ct) - u[1] * st) * r[0] + (u[2] * u[1] * (1 - ct) + u[0] * st) * r[1] + (u[2] * u[2] * (1 - ct) + ct) * r[2];
}

// Beam CDF as MCmatlab.c:538-576 builds it: a single value is a code (-1 - code), a sampled
// distribution becomes its trapezoid-rule CDF (r-weighted for radial distributions).
std::vector<float> beam_cdf(const mcb_distr &d, bool radial) {
  std::vector<float> o(std::max<int64_t>(d.n, 1));
  if (d.n == 1) {
    o[0] = (float)(-1.0 - d.values[0]);
  } else {
    std::vector<double> c(d.n);
    c[0] = 0;
    for (int64_t k = 1; k < d.n; k++)
      c[k] = c[k - 1] + (radial ? k - 1 : 1) * d.values[k - 1] + (radial ? k : 1) * d.values[k];
    for (int64_t k = 0; k < d.n; k++) o[k] = (float)(k ? c[k] / c[d.n - 1] : 0.0);
  }
  return o;
}

// per-wavelength device counters: launched, collected, (unused), failed launches, free-step cuts
// and their weight (FP64 bits)
constexpr int kCtr = 6;

struct ModelPlan {
  const mcb_mc_model *m;
  mcb_mc_result *r;
  long long L;
  int nL;
  bool useS;
  // per wavelength
  std::vector<unsigned long long> nPackets;
  std::vector<double> power;
  // device pointers
  uint8_t *M0 = nullptr;
  float4 *nrm = nullptr;
  float4 *med = nullptr;     // [nL][nM]
  int *cdfidx = nullptr;     // [nL][nM]
  float *CDFs = nullptr;
  float *beam = nullptr;     // FP1 | FP2 | AI1 | AI2
  double *S = nullptr;       // [nL][L+1]
  double *accNFR = nullptr, *accImg = nullptr, *accFF = nullptr, *accNI = nullptr;
  unsigned long long *ctr = nullptr;  // [nL][kCtr]
  long long Lim = 0, Lff = 0, Lx = 0, Ly = 0, Lz = 0, Lzn = 0, niPer = 0;
  std::vector<Inst> insts;   // one per wavelength
};

mcb_status validate(mcb_ctx *ctx, const mcb_mc_model *m) {
  if (!m) return set_error(ctx, MCB_EINVAL, "model is NULL");
  if (m->nx < 2 || m->ny < 2 || m->nz < 2) return set_error(ctx, MCB_EINVAL, "grid dimensions must be > 1");
  const long long L = (long long)m->nx * m->ny * m->nz;
  if (L > 2147483647ll) return set_error(ctx, MCB_EINVAL, "grid has more than 2^31-1 voxels");
  if (!(m->dx > 0 && m->dy > 0 && m->dz > 0)) return set_error(ctx, MCB_EINVAL, "voxel sizes must be positive");
  if (!m->M) return set_error(ctx, MCB_EINVAL, "M is NULL");
  if (m->nM < 1 || m->nM > 256) return set_error(ctx, MCB_EINVAL, "nM must be in [1, 256]");
  if (m->nL < 1) return set_error(ctx, MCB_EINVAL, "nL must be >= 1");
  if (!m->mua || !m->mus || !m->g || !m->n || !m->CDFidx || !m->spectrum)
    return set_error(ctx, MCB_EINVAL, "media tables or spectrum missing");
  if (m->boundaryType < 0 || m->boundaryType > 3) return set_error(ctx, MCB_EINVAL, "boundaryType must be 0..3");
  if (!m->sourceDistribution && (m->sourceType < 0 || m->sourceType > 5))
    return set_error(ctx, MCB_EINVAL, "sourceType must be 0..5");
  const bool timed = std::isnan(m->nPhotonsRequested);
  if (!timed && !(m->nPhotonsRequested >= 1)) return set_error(ctx, MCB_EINVAL, "nPhotonsRequested must be >= 1 or NaN");
  if (timed && !(m->simulationTimeRequested > 0))
    return set_error(ctx, MCB_EINVAL, "simulationTimeRequested must be positive for a timed run");
  if (!m->sourceDistribution && m->sourceType >= 4) {
    const mcb_distr *ds[2] = {m->sourceType == 4 ? &m->FPID_radial : &m->FPID_X,
                              m->sourceType == 4 ? &m->AID_radial : &m->AID_X};
    for (auto d : ds)
      if (!d->values || d->n < 1) return set_error(ctx, MCB_EINVAL, "beam distribution missing");
    if (m->sourceType == 5 && (!m->FPID_Y.values || m->FPID_Y.n < 1 || !m->AID_Y.values || m->AID_Y.n < 1))
      return set_error(ctx, MCB_EINVAL, "Y beam distribution missing");
  }
  bool anyCustom = false, mismatched = false;
  for (int k = 0; k < m->nM * m->nL; k++) {
    if (!(m->mua[k] > 0) || !std::isfinite(m->mua[k])) return set_error(ctx, MCB_EINVAL, "mua must be finite and positive");
    if (!(m->mus[k] > 0) || !std::isfinite(m->mus[k])) return set_error(ctx, MCB_EINVAL, "mus must be finite and positive");
    if (std::isnan(m->g[k])) anyCustom = true;
    if (!(m->n[k] >= 1)) return set_error(ctx, MCB_EINVAL, "n must be >= 1");
    if (m->n[k] != m->n[k % m->nM]) mismatched = true;
  }
  for (int k = 1; k < m->nM; k++)
    if (m->n[k] != m->n[0]) mismatched = true;
  if (anyCustom && (!m->CDFs || m->nCDFelems < 201)) return set_error(ctx, MCB_EINVAL, "custom phase functions need CDFs");
  for (int k = 0; k < m->nM * m->nL; k++)
    if (std::isnan(m->g[k]) && !(m->CDFidx[k] >= 0 && (m->CDFidx[k] + 1) * 201 <= (double)m->nCDFelems))
      return set_error(ctx, MCB_EINVAL, "CDFidx out of range for a custom phase function");
  if (!m->sourceDistribution && m->sourceType >= 4) {
    const mcb_distr *all[4] = {m->sourceType == 4 ? &m->FPID_radial : &m->FPID_X, &m->FPID_Y,
                               m->sourceType == 4 ? &m->AID_radial : &m->AID_X, &m->AID_Y};
    for (int q = 0; q < (m->sourceType == 5 ? 4 : 4); q++) {
      if (m->sourceType == 4 && (q == 1 || q == 3)) continue;
      const mcb_distr *d = all[q];
      if (d->n == 1) {
        const double c = d->values[0];
        const bool angular = q >= 2;
        if (!(c == 0 || c == 1 || (angular && c == 2)))
          return set_error(ctx, MCB_EINVAL, "beam distribution code must be 0, 1%s", angular ? " or 2" : "");
      } else {
        for (int64_t k = 0; k < d->n; k++)
          if (!(d->values[k] >= 0) || !std::isfinite(d->values[k]))
            return set_error(ctx, MCB_EINVAL, "beam distributions must be finite and non-negative");
      }
      if (q < 2 && !(d->width >= 0)) return set_error(ctx, MCB_EINVAL, "focal plane width must be >= 0");
    }
  }
  if (m->sourceDistribution) {
    const long long LL = (long long)m->nx * m->ny * m->nz * m->nL;
    for (long long k = 0; k < LL; k++)
      if (!(m->sourceDistribution[k] >= 0) || !std::isfinite(m->sourceDistribution[k]))
        return set_error(ctx, MCB_EINVAL, "sourceDistribution must be finite and non-negative");
  }
  for (long long k = 0; k < L; k++)
    if (m->M[k] < 1 || m->M[k] > m->nM) return set_error(ctx, MCB_EINVAL, "M holds a medium index outside 1..nM");
  if (mismatched && !m->interfaceNormals)
    return set_error(ctx, MCB_EINVAL, "refractive indices differ between media but interfaceNormals is NULL");
  if (m->useLightCollector && m->LC_res < 1 && std::isfinite(m->LC_f))
    return set_error(ctx, MCB_EINVAL, "light collector resolution must be >= 1");
  if (m->farFieldRes < 0) return set_error(ctx, MCB_EINVAL, "farFieldRes must be >= 0");
  return MCB_OK;
}

size_t plan_bytes(const mcb_mc_model *m) {
  const long long L = (long long)m->nx * m->ny * m->nz;
  const int nL = m->nL;
  size_t b = 0;
  auto add = [&](size_t x) { b += ((x + 255) & ~(size_t)255) + 256; };
  add(L);                                       // M (1-based upload)
  add(L);                                       // M0
  if (m->interfaceNormals) add(8 * L), add(16 * L);
  add(16 * (size_t)m->nM * nL), add(4 * (size_t)m->nM * nL);
  add(4 * (size_t)std::max<int64_t>(m->nCDFelems, 1));
  add(4 * (size_t)(std::max<int64_t>(m->FPID_radial.n, 1) + std::max<int64_t>(m->FPID_X.n, 1) + std::max<int64_t>(m->FPID_Y.n, 1) +
                   std::max<int64_t>(m->AID_radial.n, 1) + std::max<int64_t>(m->AID_X.n, 1) + std::max<int64_t>(m->AID_Y.n, 1) + 8));
  if (m->sourceDistribution) add(8 * (size_t)(L + 1) * nL);
  const long long res = m->LC_res, nT = m->LC_nTimeBins ? m->LC_nTimeBins + 2 : 1;
  if (m->calcNFR) add(8 * (size_t)L * nL);
  if (m->useLightCollector) add(8 * (size_t)res * res * nT * nL);
  if (m->farFieldRes) add(8 * (size_t)m->farFieldRes * m->farFieldRes * nL);
  const long long nx = m->nx, ny = m->ny, nz = m->nz;
  add(8 * (size_t)(2 * ny * nz + 2 * nx * nz + nx * ny + 25 * nx * ny) * nL);
  add(8 * kCtr * (size_t)nL);
  add(sizeof(Inst) * nL + 8 * (nL + 1));
  // float staging for outputs
  size_t fo = 0;
  if (m->calcNFR) fo += (size_t)L * nL;
  if (m->useLightCollector) fo += (size_t)res * res * nT * nL;
  if (m->farFieldRes) fo += (size_t)m->farFieldRes * m->farFieldRes * nL;
  fo += (size_t)(2 * ny * nz + 2 * nx * nz + nx * ny + 25 * nx * ny) * nL;
  add(4 * fo);
  return b;
}

// Copies inputs and builds the instance table of one model inside the arena.
// Offsets (in doubles) of the blocks of mcb_mc_result.tallies; the accumulator sizes are those
// build_plan gives the plan's device accumulators.
struct TallyLayout {
  long long nfr, img, ff, ni, cnt, total;
};

TallyLayout tally_layout(const mcb_mc_model *m) {
  const long long nx = m->nx, ny = m->ny, nz = m->nz, L = nx * ny * nz, nL = m->nL;
  const bool useS = m->sourceDistribution != nullptr;
  const long long res = m->LC_res, nT = (!useS && m->LC_nTimeBins) ? m->LC_nTimeBins + 2 : 1;
  const long long Lim = m->useLightCollector ? res * res * nT : 0, Lff = (long long)m->farFieldRes * m->farFieldRes;
  const long long Lzn = m->boundaryType == 2 ? nx * ny * kKillRange * kKillRange : nx * ny;
  const long long niPer = 2 * ny * nz + 2 * nx * nz + nx * ny + Lzn;
  TallyLayout t;
  long long o = 0;
  t.nfr = o;
  o += m->calcNFR ? L * nL : 0;
  t.img = o;
  o += Lim * nL;
  t.ff = o;
  o += Lff * nL;
  t.ni = o;
  o += niPer * nL;
  t.cnt = o;
  o += 2 * nL;
  t.total = o;
  return t;
}

mcb_status build_plan(mcb_ctx *ctx, Arena &ar, ModelPlan &pl, uint32_t stream) {
  const mcb_mc_model *m = pl.m;
  cudaStream_t st = ctx->stream;
  const long long L = (long long)m->nx * m->ny * m->nz;
  pl.L = L;
  pl.nL = m->nL;
  pl.useS = m->sourceDistribution != nullptr;
  const int nM = m->nM, nL = m->nL;
  const int grid = ctx->num_sms * 8;
  // geometry
  uint8_t *M1 = ar.take<uint8_t>(L);
  pl.M0 = ar.take<uint8_t>(L);
  if (ar.overflow) return set_error(ctx, MCB_ENOMEM, "internal: device arena too small");
  MCB_CUDA(ctx, cudaMemcpyAsync(M1, m->M, L, cudaMemcpyHostToDevice, st));
  to_zero_based_kernel<<<grid, 256, 0, st>>>(M1, pl.M0, L);
  if (m->interfaceNormals) {
    float2 *raw = ar.take<float2>(L);
    pl.nrm = ar.take<float4>(L);
    if (ar.overflow) return set_error(ctx, MCB_ENOMEM, "internal: device arena too small");
    MCB_CUDA(ctx, cudaMemcpyAsync(raw, m->interfaceNormals, 8 * L, cudaMemcpyHostToDevice, st));
    normals_kernel<<<grid, 256, 0, st>>>(raw, pl.nrm, L);
  }
  // media tables per wavelength
  std::vector<float4> med((size_t)nM * nL);
  std::vector<int> cdx((size_t)nM * nL);
  for (int iL = 0; iL < nL; iL++)
    for (int k = 0; k < nM; k++) {
      const size_t q = k + (size_t)iL * nM;
      med[q] = make_float4((float)m->mua[q], (float)m->mus[q], (float)m->g[q], (float)m->n[q]);
      cdx[q] = std::isnan(m->CDFidx[q]) ? 0 : (int)(unsigned char)m->CDFidx[q];
    }
  pl.med = ar.take<float4>(med.size());
  pl.cdfidx = ar.take<int>(cdx.size());
  pl.CDFs = ar.take<float>(std::max<int64_t>(m->nCDFelems, 1));
  if (ar.overflow) return set_error(ctx, MCB_ENOMEM, "internal: device arena too small");
  MCB_CUDA(ctx, cudaMemcpyAsync(pl.med, med.data(), med.size() * sizeof(float4), cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(pl.cdfidx, cdx.data(), cdx.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  std::vector<float> cdfs(std::max<int64_t>(m->nCDFelems, 1), 0.f);
  for (int64_t k = 0; k < m->nCDFelems; k++) cdfs[k] = (float)m->CDFs[k];
  MCB_CUDA(ctx, cudaMemcpyAsync(pl.CDFs, cdfs.data(), cdfs.size() * 4, cudaMemcpyHostToDevice, st));
  // beam
  std::vector<float> FP1{0.f}, FP2{0.f}, AI1{0.f}, AI2{0.f};
  if (!pl.useS && m->sourceType >= 4) {
    FP1 = beam_cdf(m->sourceType == 4 ? m->FPID_radial : m->FPID_X, m->sourceType == 4);
    AI1 = beam_cdf(m->sourceType == 4 ? m->AID_radial : m->AID_X, m->sourceType == 4);
    if (m->sourceType == 5) {
      FP2 = beam_cdf(m->FPID_Y, false);
      AI2 = beam_cdf(m->AID_Y, false);
    }
  }
  std::vector<float> beam;
  beam.insert(beam.end(), FP1.begin(), FP1.end());
  beam.insert(beam.end(), FP2.begin(), FP2.end());
  beam.insert(beam.end(), AI1.begin(), AI1.end());
  beam.insert(beam.end(), AI2.begin(), AI2.end());
  pl.beam = ar.take<float>(beam.size());
  if (pl.useS) pl.S = ar.take<double>((size_t)(L + 1) * nL);
  if (ar.overflow) return set_error(ctx, MCB_ENOMEM, "internal: device arena too small");
  MCB_CUDA(ctx, cudaMemcpyAsync(pl.beam, beam.data(), beam.size() * 4, cudaMemcpyHostToDevice, st));
  // distributed source CDFs (MCmatlab.c:626-629), per wavelength, in double
  pl.power.assign(nL, 0.0);
  if (pl.useS) {
    std::vector<double> S(L + 1);
    for (int iL = 0; iL < nL; iL++) {
      S[0] = 0;
      for (long long k = 1; k < L + 1; k++) S[k] = S[k - 1] + (double)m->sourceDistribution[(size_t)iL * L + k - 1];
      pl.power[iL] = S[L] * m->dx * m->dy * m->dz;
      const double tot = S[L];
      if (!(tot > 0)) return set_error(ctx, MCB_EINVAL, "sourceDistribution is zero at wavelength %d", iL);
      for (long long k = 1; k < L + 1; k++) S[k] /= tot;
      MCB_CUDA(ctx, cudaMemcpy(pl.S + (size_t)iL * (L + 1), S.data(), 8 * (L + 1), cudaMemcpyHostToDevice));
    }
  } else {
    for (int iL = 0; iL < nL; iL++) pl.power[iL] = m->spectrum[iL];
  }
  // accumulators
  const long long nx = m->nx, ny = m->ny, nz = m->nz;
  const long long res = m->LC_res, nT = (!pl.useS && m->LC_nTimeBins) ? m->LC_nTimeBins + 2 : 1;
  pl.Lim = m->useLightCollector ? res * res * nT : 0;
  pl.Lff = (long long)m->farFieldRes * m->farFieldRes;
  pl.Lx = ny * nz;
  pl.Ly = nx * nz;
  pl.Lz = nx * ny;
  pl.Lzn = m->boundaryType == 2 ? nx * ny * kKillRange * kKillRange : nx * ny;
  pl.niPer = 2 * pl.Lx + 2 * pl.Ly + pl.Lz + pl.Lzn;
  if (m->calcNFR) pl.accNFR = ar.take<double>((size_t)L * nL);
  if (pl.Lim) pl.accImg = ar.take<double>((size_t)pl.Lim * nL);
  if (pl.Lff) pl.accFF = ar.take<double>((size_t)pl.Lff * nL);
  pl.accNI = ar.take<double>((size_t)pl.niPer * nL);
  pl.ctr = ar.take<unsigned long long>(kCtr * (size_t)nL);
  if (ar.overflow) return set_error(ctx, MCB_ENOMEM, "internal: device arena too small");
  if (pl.accNFR) MCB_CUDA(ctx, cudaMemsetAsync(pl.accNFR, 0, 8 * (size_t)L * nL, st));
  if (pl.accImg) MCB_CUDA(ctx, cudaMemsetAsync(pl.accImg, 0, 8 * (size_t)pl.Lim * nL, st));
  if (pl.accFF) MCB_CUDA(ctx, cudaMemsetAsync(pl.accFF, 0, 8 * (size_t)pl.Lff * nL, st));
  MCB_CUDA(ctx, cudaMemsetAsync(pl.accNI, 0, 8 * (size_t)pl.niPer * nL, st));
  MCB_CUDA(ctx, cudaMemsetAsync(pl.ctr, 0, 8 * kCtr * (size_t)nL, st));

  // beam basis (MCmatlab.c:579-589)
  const double tb = pl.useS ? 0 : m->theta, pb = pl.useS ? 0 : m->phi, psib = pl.useS ? 0 : m->psi;
  double u[3] = {std::sin(tb) * std::cos(pb), std::sin(tb) * std::sin(pb), std::cos(tb)};
  double w[3] = {1, 0, 0}, v[3] = {0, 0, 1};
  if (u[2] != 1) unit_cross(u, v, w);
  axis_rotate_h(w, u, psib, v);
  unit_cross(u, v, w);

  // photon split over wavelengths (MCmatlab.c:635)
  pl.nPackets.assign(nL, 0);
  const bool timed = std::isnan(m->nPhotonsRequested);
  if (!timed) {
    const unsigned long long per = (unsigned long long)(m->nPhotonsRequested / nL);
    for (int iL = 0; iL < nL; iL++)
      pl.nPackets[iL] = iL == nL - 1 ? (unsigned long long)(m->nPhotonsRequested - (double)per * (nL - 1)) : per;
  }

  pl.insts.resize(nL);
  const double f = m->LC_f;
  const bool fin = std::isfinite(f);
  for (int iL = 0; iL < nL; iL++) {
    Inst &I = pl.insts[iL];
    std::memset(&I, 0, sizeof I);
    I.n[0] = m->nx; I.n[1] = m->ny; I.n[2] = m->nz;
    I.d[0] = (float)m->dx; I.d[1] = (float)m->dy; I.d[2] = (float)m->dz;
    I.invd[0] = (float)(1.0 / m->dx); I.invd[1] = (float)(1.0 / m->dy); I.invd[2] = (float)(1.0 / m->dz);
    I.bt = m->boundaryType;
    I.ffr = m->farFieldRes;
    I.M0 = pl.M0;
    I.nrm = pl.nrm;
    I.nM = nM;
    I.med = pl.med + (size_t)iL * nM;
    I.cdfidx = pl.cdfidx + (size_t)iL * nM;
    I.CDFs = pl.CDFs;
    I.beamType = pl.useS ? 0 : m->sourceType;
    I.emitterLength = pl.useS ? 0.f : (float)m->emitterLength;
    I.FP1 = pl.beam;
    I.FP2 = I.FP1 + FP1.size();
    I.AI1 = I.FP2 + FP2.size();
    I.AI2 = I.AI1 + AI1.size();
    I.LFP1 = (int)FP1.size(); I.LFP2 = (int)FP2.size(); I.LAI1 = (int)AI1.size(); I.LAI2 = (int)AI2.size();
    if (!pl.useS) {
      I.FPw1 = (float)(m->sourceType == 5 ? m->FPID_X.width : m->FPID_radial.width);
      I.AIw1 = (float)(m->sourceType == 5 ? m->AID_X.width : m->AID_radial.width);
      I.FPw2 = (float)(m->sourceType == 5 ? m->FPID_Y.width : 0.0);
      I.AIw2 = (float)(m->sourceType == 5 ? m->AID_Y.width : 0.0);
    }
    I.S = pl.useS ? pl.S + (size_t)iL * (L + 1) : nullptr;
    I.focus[0] = pl.useS ? 0.f : (float)m->xFocus;
    I.focus[1] = pl.useS ? 0.f : (float)m->yFocus;
    I.focus[2] = pl.useS ? 0.f : (float)m->zFocus;
    for (int k = 0; k < 3; k++) { I.u[k] = (float)u[k]; I.v[k] = (float)v[k]; I.w[k] = (float)w[k]; }
    I.useLC = m->useLightCollector;
    I.lcFinite = fin;
    I.LCth = (float)m->LC_theta;
    I.LCph = (float)m->LC_phi;
    I.LCf = (float)f;
    I.LCdiam = (float)m->LC_diam;
    I.LCfs = (float)(fin ? m->LC_fieldSize : m->LC_NA);
    I.LCr[0] = (float)(m->LC_x - (fin ? f * std::sin(m->LC_theta) * std::cos(m->LC_phi) : 0));
    I.LCr[1] = (float)(m->LC_y - (fin ? f * std::sin(m->LC_theta) * std::sin(m->LC_phi) : 0));
    I.LCr[2] = (float)(m->LC_z - (fin ? f * std::cos(m->LC_theta) : 0));
    I.LCres0 = m->LC_res;
    I.LCres1 = (int)nT;
    I.tStart = pl.useS ? 0.f : (float)m->LC_tStart;
    I.tEnd = pl.useS ? 0.f : (float)m->LC_tEnd;
    I.minS = inf_cast(m->DC_minScatterings); I.maxS = inf_cast(m->DC_maxScatterings);
    I.minRefr = inf_cast(m->DC_minRefractions); I.maxRefr = inf_cast(m->DC_maxRefractions);
    I.minRefl = inf_cast(m->DC_minReflections); I.maxRefl = inf_cast(m->DC_maxReflections);
    I.minI = inf_cast(m->DC_minInterfaceTransitions); I.maxI = inf_cast(m->DC_maxInterfaceTransitions);
    I.minIdx = inf_cast(m->DC_minSubmediaIdx) - 1;
    I.maxIdx = inf_cast(m->DC_maxSubmediaIdx) - 1;
    I.onlyCollected = m->DC_onlyCollected;
    I.eol = m->DC_evaluateOnlyAtEndOfLife;
    I.crit = 1;
    if (I.minS == 0 && I.maxS == 0xFFFFFFFFu && I.minRefr == 0 && I.maxRefr == 0xFFFFFFFFu && I.minRefl == 0 &&
        I.maxRefl == 0xFFFFFFFFu && I.minI == 0 && I.maxI == 0xFFFFFFFFu && !I.onlyCollected) {
      I.eol = 0;  // MCmatlab.c:418-424
      I.crit = 0;
    }
    I.NFR = pl.accNFR ? pl.accNFR + (size_t)iL * L : nullptr;
    I.image = pl.accImg ? pl.accImg + (size_t)iL * pl.Lim : nullptr;
    I.FF = pl.accFF ? pl.accFF + (size_t)iL * pl.Lff : nullptr;
    double *ni = pl.accNI + (size_t)iL * pl.niPer;
    if (m->boundaryType == 1) {
      I.NIxp = ni; I.NIxn = ni + pl.Lx; I.NIyp = ni + 2 * pl.Lx; I.NIyn = I.NIyp + pl.Ly;
      I.NIzp = I.NIyn + pl.Ly; I.NIzn = I.NIzp + pl.Lz;
    } else if (m->boundaryType == 2) {
      I.NIzn = ni;
    } else if (m->boundaryType == 3) {
      I.NIzp = ni; I.NIzn = ni + pl.Lz;
    }
    I.ctr = pl.ctr + kCtr * iL;
    I.key0 = (uint32_t)m->seed;
    I.key1 = (uint32_t)(m->seed >> 32);
    I.ctr2hi = (uint32_t)iL << 16;
    // streams are keyed by the model's seed only, so a model gives the same packets whether it
    // runs alone or inside a batch (the batch slot is not part of the counter)
    I.stream = 0;
    (void)stream;
    I.count = pl.nPackets[iL];
    I.pOff = m->packetOffset;
    I.pStride = m->packetStride ? m->packetStride : 1;
  }
  return MCB_OK;
}

// Dynamic shared memory of the gradient kernel: the block's radial-bin and box sums (FP64) and
// per-thread columns of L_m, k_m and the box partial sums (FP32).
size_t grad_smem_bytes(int nM, int nR, int threads) {
  return 8 * (size_t)(nR * (1 + 2 * nM) + 1 + 2 * nM) + 4 * (size_t)threads * (4 * nM + 1 + 2 * nM);
}

// Launch-parameter class: voxels in powers of 4 (0..15), +16 gradient, +32 batched.
int size_class(long long voxels, bool grad, bool batched) {
  int c = 0;
  while (c < 15 && (1ll << (2 * (c + 1))) <= voxels) c++;
  return c + (grad ? 16 : 0) + (batched ? 32 : 0);
}

// The autotuner's override, else the class's tuned parameters, else the autotuner's choices on the
// 100^3 cube (refill 16, scatter 8: 6.83 ms for 1e6 packets against 7.14 ms at 8, 8) and on the
// 256^3 gradient cube (12, 12).
mcb_mc_launch launch_params(const mcb_ctx *ctx, int cls, bool grad) {
  if (ctx->force.refillMin > 0) return ctx->force;
  const auto it = ctx->tuned.find(cls);
  if (it != ctx->tuned.end()) return it->second;
  return grad ? mcb_mc_launch{12, 12} : mcb_mc_launch{16, 8};
}

mcb_status launch_transport(mcb_ctx *ctx, Arena &ar, const std::vector<Inst> &insts, bool openEnded,
                            unsigned long long collectTarget, double seconds, unsigned long long *stepsOut,
                            float *msOut, int *statusOut, bool grad = false) {
  cudaStream_t st = ctx->stream;
  const int n = (int)insts.size();
  std::vector<unsigned long long> first(n + 1, 0);
  for (int k = 0; k < n; k++) first[k + 1] = first[k] + insts[k].count;
  std::vector<Inst> host = insts;
  for (int k = 0; k < n; k++) host[k].first = first[k];
  Inst *dInst = ar.take<Inst>(n);
  unsigned long long *dFirst = ar.take<unsigned long long>(n + 1);
  unsigned long long *scratch = ar.take<unsigned long long>(4);  // [0] next packet, [1] steps, [2] status, [3] clock
  if (ar.overflow) return set_error(ctx, MCB_ENOMEM, "internal: device arena too small");
  MCB_CUDA(ctx, cudaMemcpyAsync(dInst, host.data(), sizeof(Inst) * n, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(dFirst, first.data(), 8 * (n + 1), cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemsetAsync(scratch, 0, 32, st));
  KernelArgs a;
  a.insts = dInst;
  a.instFirst = dFirst;
  a.nInst = n;
  a.nextPacket = scratch;
  a.steps = scratch + 1;
  a.status = (int *)(scratch + 2);
  a.totalPackets = first[n];
  a.openEnded = openEnded ? 1 : 0;
  a.collectTarget = collectTarget;
  a.cancel = ctx->cancel_dev;
  a.deadlineNs = 0;
  {
    long long vox = 0;
    for (const Inst &I : insts) vox = std::max(vox, (long long)I.n[0] * I.n[1] * I.n[2]);
    const mcb_mc_launch L = launch_params(ctx, size_class(vox, grad, n > 1), grad);
    a.refillMin = L.refillMin;
    a.scatterMin = L.scatterMin;
  }
  const size_t dynSmem = grad ? grad_smem_bytes(insts[0].nM, insts[0].nR, 256) : 0;
  if (grad)
    MCB_CUDA(ctx, cudaFuncSetAttribute(transport_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dynSmem));
  int blocksPerSm = 0;
  MCB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocksPerSm, grad ? transport_kernel<true> : transport_kernel<false>, 256, dynSmem));
  if (blocksPerSm < 1) blocksPerSm = 1;
  const int grid = ctx->num_sms * blocksPerSm;
  if (ar.overflow) return set_error(ctx, MCB_ENOMEM, "internal: device arena too small");
  if (openEnded && seconds > 0) {
    // the deadline is taken on the device clock (%globaltimer, ns) right before the launch
    unsigned long long now = 0;
    unsigned long long *dNow = scratch + 3;
    read_globaltimer<<<1, 1, 0, st>>>(dNow);
    MCB_CUDA(ctx, cudaMemcpyAsync(&now, dNow, 8, cudaMemcpyDeviceToHost, st));
    MCB_CUDA(ctx, cudaStreamSynchronize(st));
    a.deadlineNs = now + (unsigned long long)(seconds * 1e9);
  }
  MCB_CUDA(ctx, cudaEventRecord(ctx->ev0, st));
  if (grad) transport_kernel<true><<<grid, 256, dynSmem, st>>>(a);
  else transport_kernel<false><<<grid, 256, 0, st>>>(a);
  MCB_CUDA(ctx, cudaGetLastError());
  MCB_CUDA(ctx, cudaEventRecord(ctx->ev1, st));
  unsigned long long tail[3];
  MCB_CUDA(ctx, cudaMemcpyAsync(tail, scratch, 24, cudaMemcpyDeviceToHost, st));
  MCB_CUDA(ctx, cudaStreamSynchronize(st));
  float ms = 0.f;
  MCB_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  *stepsOut += tail[1];
  *msOut += ms;
  *statusOut |= (int)tail[2];
  return MCB_OK;
}

mcb_status finish_plan(mcb_ctx *ctx, Arena &ar, ModelPlan &pl, double *nPhCum, double *nColCum) {
  cudaStream_t st = ctx->stream;
  const mcb_mc_model *m = pl.m;
  mcb_mc_result *r = pl.r;
  const int nL = pl.nL;
  const long long L = pl.L;
  const int grid = ctx->num_sms * 8;
  std::vector<unsigned long long> ctr(kCtr * (size_t)nL);
  r->freeStepCuts = r->freeStepCutWeight = 0.0;
  MCB_CUDA(ctx, cudaMemcpyAsync(ctr.data(), pl.ctr, 8 * ctr.size(), cudaMemcpyDeviceToHost, st));
  if (r->tallies) {
    // the FP64 tallies as accumulated (the normalisation below reads them, it does not change them)
    const TallyLayout t = tally_layout(m);
    if (pl.accNFR) MCB_CUDA(ctx, cudaMemcpyAsync(r->tallies + t.nfr, pl.accNFR, 8 * (size_t)L * nL, cudaMemcpyDeviceToHost, st));
    if (pl.accImg) MCB_CUDA(ctx, cudaMemcpyAsync(r->tallies + t.img, pl.accImg, 8 * (size_t)pl.Lim * nL, cudaMemcpyDeviceToHost, st));
    if (pl.accFF) MCB_CUDA(ctx, cudaMemcpyAsync(r->tallies + t.ff, pl.accFF, 8 * (size_t)pl.Lff * nL, cudaMemcpyDeviceToHost, st));
    MCB_CUDA(ctx, cudaMemcpyAsync(r->tallies + t.ni, pl.accNI, 8 * (size_t)pl.niPer * nL, cudaMemcpyDeviceToHost, st));
  }
  MCB_CUDA(ctx, cudaStreamSynchronize(st));
  if (r->tallies) {
    const TallyLayout t = tally_layout(m);
    for (int iL = 0; iL < nL; iL++) {
      r->tallies[t.cnt + 2 * iL] = (double)ctr[kCtr * iL];
      r->tallies[t.cnt + 2 * iL + 1] = (double)ctr[kCtr * iL + 1];
    }
  }
  const double V = m->dx * m->dy * m->dz;
  float *stage = ar.take<float>(std::max<long long>(std::max<long long>(L, pl.Lim), std::max<long long>(pl.Lff, pl.niPer)));
  if (ar.overflow) return set_error(ctx, MCB_ENOMEM, "internal: device arena too small");
  for (int iL = 0; iL < nL; iL++) {
    const double nPh = (double)ctr[kCtr * iL], nCol = (double)ctr[kCtr * iL + 1];
    *nPhCum += nPh;
    *nColCum += nCol;
    double cutW;
    std::memcpy(&cutW, &ctr[kCtr * iL + 5], 8);
    r->freeStepCuts += (double)ctr[kCtr * iL + 4];
    r->freeStepCutWeight += cutW;
    // normfactor (MCmatlablib.c:1193-1198)
    double nf = nPh / pl.power[iL];
    if (pl.useS) nf /= pl.power[iL];
    else if (m->sourceType == 2 && (m->boundaryType == 0 || m->boundaryType == 2)) nf /= kKillRange * kKillRange;
    if (nPh == 0) nf = 1.0;  // nothing launched: tallies are zero
    if (pl.accNFR && r->NFR) {
      normalize_nfr_kernel<<<grid, 256, 0, st>>>(pl.accNFR + (size_t)iL * L, pl.M0, pl.med + (size_t)iL * m->nM, V * nf, stage, L);
      MCB_CUDA(ctx, cudaMemcpyAsync(r->NFR + (size_t)iL * L, stage, 4 * L, cudaMemcpyDeviceToHost, st));
      MCB_CUDA(ctx, cudaStreamSynchronize(st));
    }
    if (pl.accFF && r->farField) {
      scale_kernel<<<grid, 256, 0, st>>>(pl.accFF + (size_t)iL * pl.Lff, 1.0 / nf, stage, pl.Lff);
      MCB_CUDA(ctx, cudaMemcpyAsync(r->farField + (size_t)iL * pl.Lff, stage, 4 * pl.Lff, cudaMemcpyDeviceToHost, st));
      MCB_CUDA(ctx, cudaStreamSynchronize(st));
    }
    if (pl.accImg && r->image) {
      const long long Lp = (long long)m->LC_res * m->LC_res;
      const double fs = std::isfinite(m->LC_f) ? m->LC_fieldSize : m->LC_NA;
      const double inv = Lp > 1 ? 1.0 / (fs * fs / Lp * nf) : 1.0 / nf;
      scale_kernel<<<grid, 256, 0, st>>>(pl.accImg + (size_t)iL * pl.Lim, inv, stage, pl.Lim);
      MCB_CUDA(ctx, cudaMemcpyAsync(r->image + (size_t)iL * pl.Lim, stage, 4 * pl.Lim, cudaMemcpyDeviceToHost, st));
      MCB_CUDA(ctx, cudaStreamSynchronize(st));
    }
    const double *ni = pl.accNI + (size_t)iL * pl.niPer;
    auto face = [&](const double *src, float *dst, long long cnt, double area) -> mcb_status {
      if (!dst) return MCB_OK;
      scale_kernel<<<grid, 256, 0, st>>>(src, 1.0 / (area * nf), stage, cnt);
      MCB_CUDA(ctx, cudaMemcpyAsync(dst + (size_t)iL * cnt, stage, 4 * cnt, cudaMemcpyDeviceToHost, st));
      MCB_CUDA(ctx, cudaStreamSynchronize(st));
      return MCB_OK;
    };
    if (m->boundaryType == 1) {
      MCB_TRY(face(ni, r->NI_xpos, pl.Lx, m->dy * m->dz));
      MCB_TRY(face(ni + pl.Lx, r->NI_xneg, pl.Lx, m->dy * m->dz));
      MCB_TRY(face(ni + 2 * pl.Lx, r->NI_ypos, pl.Ly, m->dx * m->dz));
      MCB_TRY(face(ni + 2 * pl.Lx + pl.Ly, r->NI_yneg, pl.Ly, m->dx * m->dz));
      MCB_TRY(face(ni + 2 * pl.Lx + 2 * pl.Ly, r->NI_zpos, pl.Lz, m->dx * m->dy));
      MCB_TRY(face(ni + 2 * pl.Lx + 2 * pl.Ly + pl.Lz, r->NI_zneg, pl.Lz, m->dx * m->dy));
    } else if (m->boundaryType == 2) {
      MCB_TRY(face(ni, r->NI_zneg, pl.Lzn, m->dx * m->dy));
    } else if (m->boundaryType == 3) {
      MCB_TRY(face(ni, r->NI_zpos, pl.Lz, m->dx * m->dy));
      MCB_TRY(face(ni + pl.Lz, r->NI_zneg, pl.Lz, m->dx * m->dy));
    }
  }
  return MCB_OK;
}

}  // namespace

static mcb_status run_models(mcb_ctx *ctx, int n, const mcb_mc_model *const *models, mcb_mc_result *const *results,
                             const mcb_mc_objectives *obj = nullptr, mcb_mc_grad_result *grad = nullptr) {
  using namespace mcb;
  for (int k = 0; k < n; k++) {
    MCB_TRY(validate(ctx, models[k]));
    if (!results[k]) return set_error(ctx, MCB_EINVAL, "result %d is NULL", k);
  }
  const bool gradRun = obj != nullptr;
  if (gradRun) {
    const mcb_mc_model *m = models[0];
    if (n != 1) return set_error(ctx, MCB_EINVAL, "gradient runs take one model");
    if (m->nL != 1) return set_error(ctx, MCB_EINVAL, "gradient runs need a single wavelength");
    if (m->nM > kGradMedia) return set_error(ctx, MCB_EINVAL, "gradient runs support at most %d media", kGradMedia);
    if (std::isnan(m->nPhotonsRequested) || m->requestCollectedPhotons)
      return set_error(ctx, MCB_EINVAL, "gradient runs need a fixed launched-packet count");
    if (!(m->DC_minScatterings == 0 && std::isinf(m->DC_maxScatterings) && m->DC_minRefractions == 0 &&
          std::isinf(m->DC_maxRefractions) && m->DC_minReflections == 0 && std::isinf(m->DC_maxReflections) &&
          m->DC_minInterfaceTransitions == 0 && std::isinf(m->DC_maxInterfaceTransitions) && !m->DC_onlyCollected))
      return set_error(ctx, MCB_EINVAL, "gradient runs need default deposition criteria");
    if (obj->nRadialBins < 0 || obj->nRadialBins > 64) return set_error(ctx, MCB_EINVAL, "nRadialBins must be 0..64");
    if (obj->nRadialBins > 0 && !(obj->radialBinWidth > 0)) return set_error(ctx, MCB_EINVAL, "radialBinWidth must be > 0");
    if (!grad) return set_error(ctx, MCB_EINVAL, "grad result is NULL");
  }
  MCB_CUDA(ctx, cudaSetDevice(ctx->device));
  size_t bytes = 1 << 20;
  for (int k = 0; k < n; k++) bytes += plan_bytes(models[k]);
  bytes += (size_t)(sizeof(Inst) + 16) * 64 * (n + 1);
  for (int k = 0; k < n; k++)
    if (models[k]->nExamplePaths > 0 && results[k]->examplePaths) bytes += 32 * (size_t)results[k]->examplePathsCap + 4096;
  void *base = nullptr;
  MCB_TRY(pool_get(ctx, SLOT_MC_INST, bytes, &base));
  Arena ar{(char *)base, bytes, 0};
  std::vector<ModelPlan> plans(n);
  for (int k = 0; k < n; k++) {
    plans[k].m = models[k];
    plans[k].r = results[k];
    MCB_TRY(build_plan(ctx, ar, plans[k], (uint32_t)k));
  }
  double *gR = nullptr, *gF = nullptr;
  int nGR = 0, nGM = 0, box[6] = {0, 0, 0, 0, 0, 0};
  if (gradRun) {
    const mcb_mc_model *m = models[0];
    nGM = m->nM;
    nGR = obj->nRadialBins;
    const int nn[3] = {m->nx, m->ny, m->nz};
    for (int q = 0; q < 6; q++) box[q] = std::min(std::max(obj->box[q], 0), nn[q / 2]);
    gR = ar.take<double>(std::max(1, nGR * (1 + 2 * nGM)));
    gF = ar.take<double>(1 + 2 * nGM);
    if (ar.overflow) return set_error(ctx, MCB_ENOMEM, "internal: device arena too small");
    MCB_CUDA(ctx, cudaMemsetAsync(gR, 0, 8 * (size_t)std::max(1, nGR * (1 + 2 * nGM)), ctx->stream));
    MCB_CUDA(ctx, cudaMemsetAsync(gF, 0, 8 * (size_t)(1 + 2 * nGM), ctx->stream));
    Inst &I = plans[0].insts[0];
    I.nR = nGR;
    I.rbin = (float)obj->radialBinWidth;
    for (int q = 0; q < 6; q++) I.box[q] = box[q];
    I.gR = gR;
    I.gF = gF;
  }
  const bool single = n == 1;
  const mcb_mc_model *m0 = models[0];
  const bool timed = single && std::isnan(m0->nPhotonsRequested);
  const bool collected = single && !timed && m0->requestCollectedPhotons;
  unsigned long long steps = 0;
  float ms = 0.f;
  int status = 0;
  if (!single) {
    for (int k = 0; k < n; k++)
      if (std::isnan(models[k]->nPhotonsRequested) || models[k]->requestCollectedPhotons)
        return set_error(ctx, MCB_EINVAL, "batched runs need fixed launched-packet counts");
  }
  if (timed || collected) {
    // open-ended modes run wavelength by wavelength (MCmatlab.c:617-636)
    ModelPlan &pl = plans[0];
    double colSoFar = 0;
    for (int iL = 0; iL < pl.nL; iL++) {
      std::vector<Inst> one{pl.insts[iL]};
      one[0].count = ~0ull >> 1;
      unsigned long long target = 0;
      if (collected) {
        const unsigned long long per = (unsigned long long)(m0->nPhotonsRequested / pl.nL);
        target = iL == pl.nL - 1 ? (unsigned long long)(m0->nPhotonsRequested - colSoFar) : per;
      }
      const double secs = timed ? m0->simulationTimeRequested * 60.0 / pl.nL : 0.0;
      const size_t mark = ar.used;
      MCB_TRY(launch_transport(ctx, ar, one, true, target, secs, &steps, &ms, &status));
      ar.used = mark;
      unsigned long long c[4];
      MCB_CUDA(ctx, cudaMemcpy(c, pl.ctr + kCtr * iL, 32, cudaMemcpyDeviceToHost));
      colSoFar += (double)c[1];
      if (status & 1) break;
    }
  } else {
    std::vector<Inst> all;
    for (auto &pl : plans) all.insert(all.end(), pl.insts.begin(), pl.insts.end());
    const size_t mark = ar.used;
    MCB_TRY(launch_transport(ctx, ar, all, false, 0, 0.0, &steps, &ms, &status, gradRun));
    ar.used = mark;
  }
  for (int k = 0; k < n; k++) {
    double nPh = 0, nCol = 0;
    const size_t mark = ar.used;
    MCB_TRY(finish_plan(ctx, ar, plans[k], &nPh, &nCol));
    ar.used = mark;
    mcb_mc_result *r = results[k];
    r->nPhotons = nPh;
    r->nPhotonsCollected = nCol;
    r->nThreads = (double)ctx->num_sms;  // one persistent grid; reported per SM like the MEX reports threads
    r->simulationTime = ms / 60000.0;
    r->propagationSteps = single ? steps : 0;
    r->kernelMs = ms;
    ctx->lastKernelMs = ms;
    r->examplePathsN = 0;
    const mcb_mc_model *m = models[k];
    if (m->nExamplePaths > 0 && r->examplePaths && r->examplePathsCap > 0) {
      const size_t mark2 = ar.used;
      double *dPaths = ar.take<double>(4 * (size_t)r->examplePathsCap);
      long long *dN = ar.take<long long>(1);
      Inst *dI = ar.take<Inst>(1);
      if (ar.overflow) {
        // grow the arena for the path buffer on the next call; report no paths now
        r->examplePathsN = 0;
        ar.used = mark2;
        ar.overflow = false;
        continue;
      }
      Inst I0 = plans[k].insts[0];
      I0.first = 0;
      MCB_CUDA(ctx, cudaMemcpyAsync(dI, &I0, sizeof(Inst), cudaMemcpyHostToDevice, ctx->stream));
      const unsigned long long maxP = plans[k].nPackets[0] ? plans[k].nPackets[0] : (unsigned long long)nPh;
      example_paths_kernel<<<1, 32, 0, ctx->stream>>>(dI, m->nExamplePaths, maxP, dPaths, r->examplePathsCap, dN);
      MCB_CUDA(ctx, cudaGetLastError());
      long long nOut = 0;
      MCB_CUDA(ctx, cudaMemcpyAsync(&nOut, dN, 8, cudaMemcpyDeviceToHost, ctx->stream));
      MCB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      if (nOut > 0)
        MCB_CUDA(ctx, cudaMemcpy(r->examplePaths, dPaths, 32 * (size_t)nOut, cudaMemcpyDeviceToHost));
      r->examplePathsN = nOut;
      ar.used = mark2;
    }
  }
  if (gradRun) {
    // normalisation as for NI (per unit area) and NFR (per voxel volume), MCmatlablib.c:1193-1243
    const mcb_mc_model *m = models[0];
    std::vector<double> hR(std::max(1, nGR * (1 + 2 * nGM))), hF(1 + 2 * nGM);
    MCB_CUDA(ctx, cudaMemcpy(hR.data(), gR, 8 * hR.size(), cudaMemcpyDeviceToHost));
    MCB_CUDA(ctx, cudaMemcpy(hF.data(), gF, 8 * hF.size(), cudaMemcpyDeviceToHost));
    const double power = plans[0].power[0];
    double nf = results[0]->nPhotons / power;
    if (plans[0].useS) nf /= power;
    else if (m->sourceType == 2 && (m->boundaryType == 0 || m->boundaryType == 2)) nf /= kKillRange * kKillRange;
    if (results[0]->nPhotons == 0) nf = 1.0;
    const double w = obj->radialBinWidth;
    for (int b = 0; b < nGR; b++) {
      const double area = 3.14159265358979323846 * w * w * ((b + 1.0) * (b + 1.0) - (double)b * b);
      const double sc = 1.0 / (area * nf);
      const double *row = hR.data() + b * (1 + 2 * nGM);
      if (grad->R) grad->R[b] = row[0] * sc;
      for (int q = 0; q < nGM; q++) {
        if (grad->dR_dmua) grad->dR_dmua[b + nGR * q] = row[1 + q] * sc;
        if (grad->dR_dmus) grad->dR_dmus[b + nGR * q] = row[1 + nGM + q] * sc;
      }
    }
    const double nbox = (double)std::max(0, box[1] - box[0]) * std::max(0, box[3] - box[2]) * std::max(0, box[5] - box[4]);
    const double sF = nbox > 0 ? 1.0 / (m->dx * m->dy * m->dz * nf * nbox) : 0.0;
    grad->F = hF[0] * sF;
    for (int q = 0; q < nGM; q++) {
      if (grad->dF_dmua) grad->dF_dmua[q] = hF[1 + q] * sF;
      if (grad->dF_dmus) grad->dF_dmus[q] = hF[1 + nGM + q] * sF;
    }
  }
  if (status & 1) return set_error(ctx, MCB_ECANCELLED, "run cancelled");
  if (status & 2) {
    bool any = false;
    for (int k = 0; k < n; k++) any |= results[k]->nPhotons > 0;
    if (!any) return set_error(ctx, MCB_ELAUNCH, "all photons launch outside the allowed region; check the model definition");
  }
  return MCB_OK;
}

extern "C" mcb_status mcb_mc_run(mcb_ctx *ctx, const mcb_mc_model *model, mcb_mc_result *result) {
  if (!ctx) return MCB_EINVAL;
  const mcb_mc_model *ms[1] = {model};
  mcb_mc_result *rs[1] = {result};
  return run_models(ctx, 1, ms, rs);
}

extern "C" mcb_status mcb_mc_grad(mcb_ctx *ctx, const mcb_mc_model *model, const mcb_mc_objectives *objectives,
                                  mcb_mc_result *result, mcb_mc_grad_result *grad) {
  if (!ctx) return MCB_EINVAL;
  if (!objectives) return mcb::set_error(ctx, MCB_EINVAL, "objectives is NULL");
  const mcb_mc_model *ms[1] = {model};
  mcb_mc_result *rs[1] = {result};
  return run_models(ctx, 1, ms, rs, objectives, grad);
}

extern "C" int32_t mcb_mc_size_class(const mcb_mc_model *model, int32_t gradient, int32_t batched) {
  if (!model) return -1;
  return size_class((long long)model->nx * model->ny * model->nz, gradient != 0, batched != 0);
}

namespace mcb {
// Tuning file: one line per (GPU name, class): "<name>\t<class>\t<refillMin>\t<scatterMin>".
void tune_file_load(mcb_ctx *ctx) {
  const char *path = std::getenv("MCB_TUNE_FILE");
  if (!path || !*path) return;
  FILE *f = std::fopen(path, "r");
  if (!f) return;
  char line[512];
  while (std::fgets(line, sizeof line, f)) {
    char *tab = std::strchr(line, '\t');
    if (!tab) continue;
    *tab = 0;
    int cls = 0, r = 0, s = 0;
    if (ctx->gpuName == line && std::sscanf(tab + 1, "%d %d %d", &cls, &r, &s) == 3 && r >= 1 && r <= 32 && s >= 1 &&
        s <= 32)
      ctx->tuned[cls] = mcb_mc_launch{r, s};
  }
  std::fclose(f);
}

void tune_file_store(const mcb_ctx *ctx, int cls, const mcb_mc_launch &L) {
  const char *path = std::getenv("MCB_TUNE_FILE");
  if (!path || !*path) return;
  std::vector<std::string> keep;
  if (FILE *f = std::fopen(path, "r")) {
    char line[512];
    char key[320];
    std::snprintf(key, sizeof key, "%s\t%d\t", ctx->gpuName.c_str(), cls);
    while (std::fgets(line, sizeof line, f))
      if (std::strncmp(line, key, std::strlen(key)) != 0) keep.push_back(line);
    std::fclose(f);
  }
  if (FILE *f = std::fopen(path, "w")) {
    for (const std::string &l : keep) std::fputs(l.c_str(), f);
    std::fprintf(f, "%s\t%d\t%d\t%d\n", ctx->gpuName.c_str(), cls, L.refillMin, L.scatterMin);
    std::fclose(f);
  }
}
}  // namespace mcb

extern "C" mcb_status mcb_mc_autotune(mcb_ctx *ctx, const mcb_mc_model *model, double calibrationPackets, int32_t gradient,
                                      mcb_mc_launch *chosen, double *table) {
  using namespace mcb;
  if (!ctx) return MCB_EINVAL;
  MCB_TRY(validate(ctx, model));
  if (!(calibrationPackets >= 1)) return set_error(ctx, MCB_EINVAL, "calibrationPackets must be >= 1");
  mcb_mc_model m = *model;
  m.nPhotonsRequested = calibrationPackets;
  m.requestCollectedPhotons = 0;
  m.nExamplePaths = 0;
  mcb_mc_result r;
  std::memset(&r, 0, sizeof r);
  mcb_mc_objectives obj;
  std::memset(&obj, 0, sizeof obj);
  mcb_mc_grad_result g;
  std::memset(&g, 0, sizeof g);
  const int cand[4] = {4, 8, 12, 16};
  mcb_mc_launch best = launch_params(ctx, -1, gradient != 0);
  double bestMs = 1e300;
  int row = 0;
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++) {
      ctx->force = mcb_mc_launch{cand[a], cand[b]};
      double ms = 1e300;
      for (int rep = 0; rep < 2; rep++) {
        const mcb_mc_model *ms1[1] = {&m};
        mcb_mc_result *rs1[1] = {&r};
        const mcb_status st = gradient ? run_models(ctx, 1, ms1, rs1, &obj, &g) : run_models(ctx, 1, ms1, rs1);
        if (st != MCB_OK) {
          ctx->force = mcb_mc_launch{0, 0};
          return st;
        }
        ms = std::min(ms, r.kernelMs);
      }
      if (table) {
        table[3 * row] = cand[a];
        table[3 * row + 1] = cand[b];
        table[3 * row + 2] = ms;
      }
      row++;
      if (ms < bestMs) {
        bestMs = ms;
        best = ctx->force;
      }
    }
  ctx->force = mcb_mc_launch{0, 0};
  const int cls = size_class((long long)m.nx * m.ny * m.nz, gradient != 0, false);
  ctx->tuned[cls] = best;
  tune_file_store(ctx, cls, best);
  if (chosen) *chosen = best;
  return MCB_OK;
}

extern "C" int64_t mcb_mc_tally_count(const mcb_mc_model *model) {
  if (!model || model->nx < 1 || model->ny < 1 || model->nz < 1 || model->nL < 1) return 0;
  return tally_layout(model).total;
}

extern "C" mcb_status mcb_mc_normalize(mcb_ctx *ctx, const mcb_mc_model *model, const double *tallies,
                                       mcb_mc_result *result) {
  using namespace mcb;
  if (!ctx) return MCB_EINVAL;
  MCB_TRY(validate(ctx, model));
  if (!tallies || !result) return set_error(ctx, MCB_EINVAL, "tallies or result is NULL");
  MCB_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t bytes = (1 << 20) + plan_bytes(model) + (size_t)(sizeof(Inst) + 16) * 64;
  void *base = nullptr;
  MCB_TRY(pool_get(ctx, SLOT_MC_INST, bytes, &base));
  Arena ar{(char *)base, bytes, 0};
  ModelPlan pl;
  pl.m = model;
  pl.r = result;
  MCB_TRY(build_plan(ctx, ar, pl, 0));
  const TallyLayout t = tally_layout(model);
  const int nL = model->nL;
  cudaStream_t st = ctx->stream;
  if (pl.accNFR) MCB_CUDA(ctx, cudaMemcpyAsync(pl.accNFR, tallies + t.nfr, 8 * (size_t)pl.L * nL, cudaMemcpyHostToDevice, st));
  if (pl.accImg) MCB_CUDA(ctx, cudaMemcpyAsync(pl.accImg, tallies + t.img, 8 * (size_t)pl.Lim * nL, cudaMemcpyHostToDevice, st));
  if (pl.accFF) MCB_CUDA(ctx, cudaMemcpyAsync(pl.accFF, tallies + t.ff, 8 * (size_t)pl.Lff * nL, cudaMemcpyHostToDevice, st));
  MCB_CUDA(ctx, cudaMemcpyAsync(pl.accNI, tallies + t.ni, 8 * (size_t)pl.niPer * nL, cudaMemcpyHostToDevice, st));
  std::vector<unsigned long long> c(kCtr * (size_t)nL, 0ull);
  for (int iL = 0; iL < nL; iL++) {
    const double a = tallies[t.cnt + 2 * iL], b = tallies[t.cnt + 2 * iL + 1];
    if (!(a >= 0 && b >= 0 && a < 1.8e19 && b < 1.8e19)) return set_error(ctx, MCB_EINVAL, "packet counts out of range");
    c[kCtr * iL] = (unsigned long long)a;
    c[kCtr * iL + 1] = (unsigned long long)b;
  }
  MCB_CUDA(ctx, cudaMemcpyAsync(pl.ctr, c.data(), 8 * c.size(), cudaMemcpyHostToDevice, st));
  double *keep = result->tallies;
  result->tallies = nullptr;
  double nPh = 0, nCol = 0;
  const mcb_status rc = finish_plan(ctx, ar, pl, &nPh, &nCol);
  result->tallies = keep;
  MCB_TRY(rc);
  result->nPhotons = nPh;
  result->nPhotonsCollected = nCol;
  result->nThreads = 0;
  result->simulationTime = 0;
  result->propagationSteps = 0;
  result->kernelMs = 0;
  result->examplePathsN = 0;
  return MCB_OK;
}

extern "C" mcb_status mcb_mc_run_batch(mcb_ctx *ctx, int32_t n, const mcb_mc_model *const *models,
                                       mcb_mc_result *const *results) {
  if (!ctx) return MCB_EINVAL;
  if (n < 1 || !models || !results) return mcb::set_error(ctx, MCB_EINVAL, "empty batch");
  return run_models(ctx, n, models, results);
}
