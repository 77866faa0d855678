/*
 * mc_oracle.c — FP64 CPU restatement of the reference photon-packet transport.
 *
 * TEST INFRASTRUCTURE ONLY (the checker). Restates the reference MC MEX
 * (+MCmatlab/src/MCmatlab.c and +MCmatlab/src/MCmatlablib.c) in double precision,
 * with one change: the random numbers come from the counter-based Philox stream
 * described in philox.h (one stream per packet) instead of dSFMT seeded from the
 * clock. Everything else follows the reference function by function:
 *
 *   marshalling, beam CDFs, beam basis   MCmatlab.c:317-616
 *   wavelength loop, photon split        MCmatlab.c:617-636, :752
 *   packet loop                          MCmatlab.c:245-265 (threadInitAndLoop)
 *   launchPhoton (6 source types, S)     MCmatlablib.c:519-732
 *   propagatePhoton                      MCmatlablib.c:1019-1119
 *   getInterpolatedNormal / getNormal    MCmatlablib.c:909-1014
 *   checkEscape                          MCmatlablib.c:821-889
 *   formImage / formFarField / edges     MCmatlablib.c:737-816
 *   getNewj / getNewVoxelProperties      MCmatlablib.c:281-285, :894-904
 *   checkRoulette / scatterPhoton        MCmatlablib.c:1124-1184
 *   depositionCriteriaMet                MCmatlablib.c:126-136
 *   normalizeDepositionAndResetO         MCmatlablib.c:1186-1250
 *   Lambert W(-1) for the LG01 beam      written from Corless et al. (1996), eq. 5.9 Halley
 *                                        iteration, not from the reference's GSL-derived lambert.c
 *
 * Packets run in parallel with OpenMP; each packet's random stream depends only on its
 * id, so results do not depend on the thread count apart from FP64 summation order.
 */
#include <math.h>
#include <float.h>
#include <limits.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/mcb200.h"
#include "philox.h"

#define O_C 29979245800.0
#define O_THRESHOLD 0.01
#define O_CHANCE 0.1
#define O_KILLRANGE 5
#define O_CDFSIZE 201
#define O_PI 3.14159265358979323846

typedef struct {
  long n[3];
  double d[3];
  int bt; /* boundaryType */
  long ffr;
  const uint8_t *M0; /* 0-based */
  const float *normals;
  int nM;
  double *mua, *mus, *g, *RI;
  int *cdfidx;
  const double *CDFs;
  /* source */
  int beamType;
  double emitterLength;
  double *FP1, *FP2, *AI1, *AI2;
  long LFP1, LFP2, LAI1, LAI2;
  double FPw1, FPw2, AIw1, AIw2;
  double *S;
  double power;
  double focus[3], u[3], v[3], w[3];
  /* light collector */
  int useLC;
  double LCr[3], LCth, LCph, LCf, LCdiam, LCfs;
  long LCres[2];
  double tStart, tEnd;
  /* deposition criteria */
  unsigned long minS, maxS, minRefr, maxRefr, minRefl, maxRefl, minI, maxI, minIdx, maxIdx;
  bool onlyCollected, eol;
  /* accumulators */
  double *NFR, *image, *FF, *NIxp, *NIxn, *NIyp, *NIyn, *NIzp, *NIzn;
  unsigned long long nPhotons, nPhotonsCollected;
  double cuts, cutW; /* packets ended by the free-step limit and their weight (all wavelengths) */
  /* example-path recording (one thread, packets 0, 1, 2, ... of the first wavelength): columns of
   * (x, y, z, weight), NaN-separated (MCmatlablib.c:465-514); pn > pcap marks an overflow */
  double *pdata;
  long pcap, pn;
  int pstarted;
  unsigned long long steps;
  uint32_t key[2];
  uint32_t stream;
  uint32_t iL;
  int aborting;
  /* perturbation MC (gradient runs) */
  int grad, nGM, nR;
  /* sharding: packet k of this run uses the stream of packet pOff + k * pStride */
  uint64_t pOff, pStride;
  double rbin;
  int box[6];
  double *gR, *gF;
} orc_mc;

typedef struct {
  double i[3], u[3], D[3];
  long j;
  double mua, mus, g, RI;
  int CDFidx;
  double stepLeft, weight, time;
  bool insideVolume, alive, sameVoxel;
  uint64_t pid;
  uint32_t draw;
  uint32_t buf[4];
  uint32_t bufblock;
  long recSize, recN;
  long *jrec;
  double *wrec;
  unsigned long scat, refr, refl, itr;
  int kec; /* 0 killed, 1 escaped, 2 collected */
  unsigned long long steps;
  unsigned long psteps; /* sub-steps since launch or the last scattering event */
  double L[10], k[10]; /* path length and scattering count per medium (gradient runs) */
  int inbox;
} orc_photon;

static double rnd(const orc_mc *R, orc_photon *P) {
  uint32_t blk = P->draw >> 2;
  if (P->draw == 0 || blk != P->bufblock) {
    uint32_t ctr[4] = {blk, (uint32_t)P->pid, (uint32_t)((P->pid >> 32) & 0xFFFFu) | (R->iL << 16), R->stream};
    orc_philox4x32_10(ctr, R->key, P->buf);
    P->bufblock = blk;
  }
  double u = orc_u01(P->buf[P->draw & 3]);
  P->draw++;
  return u;
}

static inline double sqr(double x) { return x * x; }

static void unitcross(const double *a, const double *b, double *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
  double nrm = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
  for (int k = 0; k < 3; k++) c[k] /= nrm;
}

static void rotate(const double *r, const double *u, double th, double *o) {
  double st = sin(th), ct = cos(th);
  o[0] = (u[0] * u[0] * (1 - ct) + ct) * r[0] + (u[0] * u[1] * (1 - ct) - u[2] * st) * r[1] + (u[0] * u[2] * (1 - ct) + u[1] * st) * r[2];
  o[1] = (u[1] * u[0] * (1 - ct) + u[2] * st) * r[0] + (u[1] * u[1] * (1 - ct) + ct) * r[1] + (u[1] * u[2] * (1 - ct) - u[0] * st) * r[2];
  o[2] = (u[2] * u[0] * (1 - ct) - u[1] * st) * r[0] + (u[2] * u[1] * (1 - ct) + u[0] * st) * r[1] + (u[2] * u[2] * (1 - ct) + ct) * r[2];
}

static void toLC(const double *r, double th, double ph, double *o) {
  o[0] = sin(ph) * r[0] - cos(ph) * r[1];
  o[1] = cos(th) * cos(ph) * r[0] + cos(th) * sin(ph) * r[1] - sin(th) * r[2];
  o[2] = sin(th) * cos(ph) * r[0] + sin(th) * sin(ph) * r[1] + cos(th) * r[2];
}

/* index j in [0, N-1] with D[j] < r <= D[j+1] for a nondecreasing D[0..N] (MCmatlablib.c:263-276) */
static long bsearch_cdf(double r, long N, const double *D) {
  long lo = 0, hi = N; /* find first k in [1, N] with D[k] >= r */
  while (lo + 1 < hi) {
    long mid = (lo + hi) / 2;
    if (D[mid] >= r) hi = mid; else lo = mid;
  }
  return lo;
}

/* Lambert W, branch -1, for x in [-1/e, 0): Corless et al. (1996) initial guesses + Halley iteration (eq. 5.9) */
static double lambert_wm1(double x) {
  if (x >= 0.0) return 0.0;
  const double em1 = exp(-1.0);
  double w;
  if (x < -em1) return -1.0;
  if (x < -0.25) {
    double p = -sqrt(2.0 * (exp(1.0) * x + 1.0));
    w = -1.0 + p - p * p / 3.0 + 11.0 / 72.0 * p * p * p;
  } else {
    double L1 = log(-x), L2 = log(-L1);
    w = L1 - L2 + L2 / L1;
  }
  for (int it = 0; it < 40; it++) {
    double ew = exp(w);
    double f = w * ew - x;
    double wp1 = w + 1.0;
    if (wp1 == 0.0) break;
    double dw = f / (ew * wp1 - (w + 2.0) * f / (2.0 * wp1));
    w -= dw;
    if (fabs(dw) <= 4.0 * DBL_EPSILON * fmax(1.0, fabs(w))) break;
  }
  return w;
}

static bool criteria(const orc_mc *R, const orc_photon *P) {
  bool killed = !P->alive && P->kec == 0;
  return P->scat >= R->minS && (killed ? ULONG_MAX : P->scat) <= R->maxS &&
         P->refr >= R->minRefr && (killed ? ULONG_MAX : P->refr) <= R->maxRefr &&
         P->refl >= R->minRefl && (killed ? ULONG_MAX : P->refl) <= R->maxRefl &&
         P->itr >= R->minI && (killed ? ULONG_MAX : P->itr) <= R->maxI &&
         (R->onlyCollected ? P->kec == 2 : true);
}

static inline void add(double *p, double v) {
#pragma omp atomic
  *p += v;
}

static long newj(const orc_mc *R, const double *i) {
  long c[3];
  for (int k = 0; k < 3; k++) c[k] = i[k] < 0 ? 0 : (i[k] >= R->n[k] ? R->n[k] - 1 : (long)floor(i[k]));
  return c[2] * R->n[0] * R->n[1] + c[1] * R->n[0] + c[0];
}

static int box_of(const orc_mc *R, const double *i) {
  long c[3];
  for (int k = 0; k < 3; k++) c[k] = i[k] < 0 ? 0 : (i[k] >= R->n[k] ? R->n[k] - 1 : (long)floor(i[k]));
  return c[0] >= R->box[0] && c[0] < R->box[1] && c[1] >= R->box[2] && c[1] < R->box[3] && c[2] >= R->box[4] &&
         c[2] < R->box[5];
}

static void voxel_props(const orc_mc *R, orc_photon *P) {
  P->j = newj(R, P->i);
  if (R->grad) P->inbox = box_of(R, P->i);
  int m = R->M0[P->j];
  P->mua = R->mua[m];
  P->mus = R->mus[m];
  P->g = R->g[m];
  P->CDFidx = R->cdfidx[m];
}

static bool inside(const orc_mc *R, const double *i) {
  return i[0] < R->n[0] && i[0] >= 0 && i[1] < R->n[1] && i[1] >= 0 && i[2] < R->n[2] && i[2] >= 0;
}

static void set_D(const orc_mc *R, orc_photon *P) {
  for (int k = 0; k < 3; k++)
    P->D[k] = P->u[k] != 0 ? (floor(P->i[k]) + (P->u[k] > 0) - P->i[k]) * R->d[k] / P->u[k] : INFINITY;
}

static double start_time_focus(const orc_mc *R, const orc_photon *P, const double *tgt) {
  return -P->RI / O_C * sqrt(sqr((P->i[0] - R->n[0] / 2.0) * R->d[0] - tgt[0]) + sqr((P->i[1] - R->n[1] / 2.0) * R->d[1] - tgt[1]) +
                             sqr(P->i[2] * R->d[2] - tgt[2]));
}

static void launch(orc_mc *R, orc_photon *P) {
  P->sameVoxel = false;
  P->weight = 1;
  P->recN = 0;
  P->kec = 0;
  long attempts = 0;
  double tgt[3] = {0, 0, 0}, w0[3], X, Y, r, phi, tx, ty, ct, stt;
  do {
    if (R->S) {
      long j = bsearch_cdf(rnd(R, P), R->n[0] * R->n[1] * R->n[2], R->S);
      P->i[0] = j % R->n[0] + 1 - rnd(R, P);
      P->i[1] = j / R->n[0] % R->n[1] + 1 - rnd(R, P);
      P->i[2] = j / R->n[0] / R->n[1] + 1 - rnd(R, P);
      ct = 1 - 2 * rnd(R, P);
      stt = sqrt(1 - ct * ct);
      phi = 2 * O_PI * rnd(R, P);
      P->u[0] = stt * cos(phi);
      P->u[1] = stt * sin(phi);
      P->u[2] = ct;
      P->j = newj(R, P->i);
      P->RI = R->RI[R->M0[P->j]];
      P->time = 0;
    } else switch (R->beamType) {
      case 0:
        P->i[0] = (R->focus[0] - R->focus[2] * R->u[0] / R->u[2]) / R->d[0] + R->n[0] / 2.0;
        P->i[1] = (R->focus[1] - R->focus[2] * R->u[1] / R->u[2]) / R->d[1] + R->n[1] / 2.0;
        P->i[2] = 0;
        for (int k = 0; k < 3; k++) P->u[k] = R->u[k];
        P->j = newj(R, P->i);
        P->RI = R->RI[R->M0[P->j]];
        P->time = start_time_focus(R, P, R->focus);
        break;
      case 1:
        r = rnd(R, P);
        P->i[0] = (R->focus[0] + R->u[0] * (r - 0.5) * R->emitterLength) / R->d[0] + R->n[0] / 2.0;
        P->i[1] = (R->focus[1] + R->u[1] * (r - 0.5) * R->emitterLength) / R->d[1] + R->n[1] / 2.0;
        P->i[2] = (R->focus[2] + R->u[2] * (r - 0.5) * R->emitterLength) / R->d[2];
        ct = 1 - 2 * rnd(R, P);
        stt = sqrt(1 - ct * ct);
        phi = 2 * O_PI * rnd(R, P);
        P->u[0] = stt * cos(phi);
        P->u[1] = stt * sin(phi);
        P->u[2] = ct;
        P->j = newj(R, P->i);
        P->RI = R->RI[R->M0[P->j]];
        P->time = 0;
        break;
      case 2: {
        double span = (R->bt == 1 || R->bt == 3) ? 1 : O_KILLRANGE;
        P->i[0] = span * R->n[0] * (rnd(R, P) - 0.5) + R->n[0] / 2.0;
        P->i[1] = span * R->n[1] * (rnd(R, P) - 0.5) + R->n[1] / 2.0;
        P->i[2] = 0;
        for (int k = 0; k < 3; k++) P->u[k] = R->u[k];
        P->j = newj(R, P->i);
        P->RI = R->RI[R->M0[P->j]];
        P->time = P->RI / O_C * ((P->i[0] - R->n[0] / 2.0) * R->d[0] * R->u[0] + (P->i[1] - R->n[1] / 2.0) * R->d[1] * R->u[1] +
                                 P->i[2] * R->d[2] * R->u[2]);
        break;
      }
      case 3:
        phi = rnd(R, P) * 2 * O_PI;
        rotate(R->v, R->u, phi, w0);
        r = R->FPw1 * sqrt((lambert_wm1(-rnd(R, P) * exp(-1.0)) + 1) / (-2)) / 1.50087;
        for (int k = 0; k < 3; k++) tgt[k] = R->focus[k] + r * w0[k];
        phi = R->AIw1 * sqrt((lambert_wm1(-rnd(R, P) * exp(-1.0)) + 1) / (-2)) / 1.50087;
        rotate(R->u, w0, phi, P->u);
        P->i[0] = (tgt[0] - tgt[2] * P->u[0] / P->u[2]) / R->d[0] + R->n[0] / 2.0;
        P->i[1] = (tgt[1] - tgt[2] * P->u[1] / P->u[2]) / R->d[1] + R->n[1] / 2.0;
        P->i[2] = 0;
        P->j = newj(R, P->i);
        P->RI = R->RI[R->M0[P->j]];
        P->time = start_time_focus(R, P, tgt);
        break;
      case 4:
        rotate(R->v, R->u, rnd(R, P) * 2 * O_PI, w0);
        if (R->FP1[0] == -1) r = R->FPw1 * sqrt(rnd(R, P));
        else if (R->FP1[0] == -2) r = R->FPw1 * sqrt(-0.5 * log(rnd(R, P)));
        else {
          double a = rnd(R, P);
          r = R->FPw1 * (bsearch_cdf(a, R->LFP1 - 1, R->FP1) + rnd(R, P)) / (R->LFP1 - 1);
        }
        for (int k = 0; k < 3; k++) tgt[k] = R->focus[k] + r * w0[k];
        rotate(R->v, R->u, rnd(R, P) * 2 * O_PI, w0);
        if (R->AI1[0] == -1) phi = atan(tan(R->AIw1) * sqrt(rnd(R, P)));
        else if (R->AI1[0] == -2) phi = atan(tan(R->AIw1) * sqrt(-0.5 * log(rnd(R, P))));
        else if (R->AI1[0] == -3) phi = asin(sqrt(rnd(R, P)));
        else {
          double a = rnd(R, P);
          phi = atan(tan(R->AIw1) * (bsearch_cdf(a, R->LAI1 - 1, R->AI1) + rnd(R, P)) / (R->LAI1 - 1));
        }
        rotate(R->u, w0, phi, P->u);
        P->i[0] = (tgt[0] - tgt[2] * P->u[0] / P->u[2]) / R->d[0] + R->n[0] / 2.0;
        P->i[1] = (tgt[1] - tgt[2] * P->u[1] / P->u[2]) / R->d[1] + R->n[1] / 2.0;
        P->i[2] = 0;
        P->j = newj(R, P->i);
        P->RI = R->RI[R->M0[P->j]];
        P->time = start_time_focus(R, P, tgt);
        break;
      case 5: {
        if (R->FP1[0] == -1) X = R->FPw1 * (rnd(R, P) * 2 - 1);
        else if (R->FP1[0] == -2) { double a = rnd(R, P); X = R->FPw1 * sqrt(-0.5 * log(a)) * cos(2 * O_PI * rnd(R, P)); }
        else { double a = rnd(R, P); X = R->FPw1 * ((bsearch_cdf(a, R->LFP1 - 1, R->FP1) + rnd(R, P)) / (R->LFP1 - 1) * 2 - 1); }
        if (R->FP2[0] == -1) Y = R->FPw2 * (rnd(R, P) * 2 - 1);
        else if (R->FP2[0] == -2) { double a = rnd(R, P); Y = R->FPw2 * sqrt(-0.5 * log(a)) * cos(2 * O_PI * rnd(R, P)); }
        else { double a = rnd(R, P); Y = R->FPw2 * ((bsearch_cdf(a, R->LFP2 - 1, R->FP2) + rnd(R, P)) / (R->LFP2 - 1) * 2 - 1); }
        for (int k = 0; k < 3; k++) tgt[k] = R->focus[k] + X * R->v[k] + Y * R->w[k];
        if (R->AI1[0] == -3) {
          rotate(R->v, R->u, rnd(R, P) * 2 * O_PI, w0);
          rotate(R->u, w0, asin(sqrt(rnd(R, P))), P->u);
        } else {
          /* MCmatlablib.c:678-688: custom angular X/Y distributions are scaled by L (not L-1) */
          if (R->AI1[0] == -1) tx = tan(R->AIw1) * (rnd(R, P) * 2 - 1);
          else if (R->AI1[0] == -2) { double a = rnd(R, P); tx = tan(R->AIw1) * sqrt(-0.5 * log(a)) * cos(2 * O_PI * rnd(R, P)); }
          else { double a = rnd(R, P); tx = tan(R->AIw1) * ((bsearch_cdf(a, R->LAI1 - 1, R->AI1) + rnd(R, P)) / R->LAI1 * 2 - 1); }
          if (R->AI2[0] == -1) ty = tan(R->AIw2) * (rnd(R, P) * 2 - 1);
          else if (R->AI2[0] == -2) { double a = rnd(R, P); ty = tan(R->AIw2) * sqrt(-0.5 * log(a)) * cos(2 * O_PI * rnd(R, P)); }
          else { double a = rnd(R, P); ty = tan(R->AIw2) * ((bsearch_cdf(a, R->LAI2 - 1, R->AI2) + rnd(R, P)) / R->LAI2 * 2 - 1); }
          rotate(R->v, R->u, atan2(tx, ty), w0);
          rotate(R->u, w0, atan(sqrt(tx * tx + ty * ty)), P->u);
        }
        P->i[0] = (tgt[0] - tgt[2] * P->u[0] / P->u[2]) / R->d[0] + R->n[0] / 2.0;
        P->i[1] = (tgt[1] - tgt[2] * P->u[1] / P->u[2]) / R->d[1] + R->n[1] / 2.0;
        P->i[2] = 0;
        P->j = newj(R, P->i);
        P->RI = R->RI[R->M0[P->j]];
        P->time = start_time_focus(R, P, tgt);
        break;
      }
    }
    const double h = O_KILLRANGE / 2.0;
    switch (R->bt) {
      case 0:
        P->alive = fabs(P->i[0] / R->n[0] - 0.5) < h && fabs(P->i[1] / R->n[1] - 0.5) < h && fabs(P->i[2] / R->n[2] - 0.5) < h;
        break;
      case 2:
        P->alive = fabs(P->i[0] / R->n[0] - 0.5) < h && fabs(P->i[1] / R->n[1] - 0.5) < h && P->i[2] / R->n[2] - 0.5 < h && P->i[2] >= 0;
        break;
      default:
        P->alive = inside(R, P->i);
        break;
    }
  } while (!P->alive && ++attempts < 1000000);
  if (attempts >= 1000000) R->aborting = 1;
  set_D(R, P);
  P->insideVolume = inside(R, P->i);
  P->stepLeft = -log(rnd(R, P));
  P->scat = P->refr = P->refl = P->itr = 0;
}

static void interp_normal(const orc_mc *R, const orc_photon *P, long jn, double *nv) {
  /* MCmatlablib.c:920-1013. The coerced index is truncated to an integer before the
   * "- 0.5" (it is declared long), so every weight evaluates to 0.5: the normal is the
   * equal-weight sum over the 2x2x2 block {k-1, k}^3 of voxels with the new voxel's RI. */
  long kc[3];
  for (int k = 0; k < 3; k++) kc[k] = (long)(P->i[k] < 0 ? 0 : (P->i[k] >= R->n[k] ? R->n[k] - 1 : P->i[k]));
  long i0[3];
  double wt[3];
  for (int k = 0; k < 3; k++) {
    i0[k] = (long)floor(kc[k] - 0.5);
    wt[k] = kc[k] - 0.5 - i0[k];
  }
  double ri = R->RI[R->M0[jn]];
  nv[0] = nv[1] = nv[2] = 0;
  for (int cz = 0; cz < 2; cz++)
    for (int cy = 0; cy < 2; cy++)
      for (int cx = 0; cx < 2; cx++) {
        long jx = i0[0] + cx, jy = i0[1] + cy, jz = i0[2] + cz;
        if ((cx == 0 ? jx < 0 : i0[0] >= R->n[0] - 1) || (cy == 0 ? jy < 0 : i0[1] >= R->n[1] - 1) ||
            (cz == 0 ? jz < 0 : i0[2] >= R->n[2] - 1))
          continue;
        long jc = jx + jy * R->n[0] + jz * R->n[0] * R->n[1];
        if (R->RI[R->M0[jc]] != ri) continue;
        double th = R->normals[2 * jc], ph = R->normals[2 * jc + 1];
        double wgt = (cx ? wt[0] : 1 - wt[0]) * (cy ? wt[1] : 1 - wt[1]) * (cz ? wt[2] : 1 - wt[2]);
        nv[0] += wgt * sin(th) * cos(ph);
        nv[1] += wgt * sin(th) * sin(ph);
        nv[2] += wgt * cos(th);
      }
  double nrm = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
  nv[0] /= nrm;
  nv[1] /= nrm;
  nv[2] /= nrm;
}

/* (e^{-x} - (1 - e^{-x}) / x) / x, by its Taylor series -1/2 + x/3 - x^2/8 + x^3/30 - x^4/144
 * where the direct form cancels */
static double self_phi(double x) {
  if (x < 0.05) return -0.5 + x * (1.0 / 3.0 - x * (0.125 - x * (1.0 / 30.0 - x / 144.0)));
  return (exp(-x) + expm1(-x) / x) / x;
}

static void propagate(orc_mc *R, orc_photon *P) {
  const int mj = R->M0[P->j];
  const double wpre = P->weight;
  P->sameVoxel = true;
  P->steps++;
  double s = fmin(P->stepLeft / P->mus, fmin(P->D[0], fmin(P->D[1], P->D[2])));
  P->stepLeft = s == P->stepLeft / P->mus ? 0 : P->stepLeft - s * P->mus;
  P->time += s * P->RI / O_C;
  for (int k = 0; k < 3; k++) {
    long io = (long)floor(P->i[k]);
    if (s == P->D[k]) {
      P->i[k] = P->u[k] > 0 ? io + 1 : io - DBL_EPSILON * (labs(io) + 1);
      P->D[k] = R->d[k] / fabs(P->u[k]);
      P->sameVoxel = false;
    } else {
      P->i[k] += s * P->u[k] / R->d[k];
      if ((long)floor(P->i[k]) != io) P->i[k] = P->u[k] > 0 ? io + 1 - DBL_EPSILON * (labs(io) + 1) : io;
      P->D[k] -= s;
    }
  }
  if (!P->sameVoxel) {
    long jn = newj(R, P->i);
    int mn = R->M0[jn];
    double mu = P->RI / R->RI[mn];
    if (mu != 1) {
      double nv[3];
      interp_normal(R, P, jn, nv);
      double cin = nv[0] * P->u[0] + nv[1] * P->u[1] + nv[2] * P->u[2];
      if (cin > 0) {
        double cos2 = 1 - mu * mu * (1 - cin * cin);
        bool refl;
        if (cos2 > 0) {
          double co = sqrt(cos2);
          double Rf = sqr((mu * cin - co) / (mu * cin + co)) / 2 + sqr((mu * co - cin) / (mu * co + cin)) / 2;
          refl = rnd(R, P) <= Rf;
        } else refl = true;
        if (refl) {
          for (int k = 0; k < 3; k++) P->u[k] -= 2 * nv[k] * cin;
          set_D(R, P);
          if ((unsigned long)mn >= R->minIdx && (unsigned long)mn <= R->maxIdx) P->refl++;
        } else {
          double nc = sqrt(cos2) - mu * cin;
          for (int k = 0; k < 3; k++) P->u[k] = nc * nv[k] + mu * P->u[k];
          set_D(R, P);
          P->RI = R->RI[mn];
          if ((unsigned long)mn >= R->minIdx && (unsigned long)mn <= R->maxIdx) {
            P->refr++;
            P->itr++;
          }
        }
      }
    } else if (mn != R->M0[P->j] && R->RI[R->M0[P->j]] == P->RI) {
      if ((unsigned long)mn >= R->minIdx && (unsigned long)mn <= R->maxIdx) P->itr++;
    }
  }
  double absorb = -P->weight * expm1(-P->mua * s);
  P->weight -= absorb;
  if (R->grad) {
    if (P->insideVolume && P->inbox) {
      /* c(mua) = w (1 - e^{-mua s}) / mua; dc/dmua = w s^2 phi(mua s) (self_phi); the score for
       * mus counts the interaction that ends this step when the free path ran out here */
      const double mua = P->mua, c = absorb / mua;
      const double dself = wpre * s * s * self_phi(mua * s);
      const double kself = P->stepLeft > 0 ? 0.0 : 1.0;
      add(&R->gF[0], c);
      for (int m = 0; m < R->nGM; m++) {
        const double Lincl = P->L[m] + (m == mj ? s : 0.0);
        const double kincl = P->k[m] + (m == mj ? kself : 0.0);
        add(&R->gF[1 + m], -P->L[m] * c + (m == mj ? dself : 0.0));
        add(&R->gF[1 + R->nGM + m], (kincl / R->mus[m] - Lincl) * c);
      }
    }
    P->L[mj] += s;
  }
  if (P->insideVolume) {
    if (!R->eol) {
      if (R->NFR && criteria(R, P)) add(&R->NFR[P->j], absorb);
    } else {
      if (P->recN == P->recSize) {
        P->recSize = P->recSize ? 2 * P->recSize : 1000;
        P->jrec = (long *)realloc(P->jrec, P->recSize * sizeof(long));
        P->wrec = (double *)realloc(P->wrec, P->recSize * sizeof(double));
      }
      P->jrec[P->recN] = P->j;
      P->wrec[P->recN] = absorb;
      P->recN++;
    }
  }
}

static void form_image(orc_mc *R, orc_photon *P) {
  double U[3];
  toLC(P->u, R->LCth, R->LCph, U);
  if (U[2] < 0) {
    double resc[3] = {(P->i[0] - R->n[0] / 2.0) * R->d[0] - R->LCr[0], (P->i[1] - R->n[1] / 2.0) * R->d[1] - R->LCr[1],
                      P->i[2] * R->d[2] - R->LCr[2]};
    double Re[3];
    toLC(resc, R->LCth, R->LCph, Re);
    if (Re[2] > 0) {
      double RL0 = Re[0] - Re[2] * U[0] / U[2], RL1 = Re[1] - Re[2] * U[1] / U[2];
      if (sqrt(RL0 * RL0 + RL1 * RL1) < R->LCdiam / 2) {
        if (isfinite(R->LCf)) {
          double RI0 = RL0 + R->LCf * U[0] / U[2], RI1 = RL1 + R->LCf * U[1] / U[2];
          if (sqrt(RI0 * RI0 + RI1 * RI1) < R->LCfs / 2) {
            long Xi = (long)(R->LCres[0] * (RI0 / R->LCfs + 0.5));
            long Yi = (long)(R->LCres[0] * (RI1 / R->LCfs + 0.5));
            long ti = 0;
            if (R->LCres[1] > 1) {
              long v = (long)(1 + (R->LCres[1] - 2) * (P->time - (Re[2] - R->LCf) / U[2] * P->RI / O_C - R->tStart) / (R->tEnd - R->tStart));
              ti = v < 0 ? 0 : (v > R->LCres[1] - 1 ? R->LCres[1] - 1 : v);
            }
            P->kec = 2;
            if (criteria(R, P)) {
              add(&R->image[Xi + Yi * R->LCres[0] + ti * R->LCres[0] * R->LCres[0]], P->weight);
#pragma omp atomic
              R->nPhotonsCollected++;
            }
          }
        } else {
          double thFF = atan(-sqrt(U[0] * U[0] + U[1] * U[1]) / U[2]);
          if (thFF < asin(fmin(1.0, R->LCfs))) {
            long ti = 0;
            if (R->LCres[1] > 1) {
              long v = (long)(1 + (R->LCres[1] - 2) * (P->time - Re[2] / U[2] * P->RI / O_C - R->tStart) / (R->tEnd - R->tStart));
              ti = v < 0 ? 0 : (v > R->LCres[1] - 1 ? R->LCres[1] - 1 : v);
            }
            P->kec = 2;
            if (criteria(R, P)) {
              add(&R->image[ti], P->weight);
#pragma omp atomic
              R->nPhotonsCollected++;
            }
          }
        }
      }
    }
  }
}

static void edge_fluxes(orc_mc *R, const orc_photon *P) {
  const long *n = R->n;
  if (R->bt == 1) {
    if (P->i[2] < 0) add(&R->NIzn[(long)P->i[0] + n[0] * (long)P->i[1]], P->weight);
    else if (P->i[2] >= n[2]) add(&R->NIzp[(long)P->i[0] + n[0] * (long)P->i[1]], P->weight);
    else if (P->i[1] < 0) add(&R->NIyn[(long)P->i[0] + n[0] * (long)P->i[2]], P->weight);
    else if (P->i[1] >= n[1]) add(&R->NIyp[(long)P->i[0] + n[0] * (long)P->i[2]], P->weight);
    else if (P->i[0] < 0) add(&R->NIxn[(long)P->i[1] + n[1] * (long)P->i[2]], P->weight);
    else if (P->i[0] >= n[0]) add(&R->NIxp[(long)P->i[1] + n[1] * (long)P->i[2]], P->weight);
  } else if (R->bt == 2) {
    if (P->i[2] < 0)
      add(&R->NIzn[(long)(P->i[0] + n[0] * (O_KILLRANGE - 1) / 2.0) + (O_KILLRANGE * n[0]) * ((long)(P->i[1] + n[1] * (O_KILLRANGE - 1) / 2.0))],
          P->weight);
  } else {
    if (P->i[2] < 0) add(&R->NIzn[(long)P->i[0] + n[0] * (long)P->i[1]], P->weight);
    else if (P->i[2] >= n[2]) add(&R->NIzp[(long)P->i[0] + n[0] * (long)P->i[1]], P->weight);
  }
}

/* Returns whether the packet was wrapped to the opposite face (cyclic boundaries). */
static int check_escape(orc_mc *R, orc_photon *P) {
  bool esc = false;
  int tele = 0;
  const double h = O_KILLRANGE / 2.0;
  const long *n = R->n;
  switch (R->bt) {
    case 0:
      P->alive = fabs(P->i[0] / n[0] - 0.5) < h && fabs(P->i[1] / n[1] - 0.5) < h && fabs(P->i[2] / n[2] - 0.5) < h;
      break;
    case 1:
      P->alive = inside(R, P->i);
      esc = !P->alive && P->RI == 1;
      break;
    case 2:
      P->alive = fabs(P->i[0] / n[0] - 0.5) < h && fabs(P->i[1] / n[1] - 0.5) < h && P->i[2] / n[2] - 0.5 < h && P->i[2] >= 0;
      esc = P->i[2] < 0 && P->RI == 1;
      break;
    case 3: {
      bool tooOld = P->time > 1000 / O_C * sqrt(sqr(R->d[0] * n[0]) + sqr(R->d[1] * n[1]));
      P->alive = P->i[2] < n[2] && P->i[2] >= 0 && !tooOld;
      esc = !P->alive && P->RI == 1 && !tooOld;
      if (P->i[0] >= n[0]) { P->i[0] = 0; tele = 1; }
      if (P->i[0] < 0) { P->i[0] = n[0] * (1 - DBL_EPSILON); tele = 1; }
      if (P->i[1] >= n[1]) { P->i[1] = 0; tele = 1; }
      if (P->i[1] < 0) { P->i[1] = n[1] * (1 - DBL_EPSILON); tele = 1; }
      break;
    }
  }
  P->insideVolume = inside(R, P->i);
  if (esc) {
    P->kec = 1;
    if (R->image) form_image(R, P);
    if (R->FF && criteria(R, P)) {
      double th = (1 - DBL_EPSILON) * acos(P->u[2]);
      double ph = (1 - DBL_EPSILON) * (O_PI + atan2(P->u[1], P->u[0]));
      add(&R->FF[(long)floor(th / O_PI * R->ffr) + R->ffr * (long)floor(ph / (2 * O_PI) * R->ffr)], P->weight);
    }
  }
  if (!P->alive && R->bt && criteria(R, P)) edge_fluxes(R, P);
  if (R->grad && !P->alive && P->kec != 0 && P->i[2] < 0 && R->nR > 0) {
    const double x = (P->i[0] - R->n[0] / 2.0) * R->d[0], y = (P->i[1] - R->n[1] / 2.0) * R->d[1];
    const long b = (long)(sqrt(x * x + y * y) / R->rbin);
    if (b < R->nR) {
      double *row = R->gR + b * (1 + 2 * R->nGM);
      const double W = P->weight;
      add(row, W);
      for (int m = 0; m < R->nGM; m++) {
        add(row + 1 + m, -P->L[m] * W);
        add(row + 1 + R->nGM + m, (P->k[m] / R->mus[m] - P->L[m]) * W);
      }
    }
  }
  return tele;
}

static void scatter(orc_mc *R, orc_photon *P) {
  double ct;
  if (R->grad) P->k[R->M0[P->j]] += 1.0;
  if (isnan(P->g)) {
    double a = rnd(R, P);
    long jt = bsearch_cdf(a, O_CDFSIZE - 1, R->CDFs + (long)P->CDFidx * O_CDFSIZE);
    ct = cos((jt + rnd(R, P)) * O_PI / (O_CDFSIZE - 1));
  } else {
    double g = P->g;
    if (fabs(g) == 1.0) ct = g;
    else if (fabs(g) <= sqrt(DBL_EPSILON)) ct = 2 * rnd(R, P) - 1;
    else ct = (1 + g * g - sqr((1 - g * g) / (1 - g + 2 * g * rnd(R, P)))) / (2 * g);
  }
  double st = sqrt(1 - ct * ct);
  double phi = 2 * O_PI * rnd(R, P);
  double cp = cos(phi), sp = sin(phi);
  if (fabs(P->u[2]) < 1) {
    double q = sqrt(P->u[0] * P->u[0] + P->u[1] * P->u[1]);
    double ux = st * (P->u[0] * P->u[2] * cp - P->u[1] * sp) / q + P->u[0] * ct;
    double uy = st * (P->u[1] * P->u[2] * cp + P->u[0] * sp) / q + P->u[1] * ct;
    P->u[2] = -st * cp * q + P->u[2] * ct;
    P->u[1] = uy;
    P->u[0] = ux;
  } else {
    P->u[0] = st * cp;
    P->u[1] = st * sp;
    P->u[2] = ct * (P->u[2] >= 0 ? 1 : -1);
  }
  set_D(R, P);
  P->stepLeft = -log(rnd(R, P));
  int m = R->M0[P->j];
  if ((unsigned long)m >= R->minIdx && (unsigned long)m <= R->maxIdx) P->scat++;
}

/* sub-steps without a scattering event after which a packet ends as killed: the transport's
 * guard against packets caught in endless reflections in non-scattering regions (the reference
 * has no limit) */
#define ORC_MAX_FREE_STEPS 20000UL

/* addToPhotonPath (MCmatlablib.c:479-504): nanCols NaN columns, then the packet's position and
 * weight */
static void path_add(orc_mc *R, const orc_photon *P, int nanCols) {
  if (R->pn + nanCols + 1 > R->pcap) {
    R->pn = R->pcap + 1;
    return;
  }
  for (int c = 0; c < nanCols; c++) {
    for (int r = 0; r < 4; r++) R->pdata[4 * R->pn + r] = NAN;
    R->pn++;
  }
  R->pdata[4 * R->pn + 0] = (P->i[0] - R->n[0] / 2.0) * R->d[0];
  R->pdata[4 * R->pn + 1] = (P->i[1] - R->n[1] / 2.0) * R->d[1];
  R->pdata[4 * R->pn + 2] = P->i[2] * R->d[2];
  R->pdata[4 * R->pn + 3] = P->weight;
  R->pn++;
  R->pstarted = 1;
}

/* updatePaths (MCmatlablib.c:507-514); a no-op outside example-path recording */
static void path_update(orc_mc *R, orc_photon *P, int teleported) {
  if (!R->pdata || R->pn > R->pcap) return;
  if (R->eol || criteria(R, P)) path_add(R, P, R->pstarted ? (teleported ? 1 : 0) : 2);
}

static void run_packet(orc_mc *R, orc_photon *P, uint64_t pid) {
  P->pid = pid;
  P->draw = 0;
  P->bufblock = 0xFFFFFFFFu;
  launch(R, P);
  P->psteps = 0;
  for (int m = 0; m < 10; m++) P->L[m] = P->k[m] = 0.0;
  if (P->alive) {
    path_update(R, P, 0);
    voxel_props(R, P);
#pragma omp atomic
    R->nPhotons++;
  }
  while (P->alive) {
    while (P->alive && P->stepLeft > 0) {
      propagate(R, P);
      path_update(R, P, 0);
      if (!P->sameVoxel) {
        if (check_escape(R, P) && (R->eol || criteria(R, P))) path_update(R, P, 1);
        if (P->alive) voxel_props(R, P);
      }
      if (++P->psteps >= ORC_MAX_FREE_STEPS) {
        P->alive = false;
#pragma omp atomic
        R->cuts += 1.0;
#pragma omp atomic
        R->cutW += P->weight;
      }
    }
    if (P->alive && P->weight < O_THRESHOLD) {
      if (rnd(R, P) <= O_CHANCE) P->weight /= O_CHANCE;
      else P->alive = false;
    }
    if (P->alive) {
      P->psteps = 0;
      scatter(R, P);
      path_update(R, P, 0);
    }
  }
  if (R->eol && criteria(R, P) && R->NFR)
    for (long k = 0; k < P->recN; k++) add(&R->NFR[P->jrec[k]], P->weight * P->wrec[k]);
}

/* Example paths: packets 0, 1, 2, ... (of the unsharded stream) replayed one after another with
 * their vertices recorded, until nPaths paths are finished (MCmatlab.c:270-278: a path whose
 * end-of-life criteria fail is deleted). Tallies the replay makes are the caller's to discard. */
static long record_paths(orc_mc *R, long nPaths, uint64_t maxP, double *data, long cap) {
  orc_photon P;
  memset(&P, 0, sizeof P);
  R->pdata = data;
  R->pcap = cap;
  R->pn = 0;
  long finished = 0;
  for (uint64_t pid = 0; pid < maxP && finished < nPaths && R->pn <= cap; pid++) {
    const long startN = R->pn;
    R->pstarted = 0;
    run_packet(R, &P, pid);
    if (R->pstarted) {
      if (R->eol && !criteria(R, &P)) R->pn = startN;
      else finished++;
    }
  }
  free(P.jrec);
  free(P.wrec);
  R->pdata = NULL;
  return R->pn > cap ? cap : R->pn;
}

static unsigned long infcast(double x) { return isinf(x) ? ULONG_MAX : (unsigned long)x; }

/* CDF of a beam distribution (MCmatlab.c:538-576): a code becomes -1-code, a sampled
 * distribution is integrated with the trapezoid rule (r-weighted when radial). */
static double *beam_cdf(const mcb_distr *d, int radial, long *L) {
  *L = d->n;
  double *o = (double *)malloc(sizeof(double) * (d->n > 0 ? d->n : 1));
  if (d->n == 1) {
    o[0] = -1 - d->values[0];
  } else {
    o[0] = 0;
    for (long k = 1; k < d->n; k++)
      o[k] = o[k - 1] + (radial ? k - 1 : 1) * d->values[k - 1] + (radial ? k : 1) * d->values[k];
    for (long k = 1; k < d->n; k++) o[k] /= o[d->n - 1];
  }
  return o;
}

/* Runs the whole MEX-equivalent computation; with obj != NULL also the perturbation-MC
 * objectives and derivatives (one wavelength, nM <= 8). nthreads <= 0: all available. */
static int mc_run_impl(const mcb_mc_model *in, mcb_mc_result *out, int nthreads, const mcb_mc_objectives *obj,
                       mcb_mc_grad_result *gres) {
  orc_mc R;
  memset(&R, 0, sizeof R);
  if (obj) {
    if (in->nL != 1 || in->nM > 10) return -2;
    R.grad = 1;
    R.nGM = in->nM;
    R.nR = obj->nRadialBins;
    R.rbin = obj->radialBinWidth;
    const long nn[3] = {in->nx, in->ny, in->nz};
    for (int q = 0; q < 6; q++) R.box[q] = (int)(obj->box[q] < 0 ? 0 : (obj->box[q] > nn[q / 2] ? nn[q / 2] : obj->box[q]));
    R.gR = (double *)calloc((size_t)(R.nR > 0 ? R.nR : 1) * (1 + 2 * R.nGM), sizeof(double));
    R.gF = (double *)calloc(1 + 2 * R.nGM, sizeof(double));
  }
  const long L = (long)in->nx * in->ny * in->nz;
  R.n[0] = in->nx; R.n[1] = in->ny; R.n[2] = in->nz;
  R.d[0] = in->dx; R.d[1] = in->dy; R.d[2] = in->dz;
  R.bt = in->boundaryType;
  R.ffr = in->farFieldRes;
  uint8_t *M0 = (uint8_t *)malloc(L);
  for (long k = 0; k < L; k++) M0[k] = (uint8_t)(in->M[k] - 1);
  R.M0 = M0;
  R.normals = in->interfaceNormals;
  R.nM = in->nM;
  R.mua = (double *)malloc(sizeof(double) * in->nM);
  R.mus = (double *)malloc(sizeof(double) * in->nM);
  R.g = (double *)malloc(sizeof(double) * in->nM);
  R.RI = (double *)malloc(sizeof(double) * in->nM);
  R.cdfidx = (int *)malloc(sizeof(int) * in->nM);
  R.CDFs = in->CDFs;
  R.key[0] = (uint32_t)in->seed;
  R.key[1] = (uint32_t)(in->seed >> 32);
  R.stream = 0;
  const bool useS = in->sourceDistribution != NULL;
  R.beamType = useS ? 0 : in->sourceType;
  R.emitterLength = useS ? 0 : in->emitterLength;
  long l;
  if (!useS && in->sourceType >= 4) {
    R.FP1 = beam_cdf(in->sourceType == 4 ? &in->FPID_radial : &in->FPID_X, in->sourceType == 4, &R.LFP1);
    R.AI1 = beam_cdf(in->sourceType == 4 ? &in->AID_radial : &in->AID_X, in->sourceType == 4, &R.LAI1);
    if (in->sourceType == 5) {
      R.FP2 = beam_cdf(&in->FPID_Y, 0, &R.LFP2);
      R.AI2 = beam_cdf(&in->AID_Y, 0, &R.LAI2);
    }
  }
  /* widths are read for every source type (MCmatlab.c:595-606) */
  if (!useS) {
    R.FPw1 = in->sourceType == 5 ? in->FPID_X.width : in->FPID_radial.width;
    R.AIw1 = in->sourceType == 5 ? in->AID_X.width : in->AID_radial.width;
    R.FPw2 = in->sourceType == 5 ? in->FPID_Y.width : 0;
    R.AIw2 = in->sourceType == 5 ? in->AID_Y.width : 0;
  }
  (void)l;
  /* beam basis u, v, w (MCmatlab.c:579-589) */
  double tb = useS ? 0 : in->theta, pb = useS ? 0 : in->phi, psib = useS ? 0 : in->psi;
  double u[3] = {sin(tb) * cos(pb), sin(tb) * sin(pb), cos(tb)};
  double w[3] = {1, 0, 0}, v[3] = {0, 0, 1};
  if (u[2] != 1) unitcross(u, v, w);
  rotate(w, u, psib, v);
  unitcross(u, v, w);
  for (int k = 0; k < 3; k++) { R.u[k] = u[k]; R.v[k] = v[k]; R.w[k] = w[k]; }
  R.focus[0] = useS ? 0 : in->xFocus;
  R.focus[1] = useS ? 0 : in->yFocus;
  R.focus[2] = useS ? 0 : in->zFocus;
  /* light collector (MCmatlab.c:427-448) */
  R.useLC = in->useLightCollector;
  double f = in->LC_f;
  long nTB = useS ? 0 : in->LC_nTimeBins;
  R.LCth = in->LC_theta; R.LCph = in->LC_phi; R.LCf = f; R.LCdiam = in->LC_diam;
  R.LCfs = isfinite(f) ? in->LC_fieldSize : in->LC_NA;
  R.LCr[0] = in->LC_x - (isfinite(f) ? f * sin(R.LCth) * cos(R.LCph) : 0);
  R.LCr[1] = in->LC_y - (isfinite(f) ? f * sin(R.LCth) * sin(R.LCph) : 0);
  R.LCr[2] = in->LC_z - (isfinite(f) ? f * cos(R.LCth) : 0);
  R.LCres[0] = in->LC_res;
  R.LCres[1] = nTB ? nTB + 2 : 1;
  R.tStart = useS ? 0 : in->LC_tStart;
  R.tEnd = useS ? 0 : in->LC_tEnd;
  /* deposition criteria (MCmatlab.c:402-424) */
  R.minS = infcast(in->DC_minScatterings); R.maxS = infcast(in->DC_maxScatterings);
  R.minRefr = infcast(in->DC_minRefractions); R.maxRefr = infcast(in->DC_maxRefractions);
  R.minRefl = infcast(in->DC_minReflections); R.maxRefl = infcast(in->DC_maxReflections);
  R.minI = infcast(in->DC_minInterfaceTransitions); R.maxI = infcast(in->DC_maxInterfaceTransitions);
  R.minIdx = infcast(in->DC_minSubmediaIdx) - 1; R.maxIdx = infcast(in->DC_maxSubmediaIdx) - 1;
  R.onlyCollected = in->DC_onlyCollected;
  R.eol = in->DC_evaluateOnlyAtEndOfLife;
  R.pOff = in->packetOffset;
  R.pStride = in->packetStride ? in->packetStride : 1;
  if (R.minS == 0 && R.maxS == ULONG_MAX && R.minRefr == 0 && R.maxRefr == ULONG_MAX && R.minRefl == 0 &&
      R.maxRefl == ULONG_MAX && R.minI == 0 && R.maxI == ULONG_MAX && !R.onlyCollected)
    R.eol = false;
  /* accumulators */
  long Lff = R.ffr * R.ffr, Lim = R.useLC ? R.LCres[0] * R.LCres[0] * R.LCres[1] : 0;
  long Lx = in->ny * in->nz, Ly = in->nx * in->nz, Lz = in->nx * in->ny;
  R.NFR = in->calcNFR ? (double *)calloc(L, sizeof(double)) : NULL;
  R.image = R.useLC ? (double *)calloc(Lim, sizeof(double)) : NULL;
  R.FF = R.ffr ? (double *)calloc(Lff, sizeof(double)) : NULL;
  if (R.bt == 1) {
    R.NIxp = (double *)calloc(Lx, 8); R.NIxn = (double *)calloc(Lx, 8);
    R.NIyp = (double *)calloc(Ly, 8); R.NIyn = (double *)calloc(Ly, 8);
  }
  if (R.bt == 1 || R.bt == 3) R.NIzp = (double *)calloc(Lz, 8);
  long Lzn = R.bt == 2 ? Lz * O_KILLRANGE * O_KILLRANGE : Lz;
  if (R.bt != 0) R.NIzn = (double *)calloc(Lzn, 8);
  double *S = useS ? (double *)malloc(sizeof(double) * (L + 1)) : NULL;
  const double V = in->dx * in->dy * in->dz;
  double nPhCum = 0, nColCum = 0;
  unsigned long long steps = 0;
  int nL = in->nL;
  bool timed = isnan(in->nPhotonsRequested);
  if (timed) return -1; /* the oracle runs fixed packet counts only */
#ifdef _OPENMP
  int nth = nthreads > 0 ? nthreads : omp_get_max_threads();
#else
  int nth = 1;
  (void)nthreads;
#endif
  out->examplePathsN = 0;
  for (int iL = 0; iL < nL; iL++) {
    for (int m = 0; m < in->nM; m++) {
      R.mua[m] = in->mua[m + (long)iL * in->nM];
      R.mus[m] = in->mus[m + (long)iL * in->nM];
      R.g[m] = in->g[m + (long)iL * in->nM];
      R.RI[m] = in->n[m + (long)iL * in->nM];
      R.cdfidx[m] = (int)(unsigned char)in->CDFidx[m + (long)iL * in->nM];
    }
    R.iL = (uint32_t)iL;
    if (useS) {
      S[0] = 0;
      for (long k = 1; k < L + 1; k++) S[k] = S[k - 1] + (double)in->sourceDistribution[(long)iL * L + k - 1];
      R.power = S[L] * in->dx * in->dy * in->dz;
      for (long k = 1; k < L + 1; k++) S[k] /= S[L];
      R.S = S;
    } else {
      R.power = in->spectrum[iL];
    }
    unsigned long long nReq = (unsigned long long)(iL == nL - 1 ? in->nPhotonsRequested - (in->requestCollectedPhotons ? nColCum : nPhCum)
                                                                : in->nPhotonsRequested / nL);
    R.nPhotons = R.nPhotonsCollected = 0;
    R.aborting = 0;
    if (in->requestCollectedPhotons) {
      /* keep launching until enough packets were collected; packets run in id order */
      uint64_t next = 0;
#pragma omp parallel num_threads(nth)
      {
        orc_photon P;
        memset(&P, 0, sizeof P);
        for (;;) {
          uint64_t pid;
#pragma omp atomic capture
          pid = next++;
          unsigned long long col;
#pragma omp atomic read
          col = R.nPhotonsCollected;
          if (col >= nReq || R.aborting) break;
          run_packet(&R, &P, R.pOff + R.pStride * pid);
        }
#pragma omp atomic
        steps += P.steps;
        free(P.jrec);
        free(P.wrec);
      }
    } else {
#pragma omp parallel num_threads(nth)
      {
        orc_photon P;
        memset(&P, 0, sizeof P);
#pragma omp for schedule(dynamic, 64)
        for (long long pid = 0; pid < (long long)nReq; pid++) {
          if (R.aborting) continue;
          run_packet(&R, &P, R.pOff + R.pStride * (uint64_t)pid);
        }
#pragma omp atomic
        steps += P.steps;
        free(P.jrec);
        free(P.wrec);
      }
    }
    nPhCum += (double)R.nPhotons;
    nColCum += (double)R.nPhotonsCollected;
    /* normalizeDepositionAndResetO (MCmatlablib.c:1186-1250) */
    double nf = (double)R.nPhotons / R.power;
    if (useS) nf /= R.power;
    else if (R.beamType == 2 && (R.bt == 0 || R.bt == 2)) nf /= O_KILLRANGE * O_KILLRANGE;
    if (R.NFR && out->NFR)
      for (long k = 0; k < L; k++) {
        out->NFR[k + (long)iL * L] = (float)(R.NFR[k] / (V * nf * R.mua[M0[k]]));
        R.NFR[k] = 0;
      }
    if (R.FF && out->farField)
      for (long k = 0; k < Lff; k++) {
        out->farField[k + (long)iL * Lff] = (float)(R.FF[k] / nf);
        R.FF[k] = 0;
      }
    if (R.image && out->image) {
      long Lp = R.LCres[0] * R.LCres[0];
      for (long k = 0; k < Lim; k++) {
        out->image[k + (long)iL * Lim] = (float)(Lp > 1 ? R.image[k] / (R.LCfs * R.LCfs / Lp * nf) : R.image[k] / nf);
        R.image[k] = 0;
      }
    }
#define NORM(arr, dst, cnt, area)                                                 \
  if (arr) {                                                                      \
    for (long k = 0; k < (cnt); k++) {                                            \
      if (dst) (dst)[k + (long)iL * (cnt)] = (float)((arr)[k] / ((area) * nf));  \
      (arr)[k] = 0;                                                               \
    }                                                                             \
  }
    NORM(R.NIxp, out->NI_xpos, Lx, in->dy * in->dz)
    NORM(R.NIxn, out->NI_xneg, Lx, in->dy * in->dz)
    NORM(R.NIyp, out->NI_ypos, Ly, in->dx * in->dz)
    NORM(R.NIyn, out->NI_yneg, Ly, in->dx * in->dz)
    NORM(R.NIzp, out->NI_zpos, Lz, in->dx * in->dy)
    NORM(R.NIzn, out->NI_zneg, Lzn, in->dx * in->dy)
#undef NORM
    if (iL == 0 && in->nExamplePaths > 0 && out->examplePaths && out->examplePathsCap > 0 && !R.grad) {
      const unsigned long long nPh0 = R.nPhotons, nCol0 = R.nPhotonsCollected;
      const double cuts0 = R.cuts, cutW0 = R.cutW;
      out->examplePathsN = record_paths(&R, (long)in->nExamplePaths, nPh0, out->examplePaths, (long)out->examplePathsCap);
      /* discard the replay's tallies and counts */
      if (R.NFR) memset(R.NFR, 0, sizeof(double) * L);
      if (R.image) memset(R.image, 0, sizeof(double) * Lim);
      if (R.FF) memset(R.FF, 0, sizeof(double) * Lff);
      if (R.NIxp) memset(R.NIxp, 0, 8 * Lx);
      if (R.NIxn) memset(R.NIxn, 0, 8 * Lx);
      if (R.NIyp) memset(R.NIyp, 0, 8 * Ly);
      if (R.NIyn) memset(R.NIyn, 0, 8 * Ly);
      if (R.NIzp) memset(R.NIzp, 0, 8 * Lz);
      if (R.NIzn) memset(R.NIzn, 0, 8 * Lzn);
      R.nPhotons = nPh0;
      R.nPhotonsCollected = nCol0;
      R.cuts = cuts0;
      R.cutW = cutW0;
    }
    if (R.aborting) break;
  }
  if (R.grad && gres) {
    double nf = nPhCum / R.power;
    if (useS) nf /= R.power;
    else if (R.beamType == 2 && (R.bt == 0 || R.bt == 2)) nf /= O_KILLRANGE * O_KILLRANGE;
    for (int b = 0; b < R.nR; b++) {
      const double area = O_PI * R.rbin * R.rbin * ((b + 1.0) * (b + 1.0) - (double)b * b);
      const double *row = R.gR + b * (1 + 2 * R.nGM);
      if (gres->R) gres->R[b] = row[0] / (area * nf);
      for (int m = 0; m < R.nGM; m++) {
        if (gres->dR_dmua) gres->dR_dmua[b + R.nR * m] = row[1 + m] / (area * nf);
        if (gres->dR_dmus) gres->dR_dmus[b + R.nR * m] = row[1 + R.nGM + m] / (area * nf);
      }
    }
    const double nbox = (double)(R.box[1] > R.box[0] ? R.box[1] - R.box[0] : 0) * (R.box[3] > R.box[2] ? R.box[3] - R.box[2] : 0) *
                        (R.box[5] > R.box[4] ? R.box[5] - R.box[4] : 0);
    const double sc = nbox > 0 ? 1.0 / (V * nf * nbox) : 0.0;
    gres->F = R.gF[0] * sc;
    for (int m = 0; m < R.nGM; m++) {
      if (gres->dF_dmua) gres->dF_dmua[m] = R.gF[1 + m] * sc;
      if (gres->dF_dmus) gres->dF_dmus[m] = R.gF[1 + R.nGM + m] * sc;
    }
  }
  free(R.gR);
  free(R.gF);
  out->nPhotons = nPhCum;
  out->nPhotonsCollected = nColCum;
  out->nThreads = nth;
  out->simulationTime = 0;
  out->propagationSteps = steps;
  out->freeStepCuts = R.cuts;
  out->freeStepCutWeight = R.cutW;
  free(M0); free(R.mua); free(R.mus); free(R.g); free(R.RI); free(R.cdfidx);
  free(R.FP1); free(R.FP2); free(R.AI1); free(R.AI2);
  free(R.NFR); free(R.image); free(R.FF);
  free(R.NIxp); free(R.NIxn); free(R.NIyp); free(R.NIyn); free(R.NIzp); free(R.NIzn);
  free(S);
  return 0;
}

int orc_mc_run(const mcb_mc_model *in, mcb_mc_result *out, int nthreads) { return mc_run_impl(in, out, nthreads, NULL, NULL); }

int orc_mc_grad(const mcb_mc_model *in, const mcb_mc_objectives *obj, mcb_mc_result *out, mcb_mc_grad_result *g,
                int nthreads) {
  return mc_run_impl(in, out, nthreads, obj, g);
}

/* Philox known-answer access for tests */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { orc_philox4x32_10(ctr, key, out); }
double orc_lambert_wm1(double x) { return lambert_wm1(x); }
size_t orc_sizeof_mc_model(void) { return sizeof(mcb_mc_model); }
size_t orc_sizeof_mc_result(void) { return sizeof(mcb_mc_result); }
size_t orc_sizeof_heat_params(void) { return sizeof(mcb_heat_params); }
