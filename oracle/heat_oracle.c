/*
 * heat_oracle.c — FP64 CPU restatement of the reference heat stepper.
 *
 * TEST INFRASTRUCTURE ONLY (the checker). Restates, in double precision, the
 * Douglas-Gunn ADI time step of +MCmatlab/src/finiteElementHeatPropagator.c:
 *   substep1a :249-313  explicit stencil, x flux half-weighted, source added
 *   substep1b :318-390  Thomas solve along x
 *   substep2a :395-449  explicit y half-correction on T^n
 *   substep2b :454-522  Thomas solve along y
 *   substep3a :527-566  explicit z half-correction on T^n
 *   substep3b :571-647  Thomas solve along z, Arrhenius damage with the mid-step
 *                       temperature, per-medium running maximum
 *   recordTempSensors :652-664, buffer swap :667-686, driver loop :764-808
 * with the same index formulas and the same heat-sink exceptions. The reference
 * computes in float; this oracle keeps every quantity in double (coefficients and
 * inputs are read from the same float arrays), so it is the "double-precision run"
 * the GPU stepper's error is measured against.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_R 8.3144598        /* gas constant, finiteElementHeatPropagator.c:86 */
#define ORC_CELSIUSZERO 273.15 /* :87 */

static inline int sinked(int hs, long ix, long iy, long iz, long nx, long ny, long nz) {
  return hs && (ix == 0 || ix == nx - 1 || iy == 0 || iy == ny - 1 || iz == 0 || iz == nz - 1);
}

static void record_sensors(const double *T, long nx, long ny, int nS, const double *idx, const double *w,
                           double *out) {
  for (int j = 0; j < nS; j++) {
    long i = (long)idx[j];
    double wx = w[j], wy = w[j + nS], wz = w[j + 2 * nS];
    long sz = nx * ny;
    out[j] = (1 - wx) * (1 - wy) * (1 - wz) * T[i] + (1 - wx) * (1 - wy) * wz * T[i + sz] +
             (1 - wx) * wy * (1 - wz) * T[i + nx] + (1 - wx) * wy * wz * T[i + nx + sz] +
             wx * (1 - wy) * (1 - wz) * T[i + 1] + wx * (1 - wy) * wz * T[i + 1 + sz] +
             wx * wy * (1 - wz) * T[i + 1 + nx] + wx * wy * wz * T[i + 1 + nx + sz];
  }
}

/*
 * T (in/out, double [L]); Omega (in/out, double [L]) or NULL; sensorTemps [nS*(nt+1)] or NULL;
 * maxMediaTemps [nM] (initialised here to -inf). M is 0-based. Returns 0.
 */
int orc_heat_run(long nx, long ny, long nz, int nM, const uint8_t *M, const float *cf, const float *Qf,
                 const double *A, const double *E, int lightsOn, int heatSinked, long nt, double dt,
                 double *T, double *Omega, int nS, const double *sIdx, const double *sW,
                 double *sensorTemps, double *maxMediaTemps) {
  const long L = nx * ny * nz, sxy = nx * ny;
  const long nM2 = (long)nM * nM;
  double *c = (double *)malloc(sizeof(double) * nM2 * 3);
  double *T2 = (double *)malloc(sizeof(double) * L);
  double *logA = (double *)malloc(sizeof(double) * nM);
  long lmax = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
  for (long k = 0; k < nM2 * 3; k++) c[k] = cf[k];
  for (int m = 0; m < nM; m++) {
    logA[m] = log(A[m]);
    maxMediaTemps[m] = -INFINITY;
  }
  if (nS && sensorTemps) record_sensors(T, nx, ny, nS, sIdx, sW, sensorTemps);

  for (long n = 0; n < nt; n++) {
    /* 1a: explicit part, T2 = T + dt*(Q + x/2 + y + z) */
#pragma omp parallel for schedule(static)
    for (long iz = 0; iz < nz; iz++)
      for (long iy = 0; iy < ny; iy++)
        for (long ix = 0; ix < nx; ix++) {
          long i = ix + iy * nx + iz * sxy;
          double dTdt = 0;
          if (!sinked(heatSinked, ix, iy, iz, nx, ny, nz)) {
            dTdt = lightsOn ? (double)Qf[i] : 0.0;
            if (ix != 0) dTdt += (T[i - 1] - T[i]) * c[M[i] + M[i - 1] * nM] / 2;
            if (ix != nx - 1) dTdt += (T[i + 1] - T[i]) * c[M[i] + M[i + 1] * nM] / 2;
            if (iy != 0) dTdt += (T[i - nx] - T[i]) * c[M[i] + M[i - nx] * nM + nM2];
            if (iy != ny - 1) dTdt += (T[i + nx] - T[i]) * c[M[i] + M[i + nx] * nM + nM2];
            if (iz != 0) dTdt += (T[i - sxy] - T[i]) * c[M[i] + M[i - sxy] * nM + 2 * nM2];
            if (iz != nz - 1) dTdt += (T[i + sxy] - T[i]) * c[M[i] + M[i + sxy] * nM + 2 * nM2];
          }
          T2[i] = T[i] + dt * dTdt;
        }

    /* 1b: Thomas along x; 2a: explicit y; 2b: Thomas along y; 3a: explicit z; 3b: Thomas along z */
    for (int dir = 0; dir < 3; dir++) {
      const long st = dir == 0 ? 1 : (dir == 1 ? nx : sxy);
      const long nl = dir == 0 ? nx : (dir == 1 ? ny : nz);
      const long off = dir * nM2;
      if (dir > 0) {
#pragma omp parallel for schedule(static)
        for (long iz = 0; iz < nz; iz++)
          for (long iy = 0; iy < ny; iy++)
            for (long ix = 0; ix < nx; ix++) {
              long i = ix + iy * nx + iz * sxy;
              if (sinked(heatSinked, ix, iy, iz, nx, ny, nz)) continue;
              long pos = dir == 1 ? iy : iz;
              double dTdt = 0;
              if (pos != 0) dTdt -= (T[i - st] - T[i]) * c[M[i] + M[i - st] * nM + off] / 2;
              if (pos != nl - 1) dTdt -= (T[i + st] - T[i]) * c[M[i] + M[i + st] * nM + off] / 2;
              T2[i] = T2[i] + dt * dTdt;
            }
      }
      /* lines: enumerate the two other coordinates */
      long na = dir == 0 ? ny : nx, nb = dir == 2 ? ny : nz;
#pragma omp parallel
      {
        double *b = (double *)malloc(sizeof(double) * lmax);
#pragma omp for schedule(static)
        for (long ab = 0; ab < na * nb; ab++) {
          long a = ab % na, bb = ab / na;
          long ix0, iy0, iz0;
          if (dir == 0) { ix0 = 0; iy0 = a; iz0 = bb; }
          else if (dir == 1) { ix0 = a; iy0 = 0; iz0 = bb; }
          else { ix0 = a; iy0 = bb; iz0 = 0; }
          long base = ix0 + iy0 * nx + iz0 * sxy;
          for (long p = 0; p < nl; p++) {
            long i = base + p * st;
            long ix = dir == 0 ? p : ix0, iy = dir == 1 ? p : iy0, iz = dir == 2 ? p : iz0;
            b[p] = 1;
            if (!sinked(heatSinked, ix, iy, iz, nx, ny, nz)) {
              if (p < nl - 1) b[p] += dt / 2 * c[M[i] + nM * M[i + st] + off];
              if (p > 0) {
                b[p] += dt / 2 * c[M[i] + nM * M[i - st] + off];
                double w = -dt / 2 * c[M[i] + nM * M[i - st] + off] / b[p - 1];
                if (p > 1 || !heatSinked) b[p] += w * dt / 2 * c[M[i - st] + nM * M[i] + off];
                T2[i] -= w * T2[i - st];
              }
            }
          }
          for (long p = nl - 1; p >= 0; p--) {
            long i = base + p * st;
            long ix = dir == 0 ? p : ix0, iy = dir == 1 ? p : iy0, iz = dir == 2 ? p : iz0;
            if (!sinked(heatSinked, ix, iy, iz, nx, ny, nz))
              T2[i] = (T2[i] + (p == nl - 1 ? 0 : dt / 2 * c[M[i] + nM * M[i + st] + off] * T2[i + st])) / b[p];
          }
        }
        free(b);
      }
    }
    /* 3b epilogue: damage with the mid-step temperature, running maxima, then swap */
    if (Omega) {
#pragma omp parallel for schedule(static)
      for (long i = 0; i < L; i++) {
        int m = M[i];
        if (E[m] != 0)
          Omega[i] += dt * exp(logA[m] - E[m] / (ORC_R * ((T2[i] + T[i]) / 2 + ORC_CELSIUSZERO)));
      }
    }
    for (long i = 0; i < L; i++) {
      if (T2[i] > maxMediaTemps[M[i]]) maxMediaTemps[M[i]] = T2[i];
      T[i] = T2[i];
    }
    if (nS && sensorTemps) record_sensors(T, nx, ny, nS, sIdx, sW, sensorTemps + (n + 1) * nS);
  }
  free(c);
  free(T2);
  free(logA);
  return 0;
}
