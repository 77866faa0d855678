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

/* ---------------------------------------------------------------------------------------------
 * Adjoint of the DG-ADI step (no counterpart in the reference: it is the checker of the GPU
 * adjoint). The forward step above, written as linear algebra on the grid vector T:
 *   D_d   per direction d: (D_d T)_v = sum over the d-neighbours u of v of c(M_v, M_u, d)(T_u - T_v)
 *         for non-sinked v, 0 for heat-sinked v
 *   r1 = T + dt (Q + D_x T / 2 + D_y T + D_z T)     A1 = X^-1 r1,  X = I - dt/2 D_x
 *   r2 = A1 - dt/2 D_y T                             A2 = Y^-1 r2,  Y = I - dt/2 D_y
 *   r3 = A2 - dt/2 D_z T                             T' = Z^-1 r3,  Z = I - dt/2 D_z
 *   dOmega_v = dt exp(log A - E / (R ((T_v + T'_v) / 2 + 273.15)))   (media with E != 0)
 * Objective J = sum_v wd_v sum_n dOmega_v^n + sum_v wp_v max_{n=1..nt} T_v^n. The reverse sweep
 * carries lambda = dJ/dT^n: rho3 = Z^-T lambda', rho2 = Y^-T rho3, rho1 = X^-T rho2 and
 *   lambda^n = rho1 + D_x^T (dt/2 rho1) + D_y^T (dt rho1 - dt/2 rho2) + D_z^T (dt rho1 - dt/2 rho3)
 * plus the damage and peak terms; dJ/dQ = sum_n dt rho1 (non-sinked voxels, light on) and
 * dJ/dD_d = dt/2 rho1 (T + A1)^T, dt rho1 T^T + dt/2 rho2 (A2 - T)^T, dt rho1 T^T + dt/2 rho3 (T' - T)^T
 * for d = x, y, z, collected per medium pair onto c. Every state is stored (small grids only).
 * --------------------------------------------------------------------------------------------- */

typedef struct {
  long nx, ny, nz, L, sxy;
  int nM, hs;
  const uint8_t *M;
  const double *c;
  double hdt;
} adj_grid;

static long dir_stride(const adj_grid *g, int d) { return d == 0 ? 1 : (d == 1 ? g->nx : g->sxy); }
static long dir_len(const adj_grid *g, int d) { return d == 0 ? g->nx : (d == 1 ? g->ny : g->nz); }
static long dir_pos(const adj_grid *g, long v, int d) {
  return d == 0 ? v % g->nx : (d == 1 ? (v / g->nx) % g->ny : v / g->sxy);
}
static int vox_sinked(const adj_grid *g, long v) {
  long ix = v % g->nx, iy = (v / g->nx) % g->ny, iz = v / g->sxy;
  return sinked(g->hs, ix, iy, iz, g->nx, g->ny, g->nz);
}
static double cpair(const adj_grid *g, long v, long u, int d) {
  return g->c[g->M[v] + g->M[u] * g->nM + d * (long)g->nM * g->nM];
}

/* out = D_d W (out may not alias W) */
static void apply_D(const adj_grid *g, int d, const double *W, double *out) {
  const long st = dir_stride(g, d), n = dir_len(g, d);
  for (long v = 0; v < g->L; v++) {
    double s = 0;
    if (!vox_sinked(g, v)) {
      long p = dir_pos(g, v, d);
      if (p > 0) s += cpair(g, v, v - st, d) * (W[v - st] - W[v]);
      if (p < n - 1) s += cpair(g, v, v + st, d) * (W[v + st] - W[v]);
    }
    out[v] = s;
  }
}

/* out += D_d^T W */
static void add_DT(const adj_grid *g, int d, const double *W, double *out) {
  const long st = dir_stride(g, d), n = dir_len(g, d);
  for (long v = 0; v < g->L; v++) {
    if (vox_sinked(g, v)) continue;
    long p = dir_pos(g, v, d);
    if (p > 0) {
      double cc = cpair(g, v, v - st, d);
      out[v - st] += cc * W[v];
      out[v] -= cc * W[v];
    }
    if (p < n - 1) {
      double cc = cpair(g, v, v + st, d);
      out[v + st] += cc * W[v];
      out[v] -= cc * W[v];
    }
  }
}

/* Solves (I - dt/2 D_d) x = r (transpose = 0) or its transpose (transpose = 1) along every
 * d-line with the Thomas algorithm on the assembled tridiagonal rows; x may alias r. */
static void line_solve(const adj_grid *g, int d, int transpose, const double *r, double *x) {
  const long st = dir_stride(g, d), n = dir_len(g, d);
  double *sub = (double *)malloc(sizeof(double) * n), *dia = (double *)malloc(sizeof(double) * n);
  double *sup = (double *)malloc(sizeof(double) * n), *y = (double *)malloc(sizeof(double) * n);
  for (long v0 = 0; v0 < g->L; v0++) {
    if (dir_pos(g, v0, d) != 0) continue;
    for (long p = 0; p < n; p++) {
      long v = v0 + p * st;
      sub[p] = sup[p] = 0;
      dia[p] = 1;
      if (!vox_sinked(g, v)) {
        if (p > 0) {
          sub[p] = -g->hdt * cpair(g, v, v - st, d);
          dia[p] -= sub[p];
        }
        if (p < n - 1) {
          sup[p] = -g->hdt * cpair(g, v, v + st, d);
          dia[p] -= sup[p];
        }
      }
      y[p] = r[v];
    }
    if (transpose) { /* rows of the transpose: sub'_p = sup_{p-1}, sup'_p = sub_{p+1} */
      double prev = 0;
      for (long p = 0; p < n; p++) {
        double nsub = p > 0 ? prev : 0;
        prev = sup[p];
        sup[p] = p < n - 1 ? sub[p + 1] : 0;
        sub[p] = nsub;
      }
    }
    for (long p = 1; p < n; p++) {
      double w = sub[p] / dia[p - 1];
      dia[p] -= w * sup[p - 1];
      y[p] -= w * y[p - 1];
    }
    y[n - 1] /= dia[n - 1];
    for (long p = n - 2; p >= 0; p--) y[p] = (y[p] - sup[p] * y[p + 1]) / dia[p];
    for (long p = 0; p < n; p++) x[v0 + p * st] = y[p];
  }
  free(sub);
  free(dia);
  free(sup);
  free(y);
}

static double damage_rate(const adj_grid *g, const double *logA, const double *E, long v, double tmid, double *dRdT) {
  int m = g->M[v];
  if (E[m] == 0) {
    *dRdT = 0;
    return 0;
  }
  double tk = tmid + ORC_CELSIUSZERO;
  double r = exp(logA[m] - E[m] / (ORC_R * tk));
  *dRdT = r * E[m] / (ORC_R * tk * tk);
  return r;
}

/*
 * c [nM*nM*3] and Q [L] in double; T0 [L]; wd, wp [L] or NULL. J[0..2] = J, J_damage, J_peak.
 * dc [nM*nM*3], dQ [L], dT0 [L] may be NULL. Returns 0.
 */
int orc_heat_adjoint(long nx, long ny, long nz, int nM, const uint8_t *M, const double *c, const double *Q,
                     const double *A, const double *E, int lightsOn, int heatSinked, long nt, double dt,
                     const double *T0, const double *wd, const double *wp, double *J, double *dc, double *dQ,
                     double *dT0) {
  adj_grid g = {nx, ny, nz, nx * ny * nz, nx * ny, nM, heatSinked, M, c, dt / 2};
  const long L = g.L;
  double *logA = (double *)malloc(sizeof(double) * nM);
  for (int m = 0; m < nM; m++) logA[m] = log(A[m]);
  double *Ts = (double *)malloc(sizeof(double) * L * (nt + 1));
  double *A1s = (double *)malloc(sizeof(double) * L * (nt > 0 ? nt : 1));
  double *A2s = (double *)malloc(sizeof(double) * L * (nt > 0 ? nt : 1));
  double *w1 = (double *)malloc(sizeof(double) * L), *w2 = (double *)malloc(sizeof(double) * L);
  double *pk = (double *)malloc(sizeof(double) * L);
  long *pkn = (long *)malloc(sizeof(long) * L);
  memcpy(Ts, T0, sizeof(double) * L);
  for (long v = 0; v < L; v++) {
    pk[v] = -INFINITY;
    pkn[v] = -1;
  }
  double Jd = 0, Jp = 0;
  for (long n = 0; n < nt; n++) {
    const double *T = Ts + n * L;
    double *Tn1 = Ts + (n + 1) * L, *A1 = A1s + n * L, *A2 = A2s + n * L;
    /* r1 */
    for (long v = 0; v < L; v++) A1[v] = T[v] + (lightsOn && !vox_sinked(&g, v) ? dt * Q[v] : 0);
    apply_D(&g, 0, T, w1);
    for (long v = 0; v < L; v++) A1[v] += dt / 2 * w1[v];
    apply_D(&g, 1, T, w1);
    apply_D(&g, 2, T, w2);
    for (long v = 0; v < L; v++) A1[v] += dt * (w1[v] + w2[v]);
    line_solve(&g, 0, 0, A1, A1);
    for (long v = 0; v < L; v++) A2[v] = A1[v] - dt / 2 * w1[v];
    line_solve(&g, 1, 0, A2, A2);
    for (long v = 0; v < L; v++) Tn1[v] = A2[v] - dt / 2 * w2[v];
    line_solve(&g, 2, 0, Tn1, Tn1);
    for (long v = 0; v < L; v++) {
      double dr;
      if (wd && wd[v] != 0) Jd += wd[v] * dt * damage_rate(&g, logA, E, v, (T[v] + Tn1[v]) / 2, &dr);
      if (Tn1[v] > pk[v]) {
        pk[v] = Tn1[v];
        pkn[v] = n + 1;
      }
    }
  }
  if (wp)
    for (long v = 0; v < L; v++)
      if (wp[v] != 0) Jp += wp[v] * pk[v];
  J[0] = Jd + Jp;
  J[1] = Jd;
  J[2] = Jp;
  if (dc || dQ || dT0) {
    double *lam = (double *)calloc(L, sizeof(double)), *lnew = (double *)malloc(sizeof(double) * L);
    double *r1 = (double *)malloc(sizeof(double) * L), *r2 = (double *)malloc(sizeof(double) * L);
    double *r3 = (double *)malloc(sizeof(double) * L), *gd = (double *)malloc(sizeof(double) * L);
    double *q = (double *)malloc(sizeof(double) * L);
    if (dc) memset(dc, 0, sizeof(double) * nM * nM * 3);
    if (dQ) memset(dQ, 0, sizeof(double) * L);
    for (long n = nt - 1; n >= 0; n--) {
      const double *T = Ts + n * L, *Tn1 = Ts + (n + 1) * L, *A1 = A1s + n * L, *A2 = A2s + n * L;
      for (long v = 0; v < L; v++) {
        double dr = 0;
        gd[v] = 0;
        if (wd && wd[v] != 0) {
          damage_rate(&g, logA, E, v, (T[v] + Tn1[v]) / 2, &dr);
          gd[v] = wd[v] * dt * dr / 2;
        }
        r3[v] = lam[v] + gd[v] + (wp && pkn[v] == n + 1 ? wp[v] : 0);
      }
      line_solve(&g, 2, 1, r3, r3);
      line_solve(&g, 1, 1, r3, r2);
      line_solve(&g, 0, 1, r2, r1);
      for (long v = 0; v < L; v++) lnew[v] = r1[v] + gd[v];
      for (long v = 0; v < L; v++) q[v] = dt / 2 * r1[v];
      add_DT(&g, 0, q, lnew);
      for (long v = 0; v < L; v++) q[v] = dt * r1[v] - dt / 2 * r2[v];
      add_DT(&g, 1, q, lnew);
      for (long v = 0; v < L; v++) q[v] = dt * r1[v] - dt / 2 * r3[v];
      add_DT(&g, 2, q, lnew);
      if (dQ && lightsOn)
        for (long v = 0; v < L; v++)
          if (!vox_sinked(&g, v)) dQ[v] += dt * r1[v];
      if (dc) {
        for (int d = 0; d < 3; d++) {
          const long st = dir_stride(&g, d), nl = dir_len(&g, d);
          for (long v = 0; v < L; v++) {
            if (vox_sinked(&g, v)) continue;
            long p = dir_pos(&g, v, d);
            for (int side = -1; side <= 1; side += 2) {
              if ((side < 0 && p == 0) || (side > 0 && p == nl - 1)) continue;
              long u = v + side * st;
              double contrib;
              if (d == 0) contrib = dt / 2 * r1[v] * ((T[u] + A1[u]) - (T[v] + A1[v]));
              else if (d == 1)
                contrib = dt * r1[v] * (T[u] - T[v]) + dt / 2 * r2[v] * ((A2[u] - T[u]) - (A2[v] - T[v]));
              else
                contrib = dt * r1[v] * (T[u] - T[v]) + dt / 2 * r3[v] * ((Tn1[u] - T[u]) - (Tn1[v] - T[v]));
              dc[M[v] + M[u] * nM + d * (long)nM * nM] += contrib;
            }
          }
        }
      }
      double *t = lam;
      lam = lnew;
      lnew = t;
    }
    if (dT0) memcpy(dT0, lam, sizeof(double) * L);
    free(lam);
    free(lnew);
    free(r1);
    free(r2);
    free(r3);
    free(gd);
    free(q);
  }
  free(logA);
  free(Ts);
  free(A1s);
  free(A2s);
  free(w1);
  free(w2);
  free(pk);
  free(pkn);
  return 0;
}
