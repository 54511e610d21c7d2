/*
 * bve_oracle.c - CPU FP64 restatement of the reference's Biot-Savart sums and
 * RK4 driver. TEST INFRASTRUCTURE ONLY (the parity tests' reference values and
 * the timed CPU baseline); see bve_oracle.h for the parity status (pinned bit for
 * bit to the reference's own Fortran statements, run through oracle/f90).
 *
 * Every arithmetic expression keeps the reference's operand order so that a
 * strict IEEE build (gcc -O2 -ffp-contract=off, SSE2) rounds exactly as the
 * Fortran source reads:
 *   sum(a(:)*b(:))            -> ((a1*b1 + a2*b2) + a3*b3)
 *   c*vort(k)*area(k)/denom   -> (((c*vort)*area)/denom)
 *   dX/(-4.0*PI)              -> division by the double -4*pi
 *   x + s1/6 + s2/3 + ...     -> left-to-right additions of the quotients
 */
#include "bve_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* NumberKinds.f90:11 PI, rounded to double. */
static const double kPi = 3.141592653589793238462643383279502797479068098137295573004504331874296718662975536062731407582759857177734375;

/* ---------------------------------------------------------------------- */
/* Row kernels: one target row summed over all sources in ascending k.      */
/* ---------------------------------------------------------------------- */

/* Body of BVEActiveRHS for target j (PanelVelocityParallel.f90:1316-1330):
 * the two k loops skip k == j; the sums run in ascending k. */
static void active_row(const double* pv, const double* vort, const double* area, int nn, int j,
                       double d2, double out[3]) {
  const double* pj = pv + 3 * (size_t)j;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int pass = 0; pass < 2; ++pass) {
    int k0 = pass == 0 ? 0 : j + 1;
    int k1 = pass == 0 ? j : nn;
    for (int k = k0; k < k1; ++k) {
      const double* pk = pv + 3 * (size_t)k;
      double s = pk[0] * pj[0];
      s = s + pk[1] * pj[1];
      s = s + pk[2] * pj[2];
      double denom = 1.0 - s;
      if (d2 != 0.0) denom = denom + d2;
      a0 = a0 + (pj[1] * pk[2] - pj[2] * pk[1]) * vort[k] * area[k] / denom;
      a1 = a1 + (pj[2] * pk[0] - pj[0] * pk[2]) * vort[k] * area[k] / denom;
      a2 = a2 + (pj[0] * pk[1] - pj[1] * pk[0]) * vort[k] * area[k] / denom;
    }
  }
  out[0] = a0;
  out[1] = a1;
  out[2] = a2;
}

/* Body of BVEPassiveRHS (:1364-1371, d2 = 0) and BVESmoothVelocity
 * (:1403-1410, d2 = smooth*smooth): target X(:,j), all k. */
static void point_row(const double* X, const double* pv, const double* vort, const double* area,
                      int nn, int j, double d2, double out[3]) {
  const double* xj = X + 3 * (size_t)j;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int k = 0; k < nn; ++k) {
    const double* pk = pv + 3 * (size_t)k;
    double s = pk[0] * xj[0];
    s = s + pk[1] * xj[1];
    s = s + pk[2] * xj[2];
    double denom = 1.0 - s;
    if (d2 != 0.0) denom = denom + d2;
    a0 = a0 + (xj[1] * pk[2] - xj[2] * pk[1]) * vort[k] * area[k] / denom;
    a1 = a1 + (xj[2] * pk[0] - xj[0] * pk[2]) * vort[k] * area[k] / denom;
    a2 = a2 + (xj[0] * pk[1] - xj[1] * pk[0]) * vort[k] * area[k] / denom;
  }
  out[0] = a0;
  out[1] = a1;
  out[2] = a2;
}

/* ---------------------------------------------------------------------- */
/* Row-parallel driver: contiguous blocks of rows per thread, so results    */
/* never depend on the thread count (rows are independent).                 */
/* ---------------------------------------------------------------------- */

typedef struct {
  int cls; /* 0 active, 1 point */
  const int* rows; /* NULL: rows are r0..r1-1 */
  int r0, r1;
  const double* X;
  const double* pv;
  const double* vort;
  const double* area;
  int nn;
  double d2;
  double* out;  /* rows given: out[3*r]; else out[3*j] */
} row_job;

static void* row_worker(void* arg) {
  row_job* jb = (row_job*)arg;
  for (int r = jb->r0; r < jb->r1; ++r) {
    int j = jb->rows ? jb->rows[r] : r;
    double* dst = jb->out + 3 * (size_t)r;
    if (jb->cls == 0)
      active_row(jb->pv, jb->vort, jb->area, jb->nn, j, jb->d2, dst);
    else
      point_row(jb->X, jb->pv, jb->vort, jb->area, jb->nn, j, jb->d2, dst);
  }
  return NULL;
}

static void run_rows(int cls, const int* rows, int r0, int r1, const double* X, const double* pv,
                     const double* vort, const double* area, int nn, double d2, double* out,
                     int nthreads) {
  int n = r1 - r0;
  if (n <= 0) return;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > n) nthreads = n;
  row_job* jobs = (row_job*)calloc((size_t)nthreads, sizeof(row_job));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  int* start = (int*)calloc((size_t)nthreads, sizeof(int));
  int* end = (int*)calloc((size_t)nthreads, sizeof(int));
  or_load_balance(n, nthreads, start, end);
  for (int t = 0; t < nthreads; ++t) {
    row_job jb = {cls, rows, r0 + start[t], r0 + end[t], X, pv, vort, area, nn, d2, out};
    jobs[t] = jb;
  }
  for (int t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, row_worker, &jobs[t]);
  row_worker(&jobs[0]);
  for (int t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
  free(jobs);
  free(th);
  free(start);
  free(end);
}

/* ---------------------------------------------------------------------- */
/* The reference routines.                                                  */
/* ---------------------------------------------------------------------- */

static void scale_minus_4pi(double* a, size_t n) {
  const double s = -4.0 * kPi;
  for (size_t i = 0; i < n; ++i) a[i] = a[i] / s;
}

static void active_rhs_mt(double* dX, double* dVort, const double* pv, const double* vort,
                          const double* area, int nn, int i0, int i1, double omega, double delta,
                          int nthreads) {
  memset(dX, 0, sizeof(double) * 3 * (size_t)nn);
  memset(dVort, 0, sizeof(double) * (size_t)nn);
  run_rows(0, NULL, i0, i1, NULL, pv, vort, area, nn, delta * delta, dX, nthreads);
  scale_minus_4pi(dX, 3 * (size_t)nn);
  for (int j = 0; j < nn; ++j) dVort[j] = -2.0 * omega * dX[3 * (size_t)j + 2];
}

void or_active_rhs(double* dX, double* dVort, const double* pv, const double* vort,
                   const double* area, int nn, int i0, int i1, double omega, double delta) {
  active_rhs_mt(dX, dVort, pv, vort, area, nn, i0, i1, omega, delta, 1);
}

static void point_rhs_mt(double* dX, const double* X, int mm, const double* pv,
                         const double* vort, const double* area, int nn, int i0, int i1,
                         double delta, int nthreads) {
  memset(dX, 0, sizeof(double) * 3 * (size_t)mm);
  run_rows(1, NULL, i0, i1, X, pv, vort, area, nn, delta * delta, dX, nthreads);
  scale_minus_4pi(dX, 3 * (size_t)mm);
}

void or_passive_rhs(double* dX, const double* X, int mm, const double* pv, const double* vort,
                    const double* area, int nn, int i0, int i1) {
  point_rhs_mt(dX, X, mm, pv, vort, area, nn, i0, i1, 0.0, 1);
}

void or_smooth_velocity(double* dX, const double* X, int mm, const double* pv,
                        const double* vort, const double* area, int nn, int i0, int i1,
                        double smooth) {
  point_rhs_mt(dX, X, mm, pv, vort, area, nn, i0, i1, smooth, 1);
}

void or_voronoi_velocity(double* dx, double* dy, double* dz, double* dVort, const double* x,
                         const double* y, const double* z, const double* vort,
                         const double* area, int nn, int i0, int i1, double omega) {
  /* VoronoiVelocityParallel.f90:494 zeroes dx only; dy and dz keep what
   * the caller had (ZeroRK4 zeroes them between steps). */
  memset(dx, 0, sizeof(double) * (size_t)nn);
  for (int j = i0; j < i1; ++j) {
    double a0 = dx[j], a1 = dy[j], a2 = dz[j];
    for (int pass = 0; pass < 2; ++pass) {
      int k0 = pass == 0 ? 0 : j + 1;
      int k1 = pass == 0 ? j : nn;
      for (int k = k0; k < k1; ++k) {
        double denom = 1.0 - x[j] * x[k] - y[j] * y[k] - z[j] * z[k];
        a0 = a0 + (y[j] * z[k] - z[j] * y[k]) * vort[k] * area[k] / denom;
        a1 = a1 + (z[j] * x[k] - x[j] * z[k]) * vort[k] * area[k] / denom;
        a2 = a2 + (x[j] * y[k] - y[j] * x[k]) * vort[k] * area[k] / denom;
      }
    }
    dx[j] = a0;
    dy[j] = a1;
    dz[j] = a2;
  }
  const double s = -4.0 * kPi;
  for (int j = 0; j < nn; ++j) {
    dx[j] = dx[j] / s;
    dy[j] = dy[j] / s;
    dz[j] = dz[j] / s;
  }
  for (int j = 0; j < nn; ++j) dVort[j] = -2.0 * omega * dz[j];
}

void or_rows(int cls, const int* rows, int nrows, const double* X, const double* pv,
             const double* vort, const double* area, int nn, double delta, double* out,
             int nthreads) {
  run_rows(cls == 0 ? 0 : 1, rows, 0, nrows, X, pv, vort, area, nn, delta * delta, out, nthreads);
  scale_minus_4pi(out, 3 * (size_t)nrows);
}

void or_load_balance(int n, int p, int* start, int* end) {
  int chunk = n / p;
  for (int j = 0; j < p; ++j) {
    start[j] = j * chunk;
    end[j] = (j + 1) * chunk;
  }
  end[p - 1] = n;
}

void or_bve_stage(const double* xA, const double* zetaA, const double* areaA, int nA,
                  const double* xV, int nV, const double* xQ, int nQ, double omega,
                  double deltaA, double deltaV, double deltaQ, int a0, int a1, int v0,
                  int v1, int q0, int q1, double* dXA, double* dVortA, double* dXV,
                  double* dXQ, int nthreads) {
  active_rhs_mt(dXA, dVortA, xA, zetaA, areaA, nA, a0, a1, omega, deltaA, nthreads);
  point_rhs_mt(dXV, xV, nV, xA, zetaA, areaA, nA, v0, v1, deltaV, nthreads);
  point_rhs_mt(dXQ, xQ, nQ, xA, zetaA, areaA, nA, q0, q1, deltaQ, nthreads);
}

/* BVERK4, PanelVelocityParallel.f90:435-658 (one rank). */
double or_bve_rk4(double* xV, int nV, double* xA, double* zetaA, const double* areaA, int nA,
                  double* xQ, int nQ, double dt, double omega, double deltaA, double deltaV,
                  double deltaQ, const double* absVortV, double* relVortV,
                  double* kineticEnergy, int nthreads) {
  const size_t nv3 = 3 * (size_t)nV, na3 = 3 * (size_t)nA, nq3 = 3 * (size_t)nQ;
  double* inV = (double*)malloc(sizeof(double) * (nv3 ? nv3 : 1));
  double* inA = (double*)malloc(sizeof(double) * (na3 ? na3 : 1));
  double* inQ = (double*)malloc(sizeof(double) * (nq3 ? nq3 : 1));
  double* inZ = (double*)malloc(sizeof(double) * (nA ? nA : 1));
  double* sV[4];
  double* sA[4];
  double* sQ[4];
  double* sZ[4];
  for (int s = 0; s < 4; ++s) {
    sV[s] = (double*)calloc(nv3 ? nv3 : 1, sizeof(double));
    sA[s] = (double*)calloc(na3 ? na3 : 1, sizeof(double));
    sQ[s] = (double*)calloc(nq3 ? nq3 : 1, sizeof(double));
    sZ[s] = (double*)calloc(nA ? nA : 1, sizeof(double));
  }
  double totalKE = 0.0;
  /* stage input coefficient applied to the previous stage: 0, 1/2, 1/2, 1
   * (:458-462, :513-516, :555-558, :597-600) */
  for (int s = 0; s < 4; ++s) {
    if (s == 0) {
      memcpy(inV, xV, sizeof(double) * nv3);
      memcpy(inA, xA, sizeof(double) * na3);
      memcpy(inQ, xQ, sizeof(double) * nq3);
      memcpy(inZ, zetaA, sizeof(double) * (size_t)nA);
    } else if (s < 3) {
      for (size_t i = 0; i < nv3; ++i) inV[i] = xV[i] + 0.5 * sV[s - 1][i];
      for (size_t i = 0; i < na3; ++i) inA[i] = xA[i] + 0.5 * sA[s - 1][i];
      for (size_t i = 0; i < nq3; ++i) inQ[i] = xQ[i] + 0.5 * sQ[s - 1][i];
      for (int i = 0; i < nA; ++i) inZ[i] = zetaA[i] + 0.5 * sZ[s - 1][i];
    } else {
      for (size_t i = 0; i < nv3; ++i) inV[i] = xV[i] + sV[2][i];
      for (size_t i = 0; i < na3; ++i) inA[i] = xA[i] + sA[2][i];
      for (size_t i = 0; i < nq3; ++i) inQ[i] = xQ[i] + sQ[2][i];
      for (int i = 0; i < nA; ++i) inZ[i] = zetaA[i] + sZ[2][i];
    }
    or_bve_stage(inA, inZ, areaA, nA, inV, nV, inQ, nQ, omega, deltaA, deltaV, deltaQ, 0, nA, 0,
                 nV, 0, nQ, sA[s], sZ[s], sV[s], sQ[s], nthreads);
    if (s == 0) {
      /* kinetic energy, stage 1 only (:495-501) */
      double acc = 0.0;
      for (int j = 0; j < nA; ++j) {
        const double* u = sA[0] + 3 * (size_t)j;
        double ke = u[0] * u[0];
        ke = ke + u[1] * u[1];
        ke = ke + u[2] * u[2];
        if (kineticEnergy) kineticEnergy[j] = ke;
        acc = acc + ke * areaA[j];
      }
      totalKE = 0.5 * acc;
    }
    for (size_t i = 0; i < nv3; ++i) sV[s][i] = dt * sV[s][i];
    for (size_t i = 0; i < na3; ++i) sA[s][i] = dt * sA[s][i];
    for (size_t i = 0; i < nq3; ++i) sQ[s][i] = dt * sQ[s][i];
    for (int i = 0; i < nA; ++i) sZ[s][i] = dt * sZ[s][i];
  }
  /* position update (:637-644) and copy back (:650-654) */
  for (size_t i = 0; i < nv3; ++i)
    xV[i] = xV[i] + sV[0][i] / 6.0 + sV[1][i] / 3.0 + sV[2][i] / 3.0 + sV[3][i] / 6.0;
  for (size_t i = 0; i < na3; ++i)
    xA[i] = xA[i] + sA[0][i] / 6.0 + sA[1][i] / 3.0 + sA[2][i] / 3.0 + sA[3][i] / 6.0;
  for (size_t i = 0; i < nq3; ++i)
    xQ[i] = xQ[i] + sQ[0][i] / 6.0 + sQ[1][i] / 3.0 + sQ[2][i] / 3.0 + sQ[3][i] / 6.0;
  for (int i = 0; i < nA; ++i)
    zetaA[i] = zetaA[i] + sZ[0][i] / 6.0 + sZ[1][i] / 3.0 + sZ[2][i] / 3.0 + sZ[3][i] / 6.0;
  if (absVortV && relVortV)
    for (int j = 0; j < nV; ++j) relVortV[j] = absVortV[j] - 2.0 * omega * xV[3 * (size_t)j + 2];
  for (int s = 0; s < 4; ++s) {
    free(sV[s]);
    free(sA[s]);
    free(sQ[s]);
    free(sZ[s]);
  }
  free(inV);
  free(inA);
  free(inQ);
  free(inZ);
  return totalKE;
}
