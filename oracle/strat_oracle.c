/* CPU FP64 oracle of the forced (stratosphere) RK4 step - TEST
 * INFRASTRUCTURE ONLY, the reference values of the forced step's tests.
 *
 * StratosphereRK4, PanelVelocityParallel.f90:661-919, with one rank: the
 * positions of all three target classes advance by classical RK4 like
 * BVERK4, but the active vorticity is not integrated; each stage's source
 * vorticity is rebuilt from the materially conserved absolute vorticity,
 *     zeta = absVort - 2 Omega z - F(x, t_s),  t_s = t, t + dt/2, t + dt/2, t + dt
 * (:690-694, :752-755, :800-803, :847-850), and after the update the
 * relative vorticity of panels and vertices is set the same way at t + dt
 * (:908-915). F is the Juckes forcing, TracerAndVorticityDistributions.f90:
 * Juckes_Forcing :1213-1221, Juckes_A :550-566, Juckes_BVector :600-611, with
 * Latitude / atan4 from SphereGeom.f90:198-203, :213-248. */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "bve_oracle.h"

static const double PI = 3.141592653589793238462643383279502884;

double or_juckes_a(double t) {
  const double tfull = 4.0, tend = 15.0;
  const double b = PI / tfull;
  if (0.0 <= t && t < tfull) return 0.5 * (1.0 - cos(b * t));
  if (tfull <= t && t < (tend - tfull)) return 1.0;
  if ((tend - tfull) <= t && t < tend) return 0.5 * (1.0 - cos(b * (t - (tend - tfull)) + PI));
  return 0.0;
}

static double juckes_b(double lat) {
  const double th1 = PI / 3.0;
  if (lat <= 0.0) return 0.0;
  const double tan1sq = tan(th1) * tan(th1);
  return tan1sq / (tan(lat) * tan(lat)) * exp(1.0 - tan1sq / (tan(lat) * tan(lat)));
}

static double atan4(double y, double x) {
  if (x == 0.0) {
    if (y > 0.0) return PI / 2.0;
    if (y < 0.0) return 3.0 * PI / 2.0;
    return 0.0;
  }
  if (y == 0.0) return x > 0.0 ? 0.0 : PI;
  const double theta = atan2(fabs(y), fabs(x));
  if (x > 0.0 && y > 0.0) return theta;
  if (x < 0.0 && y > 0.0) return PI - theta;
  if (x < 0.0 && y < 0.0) return PI + theta;
  return 2.0 * PI - theta;
}

double or_juckes_forcing(const double* xyz, double t) {
  const double F0 = 0.3 * 4.0 * PI;
  const double lat = atan2(xyz[2], sqrt(xyz[0] * xyz[0] + xyz[1] * xyz[1]));
  const double lon = atan4(xyz[1], xyz[0]);
  return F0 * or_juckes_a(t) * juckes_b(lat) * cos(lon);
}

static void rel_vort(double* out, const double* absv, const double* x, int n, double omega,
                     double t) {
  for (int j = 0; j < n; ++j)
    out[j] = absv[j] - 2.0 * omega * x[3 * (size_t)j + 2] - or_juckes_forcing(x + 3 * (size_t)j, t);
}

double or_strat_rk4(double* xV, int nV, double* xA, const double* absVortA, double* relVortA,
                    const double* areaA, int nA, double* xQ, int nQ, const double* absVortV,
                    double* relVortV, double t, double dt, double omega, double deltaA,
                    double deltaV, double deltaQ, double* kineticEnergy, int nthreads) {
  const size_t nv3 = 3 * (size_t)nV, na3 = 3 * (size_t)nA, nq3 = 3 * (size_t)nQ;
  double* inV = (double*)malloc(sizeof(double) * (nv3 ? nv3 : 1));
  double* inA = (double*)malloc(sizeof(double) * (na3 ? na3 : 1));
  double* inQ = (double*)malloc(sizeof(double) * (nq3 ? nq3 : 1));
  double* inZ = (double*)malloc(sizeof(double) * (nA ? nA : 1));
  double* dZ = (double*)malloc(sizeof(double) * (nA ? nA : 1));
  double* sV[4];
  double* sA[4];
  double* sQ[4];
  for (int s = 0; s < 4; ++s) {
    sV[s] = (double*)calloc(nv3 ? nv3 : 1, sizeof(double));
    sA[s] = (double*)calloc(na3 ? na3 : 1, sizeof(double));
    sQ[s] = (double*)calloc(nq3 ? nq3 : 1, sizeof(double));
  }
  const double ts[4] = {t, t + 0.5 * dt, t + 0.5 * dt, t + dt};
  double totalKE = 0.0;
  for (int s = 0; s < 4; ++s) {
    if (s == 0) {
      memcpy(inV, xV, sizeof(double) * nv3);
      memcpy(inA, xA, sizeof(double) * na3);
      memcpy(inQ, xQ, sizeof(double) * nq3);
    } else if (s < 3) {
      for (size_t i = 0; i < nv3; ++i) inV[i] = xV[i] + 0.5 * sV[s - 1][i];
      for (size_t i = 0; i < na3; ++i) inA[i] = xA[i] + 0.5 * sA[s - 1][i];
      for (size_t i = 0; i < nq3; ++i) inQ[i] = xQ[i] + 0.5 * sQ[s - 1][i];
    } else {
      for (size_t i = 0; i < nv3; ++i) inV[i] = xV[i] + sV[2][i];
      for (size_t i = 0; i < na3; ++i) inA[i] = xA[i] + sA[2][i];
      for (size_t i = 0; i < nq3; ++i) inQ[i] = xQ[i] + sQ[2][i];
    }
    rel_vort(inZ, absVortA, inA, nA, omega, ts[s]);
    or_bve_stage(inA, inZ, areaA, nA, inV, nV, inQ, nQ, omega, deltaA, deltaV, deltaQ, 0, nA, 0,
                 nV, 0, nQ, sA[s], dZ, sV[s], sQ[s], nthreads);
    if (s == 0) {
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
  }
  for (size_t i = 0; i < nv3; ++i)
    xV[i] = xV[i] + sV[0][i] / 6.0 + sV[1][i] / 3.0 + sV[2][i] / 3.0 + sV[3][i] / 6.0;
  for (size_t i = 0; i < na3; ++i)
    xA[i] = xA[i] + sA[0][i] / 6.0 + sA[1][i] / 3.0 + sA[2][i] / 3.0 + sA[3][i] / 6.0;
  for (size_t i = 0; i < nq3; ++i)
    xQ[i] = xQ[i] + sQ[0][i] / 6.0 + sQ[1][i] / 3.0 + sQ[2][i] / 3.0 + sQ[3][i] / 6.0;
  if (relVortA) rel_vort(relVortA, absVortA, xA, nA, omega, t + dt);
  if (absVortV && relVortV) rel_vort(relVortV, absVortV, xV, nV, omega, t + dt);
  for (int s = 0; s < 4; ++s) {
    free(sV[s]);
    free(sA[s]);
    free(sQ[s]);
  }
  free(inV);
  free(inA);
  free(inQ);
  free(inZ);
  free(dZ);
  return totalKE;
}
