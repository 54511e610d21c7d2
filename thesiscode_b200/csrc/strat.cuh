// Juckes stratospheric forcing F(x, t) of the forced barotropic model
// (StratosphereRK4, PanelVelocityParallel.f90:661-919): the relative
// vorticity fed to the Biot-Savart sum at each RK4 stage is
//     zeta = absVort - 2 Omega z - F(x, t_stage).
// Restated from the formulas of TracerAndVorticityDistributions.f90:
//     F(x, t) = F0 A(t) B(lat) cos(lon),  F0 = 0.3 * 4 pi       (:1213-1221)
//     A(t)    = (1 - cos(pi t / 4)) / 2               0 <= t < 4
//               1                                      4 <= t < 11
//               (1 - cos(pi (t - 11) / 4 + pi)) / 2    11 <= t < 15
//               0                                      otherwise    (:550-566)
//     B(lat)  = 0 for lat <= 0, else q e^(1 - q),  q = tan^2(pi/3) / tan^2(lat)  (:600-611)
// with lat = atan2(z, sqrt(x^2 + y^2)) (SphereGeom.f90:198-203) and lon in
// [0, 2 pi) by the quadrant rules of atan4 (SphereGeom.f90:213-248).
// Transcendentals are CUDA's double-precision functions.
#pragma once

namespace tcb {

constexpr double kPi = 3.141592653589793238462643383279502884;

__host__ __device__ inline double juckes_a(double t) {
  const double tfull = 4.0, tend = 15.0, b = kPi / tfull;
  if (0.0 <= t && t < tfull) return 0.5 * (1.0 - cos(b * t));
  if (tfull <= t && t < tend - tfull) return 1.0;
  if (tend - tfull <= t && t < tend) return 0.5 * (1.0 - cos(b * (t - (tend - tfull)) + kPi));
  return 0.0;
}

__host__ __device__ inline double juckes_b(double lat) {
  if (lat <= 0.0) return 0.0;
  const double th1 = kPi / 3.0;
  const double tan1sq = tan(th1) * tan(th1);
  const double tl = tan(lat);
  return tan1sq / (tl * tl) * exp(1.0 - tan1sq / (tl * tl));
}

// atan2 mapped to [0, 2 pi) with the quadrant rules of atan4.
__host__ __device__ inline double atan4(double y, double x) {
  if (x == 0.0) {
    if (y > 0.0) return kPi / 2.0;
    if (y < 0.0) return 3.0 * kPi / 2.0;
    return 0.0;
  }
  if (y == 0.0) return x > 0.0 ? 0.0 : kPi;
  const double theta = atan2(fabs(y), fabs(x));
  if (x > 0.0 && y > 0.0) return theta;
  if (x < 0.0 && y > 0.0) return kPi - theta;
  if (x < 0.0 && y < 0.0) return kPi + theta;
  return 2.0 * kPi - theta;
}

__host__ __device__ inline double juckes_forcing(double x, double y, double z, double t) {
  const double F0 = 0.3 * 4.0 * kPi;
  const double lat = atan2(z, sqrt(x * x + y * y));
  const double lon = atan4(y, x);
  return F0 * juckes_a(t) * juckes_b(lat) * cos(lon);
}

// The relative vorticity of a forced-model stage input, evaluated in the
// reference's order: (absVort - (2 Omega) z) - F(x, t).
__host__ __device__ inline double strat_rel_vort(double abs_vort, double two_omega, double x,
                                                 double y, double z, double t) {
  return (abs_vort - two_omega * z) - juckes_forcing(x, y, z, t);
}

}  // namespace tcb
