/* A compiled host program driving the C ABI the way a Fortran BVE driver
 * drives PanelVelocityParallelModule (RHWavePanelsMPI.f90: NewGrid, initial
 * vorticity, InitializeMPIRK4, BVERK4 steps): icosahedral grid from the
 * library, GatherPanels maps, Rossby-Haurwitz wave-4 vorticity at the
 * active panels, nsteps fused RK4 steps, and checks that hold for the exact
 * flow (velocity tangent to the sphere, kinetic energy positive and nearly
 * conserved). With a CHECKPOINT path it also stops a device-resident run
 * halfway, saves it (tc_rk4_save), restores it into a new context
 * (tc_rk4_restore) and checks that the continued run ends bit for bit where
 * the uninterrupted one does. Exit status 0 = pass, 1 = check failed, 2 =
 * library error, 3 = no GPU (the library reports a CUDA error from tc_create).
 *
 * usage: bve_driver LEVEL NSTEPS PRECISION(0 = FP64, 1 = FP32C) [CHECKPOINT] */
#define _DEFAULT_SOURCE /* M_PI */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "thesiscode_b200.h"

#define CHECK(call)                                                      \
  do {                                                                   \
    int rc_ = (call);                                                    \
    if (rc_ != TC_OK) {                                                  \
      fprintf(stderr, "%s -> %d: %s\n", #call, rc_, tc_last_error());   \
      return rc_ == TC_ERR_CUDA ? 3 : 2;                                 \
    }                                                                    \
  } while (0)

int main(int argc, char** argv) {
  const int level = argc > 1 ? atoi(argv[1]) : 3;
  const int nsteps = argc > 2 ? atoi(argv[2]) : 4;
  const int precision = argc > 3 ? atoi(argv[3]) : TC_FP64;
  int np, ne, npan, nact;
  CHECK(tc_icos_grid_sizes(level, &np, &ne, &npan, &nact));
  double* px = malloc(sizeof(double) * 3 * np);
  double* px0 = malloc(sizeof(double) * 3 * np);
  double* qx = malloc(sizeof(double) * 3 * npan);
  double* qx0 = malloc(sizeof(double) * 3 * npan);
  double* qarea = malloc(sizeof(double) * npan);
  int* has_children = malloc(sizeof(int) * npan);
  int* verts = malloc(sizeof(int) * 3 * npan);
  int* nest = malloc(sizeof(int) * npan);
  int* children = malloc(sizeof(int) * 4 * npan);
  CHECK(tc_icos_grid(level, px, px0, qx, qx0, qarea, has_children, verts, nest, children));
  const int npas = npan - nact;
  int* amap = malloc(sizeof(int) * nact);
  int* pmap = malloc(sizeof(int) * (npas > 0 ? npas : 1));
  CHECK(tc_gather_maps(npan, has_children, amap, nact, pmap, npas));
  double* xA = malloc(sizeof(double) * 3 * nact);
  double* zA = malloc(sizeof(double) * nact);
  double* aA = malloc(sizeof(double) * nact);
  double* xQ = malloc(sizeof(double) * 3 * (npas > 0 ? npas : 1));
  const double Omega = 2.0 * M_PI, w = Omega / 14.0, K = Omega / 14.0;
  double area_sum = 0.0;
  for (int j = 0; j < nact; ++j) {
    const int p = amap[j];
    for (int c = 0; c < 3; ++c) xA[3 * j + c] = qx[3 * p + c];
    aA[j] = qarea[p];
    area_sum += aA[j];
    const double z = xA[3 * j + 2], lon = atan2(xA[3 * j + 1], xA[3 * j]);
    const double c2 = 1.0 - z * z;
    zA[j] = 2.0 * w * z - K * z * c2 * c2 * 30.0 * cos(4.0 * lon);
  }
  for (int j = 0; j < npas; ++j)
    for (int c = 0; c < 3; ++c) xQ[3 * j + c] = qx[3 * pmap[j] + c];
  if (fabs(area_sum - 4.0 * M_PI) > 1e-10) {
    fprintf(stderr, "total area %.15f != 4 pi\n", area_sum);
    return 1;
  }
  tc_ctx* ctx = NULL;
  CHECK(tc_create(0, precision, &ctx));
  CHECK(tc_set_omega(ctx, Omega));
  /* one BVEActiveRHS: tangency u.x = 0 */
  double* dX = malloc(sizeof(double) * 3 * nact);
  double* dV = malloc(sizeof(double) * nact);
  CHECK(tc_bs_velocity(ctx, TC_ACTIVE, NULL, nact, xA, zA, aA, nact, 0, nact, dX, dV));
  double umax = 0.0, dotmax = 0.0;
  for (int j = 0; j < nact; ++j) {
    const double* u = dX + 3 * j;
    const double un = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double d = u[0] * xA[3 * j] + u[1] * xA[3 * j + 1] + u[2] * xA[3 * j + 2];
    if (un > umax) umax = un;
    if (fabs(d) > dotmax) dotmax = fabs(d);
  }
  const double tang_tol = precision == TC_FP64 ? 1e-13 : 1e-6;
  if (!(umax > 0.0) || dotmax > tang_tol * umax) {
    fprintf(stderr, "tangency: max |u.x| = %g, max |u| = %g\n", dotmax, umax);
    return 1;
  }
  /* checkpoint round trip of the device-resident state */
  if (argc > 4 && nsteps >= 2) {
    const char* path = argv[4];
    const size_t bA = sizeof(double) * 3 * nact, bz = sizeof(double) * nact,
                 bV = sizeof(double) * 3 * np, bQ = sizeof(double) * 3 * (npas > 0 ? npas : 1);
    double *sA = malloc(bA), *sz = malloc(bz), *sV = malloc(bV), *sQ = malloc(bQ);
    double *rA = malloc(bA), *rz = malloc(bz), *rV = malloc(bV), *rQ = malloc(bQ);
    CHECK(tc_rk4_load(ctx, xA, zA, aA, nact, px, np, xQ, npas, 0));
    CHECK(tc_rk4_advance(ctx, 0.01, nsteps, NULL));
    CHECK(tc_rk4_store(ctx, sA, sz, sV, sQ, NULL, 0));
    CHECK(tc_rk4_load(ctx, xA, zA, aA, nact, px, np, xQ, npas, 0));
    CHECK(tc_rk4_advance(ctx, 0.01, nsteps / 2, NULL));
    CHECK(tc_rk4_save(ctx, path));
    tc_ctx* ctx2 = NULL;
    CHECK(tc_create(0, precision, &ctx2));
    CHECK(tc_rk4_restore(ctx2, path));
    CHECK(tc_rk4_advance(ctx2, 0.01, nsteps - nsteps / 2, NULL));
    CHECK(tc_rk4_store(ctx2, rA, rz, rV, rQ, NULL, 0));
    long long done = 0;
    CHECK(tc_rk4_steps_done(ctx2, &done));
    CHECK(tc_destroy(ctx2));
    if (done != nsteps || memcmp(sA, rA, bA) || memcmp(sz, rz, bz) || memcmp(sV, rV, bV) ||
        (npas > 0 && memcmp(sQ, rQ, sizeof(double) * 3 * npas))) {
      fprintf(stderr, "checkpoint: the restored run differs from the uninterrupted one\n");
      return 1;
    }
    printf("checkpoint round trip after %d of %d steps: identical\n", nsteps / 2, nsteps);
    free(sA), free(sz), free(sV), free(sQ), free(rA), free(rz), free(rV), free(rQ);
  }
  /* BVERK4 steps, fused on the device */
  double* tke = malloc(sizeof(double) * nsteps);
  CHECK(tc_rk4_step(ctx, xA, zA, aA, nact, px, np, xQ, npas, 0.01, nsteps, tke, NULL));
  for (int s = 0; s < nsteps; ++s) {
    if (!(tke[s] > 0.0) || fabs(tke[s] - tke[0]) > 1e-4 * tke[0]) {
      fprintf(stderr, "kinetic energy step %d: %.15g (first %.15g)\n", s, tke[s], tke[0]);
      return 1;
    }
  }
  CHECK(tc_destroy(ctx));
  printf("bve_driver level %d: %d active panels, %d steps, totalKE %.12f -> %.12f\n", level, nact,
         nsteps, tke[0], tke[nsteps - 1]);
  return 0;
}
