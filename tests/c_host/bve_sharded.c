/* A compiled host program that shards BVERK4 over ranks the way the
 * reference does (PanelVelocityParallel.f90:435-658): every rank holds the
 * whole state, computes the LoadBalance rows of each target class
 * (:167-213) for each RK4 stage, and after each stage the ranks exchange
 * rows (the reference broadcasts every rank's velocity rows, :476-489; here
 * only the next stage's packed source rows of the active panels travel).
 * Ranks are threads and the exchange is an all-gather through host memory
 * with barriers - the sequence of C-ABI calls and the data an MPI host
 * (the Fortran shim, fortran/PanelVelocityCUDA.f90) moves with
 * MPI_Allgatherv. Rank r uses device r % (number of devices).
 *
 * usage: bve_sharded IN OUT nA nV nQ NSTEPS PRECISION NRANKS DT OMEGA D_A D_V D_Q
 *   IN:  xA(3,nA) zetaA(nA) areaA(nA) xV(3,nV) xQ(3,nQ), raw doubles
 *   OUT: xA zetaA xV xQ after NSTEPS steps, then totalKE of each step
 *        (0.5 * sum(kineticEnergy * area) over all rows, as :495-501)
 * Exit status: 0 ok, 2 library error, 3 CUDA error (no GPU), 4 I/O. */
#define _DEFAULT_SOURCE
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "thesiscode_b200.h"

typedef struct {
  int nA, nV, nQ, nsteps, precision, nranks;
  double dt, omega, delta[3];
  double *xA, *zA, *aA, *xV, *xQ;    /* initial state (read by every rank) */
  double* src;                       /* all-gather buffer: packed sources, 4 doubles per row */
  double *fxA, *fzA, *fxV, *fxQ, *ke; /* gathered final state and stage-1 kinetic energy */
  double* tke;                       /* totalKE per step */
  int *a0, *a1, *v0, *v1, *q0, *q1;  /* LoadBalance ranges per rank */
  pthread_barrier_t bar;
  int status[64];
} Job;

typedef struct {
  Job* job;
  int rank;
} RankArg;

#define TRY(call)                                                           \
  do {                                                                      \
    int rc_ = (call);                                                       \
    if (rc_ != TC_OK) {                                                     \
      fprintf(stderr, "rank %d: %s -> %d: %s\n", r, #call, rc_, tc_last_error()); \
      failed = rc_ == TC_ERR_CUDA ? 3 : 2;                                  \
    }                                                                       \
  } while (0)

/* Every rank: export its rows of `which` into `buf`, wait for all, import the
 * other ranks' rows. Calls are skipped after a failure, but every rank still
 * reaches both barriers, so no rank waits forever on a failed one. */
static void allgather_rows(Job* J, tc_ctx* ctx, int r, int which, int width, const int* s,
                           const int* e, double* buf, int* failed_io) {
  int failed = *failed_io;
  if (!failed && e[r] > s[r])
    TRY(tc_rk4_copy_rows(ctx, which, s[r], e[r] - s[r], buf + (size_t)width * s[r], 0));
  if (!failed) TRY(tc_synchronize(ctx));
  pthread_barrier_wait(&J->bar);
  for (int q = 0; q < J->nranks && !failed; ++q)
    if (q != r && e[q] > s[q])
      TRY(tc_rk4_copy_rows(ctx, which, s[q], e[q] - s[q], buf + (size_t)width * s[q], 1));
  if (!failed) TRY(tc_synchronize(ctx));
  pthread_barrier_wait(&J->bar); /* nobody overwrites buf before everyone has read it */
  *failed_io = failed;
}

static void* rank_main(void* p) {
  RankArg* A = (RankArg*)p;
  Job* J = A->job;
  const int r = A->rank;
  int failed = 0, ndev = 1;
  tc_ctx* ctx = NULL;
  TRY(tc_device_count(&ndev));
  if (!failed) TRY(tc_create(r % (ndev > 0 ? ndev : 1), J->precision, &ctx));
  if (!failed) TRY(tc_set_omega(ctx, J->omega));
  if (!failed) TRY(tc_set_deltas(ctx, J->delta[0], J->delta[1], J->delta[2]));
  if (!failed)
    TRY(tc_rk4_load(ctx, J->xA, J->zA, J->aA, J->nA, J->xV, J->nV, J->nQ ? J->xQ : NULL, J->nQ, 0));
  if (!failed) TRY(tc_rk4_pack_sources(ctx));
  for (int step = 0; step < J->nsteps; ++step) {
    for (int stage = 0; stage < 4; ++stage) {
      if (!failed)
        TRY(tc_rk4_stage_range(ctx, stage, J->dt, J->a0[r], J->a1[r], J->v0[r], J->v1[r], J->q0[r],
                               J->q1[r], NULL));
      allgather_rows(J, ctx, r, TC_BUF_SOURCES, 4, J->a0, J->a1, J->src, &failed);
      if (stage == 0) {
        /* kinetic energy of stage 1: each rank's rows, gathered, summed like :500 */
        allgather_rows(J, ctx, r, TC_BUF_KE, 1, J->a0, J->a1, J->ke, &failed);
        if (r == 0) {
          double s = 0.0;
          for (int j = 0; j < J->nA; ++j) s += J->ke[j] * J->aA[j];
          J->tke[step] = 0.5 * s;
        }
      }
    }
  }
  /* the final state of every class, gathered (ScatterPanels needs all rows) */
  allgather_rows(J, ctx, r, TC_BUF_XA, 3, J->a0, J->a1, J->fxA, &failed);
  allgather_rows(J, ctx, r, TC_BUF_ZETA, 1, J->a0, J->a1, J->fzA, &failed);
  allgather_rows(J, ctx, r, TC_BUF_XV, 3, J->v0, J->v1, J->fxV, &failed);
  if (J->nQ) allgather_rows(J, ctx, r, TC_BUF_XQ, 3, J->q0, J->q1, J->fxQ, &failed);
  if (ctx) tc_destroy(ctx);
  J->status[r] = failed;
  return NULL;
}

static double* alloc_doubles(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

int main(int argc, char** argv) {
  if (argc != 14) {
    fprintf(stderr, "usage: %s IN OUT nA nV nQ NSTEPS PRECISION NRANKS DT OMEGA D_A D_V D_Q\n", argv[0]);
    return 4;
  }
  Job J;
  memset(&J, 0, sizeof J);
  J.nA = atoi(argv[3]);
  J.nV = atoi(argv[4]);
  J.nQ = atoi(argv[5]);
  J.nsteps = atoi(argv[6]);
  J.precision = atoi(argv[7]);
  J.nranks = atoi(argv[8]);
  J.dt = atof(argv[9]);
  J.omega = atof(argv[10]);
  for (int c = 0; c < 3; ++c) J.delta[c] = atof(argv[11 + c]);
  if (J.nranks < 1 || J.nranks > 64 || J.nA < 1 || J.nV < 0 || J.nQ < 0 || J.nsteps < 1) return 4;
  J.xA = alloc_doubles(3 * (size_t)J.nA);
  J.zA = alloc_doubles(J.nA);
  J.aA = alloc_doubles(J.nA);
  J.xV = alloc_doubles(3 * (size_t)J.nV);
  J.xQ = alloc_doubles(3 * (size_t)J.nQ);
  J.src = alloc_doubles(4 * (size_t)J.nA);
  J.fxA = alloc_doubles(3 * (size_t)J.nA);
  J.fzA = alloc_doubles(J.nA);
  J.fxV = alloc_doubles(3 * (size_t)J.nV);
  J.fxQ = alloc_doubles(3 * (size_t)J.nQ);
  J.ke = alloc_doubles(J.nA);
  J.tke = alloc_doubles(J.nsteps);
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 4;
  size_t got = fread(J.xA, sizeof(double), 3 * (size_t)J.nA, f) + fread(J.zA, sizeof(double), J.nA, f) +
               fread(J.aA, sizeof(double), J.nA, f) + fread(J.xV, sizeof(double), 3 * (size_t)J.nV, f) +
               fread(J.xQ, sizeof(double), 3 * (size_t)J.nQ, f);
  fclose(f);
  if (got != 5 * (size_t)J.nA + 3 * (size_t)J.nV + 3 * (size_t)J.nQ) return 4;
  /* LoadBalance of each class (:182-204) */
  int* rng[6];
  for (int k = 0; k < 6; ++k) rng[k] = (int*)calloc((size_t)J.nranks, sizeof(int));
  J.a0 = rng[0], J.a1 = rng[1], J.v0 = rng[2], J.v1 = rng[3], J.q0 = rng[4], J.q1 = rng[5];
  if (tc_load_balance(J.nA, J.nranks, J.a0, J.a1) || tc_load_balance(J.nV, J.nranks, J.v0, J.v1) ||
      tc_load_balance(J.nQ, J.nranks, J.q0, J.q1)) {
    fprintf(stderr, "tc_load_balance: %s\n", tc_last_error());
    return 2;
  }
  pthread_barrier_init(&J.bar, NULL, (unsigned)J.nranks);
  pthread_t th[64];
  RankArg args[64];
  for (int r = 0; r < J.nranks; ++r) {
    args[r].job = &J;
    args[r].rank = r;
    pthread_create(&th[r], NULL, rank_main, &args[r]);
  }
  int status = 0;
  for (int r = 0; r < J.nranks; ++r) {
    pthread_join(th[r], NULL);
    if (J.status[r] > status) status = J.status[r];
  }
  pthread_barrier_destroy(&J.bar);
  if (status) return status;
  f = fopen(argv[2], "wb");
  if (!f) return 4;
  fwrite(J.fxA, sizeof(double), 3 * (size_t)J.nA, f);
  fwrite(J.fzA, sizeof(double), J.nA, f);
  fwrite(J.fxV, sizeof(double), 3 * (size_t)J.nV, f);
  fwrite(J.fxQ, sizeof(double), 3 * (size_t)J.nQ, f);
  fwrite(J.tke, sizeof(double), J.nsteps, f);
  fclose(f);
  printf("bve_sharded: %d ranks, %d active panels, %d steps, totalKE %.12f\n", J.nranks, J.nA, J.nsteps,
         J.tke[0]);
  return 0;
}
