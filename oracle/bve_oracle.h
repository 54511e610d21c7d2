/*
 * bve_oracle.h - CPU FP64 restatement of ThesisCode's Biot-Savart / RK4 hot
 * path. TEST INFRASTRUCTURE ONLY: the reference values of the CUDA library's
 * parity tests and the CPU baseline of the benchmark. Nothing in the product links or calls it.
 *
 * Parity status: pinned against the reference's own code. The reference is
 * Fortran (ifort/Open MPI) and no Fortran compiler is available to build it,
 * so its source is run instead through oracle/f90, a translator of the
 * Fortran 90 subset its modules use, with strict IEEE double arithmetic; this
 * restatement equals the outputs of those runs bit for bit (grid, initial
 * conditions, BVERK4 and StratosphereRK4 on 1-4 ranks, the three RHS sums,
 * the Voronoi sum: tests/test_reference_source.py, fixtures
 * tests/golden/ref_*.npz). It is also checked against the known answers the
 * reference's own validation drivers check (solid-body rotation, RK4
 * time-step convergence, invariants; tests/test_oracle.py).
 *
 * Layout: a point set is x[3*k + c] (Fortran x(3,n) column-major), 0-based;
 * target ranges are half-open [i0, i1).
 */
#ifndef BVE_ORACLE_H
#define BVE_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* BVEActiveRHS, PanelVelocityParallel.f90:1287-1334. Zeroes dX(3*nn) and
 * dVort(nn), sums rows [i0,i1) over k != j, scales the whole array by
 * 1/(-4 pi) and sets dVort = -2*omega*dX(3,:). delta = 0 is the reference;
 * delta > 0 adds delta^2 to the denominator after the subtraction, the same
 * way BVESmoothVelocity does (used for one-delta-for-all-targets runs). */
void or_active_rhs(double* dX, double* dVort, const double* pv, const double* vort,
                   const double* area, int nn, int i0, int i1, double omega, double delta);

/* BVEPassiveRHS, :1337-1373 (delta = 0). */
void or_passive_rhs(double* dX, const double* X, int mm, const double* pv, const double* vort,
                    const double* area, int nn, int i0, int i1);

/* BVESmoothVelocity, :1376-1412 (denominator 1 - x.y + smooth^2). */
void or_smooth_velocity(double* dX, const double* X, int mm, const double* pv,
                        const double* vort, const double* area, int nn, int i0, int i1,
                        double smooth);

/* BVEVelocity (Voronoi, SoA), VoronoiVelocityParallel.f90:487-515: zeroes
 * only dx, loops k over all nn entries, dVort = -2*omega*dz over all nn. */
void or_voronoi_velocity(double* dx, double* dy, double* dz, double* dVort, const double* x,
                         const double* y, const double* z, const double* vort,
                         const double* area, int nn, int i0, int i1, double omega);

/* Unscaled row sums for a list of target rows (sampled parity checks at
 * sizes where the full O(N^2) oracle is too slow). cls: 0 active (row index
 * is a source index, self excluded, targets = sources), 1 vertex targets X,
 * 2 passive targets X with delta. out[3*r + c] = sum for rows[r], already
 * divided by (-4 pi) like the full routines. nthreads >= 1 splits the row
 * list into contiguous blocks. */
void or_rows(int cls, const int* rows, int nrows, const double* X, const double* pv,
             const double* vort, const double* area, int nn, double delta, double* out,
             int nthreads);

/* LoadBalance, PanelVelocityParallel.f90:167-213: contiguous chunks of n/p,
 * the last rank takes the remainder. start/end are 0-based half-open. */
void or_load_balance(int n, int p, int* start, int* end);

/* BVERK4, PanelVelocityParallel.f90:435-658 with one rank (identical to
 * PanelVelocitySerial.f90:272-425 plus the particle relVort update of :651).
 * Arrays are updated in place. absVortV/relVortV may be NULL (then :651 is
 * skipped). kineticEnergy (nA) may be NULL. Returns totalKE of stage 1.
 * nthreads >= 1 evaluates target rows in parallel; the result does not
 * depend on nthreads. */
double or_bve_rk4(double* xV, int nV, double* xA, double* zetaA, const double* areaA, int nA,
                  double* xQ, int nQ, double dt, double omega, double deltaA, double deltaV,
                  double deltaQ, const double* absVortV, double* relVortV,
                  double* kineticEnergy, int nthreads);

/* One RK4 stage's three sums (rows by LoadBalance over nthreads ranks),
 * used as the timed CPU baseline: dXA(3*nA), dVortA(nA), dXV(3*nV),
 * dXQ(3*nQ). Rows outside [a0,a1), [v0,v1), [q0,q1) are left zero. */
void or_bve_stage(const double* xA, const double* zetaA, const double* areaA, int nA,
                  const double* xV, int nV, const double* xQ, int nQ, double omega,
                  double deltaA, double deltaV, double deltaQ, int a0, int a1, int v0,
                  int v1, int q0, int q1,
                  double* dXA, double* dVortA, double* dXV, double* dXQ, int nthreads);

/* Juckes forcing F(x, t) and its time factor A(t),
 * TracerAndVorticityDistributions.f90:1213-1221, :550-566 (strat_oracle.c). */
double or_juckes_forcing(const double* xyz, double t);
double or_juckes_a(double t);

/* StratosphereRK4, PanelVelocityParallel.f90:661-919, with one rank: one
 * forced RK4 step from time t (strat_oracle.c). Positions are updated in
 * place; relVortA / relVortV (nullable) receive absVort - 2 Omega z - F(x, t+dt)
 * at the new positions. Returns totalKE of stage 1. */
double or_strat_rk4(double* xV, int nV, double* xA, const double* absVortA, double* relVortA,
                    const double* areaA, int nA, double* xQ, int nQ, const double* absVortV,
                    double* relVortV, double t, double dt, double omega, double deltaA,
                    double deltaV, double deltaQ, double* kineticEnergy, int nthreads);

/* Icosahedral triangle grid, InitIcosTriGrid + DivideTriPanel + TriPanelArea,
 * ParticlesEdgesPanels2.f90:419-645, 760-1090, 1727-1802 (icos_oracle.c).
 * Sizes (PanelMax / ParticleMax / EdgeMax, :2614-2662) for a level in [0, 11];
 * the grid with 0-based indices (-1 = none), x arrays (N, 3) = Fortran x(3, N).
 * Both return 0, or -1 on a bad level or allocation failure. */
int or_icos_sizes(int level, int* n_particles, int* n_edges, int* n_panels, int* n_active);
int or_icos_grid(int level, double* particles_x, double* particles_x0, double* panels_x,
                 double* panels_x0, double* panels_area, int* has_children, int* vertices,
                 int* nest, int* children);
/* GatherPanels maps (:1556-1619): leaf panels in index order, then divided ones. */
int or_gather_maps(int n, const int* has_children, int* active_map, int n_active,
                   int* passive_map, int n_passive);

#ifdef __cplusplus
}
#endif
#endif
