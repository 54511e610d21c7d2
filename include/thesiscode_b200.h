/*
 * thesiscode_b200.h - C ABI of the B200 (sm_100a) Biot-Savart / RK4 library.
 *
 * This is the drop-in boundary for ThesisCode's barotropic-vorticity hot
 * path: the direct O(N^2) spherical Biot-Savart velocity sum
 *
 *     u_i = -1/(4 pi) * sum_{k != i} (x_i x x_k) zeta_k A_k / (1 - x_i.x_k + delta^2)
 *
 * evaluated inside the classical RK4 step (PanelVelocityParallel.f90 and
 * PanelVelocitySerial.f90, VoronoiVelocityParallel.f90 in the reference).
 *
 * Conventions (all entry points):
 *   - reals are IEEE double (Fortran real(kreal) = kind(0.d0), NumberKinds.f90:9),
 *     integers are int32 (kint = kind(1), NumberKinds.f90:10);
 *   - a set of n points is stored as the Fortran array x(3,n), column-major,
 *     i.e. component c of point k is x[3*k + c] (0-based here);
 *   - index ranges are 0-based and half-open [i0, i1). The reference's
 *     1-based inclusive [indexStart, indexEnd] maps to i0 = indexStart-1,
 *     i1 = indexEnd;
 *   - every call returns TC_OK (0) or a negative status; none aborts or
 *     prints. tc_last_error() describes the last failure of this thread.
 *   - entry points named *_device take device pointers and run on the
 *     context's stream without synchronising; all others take host pointers
 *     and return after the results are back in host memory.
 */
#ifndef THESISCODE_B200_H
#define THESISCODE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define TC_OK 0
#define TC_ERR_ARG (-1)       /* bad size, range, pointer or enum value   */
#define TC_ERR_CUDA (-2)      /* CUDA runtime error (see tc_last_error)   */
#define TC_ERR_NONFINITE (-3) /* NaN or Inf found in an input or result   */
#define TC_ERR_TIMEOUT (-4)   /* a bounded device-side wait ran out       */
#define TC_ERR_STATE (-5)     /* call out of sequence (e.g. no state yet) */
#define TC_ERR_NOMEM (-6)     /* device or host allocation failed         */

/* ---- arithmetic of the pair sum -------------------------------------- */
#define TC_FP64 0  /* FP64 throughout; denominator rounded exactly as the
                      reference's 1 - sum(x_k*x_j) (no contraction)          */
#define TC_FP32C 1 /* FP32 pair arithmetic on tile-relative offsets with a
                      cancellation-free denominator, FP64 accumulation of
                      per-tile FP32 partial sums                              */

/* ---- visiting order of targets in the FP32C pair kernel --------------- */
#define TC_ORDER_GIVEN 0   /* the caller's order                             */
#define TC_ORDER_HILBERT 1 /* along a Hilbert curve over the cube faces (default) */

/* ---- target classes (the three RHS routines of the reference) ------- */
#define TC_ACTIVE 0  /* BVEActiveRHS  PanelVelocityParallel.f90:1287-1334:
                        targets are the sources, self pair excluded,
                        dVort = -2 Omega u_z, delta = delta_active (0)       */
#define TC_VERTEX 1  /* BVEPassiveRHS :1337-1373: particles (panel
                        vertices), delta = delta_vertex (0)                  */
#define TC_PASSIVE 2 /* BVESmoothVelocity :1376-1412: divided panels,
                        delta = smooth (0.05 by default, :27)                */

/* ---- batched ensembles (tc_batch_rk4 flags) ---------------------------- */
#define TC_BATCH_GRAPH 1    /* capture the nsteps steps in one CUDA graph     */
#define TC_BATCH_AUTOTUNE 2 /* time kernel variants x chunk lengths first     */

/* ---- end-time functionals of the adjoint ------------------------------ */
#define TC_J_ENSTROPHY 0 /* J = sum_j zeta_j^2 A_j over the active panels  */
#define TC_J_PROBE 1     /* J = zeta of one active panel                   */

/* ---- throughput probe kinds (tc_probe_peak) --------------------------- */
#define TC_PROBE_FFMA 0
#define TC_PROBE_FFMA2 1
#define TC_PROBE_DFMA 2
#define TC_PROBE_RCP32 3
#define TC_PROBE_RCP64 4
#define TC_PROBE_DDIV 5
#define TC_PROBE_F2F 6
#define TC_PROBE_FAR_PAIRS 7 /* the FP32C pair loop's far step alone, pairs/s */

typedef struct tc_ctx tc_ctx;

/* ---- library --------------------------------------------------------- */
const char* tc_version(void);
/* Message of the last failed call on this thread ("" if none). */
const char* tc_last_error(void);

/* Measured operations/s of one CUDA-core pipe on `device` (roofline
 * denominator). No counterpart in the reference (it has no GPU code). */
int tc_probe_peak(int device, int kind, int iters, double* ops_per_s);

/* ---- device buffers of the RK4 state (tc_rk4_device_buffer) --------- */
#define TC_BUF_SOURCES 0 /* double4 {x,y,z,zeta*A} per active panel       */
#define TC_BUF_XA 1      /* x(3,nA) of active panels                      */
#define TC_BUF_ZETA 2    /* relVort(nA) of active panels                  */
#define TC_BUF_XV 3      /* x(3,nV) of particles                          */
#define TC_BUF_XQ 4      /* x(3,nQ) of divided (passive) panels           */
#define TC_BUF_KE 5      /* kineticEnergy(nA), stage 1 of the last step   */

/* ---- context: the module state of PanelVelocityParallelModule -------- */
/* Replaces InitializeMPIRK4 (PanelVelocityParallel.f90:126-164) for one
 * rank: binds a device and the pair arithmetic (TC_FP64 / TC_FP32C). */
int tc_create(int device, int precision, tc_ctx** out);
/* FinalizeMPIRK4 (:216-230): frees every device buffer. */
int tc_destroy(tc_ctx* ctx);
/* Run on a caller's cudaStream_t (default: the legacy default stream). */
int tc_set_stream(tc_ctx* ctx, void* cuda_stream);
int tc_synchronize(tc_ctx* ctx);
int tc_set_precision(tc_ctx* ctx, int precision);
int tc_get_precision(tc_ctx* ctx, int* precision);
/* SetOmega (TracerAndVorticityDistributions.f90:136-139); default 2*pi. */
int tc_set_omega(tc_ctx* ctx, double omega);
int tc_get_omega(tc_ctx* ctx, double* omega);
/* SetSmooth / GetSmooth (PanelVelocityParallel.f90:96-105): delta of the
 * TC_PASSIVE class (default 0.05, :27). */
int tc_set_smooth(tc_ctx* ctx, double smooth);
int tc_get_smooth(tc_ctx* ctx, double* smooth);
/* FP32C only: visit targets in the caller's order or along a Hilbert curve
 * over the six cube faces, continuous from face to face (default; results are
 * returned in the caller's order either way). The compensated arithmetic is
 * accurate when a CTA's targets are spatially close; the curve order
 * guarantees that for any input order. */
int tc_set_target_order(tc_ctx* ctx, int order);
/* delta of each target class (reference: 0, 0, smooth). */
int tc_set_deltas(tc_ctx* ctx, double delta_active, double delta_vertex, double delta_passive);
int tc_get_deltas(tc_ctx* ctx, double* delta3);

/* ---- one velocity sum ------------------------------------------------- */
/* BVEActiveRHS (:1287-1334), BVEPassiveRHS (:1337-1373) or
 * BVESmoothVelocity (:1376-1412) selected by target_class:
 *   X(3,m)       targets (NULL or src_x for TC_ACTIVE, then m == n)
 *   src_x(3,n), vort(n), area(n)   active panels (sources)
 *   [i0,i1)      target rows computed; dX rows outside are set to 0
 *   dX(3,m)      velocity, dVort(m) = -2*Omega*dX(3,:) (TC_ACTIVE only,
 *                nullable)
 * Host pointers; returns after dX/dVort are written. */
int tc_bs_velocity(tc_ctx* ctx, int target_class, const double* X, int m, const double* src_x,
                   const double* vort, const double* area, int n, int i0, int i1, double* dX,
                   double* dVort);
/* Same with device pointers, asynchronous on the context's stream. */
int tc_bs_velocity_device(tc_ctx* ctx, int target_class, const double* X, int m,
                          const double* src_x, const double* vort, const double* area, int n,
                          int i0, int i1, double* dX, double* dVort);

/* Allocation-free form of tc_bs_velocity_device (no counterpart in the
 * reference), for callers that cannot let the library allocate device memory
 * during the call: applications whose device memory is owned by their own
 * pool, and stepping loops that cannot take cudaMalloc's implicit device
 * synchronisation. Same arguments and result: FP32C keeps the library's
 * visiting order of the targets (tc_set_target_order), so its accuracy does not
 * depend on the order the caller stores them in, and the source chunking is
 * tc_bs_velocity_device's, capped by the space left. The scratch is a 32 MiB
 * array compiled into the library (held by every GPU that loads it): sources
 * 32*n bytes, partial sums 24*m per chunk and, for FP32C in the visiting
 * order, about 4*m + 20*(i1 - i0) for the order; a call for which one chunk
 * does not fit returns TC_ERR_ARG. The first call on a device (and the first
 * after its context was re-created) looks the array's address up: make it
 * before any stream capture. Calls share the array, so calls that overlap on
 * the GPU race. */
int tc_bs_velocity_device_noalloc(tc_ctx* ctx, int target_class, const double* X, int m,
                                  const double* src_x, const double* vort, const double* area,
                                  int n, int i0, int i1, double* dX, double* dVort);

/* ---- Voronoi generators, SoA (VoronoiVelocityParallel.f90) ------------ */
/* BVEVelocity (:487-515) on x(n), y(n), z(n): rows [i0,i1) summed over all n
 * sources (unused N_Max slots have vort = area = 0), self excluded. As in the
 * reference only dx is zeroed first: dy and dz add to what the caller holds,
 * then all three are divided by (-4 pi) over the whole arrays, and
 * dVort = -2 Omega dz over all rows (nullable). */
int tc_bs_velocity_soa(tc_ctx* ctx, const double* x, const double* y, const double* z,
                       const double* vort, const double* area, int n, int i0, int i1, double* dx,
                       double* dy, double* dz, double* dVort);
int tc_bs_velocity_soa_device(tc_ctx* ctx, const double* x, const double* y, const double* z,
                              const double* vort, const double* area, int n, int i0, int i1,
                              double* dx, double* dy, double* dz, double* dVort);
/* Voronoi BVERK4 (:304-478) without the Delaunay/Voronoi rebuild (:480-482,
 * host-side STRIPACK in the reference): nsteps RK4 steps of the n used
 * generators, updated in place. */
int tc_rk4_soa_step(tc_ctx* ctx, double* x, double* y, double* z, double* relVort,
                    const double* area, int n, double dt, int nsteps, double* totalKE,
                    double* kineticEnergy);

/* ---- RK4 (BVERK4, PanelVelocityParallel.f90:435-658) ------------------ */
/* The drop-in step on host arrays (the gathered active panels, the
 * particles and the divided panels, GatherPanels order): nsteps classical
 * RK4 steps of size dt fused on the device; xA, zetaA, xV, xQ are updated
 * in place (areas frozen, :452). totalKE[nsteps] (nullable) receives each
 * step's stage-1 kinetic energy 0.5*sum(|u|^2 A) (:495-501),
 * kineticEnergy[nA] (nullable) the per-panel |u|^2 of the last step. */
int tc_rk4_step(tc_ctx* ctx, double* xA, double* zetaA, const double* areaA, int nA, double* xV,
                int nV, double* xQ, int nQ, double dt, int nsteps, double* totalKE,
                double* kineticEnergy);
/* Same with device arrays (totalKE stays a host array). */
int tc_rk4_step_device(tc_ctx* ctx, double* xA, double* zetaA, const double* areaA, int nA,
                       double* xV, int nV, double* xQ, int nQ, double dt, int nsteps,
                       double* totalKE, double* kineticEnergy);
/* tc_rk4_advance replays steps 1..nsteps-1 from a CUDA graph (captured once
 * per shape, step, parameters and buffer addresses) when a step is small
 * enough for launch overhead to matter: mode 0 never, 1 (default) when a step
 * has at most 4.1e10 interactions (level 6) and nsteps >= 3, 2 always (nsteps
 * >= 3). Results are bitwise those of the launch-by-launch path. */
int tc_set_rk4_graphs(tc_ctx* ctx, int mode);
/* StratosphereRK4 (PanelVelocityParallel.f90:661-919): nsteps forced RK4
 * steps from time t. Positions of the three classes advance like tc_rk4_step;
 * the active vorticity is not integrated: each stage's source vorticity is
 * absVortA - 2 Omega z - F(x, t_s) with the Juckes forcing F
 * (TracerAndVorticityDistributions.f90:1213-1221) at t_s = t, t + dt/2,
 * t + dt/2, t + dt (:690-694, :752-755, :800-803, :847-850). On return
 * relVortA[nA] and relVortV[nV] (nullable; relVortV needs absVortV) hold
 * absVort - 2 Omega z - F(x, t + nsteps dt) at the new positions (:908-915).
 * totalKE / kineticEnergy as for tc_rk4_step. Step k starts at t + k dt. */
int tc_strat_rk4_step(tc_ctx* ctx, double* xA, const double* absVortA, double* relVortA,
                      const double* areaA, int nA, double* xV, const double* absVortV,
                      double* relVortV, int nV, double* xQ, int nQ, double t, double dt,
                      int nsteps, double* totalKE, double* kineticEnergy);
/* Device-resident state: load once (InitRK4 + GatherPanels copy, :236-318),
 * advance any number of steps, store when the caller needs the arrays. */
int tc_rk4_load(tc_ctx* ctx, const double* xA, const double* zetaA, const double* areaA, int nA,
                const double* xV, int nV, const double* xQ, int nQ, int on_device);
int tc_rk4_advance(tc_ctx* ctx, double dt, int nsteps, double* totalKE);
int tc_rk4_store(tc_ctx* ctx, double* xA, double* zetaA, double* xV, double* xQ,
                 double* kineticEnergy, int on_device);
/* ResetRK4 (:321-372): frees the state; call after a remesh changes N. */
int tc_reset_rk4(tc_ctx* ctx);
/* Checkpoint and restart (no counterpart in the reference, whose drivers keep
 * no restart files). tc_rk4_save writes the loaded state to `path`: the
 * positions of the three classes, zetaA, areaA, Omega, the deltas, the step
 * count and, for a forced run, absVortA/absVortV and its clock. It writes
 * `path`.tmp and renames it, so an interrupted save leaves any earlier file
 * whole. The format is a fixed header, the arrays, and an FNV-1a checksum
 * (csrc/checkpoint.cu).
 * tc_rk4_restore loads such a file into ctx as tc_rk4_load would, and also
 * sets Omega, the deltas, the step count and the forced run's clock.
 * tc_rk4_advance then continues bit for bit as the run that wrote the file
 * would have, given the same precision, which is the context's own and is
 * not changed. A missing, truncated or corrupted file (bad magic, sizes or
 * checksum) returns TC_ERR_ARG and leaves the context's state as it was. */
int tc_rk4_save(tc_ctx* ctx, const char* path);
int tc_rk4_restore(tc_ctx* ctx, const char* path);
/* Validates a checkpoint file the way tc_rk4_restore does (no GPU needed) and
 * reports its sizes, whether it holds a forced run, and its step count. Every
 * output may be NULL. */
int tc_rk4_checkpoint_info(const char* path, int* nA, int* nV, int* nQ, int* forced,
                           long long* steps);
/* Steps advanced since the state was loaded (tc_rk4_advance / tc_rk4_step),
 * counting those recorded in a restored checkpoint. */
int tc_rk4_steps_done(tc_ctx* ctx, long long* steps);

/* ---- adjoint (no counterpart in the reference) ------------------------- */
/* Gradient of J(T), T = nsteps*dt, with respect to the initial state of the
 * active panels, through nsteps RK4 steps of the active panels (the only ones
 * that feed back; particles and divided panels are passive): the discrete
 * adjoint of the step (exact gradient of the RK4 map), FP64, state
 * checkpointed every ckpt_every steps and stage inputs recomputed per
 * segment. Host arrays: xA0(3,nA), zetaA0, areaA in; J, g_zeta0(nA),
 * g_x0(3,nA) out. Replaces the context's loaded RK4 state. */
int tc_rk4_adjoint(tc_ctx* ctx, const double* xA0, const double* zetaA0, const double* areaA,
                   int nA, double dt, int nsteps, int ckpt_every, int functional, int probe,
                   double* J, double* g_zeta0, double* g_x0);
/* Vector-Jacobian product of the whole trajectory: given cotangents gT_x[3nA]
 * and gT_zeta[nA] (either nullable, not both) on the state after nsteps RK4
 * steps, g_x0 / g_zeta0 = (d state(T) / d state(0))^T applied to them, and J =
 * gT_x . x(T) + gT_zeta . zeta(T). Same checkpointing and errors as
 * tc_rk4_adjoint (no reference counterpart). */
int tc_rk4_vjp(tc_ctx* ctx, const double* xA0, const double* zetaA0, const double* areaA, int nA,
               double dt, int nsteps, int ckpt_every, const double* gT_x, const double* gT_zeta,
               double* J, double* g_zeta0, double* g_x0);
/* How each stage's vector-Jacobian product visits the pairs: 3 to 6 = one
 * row-major pass computing both sides' row sums (3: one row per thread,
 * 4: two rows per thread; 5 and 6: the same with a one-step Newton
 * reciprocal, relative error the square of the rcp.approx.f64 seed's; 7:
 * three rows per thread, one-step Newton), 0 = two
 * passes (target side, transposed source side), 1 and 2 = one pass with
 * in-block column reductions (256 threads x 2 targets, or 128 x 4). Default 6.
 * Modes 0-4 give the same gradient to FP64 rounding; 5-7 differ from them
 * by the seed's squared error (below 1e-13 of the gradient's scale). */
int tc_set_adjoint_mode(tc_ctx* ctx, int mode);
/* Device time (ms) of the last tc_rk4_adjoint call: ms3[0] forward sweep
 * with checkpoints, ms3[1] recomputation of checkpoint segments, ms3[2]
 * backward sweep. */
int tc_adjoint_phase_ms(tc_ctx* ctx, double* ms3);

/* ---- batched ensembles (no counterpart in the reference) --------------- */
/* `count` independent particle sets stored back to back (host arrays):
 * instance b owns active rows [sum_{c<b} nA[c], +nA[b]) of xA(3,*), zetaA,
 * areaA and vertex rows [sum_{c<b} nV[c], +nV[b]) of xV(3,*); each evolves
 * as its own BVERK4 (its active panels are its only sources) for nsteps
 * steps, updated in place. totalKE[nsteps*count] (step-major) receives each
 * instance's stage-1 kinetic energy. The pair work of all instances runs in
 * one persistent launch per stage; TC_BATCH_GRAPH replays all steps as one
 * CUDA graph, TC_BATCH_AUTOTUNE times the kernel variants and source-chunk
 * lengths on the batch first (cached per batch shape). */
int tc_batch_rk4(tc_ctx* ctx, int count, const int* nA, const int* nV, double* xA, double* zetaA,
                 const double* areaA, double* xV, double dt, int nsteps, double* totalKE,
                 int flags);
/* Variant, source-chunk length and work-item count of the last batch. */
int tc_batch_info(tc_ctx* ctx, int* variant, int* chunk_len, int* n_items);

/* ---- stage primitives for target-sharded multi-rank runs -------------- */
/* Pack stage-1 sources of the loaded state into TC_BUF_SOURCES. */
int tc_rk4_pack_sources(tc_ctx* ctx);
/* One stage (0..3) for the target rows [a0,a1) x [v0,v1) x [q0,q1)
 * (LoadBalance ranges, :167-213). Reads every row of TC_BUF_SOURCES, writes
 * the rows [a0,a1) of the next stage's sources; a rank exchanges those rows
 * (the reference's per-stage MPI_BCAST loop, :476-489) before the next
 * stage. total_ke_device (device, nullable): stage-0 0.5*sum(KE*A) of the
 * rank's active rows. */
int tc_rk4_stage_range(tc_ctx* ctx, int stage, double dt, int a0, int a1, int v0, int v1, int q0,
                       int q1, double* total_ke_device);
int tc_rk4_device_buffer(tc_ctx* ctx, int which, void** ptr);
/* Copy rows [row0, row0+nrows) of an RK4 device buffer (TC_BUF_*) to
 * (to_buffer = 0) or from (to_buffer = 1) memory at ptr, device or host
 * memory, on the context's stream (tc_synchronize before reading a host
 * copy): the exchange unit of a target-sharded run. */
int tc_rk4_copy_rows(tc_ctx* ctx, int which, int row0, int nrows, void* ptr, int to_buffer);
/* LoadBalance (PanelVelocityParallel.f90:167-213; the partition at :182-204):
 * contiguous chunks of n / num_procs rows, the last rank takes the
 * remainder; 0-based half-open [index_start[r], index_end[r]) per rank. */
int tc_load_balance(int n, int num_procs, int* index_start, int* index_end);
/* Number of visible CUDA devices (no counterpart: the reference runs on
 * CPUs); a sharded run maps rank r to device r % count. */
int tc_device_count(int* count);

/* ---- pair-kernel variants (no counterpart in the reference) ------------ */
/* Number of compiled launch shapes for a precision, and their parameters:
 * info8 = {threads, targets/thread, sources/tile, FP32 flush length (FP64:
 * 1 fused denominator, 0 rounded like the reference), min CTAs/SM, unroll,
 * targets/CTA, form}. FP32C form: bit 3 = source-paired kernel (set in every
 * variant: the two lanes of each f32x2 instruction carry two sources of one
 * target), bit 1 = FP64 accumulators in shared memory, bit 2 = hi/lo
 * near-pair offsets (the accurate variants), bits 8-9 = log2 of the flush
 * lengths between flushes in tiles whose every source is far. FP64 form: 0. */
int tc_pair_variant_count(int precision, int* count);
int tc_pair_variant_info(int precision, int id, int* info8);
/* Select a variant. By default the variant is chosen per launch by problem
 * size. For FP32C: variant 1 below 131,072 sources, 0 above. For FP64:
 * variant 2, or variant 6 (the same shape with 32-source tiles and chunks of
 * any multiple of 32 sources) for launches that would fill less than 90% of
 * one wave of CTAs with whole 256-source chunks. Selecting a variant turns
 * the automatic choice off; id = -1 turns it back on. tc_get_pair_variant
 * returns the variant in use (with the automatic choice: the one last
 * used). */
int tc_set_pair_variant(tc_ctx* ctx, int precision, int id);
int tc_get_pair_variant(tc_ctx* ctx, int precision, int* id);

/* ---- instrumentation (no counterpart in the reference) ----------------- */
/* Record CUDA events around every pair-kernel launch on the context's
 * stream (off by default). */
int tc_stats_enable_timing(tc_ctx* ctx, int on);
/* Kernels launched, pair-kernel launches, pairs evaluated and summed
 * pair-kernel event time (ms) since the last reset; reset != 0 zeroes them. */
int tc_stats(tc_ctx* ctx, int reset, long long* launches, long long* pair_launches,
             long long* pair_interactions, double* pair_ms);

/* ---- index checks (checked build; the reference's commented-out ifort
 * flags -check bounds -check pointers, Makefile:7) ---------------------- */
/* The same sources compiled with -DTC_BOUNDS_CHECK=1 give
 * libthesiscode_b200_checked.so (`python -m thesiscode_b200.build --checked`).
 * In it the pair kernels (single and batched), source packing, the
 * velocity and RK4 stage epilogues, the FP32C visiting-order keys and the
 * adjoint's row pass (the default adjoint mode) check every global-memory
 * index against its array's extent. That extent is the library's own allocation, or the size the
 * caller declared. An index outside it is not accessed: a load reads 0 and
 * a store is skipped. The first such index goes into the device's record.
 * Other kernels (the adjoint's other modes, grid, Voronoi adapters) are not
 * checked. */
#define TC_BC_PAIR_X 1        /* pair kernels: target positions (points)       */
#define TC_BC_PAIR_PERM 2     /* pair kernels: target visiting order           */
#define TC_BC_PAIR_SRC 3      /* pair kernels: packed sources                  */
#define TC_BC_PAIR_OUT 4      /* pair kernels: partial-sum stores (doubles)    */
#define TC_BC_BATCH_SEG 5     /* batched pair kernels: segment table           */
#define TC_BC_PACK_IN 6       /* packing: positions, vorticity, area (points)  */
#define TC_BC_PACK_OUT 7      /* packing: packed-source stores                 */
#define TC_BC_EPI_PERM 8      /* velocity epilogue: visiting order             */
#define TC_BC_EPI_X 9         /* velocity epilogue: target positions (points)  */
#define TC_BC_EPI_PARTIAL 10  /* velocity epilogue: partial sums (doubles)     */
#define TC_BC_EPI_OUT 11      /* velocity epilogue: dX / dVort stores (points) */
#define TC_BC_STAGE_PERM 12   /* stage epilogue: visiting orders               */
#define TC_BC_STAGE_STATE 13  /* stage epilogue: a class's state arrays        */
#define TC_BC_STAGE_PARTIAL 14 /* stage epilogue: partial sums (doubles)       */
#define TC_BC_STAGE_CHUNKS 15 /* stage epilogue: per-row chunk counts (batch)  */
#define TC_BC_STAGE_ACTIVE 16 /* stage epilogue: active-only arrays            */
#define TC_BC_STAGE_KEBLOCK 17 /* stage epilogue: per-block KE sums            */
#define TC_BC_ADJ_ROW_IN 18   /* adjoint row pass: per-panel inputs            */
#define TC_BC_ADJ_ROW_OUT 19  /* adjoint row pass: partial-sum stores          */
#define TC_BC_ADJ_COMBINE 20  /* adjoint row combination: partial-sum reads    */
#define TC_BC_ORDER_X 21      /* visiting-order keys: per-target inputs        */
#define TC_BC_ORDER_KEYS 22   /* visiting-order keys: key and index stores     */
#define TC_BC_BATCH_KE 23     /* batched runs: per-instance KE sums' reads     */
/* 1 in the checked library, 0 in the release library. */
int tc_bounds_checked(void);
/* Waits for the device, then reads its record: rec[0] = violations since the
 * last reset, rec[1] = TC_BC_* site of the first one, rec[2] = its index,
 * rec[3] = the extent it was checked against. reset != 0 clears the record.
 * Every context on the device shares the one record. The release library
 * gives all zeros. */
int tc_bounds_status(int device, long long rec[4], int reset);
/* Checked library only; the release library returns TC_ERR_STATE. Launches made
 * after the call declare at most `cap` elements for `site` (0: every site),
 * while the arrays keep their size. So the checks can be seen firing on
 * accesses that still lie inside the real allocation. cap < 0 removes the
 * cap. A CUDA graph captured earlier keeps the extents it was captured
 * with. */
int tc_bounds_cap(tc_ctx* ctx, int site, long long cap);

/* ---- icosahedral grid (input generator) ------------------------------- */
/* PanelMax / ParticleMax / EdgeMax (ParticlesEdgesPanels2.f90:2614-2662)
 * and the number of leaf panels, 20*4^level. level in [0, 11]. */
int tc_icos_grid_sizes(int level, int* n_particles, int* n_edges, int* n_panels, int* n_active);
/* InitIcosTriGrid (:419-645) with DivideTriPanel (:760-1090) and
 * TriPanelArea (:1727-1802): particle and panel arrays in the reference's
 * numbering (0-based). Optional outputs may be NULL. */
int tc_icos_grid(int level, double* particles_x, double* particles_x0, double* panels_x,
                 double* panels_x0, double* panels_area, int* panels_has_children,
                 int* panels_vertices, int* panels_nest, int* panels_children);
/* The same grid generated on the GPU of ctx (no counterpart in the
 * reference, whose generator runs on the host): every output is a device
 * pointer on ctx's device, written on ctx's stream; the call returns when the
 * grid is complete. Particle positions, panel centres and all index arrays
 * equal tc_icos_grid's bit for bit; areas agree to a few ulps (CUDA's atan2
 * and tan). particles_x, panels_x and panels_area are required. */
int tc_icos_grid_device(tc_ctx* ctx, int level, double* particles_x, double* particles_x0,
                        double* panels_x, double* panels_x0, double* panels_area,
                        int* panels_has_children, int* panels_vertices, int* panels_nest,
                        int* panels_children);
/* GatherPanels index maps (:1556-1619), 0-based. */
int tc_gather_maps(int n, const int* has_children, int* active_map, int n_active,
                   int* passive_map, int n_passive);

#ifdef __cplusplus
}
#endif
#endif /* THESISCODE_B200_H */
