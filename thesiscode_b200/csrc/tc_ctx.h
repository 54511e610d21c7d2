// The library context: what PanelVelocityParallelModule keeps as module
// state (`save` variables, PanelVelocityParallel.f90:25-71: smooth, the RK4
// scratch arrays, kineticEnergy, totalKE) plus the device, stream and
// launch configuration. Explicit instead of global, so the ABI is reentrant.
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <vector>

#include "bs_core.cuh"
#include "tc_internal.h"

namespace tcb {

// A growable device allocation owned by the context.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  int ensure(size_t need);  // grows (never shrinks); contents are not kept
  void release();
  template <class T>
  T* as() const { return static_cast<T*>(ptr); }
};

// Launch shape of one pair-kernel variant.
struct PairCfg {
  int nt;     // threads per CTA
  int tpt;    // targets per thread
  int ts;     // sources per shared-memory tile
  int tb() const { return nt * tpt; }
};

// One compiled pair-kernel shape.
struct PairVariant {
  int precision;
  int nt, tpt, ts, flush, minb, unroll;
  void (*launch)(dim3 grid, cudaStream_t stream, const PairLaunch& P);
  const void* fn;
  void (*launch_batch)(int grid, cudaStream_t stream, const BatchLaunch& B);
  const void* fn_batch;
  int form;  // FP32C: bit 3 source-paired form (every variant), bit 1 shared-memory FP64 accumulators, bit 2 hi/lo near offsets, bits 8-9 log2 of flush lengths per flush in all-far tiles. FP64: 0
};

// Target segment as the host describes it before tiles are assigned.
struct SegDesc {
  const double* x;
  const int* perm;  // visiting order of [i0, i1) (FP32C only; null: as stored)
  int i0, i1;
  int out_offset;
  int self_offset;
  double d2;
  long long x_len;     // points in x (its allocation or the caller's declared size)
  long long perm_len;  // entries in perm
};

// RK4 state and scratch kept on the device between calls (the reference's
// activePanelsInput/Stage1..4/newActivePanelsX family, :34-71, laid out for
// the fused stage epilogue: only the running sum of the stages is kept).
struct Rk4State {
  int nA = 0, nV = 0, nQ = 0;
  bool ready = false;
  DevBuf x0A, z0, areaA, x0V, x0Q;      // state at the start of the step
  DevBuf xiA, ziA, xiV, xiQ;            // stage inputs (targets / sources)
  DevBuf newA, newZ, newV, newQ;        // running x + k1/6 + k2/3 + ...
  DevBuf src;                           // packed sources of the current stage
  DevBuf ke;                            // kineticEnergy(nA), stage 1
  DevBuf keBlocks;                      // per-block partial sums of KE*A
  DevBuf totalKE;                       // one value per step
  DevBuf permA, permV, permQ;           // FP32C visiting orders (cube-face Hilbert), per class
  bool ordered = false;                 // perm* hold orders of the current stage ranges
  int order_range[6] = {0, 0, 0, 0, 0, 0};
  // forced (stratosphere) model: source vorticity rebuilt each stage from absA
  bool strat = false;
  DevBuf absA, absV;                    // absolute vorticity of panels and vertices
  double t0 = 0.0;                      // time at the start of step 0
  double strat_dt = 0.0;                // step length of the forced run
  long long step = 0;                   // steps completed since t0
  long long steps_total = 0;            // steps advanced since the state was loaded (checkpoints)
};

}  // namespace tcb

struct tc_batch_plan;            // batched-ensemble plan (batch.cu)
struct tc_advance_graph;         // captured RK4 steps of tc_rk4_advance (api.cu)
void tc_advance_graph_free(tc_ctx* ctx);
void tc_batch_free(tc_ctx* ctx);

struct tc_ctx {
  int device = 0;
  int precision = TC_FP64;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 148;
  double omega = 6.283185307179586476925286766559;  // 2*pi, TracerAndVorticityDistributions.f90:34-35
  double delta[3] = {0.0, 0.0, 0.05};               // ACTIVE, VERTEX, PASSIVE (smooth, :27)
  tcb::PairCfg cfg64{256, 2, 256};
  tcb::PairCfg cfg32{256, 4, 256};
  int var64 = 2, var32 = 0;  // pair-kernel variants in use (see kVariants64/32)
  bool auto32 = true;  // FP32C variant chosen per launch by problem size (tc_set_pair_variant turns it off)
  bool auto64 = true;  // FP64: 32-source tiles for launches too small to fill a wave (likewise)
  int slots64_default = 0;  // resident CTAs per GPU of the default FP64 variant
  int target_order = TC_ORDER_HILBERT;  // FP32C visiting order of targets
  double adj_ms[3] = {0.0, 0.0, 0.0};  // last adjoint: forward sweep, recompute, backward
  int adj_mode = 6;  // adjoint VJP: 3-6 row pass, 0 two passes, 1 and 2 fused (tc_set_adjoint_mode)
  tcb::DevBuf order_buf[4];             // keys, sorted keys, indices, sort scratch
  int min_chunk = 256;    // smallest source chunk a CTA walks (one shared-memory tile)
  int max_chunks = 64;
  int slots64 = 0, slots32 = 0;  // resident CTAs per GPU for each kernel
  tcb::DevBuf partial;    // pair-kernel partial sums
  tcb::DevBuf scratch[6]; // one-call buffers (velocity entry points)
  tcb::DevBuf grid_buf[6];  // tc_icos_grid_device: edge and panel tables, prefix sums
  tcb::DevBuf check_buf;    // first non-finite index of each result array scanned on the device
  tcb::Rk4State rk;
  // instrumentation (tc_stats): kernels launched, and CUDA-event time of the
  // pair kernels when timing is on (events recorded on ctx->stream).
  long long launches = 0;
  long long pair_launches = 0;
  long long pair_interactions = 0;
  bool time_pairs = false;
  std::vector<cudaEvent_t> pair_events;  // start/stop pairs, resolved by tc_stats
  double pair_ms = 0.0;
  tc_batch_plan* batch = nullptr;
  tc_advance_graph* agraph = nullptr;
  int rk4_graphs = 1;  // tc_rk4_advance graph replay: 0 never, 1 small problems, 2 always
  // checked build: the device's violation record, and per-site caps on the declared
  // extents (tc_bounds_cap)
  tcb::BoundsRec* bc_rec = nullptr;
  bool bc_capped[tcb::BC_SITE_END] = {};
  long long bc_cap[tcb::BC_SITE_END] = {};
};

namespace tcb {
// The automatic FP64 variants: the default, and the same shape with 32-source
// tiles for launches that leave most of one wave's CTA slots empty.
constexpr int kAuto64Default = 2;
constexpr int kAuto64Small = 6;
// Checked build: the extent the kernels check `site`'s indices against, n or the
// cap tc_bounds_cap set (the smaller).
inline long long bc_extent(const tc_ctx* ctx, int site, long long n) {
  return (ctx->bc_capped[site] && ctx->bc_cap[site] < n) ? ctx->bc_cap[site] : n;
}
// Launch the pair kernel of ctx->precision over up to three target segments
// (src_len: packed sources the src allocation holds, at least n).
// Allocates ctx->partial and returns the number of source chunks in *nchunks.
int launch_pairs(tc_ctx* ctx, const SegDesc* segs, int nseg, const double4* src, int n,
                 long long src_len, int n_out, int* nchunks);
// The same with the partial sums in caller-provided memory of partial_bytes bytes (at least one
// chunk, 24 * n_out bytes); the chunk count is capped by what fits. Allocates nothing.
int launch_pairs_into(tc_ctx* ctx, const SegDesc* segs, int nseg, const double4* src, int n,
                      long long src_len, int n_out, double* partial, size_t partial_bytes,
                      int* nchunks);
// Pack {x, y, z, zeta*area} for n sources.
int launch_pack_strat(tc_ctx* ctx, double t);
int launch_strat_rel_vort(tc_ctx* ctx, const double* abs_vort, const double* x, int n, double t,
                          double* out);
// out_len: packed sources the out allocation holds (at least n).
int launch_pack(tc_ctx* ctx, const double* x, const double* zeta, const double* area, int n,
                double4* out, long long out_len);
// dX (3*m) and dVort (m, nullable) for rows [i0, i1), zero elsewhere; partial
// rows are row_offset + i. The partial sums are ctx->partial, or `partial`
// (partial_len doubles) when that is given.
int launch_velocity_epilogue(tc_ctx* ctx, const double* x, const int* perm, int m, int i0, int i1,
                             int row_offset, int n_out, int nchunks, double* dX, double* dVort,
                             const double* partial = nullptr, long long partial_len = 0);
// perm[i0..i1) <- i0..i1-1 sorted along the cube-face Hilbert curve (sphere_order.cuh);
// x holds x_len points, perm perm_len entries (a range past either is an error)
int compute_order(tc_ctx* ctx, const double* x, int i0, int i1, int* perm, long long x_len,
                  long long perm_len);
// Extents of an order computation: points in x, entries in perm, entries in each key and
// index buffer.
struct OrderExtents {
  long long x_len, perm_len, key_len;
};
// The same in caller-provided scratch (keys in/out and indices: i1 - i0 entries each; temp:
// order_sort_bytes(i1 - i0) bytes); allocates nothing.
int order_sort_bytes(int n, size_t* bytes);
int compute_order_into(tc_ctx* ctx, const double* x, int i0, int i1, int* perm, unsigned* k_in,
                       unsigned* k_out, int* v_in, void* temp, size_t temp_bytes,
                       const OrderExtents& ext);
// One RK4 stage epilogue over the three classes' ranges.
// total_ke (device, nullable) receives 0.5*sum(KE*A) of the rows in range at
// stage 0; nchunks is what launch_pairs returned for this stage.
// Batched runs pass row_nchunks (row_nchunks_len entries) and their own partial sums
// (partial_len doubles).
int launch_stage_epilogue(tc_ctx* ctx, int stage, double dt, const int range[6], int nchunks,
                          double* total_ke, const int* row_nchunks = nullptr,
                          const double* partial = nullptr, long long row_nchunks_len = 0,
                          long long partial_len = 0);
int resolve_slots(tc_ctx* ctx);
// Checked build: points ctx->bc_rec at the device's violation record (allocated on first use
// in each CUDA context).
int bounds_attach(tc_ctx* ctx);
// Unique id of the current CUDA context; 0 when the driver cannot say.
unsigned long long current_context_id();
const PairVariant* variant(int precision, int id);
int variant_count(int precision);
int select_variant(tc_ctx* ctx, int precision, int id);
// With ctx->auto32, selects the FP32C variant for a launch over n sources.
int use_fp32c_variant(tc_ctx* ctx, int n);
}  // namespace tcb
