// Host-side launch logic for the pair kernels and the epilogues that turn
// per-chunk partial sums into velocities and RK4 stage updates.
#include <algorithm>
#include <cmath>

#include "strat.cuh"
#include "tc_ctx.h"

namespace tcb {

// The reference's (-4.0_kreal*PI) (PanelVelocityParallel.f90:1332).
__constant__ double kMinus4Pi = -4.0 * 3.141592653589793238462643383279502884;

int DevBuf::ensure(size_t need) {
  if (need <= bytes && ptr) return TC_OK;
  release();
  if (need == 0) need = 16;
  cudaError_t e = cudaMalloc(&ptr, need);
  if (e != cudaSuccess) {
    ptr = nullptr;
    bytes = 0;
    tc_record_error("cudaMalloc of %zu bytes failed: %s", need, cudaGetErrorString(e));
    cudaGetLastError();
    return TC_ERR_NOMEM;
  }
  bytes = need;
  return TC_OK;
}

void DevBuf::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

// ---------------------------------------------------------------------------
// Kernel variants: the launch shapes the autotuner chooses from. FP32C
// variants differ in threads per CTA, targets per thread, FP32 partial length
// before the FP64 flush, minimum resident CTAs (register cap), source-loop
// unrolling and form bits; FP64 variants in threads and targets per thread.
// ---------------------------------------------------------------------------
constexpr int kTS = 256;

template <int NT, int TPT, int MINB, bool FUSED, int TS>
void launch64(dim3 g, cudaStream_t s, const PairLaunch& P) {
  pair_fp64_kernel<NT, TPT, TS, MINB, FUSED><<<g, NT, 0, s>>>(P);
}
template <int NT, int TPT, int MINB, bool FUSED, int TS>
void launch64b(int g, cudaStream_t s, const BatchLaunch& B) {
  pair_fp64_batch_kernel<NT, TPT, TS, MINB, FUSED><<<g, NT, 0, s>>>(B);
}
template <int NT, int T, int FLUSH, int MINB, int UNROLL, int FM>
void launch32b(int g, cudaStream_t s, const BatchLaunch& B) {
  pair_fp32c_batch_kernel<NT, T, kTS, FLUSH, MINB, UNROLL, FM><<<g, NT, 0, s>>>(B);
}
template <int NT, int T, int FLUSH, int MINB, int UNROLL, int FM>
void launch32(dim3 g, cudaStream_t s, const PairLaunch& P) {
  pair_fp32c_kernel<NT, T, kTS, FLUSH, MINB, UNROLL, FM><<<g, NT, 0, s>>>(P);
}

#define V64T(NT, TPT, MINB, FUSED, TS)                                              \
  PairVariant { TC_FP64, NT, TPT, TS, FUSED, MINB, 0, launch64<NT, TPT, MINB, FUSED, TS>, \
                (const void*)pair_fp64_kernel<NT, TPT, TS, MINB, FUSED>,                  \
                launch64b<NT, TPT, MINB, FUSED, TS>,                                        \
                (const void*)pair_fp64_batch_kernel<NT, TPT, TS, MINB, FUSED>, 0 }
#define V64(NT, TPT, MINB, FUSED) V64T(NT, TPT, MINB, FUSED, kTS)
// FP32C: T targets per thread, FP32 flush every FLUSH sources, form bits FM
#define V32(NT, T, FLUSH, MINB, UNROLL, FM)                                            \
  PairVariant { TC_FP32C, NT, T, kTS, FLUSH, MINB, UNROLL,                             \
                launch32<NT, T, FLUSH, MINB, UNROLL, FM>,                              \
                (const void*)pair_fp32c_kernel<NT, T, kTS, FLUSH, MINB, UNROLL, FM>,   \
                launch32b<NT, T, FLUSH, MINB, UNROLL, FM>,                             \
                (const void*)pair_fp32c_batch_kernel<NT, T, kTS, FLUSH, MINB, UNROLL, FM>, FM }

// FP64: the `flush` field records the denominator mode (1 = fused, 0 =
// rounded exactly like the reference).
// Variant 6 is variant 2 with 32-source tiles, for launches too small to fill
// one wave of whole 256-source chunks (chosen automatically, fp64_small).
const PairVariant kVariants64[] = {
    V64(256, 2, 5, true),  V64(256, 4, 2, true),  V64(256, 1, 6, true), V64(128, 4, 4, true),
    V64(256, 2, 5, false), V64(256, 4, 2, false), V64T(256, 1, 6, true, 32),
};
static_assert(kAuto64Default == 2 && kAuto64Small == 6, "automatic FP64 variants");
// FP32C form bits (SpForm in bs_core.cuh): 8 = source-paired form (all
// variants), 2 = FP64 accumulators in shared memory, 4 = hi/lo near offsets,
// 256 / 512 = tiles whose every source is far flushed every 2 / 4 flush
// lengths.
const PairVariant kVariants32[] = {
    // 0: default from 131,072 sources (3 targets per thread); 1: default below (2 per thread)
    V32(128, 3, 64, 6, 4, 8 | 2 | 256), V32(128, 2, 64, 6, 4, 8 | 512),
    // 2-7: the batch autotuner's other candidates (4: the 64-source far flush of 0)
    V32(128, 2, 64, 6, 4, 8 | 2 | 512), V32(128, 2, 64, 6, 4, 8 | 2 | 256),
    V32(128, 3, 64, 6, 4, 8 | 2), V32(128, 2, 64, 6, 4, 8), V32(128, 2, 64, 6, 4, 8 | 2),
    V32(128, 3, 64, 6, 2, 8 | 2),
    // 8-11: near tiles with hi/lo offsets (1e-7 at coarser grids, at a fraction of the speed)
    V32(128, 3, 64, 6, 4, 8 | 4 | 2), V32(128, 2, 64, 6, 4, 8 | 4), V32(128, 2, 64, 6, 4, 8 | 4 | 2),
    V32(128, 3, 64, 5, 4, 8 | 4 | 2),
};
constexpr int kN64 = sizeof(kVariants64) / sizeof(kVariants64[0]);
constexpr int kN32 = sizeof(kVariants32) / sizeof(kVariants32[0]);

const PairVariant* variant(int precision, int id) {
  if (precision == TC_FP64) return (id >= 0 && id < kN64) ? &kVariants64[id] : nullptr;
  return (id >= 0 && id < kN32) ? &kVariants32[id] : nullptr;
}

int variant_count(int precision) { return precision == TC_FP64 ? kN64 : kN32; }

int select_variant(tc_ctx* ctx, int precision, int id) {
  const PairVariant* v = variant(precision, id);
  if (!v) {
    tc_record_error("no pair-kernel variant %d for precision %d", id, precision);
    return TC_ERR_ARG;
  }
  int blocks = 0;
  TC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, v->fn, v->nt, 0));
  int slots = std::max(1, blocks) * ctx->num_sms;
  if (precision == TC_FP64) {
    ctx->var64 = id;
    ctx->slots64 = slots;
    ctx->cfg64 = PairCfg{v->nt, v->tpt, v->ts};
  } else {
    ctx->var32 = id;
    ctx->slots32 = slots;
    ctx->cfg32 = PairCfg{v->nt, v->tpt, v->ts};
  }
  return TC_OK;
}

// Automatic FP32C variant: below kAutoSmallSources sources (icosahedral level
// 6 and coarser) two targets per thread (variant 1: more CTAs for few
// tiles, and smaller tile patches, hence smaller FP32 offsets), above it
// three (variant 0: 2-4% faster from level 7 on); both flush all-far tiles
// less often than mixed ones (0 every 128 sources, 1.8-2.0% faster than
// every 64 at levels 7-8 with the same error; 1 every 256, 1.6% faster at
// level 6, error 6.1e-8 against 5.2e-8 on the level-6 jet).
constexpr int kAutoSmallSources = 131072;
constexpr int kAutoSmallVariant = 1;
constexpr int kAutoLargeVariant = 0;

int use_fp32c_variant(tc_ctx* ctx, int n) {
  if (!ctx->auto32) return TC_OK;
  const int want = n < kAutoSmallSources ? kAutoSmallVariant : kAutoLargeVariant;
  return want == ctx->var32 ? TC_OK : select_variant(ctx, TC_FP32C, want);
}

int resolve_slots(tc_ctx* ctx) {
  cudaDeviceProp prop;
  TC_CUDA_TRY(cudaGetDeviceProperties(&prop, ctx->device));
  ctx->num_sms = prop.multiProcessorCount;
  int blocks = 0;
  TC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &blocks, kVariants64[kAuto64Default].fn, kVariants64[kAuto64Default].nt, 0));
  ctx->slots64_default = std::max(1, blocks) * ctx->num_sms;
  int rc = select_variant(ctx, TC_FP64, ctx->var64);
  if (rc) return rc;
  return select_variant(ctx, TC_FP32C, ctx->var32);
}

// Number of source chunks: the split that best fills the resident CTA slots
// (waves of tiles x chunks), never cutting chunks below ctx->min_chunk.
static int choose_chunks(int tiles, int n, int ts, int slots, int min_chunk, int max_chunks) {
  int best = 1;
  double best_eff = 0.0;
  for (int s = 1; s <= max_chunks; ++s) {
    int len = (n + s - 1) / s;
    if (s > 1 && len < min_chunk) break;
    long long items = (long long)tiles * s;
    long long waves = (items + slots - 1) / slots;
    double eff = (double)items / (double)(waves * slots);
    if (eff > best_eff + 0.02) {
      best_eff = eff;
      best = s;
    }
    if (eff > 0.97) break;
  }
  (void)ts;
  return best;
}

// Source chunk length of an FP64 launch too small to fill the GPU with
// whole 256-source chunks (run with kAuto64Small's 32-source tiles, so that
// chunks may be any multiple of 32 sources without padding). The work items run
// in one or two waves, and each SM works through its CTAs at its FP64 pipe's
// rate. The length minimised is therefore ceil(items / SMs) x chunk length.
// Example: 5,120 sources and 31 tiles on 148 SMs. Whole-tile chunks allow at
// most 20 chunks: 620 items, 5 per SM, of 256 sources each (1,280). Chunks of
// 224 give 23 chunks: 713 items, 5 per SM, 1,120 (-12.5%).
static int fine_chunk_len(int tiles, int n, int num_sms, int slots, int max_chunks, int gran) {
  long long best_cost = -1;
  int best_len = n;
  for (int s = 1; s <= max_chunks; ++s) {
    int len = (n + s - 1) / s;
    len = (len + gran - 1) / gran * gran;
    const int chunks = (n + len - 1) / len;
    const long long items = (long long)tiles * chunks;
    if (items > 2LL * slots) break;
    const long long cost = (items + num_sms - 1) / num_sms * (long long)len;
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      best_len = len;
    }
  }
  return best_len;
}

// Chunk length of whole-tile chunks (tiles of ts sources).
static int whole_chunk_len(int tiles, int n, int ts, int slots, int min_chunk, int max_chunks) {
  const int S = choose_chunks(tiles, n, ts, slots, min_chunk, max_chunks);
  const int len = (n + S - 1) / S;
  return (len + ts - 1) / ts * ts;
}

// With the default FP64 variant's whole-tile chunks, does this launch fill
// less than 90% of one wave's CTA slots?
static bool fp64_small(const tc_ctx* ctx, int tiles, int n, int max_chunks) {
  const int slots = ctx->slots64_default;
  const int len = whole_chunk_len(tiles, n, kTS, slots, ctx->min_chunk, max_chunks);
  const long long items = (long long)tiles * ((n + len - 1) / len);
  return items * 10 < 9LL * slots;
}

// Tiles and chunking of one pair launch: the target segments, the grid and the
// chunk length (partial sums need S * 3 * n_out doubles).
static int plan_pairs(tc_ctx* ctx, const SegDesc* segs, int nseg, const double4* src, int n,
                      long long src_len, int n_out, int max_chunks, PairLaunch* P, dim3* grid) {
  const bool fp64 = ctx->precision == TC_FP64;
  if (!fp64) {
    const int rc0 = use_fp32c_variant(ctx, n);
    if (rc0) return rc0;
  }
  const PairCfg& cfg = fp64 ? ctx->cfg64 : ctx->cfg32;
  const int tb = cfg.tb();
  *P = PairLaunch{};
  int tiles = 0, k = 0;
  for (int s = 0; s < nseg; ++s) {
    int len = segs[s].i1 - segs[s].i0;
    if (len <= 0) continue;
    TargetSeg& g = P->seg[k++];
    g.x = segs[s].x;
    g.perm = fp64 ? nullptr : segs[s].perm;
    g.i0 = segs[s].i0;
    g.i1 = segs[s].i1;
    g.out_offset = segs[s].out_offset;
    g.self_offset = segs[s].self_offset;
    g.d2 = segs[s].d2;
    g.x_len = bc_extent(ctx, BC_PAIR_X, segs[s].x_len);
    g.perm_len = bc_extent(ctx, BC_PAIR_PERM, segs[s].perm_len);
    g.tile_begin = tiles;
    tiles += (len + tb - 1) / tb;
  }
  P->nseg = k;
  *grid = dim3(tiles, 0);
  if (tiles == 0 || n <= 0) return TC_OK;
  // automatic FP64 variant: the same target tiles either way, only the source tiles differ
  if (fp64 && ctx->auto64) {
    const int want = fp64_small(ctx, tiles, n, max_chunks) ? kAuto64Small : kAuto64Default;
    if (want != ctx->var64) {
      const int rc = select_variant(ctx, TC_FP64, want);
      if (rc) return rc;
    }
  }
  const PairCfg& cur = fp64 ? ctx->cfg64 : ctx->cfg32;
  const int slots = fp64 ? ctx->slots64 : ctx->slots32;
  const int chunk_len =
      (fp64 && ctx->auto64 && ctx->var64 == kAuto64Small)
          ? fine_chunk_len(tiles, n, ctx->num_sms, slots, max_chunks, cur.ts)
          : whole_chunk_len(tiles, n, cur.ts, slots, ctx->min_chunk, max_chunks);
  const int S = (n + chunk_len - 1) / chunk_len;
  P->src = src;
  P->n = n;
  P->chunk_len = chunk_len;
  P->n_out = n_out;
  P->bc = ctx->bc_rec;
  P->src_len = bc_extent(ctx, BC_PAIR_SRC, src_len);
  *grid = dim3(tiles, S);
  return TC_OK;
}

// Launches a planned pair kernel (timing events and counters as tc_stats reports them).
static int run_pairs(tc_ctx* ctx, const PairLaunch& P, dim3 grid) {
  const bool fp64 = ctx->precision == TC_FP64;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if (ctx->time_pairs) {
    TC_CUDA_TRY(cudaEventCreate(&ev[0]));
    TC_CUDA_TRY(cudaEventCreate(&ev[1]));
    TC_CUDA_TRY(cudaEventRecord(ev[0], ctx->stream));
  }
  variant(ctx->precision, fp64 ? ctx->var64 : ctx->var32)->launch(grid, ctx->stream, P);
  TC_CUDA_TRY(cudaGetLastError());
  if (ctx->time_pairs) {
    TC_CUDA_TRY(cudaEventRecord(ev[1], ctx->stream));
    ctx->pair_events.push_back(ev[0]);
    ctx->pair_events.push_back(ev[1]);
  }
  ctx->launches += 1;
  ctx->pair_launches += 1;
  for (int s = 0; s < P.nseg; ++s)
    ctx->pair_interactions += (long long)(P.seg[s].i1 - P.seg[s].i0) * P.n -
                              (P.seg[s].self_offset != kNoSelf ? (P.seg[s].i1 - P.seg[s].i0) : 0);
  return TC_OK;
}

int launch_pairs(tc_ctx* ctx, const SegDesc* segs, int nseg, const double4* src, int n,
                 long long src_len, int n_out, int* nchunks) {
  *nchunks = 0;
  PairLaunch P;
  dim3 grid;
  int rc = plan_pairs(ctx, segs, nseg, src, n, src_len, n_out, ctx->max_chunks, &P, &grid);
  if (rc || grid.y == 0) return rc;
  if ((rc = ctx->partial.ensure((size_t)grid.y * 3 * (size_t)n_out * sizeof(double)))) return rc;
  P.partial = ctx->partial.as<double>();
  P.partial_len = bc_extent(ctx, BC_PAIR_OUT, (long long)(ctx->partial.bytes / sizeof(double)));
  if ((rc = run_pairs(ctx, P, grid))) return rc;
  *nchunks = (int)grid.y;
  return TC_OK;
}

int launch_pairs_into(tc_ctx* ctx, const SegDesc* segs, int nseg, const double4* src, int n,
                      long long src_len, int n_out, double* partial, size_t partial_bytes,
                      int* nchunks) {
  *nchunks = 0;
  const size_t per_chunk = 3 * (size_t)n_out * sizeof(double);
  const size_t fit = per_chunk ? partial_bytes / per_chunk : (size_t)ctx->max_chunks;
  PairLaunch P;
  dim3 grid;
  int rc = plan_pairs(ctx, segs, nseg, src, n, src_len, n_out,
                      (int)std::max<size_t>(1, std::min<size_t>(fit, (size_t)ctx->max_chunks)), &P,
                      &grid);
  if (rc || grid.y == 0) return rc;
  if ((size_t)grid.y * per_chunk > partial_bytes) {
    tc_record_error("pair partial sums need %zu bytes, %zu given", (size_t)grid.y * per_chunk,
                    partial_bytes);
    return TC_ERR_ARG;
  }
  P.partial = partial;
  P.partial_len = bc_extent(ctx, BC_PAIR_OUT, (long long)(partial_bytes / sizeof(double)));
  if ((rc = run_pairs(ctx, P, grid))) return rc;
  *nchunks = (int)grid.y;
  return TC_OK;
}

// ---------------------------------------------------------------------------
// Packing: {x, y, z, zeta*area} per source.
// ---------------------------------------------------------------------------
// Checked build: extents of the packing's inputs (points) and output.
struct PackBounds {
  BoundsRec* rec;
  long long in_len, out_len;
};

__global__ void pack_kernel(const double* __restrict__ x, const double* __restrict__ zeta,
                            const double* __restrict__ area, int n, double4* __restrict__ out,
                            const PackBounds pb) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  if (!TC_BC(pb.rec, BC_PACK_IN, k, pb.in_len)) return;
  if (!TC_BC(pb.rec, BC_PACK_OUT, k, pb.out_len)) return;
  out[k] = make_double4(x[3 * (size_t)k], x[3 * (size_t)k + 1], x[3 * (size_t)k + 2],
                        __dmul_rn(zeta[k], area[k]));
}

// Forced model: stage-1 sources from the absolute vorticity at time t; the
// relative vorticity is also written to z0 (it is the state's zeta at t).
__global__ void pack_strat_kernel(const double* __restrict__ x, const double* __restrict__ absv,
                                  const double* __restrict__ area, int n, double two_omega,
                                  double t, double* __restrict__ zeta, double4* __restrict__ out,
                                  const PackBounds pb) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  if (!TC_BC(pb.rec, BC_PACK_IN, k, pb.in_len)) return;
  if (!TC_BC(pb.rec, BC_PACK_OUT, k, pb.out_len)) return;
  const double px = x[3 * (size_t)k], py = x[3 * (size_t)k + 1], pz = x[3 * (size_t)k + 2];
  const double z = strat_rel_vort(absv[k], two_omega, px, py, pz, t);
  zeta[k] = z;
  out[k] = make_double4(px, py, pz, __dmul_rn(z, area[k]));
}

__global__ void strat_rel_vort_kernel(const double* __restrict__ absv,
                                      const double* __restrict__ x, int n, double two_omega,
                                      double t, double* __restrict__ out, const PackBounds pb) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  if (!TC_BC(pb.rec, BC_PACK_IN, k, pb.in_len)) return;
  if (!TC_BC(pb.rec, BC_PACK_OUT, k, pb.out_len)) return;
  out[k] = strat_rel_vort(absv[k], two_omega, x[3 * (size_t)k], x[3 * (size_t)k + 1],
                          x[3 * (size_t)k + 2], t);
}

int launch_pack_strat(tc_ctx* ctx, double t) {
  Rk4State& R = ctx->rk;
  if (R.nA <= 0) return TC_OK;
  const long long in_len = (long long)std::min({R.x0A.bytes / (3 * sizeof(double)),
                                                R.absA.bytes / sizeof(double),
                                                R.areaA.bytes / sizeof(double)});
  const long long out_len =
      (long long)std::min(R.z0.bytes / sizeof(double), R.src.bytes / sizeof(double4));
  const PackBounds pb{ctx->bc_rec, bc_extent(ctx, BC_PACK_IN, in_len),
                      bc_extent(ctx, BC_PACK_OUT, out_len)};
  pack_strat_kernel<<<(R.nA + 255) / 256, 256, 0, ctx->stream>>>(
      R.x0A.as<double>(), R.absA.as<double>(), R.areaA.as<double>(), R.nA, 2.0 * ctx->omega, t,
      R.z0.as<double>(), R.src.as<double4>(), pb);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  return TC_OK;
}

int launch_strat_rel_vort(tc_ctx* ctx, const double* abs_vort, const double* x, int n, double t,
                          double* out) {
  if (n <= 0) return TC_OK;
  const PackBounds pb{ctx->bc_rec, bc_extent(ctx, BC_PACK_IN, n), bc_extent(ctx, BC_PACK_OUT, n)};
  strat_rel_vort_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(abs_vort, x, n,
                                                                  2.0 * ctx->omega, t, out, pb);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  return TC_OK;
}

int launch_pack(tc_ctx* ctx, const double* x, const double* zeta, const double* area, int n,
                double4* out, long long out_len) {
  if (n <= 0) return TC_OK;
  const PackBounds pb{ctx->bc_rec, bc_extent(ctx, BC_PACK_IN, n),
                      bc_extent(ctx, BC_PACK_OUT, out_len)};
  pack_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(x, zeta, area, n, out, pb);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  return TC_OK;
}

// ---------------------------------------------------------------------------
// Shared epilogue math.
// ---------------------------------------------------------------------------
// Sum of a partial row over the chunks; the checked build checks each read
// against partial_len doubles (site: BC_EPI_PARTIAL or BC_STAGE_PARTIAL).
__device__ __forceinline__ void reduce_row(const double* __restrict__ partial, int nchunks,
                                           size_t n_out, size_t row, double T[3],
                                           BoundsRec* rec, int site, long long partial_len) {
  T[0] = T[1] = T[2] = 0.0;
  for (int c = 0; c < nchunks; ++c) {
    const size_t o = (size_t)c * 3 * n_out + row;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const size_t j = o + (size_t)k * n_out;
      if (TC_BC(rec, site, j, partial_len)) T[k] += partial[j];
    }
  }
}

// u = (x x T) / (-4 pi): the reference divides the summed dX by (-4 pi).
__device__ __forceinline__ void velocity_from_sum(const double x[3], const double T[3],
                                                  double u[3]) {
  u[0] = (x[1] * T[2] - x[2] * T[1]) / kMinus4Pi;
  u[1] = (x[2] * T[0] - x[0] * T[2]) / kMinus4Pi;
  u[2] = (x[0] * T[1] - x[1] * T[0]) / kMinus4Pi;
}

// Thread p handles partial row p; with a visiting order perm (a permutation
// of [i0, i1)) that row belongs to target perm[p].
// Checked build: extents of the velocity epilogue's arrays.
struct EpiBounds {
  BoundsRec* rec;
  long long x_len, perm_len, partial_len, out_len;
};

__global__ void velocity_epilogue_kernel(const double* __restrict__ x, const int* __restrict__ perm,
                                         int m, int i0, int i1, int row_offset, int n_out,
                                         int nchunks, const double* __restrict__ partial,
                                         double m2omega, double* __restrict__ dX,
                                         double* __restrict__ dVort, const EpiBounds eb) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= m) return;
  const bool in_range = p >= i0 && p < i1;
  int i = p;
  if (in_range && perm) {
    if (!TC_BC(eb.rec, BC_EPI_PERM, p, eb.perm_len)) return;
    i = perm[p];
  }
  double u[3] = {0.0, 0.0, 0.0};
  if (in_range) {
    if (!TC_BC(eb.rec, BC_EPI_X, i, eb.x_len)) return;
    double xi[3] = {x[3 * (size_t)i], x[3 * (size_t)i + 1], x[3 * (size_t)i + 2]};
    double T[3];
    reduce_row(partial, nchunks, (size_t)n_out, (size_t)(row_offset + p), T, eb.rec,
               BC_EPI_PARTIAL, eb.partial_len);
    velocity_from_sum(xi, T, u);
  }
  if (!TC_BC(eb.rec, BC_EPI_OUT, i, eb.out_len)) return;
  dX[3 * (size_t)i] = u[0];
  dX[3 * (size_t)i + 1] = u[1];
  dX[3 * (size_t)i + 2] = u[2];
  if (dVort) dVort[i] = m2omega * u[2];
}

int launch_velocity_epilogue(tc_ctx* ctx, const double* x, const int* perm, int m, int i0, int i1,
                             int row_offset, int n_out, int nchunks, double* dX, double* dVort,
                             const double* partial, long long partial_len) {
  if (m <= 0) return TC_OK;
  if (!partial) {
    partial = ctx->partial.as<double>();
    partial_len = (long long)(ctx->partial.bytes / sizeof(double));
  }
  if (ctx->precision == TC_FP64) perm = nullptr;
  const EpiBounds eb{ctx->bc_rec, bc_extent(ctx, BC_EPI_X, m), bc_extent(ctx, BC_EPI_PERM, m),
                     bc_extent(ctx, BC_EPI_PARTIAL, partial_len), bc_extent(ctx, BC_EPI_OUT, m)};
  velocity_epilogue_kernel<<<(m + 255) / 256, 256, 0, ctx->stream>>>(
      x, perm, m, i0, i1, row_offset, n_out, nchunks, partial, -2.0 * ctx->omega, dX, dVort, eb);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  return TC_OK;
}

// ---------------------------------------------------------------------------
// RK4 stage epilogue (PanelVelocityParallel.f90:495-516, 545-558, 586-600,
// 628-656) fused over the three target classes:
//   k_s    = dt * u_s                         (:503-506)
//   new   += k_s / 6 or / 3                   (:637-644, evaluated left to right)
//   input  = x + {1/2, 1/2, 1} * k_s          (next stage's targets/sources)
//   active: dzeta = (-2 Omega) * u_z, same update for zeta; sources repacked
//   stage 1: kineticEnergy = u.u, per-block sums of KE*A (:495-501)
//   stage 4: the state advances to `new`.
// ---------------------------------------------------------------------------
struct StageEpi {
  int stage;
  double dt, m2omega;
  int nA, nV, nQ;
  int a0, a1, v0, v1, q0, q1;
  int n_out, nchunks;
  const double* partial;
  double *x0A, *z0, *x0V, *x0Q;
  const double* areaA;
  double *xiA, *ziA, *xiV, *xiQ;
  double *newA, *newZ, *newV, *newQ;
  double4* src;
  double* ke;
  double* keBlocks;
  const int *permA, *permV, *permQ;  // visiting orders of the three ranges (null: as stored)
  const int* row_nchunks;            // batched runs: chunks of each partial row (null: nchunks)
  const double* absA;                // forced model: absolute vorticity (null: BVE)
  double two_omega, t_next;          // forced model: 2 Omega, time of the next stage input
  // checked build: violation record and extents
  BoundsRec* rec;
  long long state_len[3];            // points in every state/stage array of each class
  long long active_len;              // entries in every active-only array
  long long perm_len[3];
  long long partial_len, chunks_len, keblock_len;
};

constexpr int kEpiThreads = 256;

__global__ void __launch_bounds__(kEpiThreads) stage_epilogue_kernel(const StageEpi E) {
  __shared__ double red[kEpiThreads];
  const int lenA = E.a1 - E.a0, lenV = E.v1 - E.v0, lenQ = E.q1 - E.q0;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  double ke_area = 0.0;
  if (r < lenA + lenV + lenQ) {
    int cls, pos;
    if (r < lenA) {
      cls = 0;
      pos = E.a0 + r;
    } else if (r < lenA + lenV) {
      cls = 1;
      pos = E.v0 + (r - lenA);
    } else {
      cls = 2;
      pos = E.q0 + (r - lenA - lenV);
    }
    const int* perm = cls == 0 ? E.permA : cls == 1 ? E.permV : E.permQ;
    int i = pos;
    bool ok = true;
    if (perm) {
      ok = TC_BC(E.rec, BC_STAGE_PERM, pos, E.perm_len[cls]);
      i = ok ? perm[pos] : 0;
    }
    ok = ok && TC_BC(E.rec, BC_STAGE_STATE, i, E.state_len[cls]);
    if (cls == 0) ok = ok && TC_BC(E.rec, BC_STAGE_ACTIVE, i, E.active_len);
    if (ok) {
      const int row = (cls == 0 ? 0 : cls == 1 ? E.nA : E.nA + E.nV) + pos;
      double* x0 = cls == 0 ? E.x0A : cls == 1 ? E.x0V : E.x0Q;
      double* xi = cls == 0 ? E.xiA : cls == 1 ? E.xiV : E.xiQ;
      double* nw = cls == 0 ? E.newA : cls == 1 ? E.newV : E.newQ;
      const double* xin = E.stage == 0 ? x0 : xi;
      const size_t b = 3 * (size_t)i;
      double xs[3] = {xin[b], xin[b + 1], xin[b + 2]};
      double T[3], u[3];
      int nch = E.nchunks;
      if (E.row_nchunks)
        nch = TC_BC(E.rec, BC_STAGE_CHUNKS, row, E.chunks_len) ? E.row_nchunks[row] : 0;
      reduce_row(E.partial, nch, (size_t)E.n_out, (size_t)row, T, E.rec, BC_STAGE_PARTIAL,
                 E.partial_len);
      velocity_from_sum(xs, T, u);
      if (cls == 0 && E.stage == 0) {
        double k2 = __dadd_rn(__dadd_rn(__dmul_rn(u[0], u[0]), __dmul_rn(u[1], u[1])),
                              __dmul_rn(u[2], u[2]));
        E.ke[i] = k2;
        ke_area = k2 * E.areaA[i];
      }
      const double div = (E.stage == 0 || E.stage == 3) ? 6.0 : 3.0;
      const double cnext = E.stage == 2 ? 1.0 : 0.5;
      double xnext[3];
      for (int c = 0; c < 3; ++c) {
        double kc = __dmul_rn(E.dt, u[c]);  // rounded like the reference's dt*stage
        double base = E.stage == 0 ? x0[b + c] : nw[b + c];
        double nv = base + kc / div;
        if (E.stage < 3) {
          nw[b + c] = nv;
          xnext[c] = x0[b + c] + (E.stage == 2 ? kc : cnext * kc);
          xi[b + c] = xnext[c];
        } else {
          x0[b + c] = nv;
          xnext[c] = nv;
        }
      }
      if (cls == 0 && E.absA) {
        // forced model (PanelVelocityParallel.f90:752-755, :800-803, :847-850, :908-911): the
        // vorticity is not integrated; the next input is rebuilt from absVort at t_next
        const double znext =
            strat_rel_vort(E.absA[i], E.two_omega, xnext[0], xnext[1], xnext[2], E.t_next);
        if (E.stage < 3)
          E.ziA[i] = znext;
        else
          E.z0[i] = znext;
        E.src[i] = make_double4(xnext[0], xnext[1], xnext[2], znext * E.areaA[i]);
      } else if (cls == 0) {
        double kz = __dmul_rn(E.dt, __dmul_rn(E.m2omega, u[2]));
        double zbase = E.stage == 0 ? E.z0[i] : E.newZ[i];
        double zn = zbase + kz / div;
        double znext;
        if (E.stage < 3) {
          E.newZ[i] = zn;
          znext = E.z0[i] + (E.stage == 2 ? kz : cnext * kz);
          E.ziA[i] = znext;
        } else {
          E.z0[i] = zn;
          znext = zn;
        }
        E.src[i] = make_double4(xnext[0], xnext[1], xnext[2], znext * E.areaA[i]);
      }
    }
  }
  if (E.stage == 0) {
    red[threadIdx.x] = ke_area;
    __syncthreads();
    for (int s = kEpiThreads / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0 && TC_BC(E.rec, BC_STAGE_KEBLOCK, blockIdx.x, E.keblock_len))
      E.keBlocks[blockIdx.x] = red[0];
  }
}

__global__ void ke_finalize_kernel(const double* __restrict__ blocks, int nblocks,
                                   double* __restrict__ out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int j = threadIdx.x; j < nblocks; j += 256) s += blocks[j];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = 0.5 * red[0];
}

// Capacity of a context buffer in elements of T.
template <class T>
static long long cap_of(const DevBuf& b) {
  return (long long)(b.bytes / sizeof(T));
}

int launch_stage_epilogue(tc_ctx* ctx, int stage, double dt, const int range[6], int nchunks,
                          double* total_ke, const int* row_nchunks, const double* partial,
                          long long row_nchunks_len, long long partial_len) {
  Rk4State& R = ctx->rk;
  StageEpi E;
  E.row_nchunks = row_nchunks;
  E.stage = stage;
  E.dt = dt;
  E.m2omega = -2.0 * ctx->omega;
  E.nA = R.nA;
  E.nV = R.nV;
  E.nQ = R.nQ;
  E.a0 = range[0];
  E.a1 = range[1];
  E.v0 = range[2];
  E.v1 = range[3];
  E.q0 = range[4];
  E.q1 = range[5];
  E.n_out = R.nA + R.nV + R.nQ;
  E.nchunks = nchunks;
  E.partial = partial ? partial : ctx->partial.as<double>();
  E.x0A = R.x0A.as<double>();
  E.z0 = R.z0.as<double>();
  E.x0V = R.x0V.as<double>();
  E.x0Q = R.x0Q.as<double>();
  E.areaA = R.areaA.as<double>();
  E.xiA = R.xiA.as<double>();
  E.ziA = R.ziA.as<double>();
  E.xiV = R.xiV.as<double>();
  E.xiQ = R.xiQ.as<double>();
  E.newA = R.newA.as<double>();
  E.newZ = R.newZ.as<double>();
  E.newV = R.newV.as<double>();
  E.newQ = R.newQ.as<double>();
  E.src = R.src.as<double4>();
  E.ke = R.ke.as<double>();
  E.keBlocks = R.keBlocks.as<double>();
  const bool ordered = ctx->precision != TC_FP64 && R.ordered;
  E.permA = ordered ? R.permA.as<int>() : nullptr;
  E.permV = ordered ? R.permV.as<int>() : nullptr;
  E.permQ = ordered ? R.permQ.as<int>() : nullptr;
  E.absA = R.strat ? R.absA.as<double>() : nullptr;
  E.two_omega = 2.0 * ctx->omega;
  E.rec = ctx->bc_rec;
  const DevBuf* cls_bufs[3][3] = {
      {&R.x0A, &R.xiA, &R.newA}, {&R.x0V, &R.xiV, &R.newV}, {&R.x0Q, &R.xiQ, &R.newQ}};
  const DevBuf* perm_bufs[3] = {&R.permA, &R.permV, &R.permQ};
  for (int c = 0; c < 3; ++c) {
    long long len = cap_of<double>(*cls_bufs[c][0]) / 3;
    for (int b = 1; b < 3; ++b) len = std::min(len, cap_of<double>(*cls_bufs[c][b]) / 3);
    E.state_len[c] = bc_extent(ctx, BC_STAGE_STATE, len);
    E.perm_len[c] = bc_extent(ctx, BC_STAGE_PERM, cap_of<int>(*perm_bufs[c]));
  }
  long long alen = cap_of<double4>(R.src);
  for (const DevBuf* b : {&R.z0, &R.ziA, &R.newZ, &R.areaA, &R.ke})
    alen = std::min(alen, cap_of<double>(*b));
  if (R.strat) alen = std::min(alen, cap_of<double>(R.absA));
  E.active_len = bc_extent(ctx, BC_STAGE_ACTIVE, alen);
  E.partial_len = bc_extent(ctx, BC_STAGE_PARTIAL, partial ? partial_len : cap_of<double>(ctx->partial));
  E.chunks_len = bc_extent(ctx, BC_STAGE_CHUNKS, row_nchunks_len);
  // stage inputs at t, t + dt/2, t + dt/2, t + dt; after stage 4 the next step's t
  const double t_step = R.t0 + (double)R.step * dt;
  E.t_next = stage < 2 ? t_step + 0.5 * dt
                       : (stage == 2 ? t_step + dt : R.t0 + (double)(R.step + 1) * dt);
  const int rows = (E.a1 - E.a0) + (E.v1 - E.v0) + (E.q1 - E.q0);
  const int blocks = std::max(1, (rows + kEpiThreads - 1) / kEpiThreads);
  if (stage == 0) {
    int rc = R.keBlocks.ensure((size_t)blocks * sizeof(double));
    if (rc) return rc;
    E.keBlocks = R.keBlocks.as<double>();
  }
  E.keblock_len = bc_extent(ctx, BC_STAGE_KEBLOCK, cap_of<double>(R.keBlocks));
  stage_epilogue_kernel<<<blocks, kEpiThreads, 0, ctx->stream>>>(E);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  if (stage == 0 && total_ke) {
    ke_finalize_kernel<<<1, 256, 0, ctx->stream>>>(E.keBlocks, blocks, total_ke);
    TC_CUDA_TRY(cudaGetLastError());
    ctx->launches += 1;
  }
  return TC_OK;
}

}  // namespace tcb
