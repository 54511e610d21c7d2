// Batched ensembles: many independent particle sets (ensemble members, grids
// of different refinement) advanced together. The instances are concatenated
// into one device RK4 state; the persistent pair kernel takes (instance,
// target tile, source chunk) work items so uneven sizes share the GPU, the
// fused stage epilogue runs unchanged on the concatenation, and the kinetic
// energy is reduced per instance. The whole nsteps-step sequence is captured
// once in a CUDA graph and replayed as one launch. A small autotuner picks
// the pair-kernel variant and the source-chunk length by timing one stage of
// the actual batch, and caches the choice per batch shape.
#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include <cstring>
#include <map>
#include <numeric>
#include <vector>

#include "sphere_order.cuh"
#include "tc_ctx.h"

using tcb::DevBuf;

namespace {

// Checked build: extents of the batch kernels' per-row arrays.
struct RowBounds {
  tcb::BoundsRec* rec;
  long long in_len;   // rows of the inputs (positions and instance ids; KE and areas)
  long long out_len;  // rows of the key and index outputs
};

// key = instance << 31 | sphere key (cube face, 2-D Hilbert index): one
// stable sort orders every instance's rows along the curve and keeps the
// instances in their ranges.
__global__ void batch_keys_kernel(const double* __restrict__ x, const int* __restrict__ row_inst,
                                  int n, unsigned long long* __restrict__ keys,
                                  int* __restrict__ idx, const RowBounds rb) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  if (!TC_BC(rb.rec, tcb::BC_ORDER_KEYS, j, rb.out_len)) return;
  const size_t b = 3 * (size_t)j;
  keys[j] = TC_BC(rb.rec, tcb::BC_ORDER_X, j, rb.in_len)
                ? ((unsigned long long)row_inst[j] << tcb::kSphereKeyBits) |
                      tcb::sphere_key(x[b], x[b + 1], x[b + 2])
                : 0ull;
  idx[j] = j;
}

// Kinetic energy of each instance: 0.5 * sum over its active rows of KE * A.
__global__ void ke_segments_kernel(const double* __restrict__ ke, const double* __restrict__ area,
                                   const int* __restrict__ off, const int* __restrict__ cnt,
                                   double* __restrict__ out, const RowBounds rb) {
  __shared__ double red[256];
  const int b = blockIdx.x;
  double s = 0.0;
  for (int j = threadIdx.x; j < cnt[b]; j += 256) {
    const int r = off[b] + j;
    if (TC_BC(rb.rec, tcb::BC_BATCH_KE, r, rb.in_len)) s += ke[r] * area[r];
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[b] = 0.5 * red[0];
}

}  // namespace

// Host-side plan of one batch shape.
struct tc_batch_plan {
  int count = 0;
  std::vector<int> nA, nV, aOff, vOff;
  int nA_tot = 0, nV_tot = 0;
  int variant = -1, chunk_len = 0, n_items = 0, slots = 0;
  DevBuf items, segs0, segs1, counters, row_nchunks, row_inst, off_d, cnt_d, keys, keys2, vals,
      sort_tmp, ke_out, partial;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = -1;
  double graph_dt = 0.0;
  std::vector<void*> graph_ptrs;  // every device buffer the graph touches, at capture time
  cudaStream_t stream = nullptr;  // used when the context runs on the (uncapturable) NULL stream
  ~tc_batch_plan() {
    if (graph) cudaGraphExecDestroy(graph);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

std::map<std::vector<int>, std::pair<int, int>> g_tuned;  // batch shape -> (variant, chunk)

int sort_batch_rows(tc_ctx* ctx, tc_batch_plan& B, const double* x, long long x_len,
                    const int* row_inst, int n, int* perm) {
  if (n <= 0) return TC_OK;
  int rc;
  if ((rc = B.keys.ensure((size_t)n * 8)) || (rc = B.keys2.ensure((size_t)n * 8)) ||
      (rc = B.vals.ensure((size_t)n * 4)))
    return rc;
  const long long in_len = std::min(x_len, (long long)(B.row_inst.bytes / sizeof(int)));
  const long long out_len = (long long)std::min(B.keys.bytes / 8, B.vals.bytes / 4);
  const RowBounds rb{ctx->bc_rec, tcb::bc_extent(ctx, tcb::BC_ORDER_X, in_len),
                     tcb::bc_extent(ctx, tcb::BC_ORDER_KEYS, out_len)};
  batch_keys_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(
      x, row_inst, n, B.keys.as<unsigned long long>(), B.vals.as<int>(), rb);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  int bits = tcb::kSphereKeyBits;
  while ((1 << (bits - tcb::kSphereKeyBits)) < B.count + 1) ++bits;
  size_t temp = 0;
  TC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp, B.keys.as<unsigned long long>(),
                                              B.keys2.as<unsigned long long>(), B.vals.as<int>(),
                                              perm, n, 0, bits, ctx->stream));
  if ((rc = B.sort_tmp.ensure(temp))) return rc;
  TC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(B.sort_tmp.ptr, temp,
                                              B.keys.as<unsigned long long>(),
                                              B.keys2.as<unsigned long long>(), B.vals.as<int>(),
                                              perm, n, 0, bits, ctx->stream));
  return TC_OK;
}

// Work items and per-row chunk counts for (variant, chunk_len); uploads them.
int build_items(tc_ctx* ctx, tc_batch_plan& B, int variant, int chunk_len) {
  const tcb::PairVariant* v = tcb::variant(ctx->precision, variant);
  const int tb = v->nt * v->tpt;
  std::vector<tcb::BatchItem> items;
  std::vector<int> rn(B.nA_tot + B.nV_tot, 0);
  for (int b = 0; b < B.count; ++b) {
    const int nch = std::max(1, (B.nA[b] + chunk_len - 1) / chunk_len);
    for (int cls = 0; cls < 2; ++cls) {
      const int off = cls == 0 ? B.aOff[b] : B.vOff[b];
      const int n = cls == 0 ? B.nA[b] : B.nV[b];
      const int row0 = cls == 0 ? off : B.nA_tot + off;
      for (int r = 0; r < n; ++r) rn[row0 + r] = B.nA[b] > 0 ? nch : 0;
      if (B.nA[b] == 0) continue;
      for (int t = off; t < off + n; t += tb)
        for (int c = 0; c < nch; ++c) {
          tcb::BatchItem it;
          it.seg = 2 * b + cls;
          it.tile0 = t;
          it.i1 = off + n;
          it.c0 = B.aOff[b] + c * chunk_len;
          it.c1 = std::min(B.aOff[b] + B.nA[b], it.c0 + chunk_len);
          it.chunk = c;
          items.push_back(it);
        }
    }
  }
  // longest first: cost = targets in the tile x sources in the chunk
  std::stable_sort(items.begin(), items.end(), [tb](const tcb::BatchItem& a, const tcb::BatchItem& b) {
    long long ca = (long long)std::min(tb, a.i1 - a.tile0) * (a.c1 - a.c0);
    long long cb = (long long)std::min(tb, b.i1 - b.tile0) * (b.c1 - b.c0);
    return ca > cb;
  });
  int rc;
  if ((rc = B.items.ensure(std::max<size_t>(1, items.size()) * sizeof(tcb::BatchItem))) ||
      (rc = B.row_nchunks.ensure(std::max<size_t>(1, rn.size()) * sizeof(int))))
    return rc;
  if (!items.empty())
    TC_CUDA_TRY(cudaMemcpyAsync(B.items.ptr, items.data(), items.size() * sizeof(tcb::BatchItem),
                                cudaMemcpyHostToDevice, ctx->stream));
  if (!rn.empty())
    TC_CUDA_TRY(cudaMemcpyAsync(B.row_nchunks.ptr, rn.data(), rn.size() * sizeof(int),
                                cudaMemcpyHostToDevice, ctx->stream));
  int max_chunks = 1;
  for (int b = 0; b < B.count; ++b)
    max_chunks = std::max(max_chunks, (B.nA[b] + chunk_len - 1) / chunk_len);
  if ((rc = B.partial.ensure((size_t)max_chunks * 3 * (B.nA_tot + B.nV_tot) * sizeof(double))))
    return rc;
  int blocks = 0;
  TC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, v->fn_batch, v->nt, 0));
  B.slots = std::max(1, blocks) * ctx->num_sms;
  B.n_items = (int)items.size();
  B.variant = variant;
  B.chunk_len = chunk_len;
  // the stream must finish with the host vectors before they go out of scope
  TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return TC_OK;
}

int upload_segments(tc_ctx* ctx, tc_batch_plan& B) {
  tcb::Rk4State& R = ctx->rk;
  const bool ord = ctx->precision == TC_FP32C && R.ordered;
  std::vector<tcb::BatchSeg> s0, s1;
  for (int b = 0; b < B.count; ++b)
    for (int cls = 0; cls < 2; ++cls) {
      tcb::BatchSeg g;
      g.perm = ord ? (cls == 0 ? R.permA.as<int>() : R.permV.as<int>()) : nullptr;
      g.out_offset = cls == 0 ? 0 : B.nA_tot;
      g.self_offset = cls == 0 ? 0 : tcb::kNoSelf;
      g.d2 = ctx->delta[cls] * ctx->delta[cls];
      g.perm_len = g.perm ? (long long)((cls == 0 ? R.permA : R.permV).bytes / sizeof(int)) : 0;
      g.x = cls == 0 ? R.x0A.as<double>() : R.x0V.as<double>();
      g.x_len = (long long)((cls == 0 ? R.x0A : R.x0V).bytes / (3 * sizeof(double)));
      s0.push_back(g);
      g.x = cls == 0 ? R.xiA.as<double>() : R.xiV.as<double>();
      g.x_len = (long long)((cls == 0 ? R.xiA : R.xiV).bytes / (3 * sizeof(double)));
      s1.push_back(g);
    }
  int rc;
  const size_t bytes = s0.size() * sizeof(tcb::BatchSeg);
  if ((rc = B.segs0.ensure(bytes)) || (rc = B.segs1.ensure(bytes))) return rc;
  TC_CUDA_TRY(cudaMemcpyAsync(B.segs0.ptr, s0.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
  TC_CUDA_TRY(cudaMemcpyAsync(B.segs1.ptr, s1.data(), bytes, cudaMemcpyHostToDevice, ctx->stream));
  TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return TC_OK;
}

int launch_batch_pairs(tc_ctx* ctx, tc_batch_plan& B, int stage) {
  const tcb::PairVariant* v = tcb::variant(ctx->precision, B.variant);
  int* counter = B.counters.as<int>() + stage;
  TC_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int), ctx->stream));
  tcb::BatchLaunch L;
  L.items = B.items.as<tcb::BatchItem>();
  L.n_items = B.n_items;
  L.counter = counter;
  L.segs = (stage == 0 ? B.segs0 : B.segs1).as<tcb::BatchSeg>();
  L.src = ctx->rk.src.as<double4>();
  L.partial = B.partial.as<double>();
  L.stride = (size_t)(B.nA_tot + B.nV_tot);
  L.bc = ctx->bc_rec;
  L.n_segs = (int)tcb::bc_extent(ctx, tcb::BC_BATCH_SEG, 2 * B.count);
  L.src_len =
      tcb::bc_extent(ctx, tcb::BC_PAIR_SRC, (long long)(ctx->rk.src.bytes / sizeof(double4)));
  L.partial_len =
      tcb::bc_extent(ctx, tcb::BC_PAIR_OUT, (long long)(B.partial.bytes / sizeof(double)));
  v->launch_batch(B.slots, ctx->stream, L);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  ctx->pair_launches += 1;
  for (int b = 0; b < B.count; ++b)
    ctx->pair_interactions += (long long)B.nA[b] * (B.nA[b] - 1) + (long long)B.nV[b] * B.nA[b];
  return TC_OK;
}

int enqueue_steps(tc_ctx* ctx, tc_batch_plan& B, double dt, int nsteps) {
  const int range[6] = {0, B.nA_tot, 0, B.nV_tot, 0, 0};
  int rc;
  for (int step = 0; step < nsteps; ++step)
    for (int s = 0; s < 4; ++s) {
      if ((rc = launch_batch_pairs(ctx, B, s))) return rc;
      if ((rc = tcb::launch_stage_epilogue(
               ctx, s, dt, range, 0, nullptr, B.row_nchunks.as<int>(), B.partial.as<double>(),
               (long long)(B.row_nchunks.bytes / sizeof(int)),
               (long long)(B.partial.bytes / sizeof(double)))))
        return rc;
      if (s == 0) {
        const long long ke_len = (long long)std::min(ctx->rk.ke.bytes, ctx->rk.areaA.bytes) /
                                 (long long)sizeof(double);
        const RowBounds rb{ctx->bc_rec, tcb::bc_extent(ctx, tcb::BC_BATCH_KE, ke_len), 0};
        ke_segments_kernel<<<B.count, 256, 0, ctx->stream>>>(
            ctx->rk.ke.as<double>(), ctx->rk.areaA.as<double>(), B.off_d.as<int>(),
            B.cnt_d.as<int>(), B.ke_out.as<double>() + (size_t)step * B.count, rb);
        TC_CUDA_TRY(cudaGetLastError());
        ctx->launches += 1;
      }
    }
  return TC_OK;
}

// Time one stage-0 pair launch of each (variant, chunk) candidate; keep the best.
// Candidate launch shapes: the default of each precision first, then the
// shapes that were fastest on some workload of the level-7 sweep, all with the
// default's accuracy (64-source FP32 flush; a 128-source flush is faster by
// about 1% and raises the error by half).
const int kTune32[] = {0, 1, 2, 3, 4, 5, 6, 7};
const int kTune64[] = {2, 0, 1, 3};

// Times one stage-0 launch of the whole batch (best of `reps`).
int time_launch(tc_ctx* ctx, tc_batch_plan& B, cudaEvent_t e0, cudaEvent_t e1, int reps,
                float* ms) {
  *ms = 1e30f;
  for (int rep = 0; rep < reps; ++rep) {
    TC_CUDA_TRY(cudaEventRecord(e0, ctx->stream));
    int rc = launch_batch_pairs(ctx, B, 0);
    if (rc) return rc;
    TC_CUDA_TRY(cudaEventRecord(e1, ctx->stream));
    TC_CUDA_TRY(cudaEventSynchronize(e1));
    float t = 0.f;
    TC_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
    *ms = std::min(*ms, t);
  }
  return TC_OK;
}

// Two passes over the candidates: the variant at a 4096-source chunk, then
// the chunk length {1024, 2048, 4096, 8192} for the winner (11 launches for
// FP32C instead of every variant x chunk); cached per batch shape.
int autotune(tc_ctx* ctx, tc_batch_plan& B) {
  std::vector<int> key = {ctx->precision, B.count};
  key.insert(key.end(), B.nA.begin(), B.nA.end());
  key.insert(key.end(), B.nV.begin(), B.nV.end());
  auto hit = g_tuned.find(key);
  if (hit != g_tuned.end()) return build_items(ctx, B, hit->second.first, hit->second.second);
  const bool fp64 = ctx->precision == TC_FP64;
  const int* cand = fp64 ? kTune64 : kTune32;
  const int ncand = fp64 ? (int)(sizeof(kTune64) / sizeof(int)) : (int)(sizeof(kTune32) / sizeof(int));
  const int chunks[] = {1024, 2048, 4096, 8192};
  cudaEvent_t e0, e1;
  TC_CUDA_TRY(cudaEventCreate(&e0));
  TC_CUDA_TRY(cudaEventCreate(&e1));
  float best = 1e30f, ms = 0.f;
  int bv = cand[0], bc = 4096, rc = TC_OK;
  for (int j = 0; j < ncand && rc == TC_OK; ++j) {
    if (cand[j] >= tcb::variant_count(ctx->precision)) continue;
    if ((rc = build_items(ctx, B, cand[j], 4096)) || (rc = time_launch(ctx, B, e0, e1, 1, &ms))) break;
    if (ms < best) {
      best = ms;
      bv = cand[j];
    }
  }
  for (int c : chunks) {
    if (rc || c == 4096) continue;
    if ((rc = build_items(ctx, B, bv, c)) || (rc = time_launch(ctx, B, e0, e1, 1, &ms))) break;
    if (ms < best) {
      best = ms;
      bc = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  g_tuned[key] = {bv, bc};
  return build_items(ctx, B, bv, bc);
}

}  // namespace

// Batched RK4 over `count` independent instances stored back to back (host
// arrays): xA(3, sum nA), zetaA, areaA (sum nA), xV(3, sum nV); instance b owns
// rows [sum_{c<b} nA_c, +nA[b]) and [sum_{c<b} nV_c, +nV[b]). Each instance
// evolves as its own BVERK4 (sources = its own active panels). totalKE:
// nsteps x count (step-major), host. flags: TC_BATCH_GRAPH, TC_BATCH_AUTOTUNE.
static int batch_rk4_impl(tc_ctx* ctx, int count, const int* nA, const int* nV, double* xA,
                          double* zetaA, const double* areaA, double* xV, double dt, int nsteps,
                          double* totalKE, int flags) {
  tc_batch_plan& B = *ctx->batch;
  const bool same_shape = B.count == count && std::equal(B.nA.begin(), B.nA.end(), nA) &&
                          std::equal(B.nV.begin(), B.nV.end(), nV);
  if (!same_shape) {
    if (B.graph) cudaGraphExecDestroy(B.graph);
    B.graph = nullptr;
    B.graph_steps = -1;
    B.variant = -1;
  }
  B.count = count;
  B.nA.assign(nA, nA + count);
  B.nV.assign(nV, nV + count);
  B.aOff.assign(count, 0);
  B.vOff.assign(count, 0);
  B.nA_tot = B.nV_tot = 0;
  for (int b = 0; b < count; ++b) {
    if (nA[b] < 0 || nV[b] < 0) return TC_ERR_ARG;
    B.aOff[b] = B.nA_tot;
    B.vOff[b] = B.nV_tot;
    B.nA_tot += nA[b];
    B.nV_tot += nV[b];
  }
  if ((B.nA_tot && (!xA || !zetaA || !areaA)) || (B.nV_tot && !xV) || (nsteps && !totalKE)) {
    tc_record_error("tc_batch_rk4: null array argument");
    return TC_ERR_ARG;
  }
  int rc = tc_rk4_load(ctx, xA, zetaA, areaA, B.nA_tot, xV, B.nV_tot, nullptr, 0, 0);
  if (rc) return rc;
  tcb::Rk4State& R = ctx->rk;
  // per-row instance ids and per-instance offsets
  std::vector<int> inst(std::max(B.nA_tot, B.nV_tot), 0), off(count), cnt(count);
  if ((rc = B.row_inst.ensure(std::max<size_t>(1, inst.size()) * sizeof(int) * 2)) ||
      (rc = B.off_d.ensure(count * sizeof(int))) || (rc = B.cnt_d.ensure(count * sizeof(int))) ||
      (rc = B.counters.ensure(4 * sizeof(int))) ||
      (rc = B.ke_out.ensure(std::max<size_t>(1, (size_t)nsteps * count) * sizeof(double))) ||
      (rc = R.permA.ensure(std::max<size_t>(1, B.nA_tot) * sizeof(int))) ||
      (rc = R.permV.ensure(std::max<size_t>(1, B.nV_tot) * sizeof(int))))
    return rc;
  for (int b = 0; b < count; ++b) {
    off[b] = B.aOff[b];
    cnt[b] = nA[b];
  }
  TC_CUDA_TRY(cudaMemcpyAsync(B.off_d.ptr, off.data(), count * sizeof(int), cudaMemcpyHostToDevice,
                              ctx->stream));
  TC_CUDA_TRY(cudaMemcpyAsync(B.cnt_d.ptr, cnt.data(), count * sizeof(int), cudaMemcpyHostToDevice,
                              ctx->stream));
  R.ordered = false;
  if (ctx->precision == TC_FP32C && ctx->target_order == TC_ORDER_HILBERT) {
    int* ri = B.row_inst.as<int>();
    for (int cls = 0; cls < 2; ++cls) {
      const int n = cls == 0 ? B.nA_tot : B.nV_tot;
      for (int b = 0; b < count; ++b) {
        const int o = cls == 0 ? B.aOff[b] : B.vOff[b], m = cls == 0 ? nA[b] : nV[b];
        std::fill(inst.begin() + o, inst.begin() + o + m, b);
      }
      TC_CUDA_TRY(cudaMemcpyAsync(ri, inst.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice,
                                  ctx->stream));
      const tcb::DevBuf& xb = cls == 0 ? R.x0A : R.x0V;
      const tcb::DevBuf& pbuf = cls == 0 ? R.permA : R.permV;
      if ((long long)(pbuf.bytes / sizeof(int)) < n) {
        tc_record_error("batch visiting order: %d rows, room for %zu", n, pbuf.bytes / sizeof(int));
        return TC_ERR_ARG;
      }
      const long long x_len = (long long)(xb.bytes / (3 * sizeof(double)));
      if ((rc = sort_batch_rows(ctx, B, xb.as<double>(), x_len, ri, n, pbuf.as<int>()))) return rc;
      TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // `inst` is reused for the next class
    }
    R.ordered = true;
    const int rng[6] = {0, B.nA_tot, 0, B.nV_tot, 0, 0};
    memcpy(R.order_range, rng, sizeof(rng));
  }
  if ((rc = upload_segments(ctx, B))) return rc;
  if ((rc = tc_rk4_pack_sources(ctx))) return rc;
  if (B.variant < 0) {
    if (flags & TC_BATCH_AUTOTUNE) {
      if ((rc = autotune(ctx, B))) return rc;
    } else {
      const int v = ctx->precision == TC_FP64 ? (ctx->auto64 ? tcb::kAuto64Default : ctx->var64)
                                              : ctx->var32;
      if ((rc = build_items(ctx, B, v, 4096))) return rc;
    }
    if ((rc = tc_rk4_pack_sources(ctx))) return rc;  // autotuning ran stage-0 launches only
  }
  // the stage-0 epilogue's per-block kinetic-energy buffer: sized before any capture
  if ((rc = R.keBlocks.ensure(((size_t)(B.nA_tot + B.nV_tot) + 255) / 256 * sizeof(double) + 16)))
    return rc;
  if (nsteps > 0) {
    const std::vector<void*> ptrs = {R.x0A.ptr, R.z0.ptr, R.areaA.ptr, R.x0V.ptr, R.xiA.ptr,
                                     R.ziA.ptr, R.xiV.ptr, R.newA.ptr, R.newZ.ptr, R.newV.ptr,
                                     R.src.ptr, R.ke.ptr, R.keBlocks.ptr, R.permA.ptr, R.permV.ptr,
                                     B.items.ptr, B.segs0.ptr, B.segs1.ptr, B.counters.ptr,
                                     B.row_nchunks.ptr, B.off_d.ptr, B.cnt_d.ptr, B.ke_out.ptr,
                                     B.partial.ptr};
    if (flags & TC_BATCH_GRAPH) {
      if (!B.graph || B.graph_steps != nsteps || B.graph_dt != dt || B.graph_ptrs != ptrs) {
        if (B.graph) cudaGraphExecDestroy(B.graph);
        B.graph = nullptr;
        cudaGraph_t g;
        TC_CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        rc = enqueue_steps(ctx, B, dt, nsteps);
        cudaError_t ce = cudaStreamEndCapture(ctx->stream, &g);
        if (rc) return rc;
        if (ce != cudaSuccess) {
          tc_record_error("graph capture failed: %s", cudaGetErrorString(ce));
          return TC_ERR_CUDA;
        }
        TC_CUDA_TRY(cudaGraphInstantiate(&B.graph, g, 0));
        cudaGraphDestroy(g);
        B.graph_steps = nsteps;
        B.graph_dt = dt;
        B.graph_ptrs = ptrs;
      }
      TC_CUDA_TRY(cudaGraphLaunch(B.graph, ctx->stream));
    } else if ((rc = enqueue_steps(ctx, B, dt, nsteps))) {
      return rc;
    }
    TC_CUDA_TRY(cudaMemcpyAsync(totalKE, B.ke_out.ptr, (size_t)nsteps * count * sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->stream));
  }
  return tc_rk4_store(ctx, xA, zetaA, xV, nullptr, nullptr, 0);
}

extern "C" int tc_batch_rk4(tc_ctx* ctx, int count, const int* nA, const int* nV, double* xA,
                            double* zetaA, const double* areaA, double* xV, double dt, int nsteps,
                            double* totalKE, int flags) {
  if (!ctx || count <= 0 || !nA || !nV || nsteps < 0 || !std::isfinite(dt)) {
    tc_record_error("tc_batch_rk4: bad arguments");
    return TC_ERR_ARG;
  }
  TcNvtxRange nvtx_batch("tc batch rk4");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return TC_ERR_CUDA;
  if (!ctx->batch) ctx->batch = new tc_batch_plan();
  tc_batch_plan& B = *ctx->batch;
  // The legacy NULL stream cannot be captured into a graph: run the batch on
  // the plan's own stream, after the work already queued on the NULL stream.
  const cudaStream_t user = ctx->stream;
  if (!user) {
    if (!B.stream) TC_CUDA_TRY(cudaStreamCreateWithFlags(&B.stream, cudaStreamNonBlocking));
    TC_CUDA_TRY(cudaStreamSynchronize(nullptr));
    ctx->stream = B.stream;
  }
  const int rc = batch_rk4_impl(ctx, count, nA, nV, xA, zetaA, areaA, xV, dt, nsteps, totalKE, flags);
  if (!user) {
    cudaStreamSynchronize(ctx->stream);
    ctx->stream = nullptr;
  }
  return rc;
}

// The variant and source-chunk length the last tc_batch_rk4 call used.
extern "C" int tc_batch_info(tc_ctx* ctx, int* variant, int* chunk_len, int* n_items) {
  if (!ctx || !ctx->batch) return TC_ERR_STATE;
  if (variant) *variant = ctx->batch->variant;
  if (chunk_len) *chunk_len = ctx->batch->chunk_len;
  if (n_items) *n_items = ctx->batch->n_items;
  return TC_OK;
}

void tc_batch_free(tc_ctx* ctx) {
  delete ctx->batch;
  ctx->batch = nullptr;
}
