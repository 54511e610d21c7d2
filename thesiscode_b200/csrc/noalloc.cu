// Allocation-free variant of tc_bs_velocity_device.
//
// Some callers of this library cannot let it allocate device memory when
// they call it: a host code whose device memory is owned entirely by its own
// pool allocator (the whole GPU pre-reserved for the model state), and
// time-stepping loops that overlap work on several streams, where cudaMalloc's
// implicit device-wide synchronisation in the middle of a step is not
// acceptable. For them, tc_bs_velocity_device_noalloc computes the same sum
// as tc_bs_velocity_device with its scratch - the packed sources and the FP64
// partial sums of the pair kernel - in a fixed array compiled into the
// library, so a call allocates nothing.
//
// The array is a file-scope static __device__ array of kNoAllocScratchBytes
// (32 MiB); every GPU that loads the library holds it until the process
// exits. A call needs 32*n (rounded up to 256) + 24*m*chunks bytes of it, so
// the largest single-chunk problem is 32*n + 24*m <= 32 MiB (for example
// 327,680 active panels with themselves as targets); larger calls are
// rejected with TC_ERR_ARG. Host code cannot use the array's name as a device
// address, so the first call on each device looks the address up with
// cudaGetSymbolAddress (with that device current) and caches it; make that
// first call before any stream capture on the device.
//
// Every call shares the array and it keeps the previous call's contents:
// the pair kernel writes every partial-sum row the epilogue reads, so nothing
// has to start at zero. Calls that overlap on the GPU (on different streams
// or from different contexts on the same device) race on the array; callers
// must order them.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "tc_ctx.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double)];

std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (which must be current).
int scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) {
    tc_record_error("tc_bs_velocity_device_noalloc: device %d out of range", device);
    return TC_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      tc_record_error("cudaGetSymbolAddress of the no-allocation scratch failed: %s",
                      cudaGetErrorString(e));
      cudaGetLastError();
      return TC_ERR_CUDA;
    }
    g_scratch_ptr[device] = p;
  }
  *out = g_scratch_ptr[device];
  return TC_OK;
}

size_t round256(size_t b) { return (b + 255) / 256 * 256; }

}  // namespace

extern "C" int tc_bs_velocity_device_noalloc(tc_ctx* ctx, int target_class, const double* X,
                                             int m, const double* src_x, const double* vort,
                                             const double* area, int n, int i0, int i1,
                                             double* dX, double* dVort) {
  if (!ctx) {
    tc_record_error("null context");
    return TC_ERR_ARG;
  }
  if (target_class != TC_ACTIVE && target_class != TC_VERTEX && target_class != TC_PASSIVE) {
    tc_record_error("target_class %d is not TC_ACTIVE/TC_VERTEX/TC_PASSIVE", target_class);
    return TC_ERR_ARG;
  }
  if (m < 0 || n < 0 || i0 < 0 || i1 < i0 || i1 > m) {
    tc_record_error("bad sizes or range (m=%d, n=%d, [%d,%d))", m, n, i0, i1);
    return TC_ERR_ARG;
  }
  if (target_class == TC_ACTIVE && ((X != nullptr && X != src_x) || m != n)) {
    tc_record_error("TC_ACTIVE targets are the sources: X = NULL or src_x, and m == n");
    return TC_ERR_ARG;
  }
  if ((n > 0 && (!src_x || !vort || !area)) || (m > 0 && !dX) ||
      (target_class != TC_ACTIVE && m > 0 && !X)) {
    tc_record_error("null array argument");
    return TC_ERR_ARG;
  }
  const size_t src_bytes = round256((size_t)n * sizeof(double4));
  const size_t row_bytes = 3 * (size_t)m * sizeof(double);
  if (src_bytes + row_bytes > kNoAllocScratchBytes) {
    tc_record_error("tc_bs_velocity_device_noalloc: n=%d sources and m=%d targets need %zu bytes "
                    "of scratch, more than the fixed %zu bytes (32*n + 24*m must fit)",
                    n, m, src_bytes + row_bytes, kNoAllocScratchBytes);
    return TC_ERR_ARG;
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    tc_record_error("cudaSetDevice(%d) failed", ctx->device);
    return TC_ERR_CUDA;
  }
  void* base = nullptr;
  int rc = scratch_address(ctx->device, &base);
  if (rc) return rc;
  if (target_class == TC_ACTIVE) X = src_x;
  double4* src = static_cast<double4*>(base);
  double* partial = reinterpret_cast<double*>(static_cast<char*>(base) + src_bytes);

  const bool fp64 = ctx->precision == TC_FP64;
  if (!fp64 && (rc = tcb::use_fp32c_variant(ctx, n))) return rc;
  const tcb::PairVariant* v = tcb::variant(ctx->precision, fp64 ? ctx->var64 : ctx->var32);
  const int tb = v->nt * v->tpt;
  const int len = i1 - i0;
  int nchunks = 0;
  if (n > 0) {
    tcb::pack_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(src_x, vort, area, n, src);
    TC_CUDA_TRY(cudaGetLastError());
  }
  if (len > 0 && n > 0) {
    // source chunks: fill the resident CTA slots in whole waves, as far as the scratch allows
    const int tiles = (len + tb - 1) / tb;
    const int slots = fp64 ? ctx->slots64 : ctx->slots32;
    const int fit = (int)std::min<size_t>((kNoAllocScratchBytes - src_bytes) / row_bytes, 64);
    int best = 1;
    double best_eff = 0.0;
    for (int s = 1; s <= fit; ++s) {
      if (s > 1 && (n + s - 1) / s < ctx->min_chunk) break;
      long long items = (long long)tiles * s;
      long long waves = (items + slots - 1) / slots;
      double eff = (double)items / (double)(waves * slots);
      if (eff > best_eff + 0.02) {
        best_eff = eff;
        best = s;
      }
    }
    int chunk_len = (n + best - 1) / best;
    chunk_len = (chunk_len + v->ts - 1) / v->ts * v->ts;
    nchunks = (n + chunk_len - 1) / chunk_len;
    tcb::PairLaunch P{};
    P.seg[0].x = X;
    P.seg[0].perm = nullptr;  // targets in the caller's order
    P.seg[0].i0 = i0;
    P.seg[0].i1 = i1;
    P.seg[0].out_offset = 0;
    P.seg[0].self_offset = target_class == TC_ACTIVE ? 0 : tcb::kNoSelf;
    P.seg[0].d2 = ctx->delta[target_class] * ctx->delta[target_class];
    P.seg[0].tile_begin = 0;
    P.nseg = 1;
    P.src = src;
    P.n = n;
    P.chunk_len = chunk_len;
    P.partial = partial;
    P.n_out = m;
    v->launch(dim3(tiles, nchunks), ctx->stream, P);
    TC_CUDA_TRY(cudaGetLastError());
  }
  if (m > 0) {
    tcb::velocity_epilogue_kernel<<<(m + 255) / 256, 256, 0, ctx->stream>>>(
        X, nullptr, m, i0, i1, 0, m, nchunks, partial, -2.0 * ctx->omega, dX,
        target_class == TC_ACTIVE ? dVort : nullptr);
    TC_CUDA_TRY(cudaGetLastError());
  }
  return TC_OK;
}
