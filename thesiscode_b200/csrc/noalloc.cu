// Allocation-free variant of tc_bs_velocity_device.
//
// Some callers of this library cannot let it allocate device memory when
// they call it: a host code whose device memory is owned entirely by its own
// pool allocator (the whole GPU pre-reserved for the model state), and
// time-stepping loops that overlap work on several streams, where cudaMalloc's
// implicit device-wide synchronisation in the middle of a step is not
// acceptable. For them, tc_bs_velocity_device_noalloc computes the same sum
// as tc_bs_velocity_device with all of its scratch - the packed sources, the
// FP64 partial sums of the pair kernel and, for FP32C, the targets' visiting
// order with its sort buffers - in a fixed array compiled into the library,
// so a call allocates nothing.
//
// The array is a file-scope static __device__ array of kNoAllocScratchBytes
// (32 MiB); every GPU that loads the library holds it until the process
// exits. A call needs 32*n bytes for the sources (each part rounded up to 256
// bytes), 24*m per source chunk for the partial sums and, for FP32C with the
// library's visiting order, 4*m for the order plus about 20 bytes per target
// in range [i0, i1) for its sort; larger calls are rejected with TC_ERR_ARG.
// The chunk count is the allocating entry point's choice, capped by what fits,
// so the two entry points give the same result whenever that choice fits.
//
// Host code cannot use the array's name as a device address: the first call
// on each device (and the first after the device's context was destroyed and
// created again) looks the address up with cudaGetSymbolAddress, with that
// device current, and caches it with the context's id; make that first call
// before any stream capture on the device.
//
// Every call shares the array and it keeps the previous call's contents:
// every buffer in it is written before it is read within a call (packed
// sources, sort keys, the order, each partial-sum row the epilogue reads), so
// nothing has to start at zero. Calls that overlap on the GPU (on different
// streams or from different contexts on the same device) race on the array;
// callers must order them.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <mutex>

#include "tc_ctx.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double)];

struct ScratchSlot {
  unsigned long long ctx_id = 0;  // id of the context the address belongs to
  void* ptr = nullptr;
};

std::mutex g_scratch_mu;
ScratchSlot g_scratch[kMaxDevices];

}  // namespace

// Unique id of the current context (cuCtxGetId, reached through the runtime so
// the library links only libcudart); 0 when the driver cannot say.
unsigned long long tcb::current_context_id() {
  static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
  static PFN_cuCtxGetId_v12000 get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f);
    cudaGetLastError();
  });
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&c) != CUDA_SUCCESS || !c ||
      get_id(c, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

namespace {

// Device address of g_noalloc_scratch on `device` (which must be current).
int scratch_address(int device, void** out) {
  if (device < 0 || device >= kMaxDevices) {
    tc_record_error("tc_bs_velocity_device_noalloc: device %d out of range", device);
    return TC_ERR_ARG;
  }
  const unsigned long long id = tcb::current_context_id();
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  ScratchSlot& s = g_scratch[device];
  // id 0 (unknown): look the address up on every call rather than trust a cached one
  if (!s.ptr || id == 0 || s.ctx_id != id) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      tc_record_error("cudaGetSymbolAddress of the no-allocation scratch failed: %s",
                      cudaGetErrorString(e));
      cudaGetLastError();
      return TC_ERR_CUDA;
    }
    s.ptr = p;
    s.ctx_id = id;
  }
  *out = s.ptr;
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
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    tc_record_error("cudaSetDevice(%d) failed", ctx->device);
    return TC_ERR_CUDA;
  }
  // layout: sources | order (perm, keys in, keys out, indices, sort temp) | partial sums
  const int len = i1 - i0;
  const bool ordered = ctx->precision == TC_FP32C && ctx->target_order == TC_ORDER_HILBERT && len > 0;
  size_t sort_bytes = 0;
  int rc;
  if (ordered && (rc = tcb::order_sort_bytes(len, &sort_bytes))) return rc;
  const size_t src_bytes = round256((size_t)n * sizeof(double4));
  const size_t perm_bytes = ordered ? round256((size_t)m * sizeof(int)) : 0;
  const size_t key_bytes = ordered ? round256((size_t)len * sizeof(unsigned)) : 0;
  const size_t order_bytes = ordered ? perm_bytes + 3 * key_bytes + round256(sort_bytes) : 0;
  const size_t chunk_bytes = 3 * (size_t)m * sizeof(double);
  const size_t fixed = src_bytes + order_bytes;
  if (fixed > kNoAllocScratchBytes || (len > 0 && n > 0 && kNoAllocScratchBytes - fixed < chunk_bytes)) {
    tc_record_error("tc_bs_velocity_device_noalloc: n=%d sources and m=%d targets need %zu bytes of "
                    "scratch, more than its fixed 32 MiB (32*n + 24*m, plus 4*m + ~20*(i1-i0) for "
                    "the FP32C visiting order, must fit)",
                    n, m, fixed + chunk_bytes, kNoAllocScratchBytes);
    return TC_ERR_ARG;
  }
  void* base = nullptr;
  if ((rc = scratch_address(ctx->device, &base))) return rc;
  char* b = static_cast<char*>(base);
  double4* src = reinterpret_cast<double4*>(b);
  int* perm = nullptr;
  if (target_class == TC_ACTIVE) X = src_x;
  if (ordered) {
    char* o = b + src_bytes;
    perm = reinterpret_cast<int*>(o);
    unsigned* k_in = reinterpret_cast<unsigned*>(o + perm_bytes);
    unsigned* k_out = reinterpret_cast<unsigned*>(o + perm_bytes + key_bytes);
    int* v_in = reinterpret_cast<int*>(o + perm_bytes + 2 * key_bytes);
    void* temp = o + perm_bytes + 3 * key_bytes;
    const tcb::OrderExtents ext{m, (long long)(perm_bytes / sizeof(int)),
                                (long long)(key_bytes / sizeof(unsigned))};
    if ((rc = tcb::compute_order_into(ctx, X, i0, i1, perm, k_in, k_out, v_in, temp, sort_bytes,
                                      ext)))
      return rc;
  }
  double* partial = reinterpret_cast<double*>(b + fixed);
  const long long src_len = (long long)(src_bytes / sizeof(double4));
  if ((rc = tcb::launch_pack(ctx, src_x, vort, area, n, src, src_len))) return rc;
  tcb::SegDesc seg{X, perm, i0, i1, 0, target_class == TC_ACTIVE ? 0 : tcb::kNoSelf,
                   ctx->delta[target_class] * ctx->delta[target_class], m,
                   perm ? (long long)(perm_bytes / sizeof(int)) : 0};
  int nchunks = 0;
  const size_t partial_bytes = kNoAllocScratchBytes - fixed;
  if ((rc = tcb::launch_pairs_into(ctx, &seg, 1, src, n, src_len, m, partial, partial_bytes,
                                   &nchunks)))
    return rc;
  return tcb::launch_velocity_epilogue(ctx, X, perm, m, i0, i1, 0, m, nchunks, dX,
                                       target_class == TC_ACTIVE ? dVort : nullptr, partial,
                                       (long long)(partial_bytes / sizeof(double)));
}
