// The checked build's violation records and their C ABI (tc_bounds_*).
//
// Each device has one record, shared by every library context on that
// device. The first library context created there allocates it (32 bytes).
// The record is kept until the process exits, or until the device's CUDA
// context is replaced (after cudaDeviceReset). The CUDA context's id is stored
// with it, so a replaced context gets a new record rather than a dead address.
// Kernels receive the record's address in their launch structures, so CUDA
// graphs captured earlier keep reporting into it. The release library
// allocates no record and passes null.
#include <mutex>

#include "tc_ctx.h"

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_bounds_mu;
tcb::BoundsRec* g_bounds[kMaxDevices] = {};
unsigned long long g_bounds_ctx[kMaxDevices] = {};  // CUDA context id of each record
}  // namespace

namespace tcb {
// Called by tc_create with ctx->device current.
int bounds_attach(tc_ctx* ctx) {
#if TC_BOUNDS_CHECK
  if (ctx->device < 0 || ctx->device >= kMaxDevices) {
    tc_record_error("checked build: device %d has no violation record slot", ctx->device);
    return TC_ERR_ARG;
  }
  const unsigned long long id = current_context_id();
  std::lock_guard<std::mutex> lock(g_bounds_mu);
  BoundsRec*& rec = g_bounds[ctx->device];
  // a record of another (replaced) CUDA context is not freed: its memory went with that
  // context (id 0: the driver cannot tell contexts apart, and the record is kept)
  if (!rec || (id != 0 && g_bounds_ctx[ctx->device] != id)) {
    void* p = nullptr;
    TC_CUDA_TRY(cudaMalloc(&p, sizeof(BoundsRec)));
    TC_CUDA_TRY(cudaMemset(p, 0, sizeof(BoundsRec)));
    TC_CUDA_TRY(cudaDeviceSynchronize());
    rec = static_cast<BoundsRec*>(p);
    g_bounds_ctx[ctx->device] = id;
  }
  ctx->bc_rec = rec;
#else
  ctx->bc_rec = nullptr;
#endif
  return TC_OK;
}
}  // namespace tcb

extern "C" int tc_bounds_checked(void) { return TC_BOUNDS_CHECK ? 1 : 0; }

extern "C" int tc_bounds_status(int device, long long rec[4], int reset) {
  if (!rec) return TC_ERR_ARG;
  rec[0] = rec[1] = rec[2] = rec[3] = 0;
  if (device < 0 || device >= kMaxDevices) {
    tc_record_error("tc_bounds_status: no device %d", device);
    return TC_ERR_ARG;
  }
  tcb::BoundsRec* d = nullptr;
  unsigned long long owner = 0;
  {
    std::lock_guard<std::mutex> lock(g_bounds_mu);
    d = g_bounds[device];
    owner = g_bounds_ctx[device];
  }
  if (!d) return TC_OK;  // release build, or no context on this device yet
  int rc = tc_set_device_checked(device);
  if (rc) {
    tc_record_error("tc_bounds_status: device %d is not available", device);
    return rc;
  }
  const unsigned long long id = tcb::current_context_id();
  if (id != 0 && id != owner) return TC_OK;  // the record's CUDA context is gone
  TC_CUDA_TRY(cudaDeviceSynchronize());
  tcb::BoundsRec h{};
  TC_CUDA_TRY(cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost));
  rec[0] = (long long)h.count;
  rec[1] = h.site;
  rec[2] = h.index;
  rec[3] = h.extent;
  if (reset) {
    TC_CUDA_TRY(cudaMemset(d, 0, sizeof(tcb::BoundsRec)));
    TC_CUDA_TRY(cudaDeviceSynchronize());
  }
  return TC_OK;
}

extern "C" int tc_bounds_cap(tc_ctx* ctx, int site, long long cap) {
  if (!ctx) return TC_ERR_ARG;
  if (!TC_BOUNDS_CHECK) {
    tc_record_error("tc_bounds_cap: this library is the release build (no index checks)");
    return TC_ERR_STATE;
  }
  if (site < 0 || site >= tcb::BC_SITE_END) {
    tc_record_error("tc_bounds_cap: no site %d", site);
    return TC_ERR_ARG;
  }
  const int s0 = site == 0 ? 1 : site, s1 = site == 0 ? tcb::BC_SITE_END : site + 1;
  for (int s = s0; s < s1; ++s) {
    ctx->bc_capped[s] = cap >= 0;
    ctx->bc_cap[s] = cap >= 0 ? cap : 0;
  }
  return TC_OK;
}
