// C ABI of libthesiscode_b200: context, parameters, the one-call velocity
// sums and the device-resident RK4 driver.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "tc_ctx.h"

using tcb::DevBuf;
using tcb::SegDesc;

namespace {

bool valid_class(int c) { return c == TC_ACTIVE || c == TC_VERTEX || c == TC_PASSIVE; }

int check_finite_host(const double* p, size_t n, const char* what) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) {
      tc_record_error("non-finite value in %s at index %zu", what, i);
      return TC_ERR_NONFINITE;
    }
  return TC_OK;
}

// Host entry points scan their inputs for NaN/Inf on the host while the GPU
// already works on the device copies, and copy results back only once the
// scan passed, so a refused call leaves the caller's arrays as they were.
// Results are scanned on the device, where they already are: only the first
// bad index of each array crosses back.
struct HostArray {
  const double* p;
  size_t n;
  const char* what;
};

int check_finite_host_all(const HostArray* a, int count) {
  int rc = TC_OK;
  for (int j = 0; j < count && !rc; ++j)
    if (a[j].p) rc = check_finite_host(a[j].p, a[j].n, a[j].what);
  return rc;
}

constexpr int kMaxScans = 4;

__global__ void first_nonfinite_kernel(const double* __restrict__ p, size_t n,
                                       unsigned long long* __restrict__ first) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride)
    if (!isfinite(p[i])) {  // the first in this thread's stride is its smallest
      atomicMin(first, (unsigned long long)i);
      break;
    }
}

// Enqueues device scans of up to kMaxScans result arrays (null or empty ones
// are skipped) into ctx->check_buf.
int scan_results_device(tc_ctx* ctx, const HostArray* a, int count) {
  if (count < 0 || count > kMaxScans) {
    tc_record_error("internal: %d result scans (at most %d)", count, kMaxScans);
    return TC_ERR_ARG;
  }
  int rc = ctx->check_buf.ensure(kMaxScans * sizeof(unsigned long long));
  if (rc) return rc;
  unsigned long long* first = ctx->check_buf.as<unsigned long long>();
  TC_CUDA_TRY(cudaMemsetAsync(first, 0xFF, kMaxScans * sizeof(unsigned long long), ctx->stream));
  for (int j = 0; j < count; ++j) {
    if (!a[j].p || a[j].n == 0) continue;
    const size_t want = (a[j].n + 255) / 256, cap = (size_t)ctx->num_sms * 8;
    first_nonfinite_kernel<<<(int)std::min(want, cap), 256, 0, ctx->stream>>>(a[j].p, a[j].n,
                                                                               first + j);
    TC_CUDA_TRY(cudaGetLastError());
    ctx->launches += 1;
  }
  return TC_OK;
}

// Reads back what scan_results_device found (synchronises the stream).
int scan_results_status(tc_ctx* ctx, const HostArray* a, int count) {
  if (count < 0 || count > kMaxScans) return TC_ERR_ARG;
  unsigned long long first[kMaxScans];
  TC_CUDA_TRY(cudaMemcpyAsync(first, ctx->check_buf.ptr, sizeof(first), cudaMemcpyDeviceToHost,
                              ctx->stream));
  TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (int j = 0; j < count; ++j)
    if (a[j].p && first[j] != ~0ull) {
      tc_record_error("non-finite value in %s at index %llu", a[j].what, first[j]);
      return TC_ERR_NONFINITE;
    }
  return TC_OK;
}

int begin(tc_ctx* ctx) {
  if (!ctx) {
    tc_record_error("null context");
    return TC_ERR_ARG;
  }
  if (cudaSetDevice(ctx->device) != cudaSuccess) {
    tc_record_error("cudaSetDevice(%d) failed", ctx->device);
    return TC_ERR_CUDA;
  }
  return TC_OK;
}

// Shared validation of one velocity call (the size checks of
// PanelVelocityParallel.f90:1299-1315 / :1348-1361 / :1387-1400, returned
// as TC_ERR_ARG instead of printed).
int check_velocity_args(int cls, const double* X, int m, const double* src_x, const double* vort,
                        const double* area, int n, int i0, int i1, const double* dX) {
  if (!valid_class(cls)) {
    tc_record_error("target_class %d is not TC_ACTIVE/TC_VERTEX/TC_PASSIVE", cls);
    return TC_ERR_ARG;
  }
  if (m < 0 || n < 0) {
    tc_record_error("negative size (m=%d, n=%d)", m, n);
    return TC_ERR_ARG;
  }
  if (cls == TC_ACTIVE && (X != nullptr && X != src_x)) {
    tc_record_error("TC_ACTIVE targets are the sources: pass X = NULL or X = src_x");
    return TC_ERR_ARG;
  }
  if (cls == TC_ACTIVE && m != n) {
    tc_record_error("TC_ACTIVE: size mismatch m=%d n=%d", m, n);
    return TC_ERR_ARG;
  }
  if (i0 < 0 || i1 < i0 || i1 > m) {
    tc_record_error("target range [%d,%d) outside [0,%d)", i0, i1, m);
    return TC_ERR_ARG;
  }
  if ((n > 0 && (!src_x || !vort || !area)) || (m > 0 && !dX) ||
      (cls != TC_ACTIVE && m > 0 && !X)) {
    tc_record_error("null array argument");
    return TC_ERR_ARG;
  }
  return TC_OK;
}

// Device part shared by the host and device entry points.
int velocity_device(tc_ctx* ctx, int cls, const double* X, int m, const double* src_x,
                    const double* vort, const double* area, int n, int i0, int i1, double* dX,
                    double* dVort) {
  if (cls == TC_ACTIVE) X = src_x;
  int rc = ctx->scratch[0].ensure((size_t)std::max(n, 1) * sizeof(double4));
  if (rc) return rc;
  double4* src = ctx->scratch[0].as<double4>();
  int* perm = nullptr;
  if (ctx->precision == TC_FP32C && ctx->target_order == TC_ORDER_HILBERT && i1 > i0) {
    if ((rc = ctx->scratch[4].ensure((size_t)m * sizeof(int)))) return rc;
    perm = ctx->scratch[4].as<int>();
    if ((rc = tcb::compute_order(ctx, X, i0, i1, perm, m, m))) return rc;
  }
  const long long src_len = (long long)(ctx->scratch[0].bytes / sizeof(double4));
  if ((rc = tcb::launch_pack(ctx, src_x, vort, area, n, src, src_len))) return rc;
  SegDesc seg{X, perm, i0, i1, 0, cls == TC_ACTIVE ? 0 : tcb::kNoSelf,
              ctx->delta[cls] * ctx->delta[cls], m,
              perm ? (long long)(ctx->scratch[4].bytes / sizeof(int)) : 0};
  int nch = 0;
  if ((rc = tcb::launch_pairs(ctx, &seg, 1, src, n, src_len, m, &nch))) return rc;
  return tcb::launch_velocity_epilogue(ctx, X, perm, m, i0, i1, 0, m, nch, dX,
                                       cls == TC_ACTIVE ? dVort : nullptr);
}

}  // namespace

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
extern "C" int tc_create(int device, int precision, tc_ctx** out) {
  if (!out) return TC_ERR_ARG;
  *out = nullptr;
  if (precision != TC_FP64 && precision != TC_FP32C) {
    tc_record_error("precision %d is not TC_FP64/TC_FP32C", precision);
    return TC_ERR_ARG;
  }
  int rc = tc_set_device_checked(device);
  if (rc) {
    tc_record_error("device %d is not available", device);
    return rc;
  }
  tc_ctx* ctx = new (std::nothrow) tc_ctx();
  if (!ctx) return TC_ERR_NOMEM;
  ctx->device = device;
  ctx->precision = precision;
  if ((rc = tcb::resolve_slots(ctx)) || (rc = tcb::bounds_attach(ctx))) {
    delete ctx;
    return rc;
  }
  *out = ctx;
  return TC_OK;
}

extern "C" int tc_destroy(tc_ctx* ctx) {
  if (!ctx) return TC_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  ctx->partial.release();
  ctx->check_buf.release();
  for (auto& b : ctx->scratch) b.release();
  tcb::Rk4State& R = ctx->rk;
  DevBuf* bufs[] = {&R.x0A, &R.z0, &R.areaA, &R.x0V, &R.x0Q, &R.xiA, &R.ziA, &R.xiV, &R.xiQ,
                    &R.newA, &R.newZ, &R.newV, &R.newQ, &R.src, &R.ke, &R.keBlocks, &R.totalKE,
                    &R.permA, &R.permV, &R.permQ};
  for (DevBuf* b : bufs) b->release();
  for (auto& b : ctx->order_buf) b.release();
  tc_batch_free(ctx);
  tc_advance_graph_free(ctx);
  for (cudaEvent_t e : ctx->pair_events) cudaEventDestroy(e);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return TC_OK;
}

extern "C" int tc_set_stream(tc_ctx* ctx, void* stream) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  ctx->own_stream = false;
  ctx->stream = static_cast<cudaStream_t>(stream);
  return TC_OK;
}

extern "C" int tc_synchronize(tc_ctx* ctx) {
  int rc = begin(ctx);
  if (rc) return rc;
  TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return TC_OK;
}

extern "C" int tc_set_precision(tc_ctx* ctx, int precision) {
  if (!ctx) return TC_ERR_ARG;
  if (precision != TC_FP64 && precision != TC_FP32C) return TC_ERR_ARG;
  ctx->precision = precision;
  return TC_OK;
}

extern "C" int tc_get_precision(tc_ctx* ctx, int* precision) {
  if (!ctx || !precision) return TC_ERR_ARG;
  *precision = ctx->precision;
  return TC_OK;
}

extern "C" int tc_set_omega(tc_ctx* ctx, double omega) {
  if (!ctx || !std::isfinite(omega)) return TC_ERR_ARG;
  ctx->omega = omega;
  return TC_OK;
}

extern "C" int tc_get_omega(tc_ctx* ctx, double* omega) {
  if (!ctx || !omega) return TC_ERR_ARG;
  *omega = ctx->omega;
  return TC_OK;
}

extern "C" int tc_set_smooth(tc_ctx* ctx, double smooth) {
  if (!ctx || !std::isfinite(smooth)) return TC_ERR_ARG;
  ctx->delta[TC_PASSIVE] = smooth;
  return TC_OK;
}

extern "C" int tc_get_smooth(tc_ctx* ctx, double* smooth) {
  if (!ctx || !smooth) return TC_ERR_ARG;
  *smooth = ctx->delta[TC_PASSIVE];
  return TC_OK;
}

extern "C" int tc_set_adjoint_mode(tc_ctx* ctx, int mode) {
  if (!ctx || mode < 0 || mode > 7) return TC_ERR_ARG;
  ctx->adj_mode = mode;
  return TC_OK;
}

extern "C" int tc_set_target_order(tc_ctx* ctx, int order) {
  if (!ctx || (order != TC_ORDER_GIVEN && order != TC_ORDER_HILBERT)) return TC_ERR_ARG;
  ctx->target_order = order;
  ctx->rk.ordered = false;
  return TC_OK;
}

extern "C" int tc_set_deltas(tc_ctx* ctx, double delta_active, double delta_vertex,
                             double delta_passive) {
  if (!ctx || !std::isfinite(delta_active) || !std::isfinite(delta_vertex) ||
      !std::isfinite(delta_passive))
    return TC_ERR_ARG;
  ctx->delta[TC_ACTIVE] = delta_active;
  ctx->delta[TC_VERTEX] = delta_vertex;
  ctx->delta[TC_PASSIVE] = delta_passive;
  return TC_OK;
}

extern "C" int tc_get_deltas(tc_ctx* ctx, double* delta3) {
  if (!ctx || !delta3) return TC_ERR_ARG;
  for (int c = 0; c < 3; ++c) delta3[c] = ctx->delta[c];
  return TC_OK;
}

// ---------------------------------------------------------------------------
// One velocity sum
// ---------------------------------------------------------------------------
extern "C" int tc_bs_velocity_device(tc_ctx* ctx, int target_class, const double* X, int m,
                                     const double* src_x, const double* vort, const double* area,
                                     int n, int i0, int i1, double* dX, double* dVort) {
  int rc = begin(ctx);
  if (rc) return rc;
  if ((rc = check_velocity_args(target_class, X, m, src_x, vort, area, n, i0, i1, dX))) return rc;
  return velocity_device(ctx, target_class, X, m, src_x, vort, area, n, i0, i1, dX, dVort);
}

extern "C" int tc_bs_velocity(tc_ctx* ctx, int target_class, const double* X, int m,
                              const double* src_x, const double* vort, const double* area, int n,
                              int i0, int i1, double* dX, double* dVort) {
  int rc = begin(ctx);
  if (rc) return rc;
  if ((rc = check_velocity_args(target_class, X, m, src_x, vort, area, n, i0, i1, dX))) return rc;
  const size_t nb = (size_t)std::max(n, 1) * sizeof(double);
  const size_t mb = (size_t)std::max(m, 1) * sizeof(double);
  if ((rc = ctx->scratch[1].ensure(3 * nb + 2 * nb)) || (rc = ctx->scratch[2].ensure(3 * mb)) ||
      (rc = ctx->scratch[3].ensure(4 * mb)))
    return rc;
  double* d_src = ctx->scratch[1].as<double>();
  double* d_vort = d_src + 3 * (size_t)std::max(n, 1);
  double* d_area = d_vort + (size_t)std::max(n, 1);
  double* d_X = ctx->scratch[2].as<double>();
  double* d_dX = ctx->scratch[3].as<double>();
  double* d_dV = d_dX + 3 * (size_t)std::max(m, 1);
  cudaStream_t s = ctx->stream;
  TC_CUDA_TRY(cudaMemcpyAsync(d_src, src_x, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s));
  TC_CUDA_TRY(cudaMemcpyAsync(d_vort, vort, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s));
  TC_CUDA_TRY(cudaMemcpyAsync(d_area, area, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (target_class != TC_ACTIVE)
    TC_CUDA_TRY(cudaMemcpyAsync(d_X, X, 3 * (size_t)m * sizeof(double), cudaMemcpyHostToDevice, s));
  rc = velocity_device(ctx, target_class, target_class == TC_ACTIVE ? nullptr : d_X, m, d_src,
                       d_vort, d_area, n, i0, i1, d_dX, d_dV);
  if (rc) return rc;
  const HostArray in[4] = {{src_x, 3 * (size_t)n, "src_x"},
                           {vort, (size_t)n, "vort"},
                           {area, (size_t)n, "area"},
                           {target_class != TC_ACTIVE ? X : nullptr, 3 * (size_t)m, "X"}};
  if ((rc = check_finite_host_all(in, 4))) {
    cudaStreamSynchronize(s);
    return rc;
  }
  const HostArray out[1] = {{d_dX, 3 * (size_t)m, "dX (result)"}};
  if ((rc = scan_results_device(ctx, out, 1))) return rc;
  TC_CUDA_TRY(cudaMemcpyAsync(dX, d_dX, 3 * (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (target_class == TC_ACTIVE && dVort)
    TC_CUDA_TRY(cudaMemcpyAsync(dVort, d_dV, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, s));
  return scan_results_status(ctx, out, 1);
}

// ---------------------------------------------------------------------------
// Voronoi SoA sum (BVEVelocity, VoronoiVelocityParallel.f90:487-515)
// ---------------------------------------------------------------------------
namespace {

__global__ void soa_to_aos_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                  const double* __restrict__ z, int n, double* __restrict__ out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  out[3 * (size_t)j] = x[j];
  out[3 * (size_t)j + 1] = y[j];
  out[3 * (size_t)j + 2] = z[j];
}

// BVEVelocity zeroes only dx (:494): dy and dz add to what the caller holds,
// and the whole arrays are divided by (-4 pi) (:510-512); dVort over all rows.
__global__ void soa_finish_kernel(const double* __restrict__ u, int n, double m2omega,
                                  double* __restrict__ dx, double* __restrict__ dy,
                                  double* __restrict__ dz, double* __restrict__ dVort) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double s = -4.0 * 3.141592653589793238462643383279502884;
  dx[j] = u[3 * (size_t)j];
  dy[j] = dy[j] / s + u[3 * (size_t)j + 1];
  dz[j] = dz[j] / s + u[3 * (size_t)j + 2];
  if (dVort) dVort[j] = m2omega * dz[j];
}

}  // namespace

extern "C" int tc_bs_velocity_soa_device(tc_ctx* ctx, const double* x, const double* y,
                                         const double* z, const double* vort, const double* area,
                                         int n, int i0, int i1, double* dx, double* dy, double* dz,
                                         double* dVort) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (n < 0 || i0 < 0 || i1 < i0 || i1 > n) {
    tc_record_error("tc_bs_velocity_soa: bad size or range (n=%d, [%d,%d))", n, i0, i1);
    return TC_ERR_ARG;
  }
  if (n > 0 && (!x || !y || !z || !vort || !area || !dx || !dy || !dz)) {
    tc_record_error("tc_bs_velocity_soa: null array argument");
    return TC_ERR_ARG;
  }
  if (n == 0) return TC_OK;
  if ((rc = ctx->scratch[5].ensure(6 * (size_t)n * sizeof(double)))) return rc;
  double* aos = ctx->scratch[5].as<double>();
  double* u = aos + 3 * (size_t)n;
  soa_to_aos_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(x, y, z, n, aos);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  if ((rc = velocity_device(ctx, TC_ACTIVE, nullptr, n, aos, vort, area, n, i0, i1, u, nullptr)))
    return rc;
  soa_finish_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(u, n, -2.0 * ctx->omega, dx, dy, dz,
                                                               dVort);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  return TC_OK;
}

extern "C" int tc_bs_velocity_soa(tc_ctx* ctx, const double* x, const double* y, const double* z,
                                  const double* vort, const double* area, int n, int i0, int i1,
                                  double* dx, double* dy, double* dz, double* dVort) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (n < 0 || (n > 0 && (!x || !y || !z || !vort || !area || !dx || !dy || !dz))) {
    tc_record_error("tc_bs_velocity_soa: bad arguments");
    return TC_ERR_ARG;
  }
  if (n == 0) return TC_OK;
  const double* in[5] = {x, y, z, vort, area};
  const size_t b = (size_t)n * sizeof(double);
  if ((rc = ctx->scratch[1].ensure(9 * b))) return rc;
  double* d = ctx->scratch[1].as<double>();
  cudaStream_t s = ctx->stream;
  for (int a = 0; a < 5; ++a)
    TC_CUDA_TRY(cudaMemcpyAsync(d + a * (size_t)n, in[a], b, cudaMemcpyHostToDevice, s));
  TC_CUDA_TRY(cudaMemcpyAsync(d + 6 * (size_t)n, dy, b, cudaMemcpyHostToDevice, s));
  TC_CUDA_TRY(cudaMemcpyAsync(d + 7 * (size_t)n, dz, b, cudaMemcpyHostToDevice, s));
  double* ddx = d + 5 * (size_t)n;
  double* ddy = d + 6 * (size_t)n;
  double* ddz = d + 7 * (size_t)n;
  double* ddv = d + 8 * (size_t)n;
  if ((rc = tc_bs_velocity_soa_device(ctx, d, d + n, d + 2 * (size_t)n, d + 3 * (size_t)n,
                                      d + 4 * (size_t)n, n, i0, i1, ddx, ddy, ddz, ddv)))
    return rc;
  const HostArray hin[5] = {{x, (size_t)n, "x"},
                            {y, (size_t)n, "y"},
                            {z, (size_t)n, "z"},
                            {vort, (size_t)n, "vort"},
                            {area, (size_t)n, "area"}};
  if ((rc = check_finite_host_all(hin, 5))) {
    cudaStreamSynchronize(s);
    return rc;
  }
  const HostArray out[1] = {{ddx, (size_t)n, "dx (result)"}};
  if ((rc = scan_results_device(ctx, out, 1))) return rc;
  TC_CUDA_TRY(cudaMemcpyAsync(dx, ddx, b, cudaMemcpyDeviceToHost, s));
  TC_CUDA_TRY(cudaMemcpyAsync(dy, ddy, b, cudaMemcpyDeviceToHost, s));
  TC_CUDA_TRY(cudaMemcpyAsync(dz, ddz, b, cudaMemcpyDeviceToHost, s));
  if (dVort) TC_CUDA_TRY(cudaMemcpyAsync(dVort, ddv, b, cudaMemcpyDeviceToHost, s));
  return scan_results_status(ctx, out, 1);
}

// ---------------------------------------------------------------------------
// RK4 driver (BVERK4, PanelVelocityParallel.f90:435-658)
// ---------------------------------------------------------------------------
namespace {

int rk4_alloc(tc_ctx* ctx, int nA, int nV, int nQ) {
  tcb::Rk4State& R = ctx->rk;
  const size_t a = (size_t)std::max(nA, 1), v = (size_t)std::max(nV, 1),
               q = (size_t)std::max(nQ, 1), D = sizeof(double);
  int rc;
  if ((rc = R.x0A.ensure(3 * a * D)) || (rc = R.z0.ensure(a * D)) || (rc = R.areaA.ensure(a * D)) ||
      (rc = R.x0V.ensure(3 * v * D)) || (rc = R.x0Q.ensure(3 * q * D)) ||
      (rc = R.xiA.ensure(3 * a * D)) || (rc = R.ziA.ensure(a * D)) ||
      (rc = R.xiV.ensure(3 * v * D)) || (rc = R.xiQ.ensure(3 * q * D)) ||
      (rc = R.newA.ensure(3 * a * D)) || (rc = R.newZ.ensure(a * D)) ||
      (rc = R.newV.ensure(3 * v * D)) || (rc = R.newQ.ensure(3 * q * D)) ||
      (rc = R.src.ensure(a * sizeof(double4))) || (rc = R.ke.ensure(a * D)))
    return rc;
  R.nA = nA;
  R.nV = nV;
  R.nQ = nQ;
  return TC_OK;
}

int check_rk4_sizes(int nA, int nV, int nQ) {
  if (nA < 0 || nV < 0 || nQ < 0) {
    tc_record_error("negative size (nA=%d, nV=%d, nQ=%d)", nA, nV, nQ);
    return TC_ERR_ARG;
  }
  return TC_OK;
}

// The host arrays tc_rk4_load copies, for the finite scan.
int rk4_host_inputs(const double* xA, const double* zetaA, const double* areaA, int nA,
                    const double* xV, int nV, const double* xQ, int nQ) {
  const HostArray in[5] = {{xA, 3 * (size_t)nA, "xA"},
                           {zetaA, (size_t)nA, "zetaA"},
                           {areaA, (size_t)nA, "areaA"},
                           {xV, 3 * (size_t)nV, "xV"},
                           {xQ, 3 * (size_t)nQ, "xQ"}};
  return check_finite_host_all(in, 5);
}

// tc_rk4_load; with scan_host = false the caller scans the host inputs itself
// (after it has queued the work on them).
int rk4_load(tc_ctx* ctx, const double* xA, const double* zetaA, const double* areaA, int nA,
             const double* xV, int nV, const double* xQ, int nQ, int on_device, bool scan_host) {
  int rc = begin(ctx);
  if (rc) return rc;
  if ((rc = check_rk4_sizes(nA, nV, nQ))) return rc;
  if ((nA && (!xA || !zetaA || !areaA)) || (nV && !xV) || (nQ && !xQ)) {
    tc_record_error("tc_rk4_load: null array argument");
    return TC_ERR_ARG;
  }
  if (!on_device && scan_host && (rc = rk4_host_inputs(xA, zetaA, areaA, nA, xV, nV, xQ, nQ)))
    return rc;
  if ((rc = rk4_alloc(ctx, nA, nV, nQ))) return rc;
  tcb::Rk4State& R = ctx->rk;
  cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const size_t D = sizeof(double);
  cudaStream_t s = ctx->stream;
  if (nA) {
    TC_CUDA_TRY(cudaMemcpyAsync(R.x0A.ptr, xA, 3 * (size_t)nA * D, kind, s));
    TC_CUDA_TRY(cudaMemcpyAsync(R.z0.ptr, zetaA, (size_t)nA * D, kind, s));
    TC_CUDA_TRY(cudaMemcpyAsync(R.areaA.ptr, areaA, (size_t)nA * D, kind, s));
  }
  if (nV) TC_CUDA_TRY(cudaMemcpyAsync(R.x0V.ptr, xV, 3 * (size_t)nV * D, kind, s));
  if (nQ) TC_CUDA_TRY(cudaMemcpyAsync(R.x0Q.ptr, xQ, 3 * (size_t)nQ * D, kind, s));
  R.ready = true;
  R.ordered = false;
  R.strat = false;
  R.steps_total = 0;
  return TC_OK;
}

}  // namespace

extern "C" int tc_rk4_load(tc_ctx* ctx, const double* xA, const double* zetaA,
                           const double* areaA, int nA, const double* xV, int nV,
                           const double* xQ, int nQ, int on_device) {
  return rk4_load(ctx, xA, zetaA, areaA, nA, xV, nV, xQ, nQ, on_device, true);
}

extern "C" int tc_rk4_store(tc_ctx* ctx, double* xA, double* zetaA, double* xV, double* xQ,
                            double* kineticEnergy, int on_device) {
  int rc = begin(ctx);
  if (rc) return rc;
  tcb::Rk4State& R = ctx->rk;
  if (!R.ready) {
    tc_record_error("tc_rk4_store: no RK4 state loaded");
    return TC_ERR_STATE;
  }
  cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const size_t D = sizeof(double);
  cudaStream_t s = ctx->stream;
  if (xA && R.nA) TC_CUDA_TRY(cudaMemcpyAsync(xA, R.x0A.ptr, 3 * (size_t)R.nA * D, kind, s));
  if (zetaA && R.nA) TC_CUDA_TRY(cudaMemcpyAsync(zetaA, R.z0.ptr, (size_t)R.nA * D, kind, s));
  if (xV && R.nV) TC_CUDA_TRY(cudaMemcpyAsync(xV, R.x0V.ptr, 3 * (size_t)R.nV * D, kind, s));
  if (xQ && R.nQ) TC_CUDA_TRY(cudaMemcpyAsync(xQ, R.x0Q.ptr, 3 * (size_t)R.nQ * D, kind, s));
  if (kineticEnergy && R.nA)
    TC_CUDA_TRY(cudaMemcpyAsync(kineticEnergy, R.ke.ptr, (size_t)R.nA * D, kind, s));
  if (!on_device) TC_CUDA_TRY(cudaStreamSynchronize(s));
  return TC_OK;
}

// One RK4 stage over the given target ranges: the pair sums of all three
// classes in one launch, then the fused stage epilogue. Sources must be
// packed in ctx->rk.src (all nA rows) before the call; the epilogue writes
// the rows [a0,a1) of the next stage's packed sources.
extern "C" int tc_rk4_stage_range(tc_ctx* ctx, int stage, double dt, int a0, int a1, int v0,
                                  int v1, int q0, int q1, double* total_ke_device) {
  int rc = begin(ctx);
  if (rc) return rc;
  tcb::Rk4State& R = ctx->rk;
  if (!R.ready) {
    tc_record_error("tc_rk4_stage_range: no RK4 state loaded");
    return TC_ERR_STATE;
  }
  if (stage < 0 || stage > 3 || a0 < 0 || a1 < a0 || a1 > R.nA || v0 < 0 || v1 < v0 ||
      v1 > R.nV || q0 < 0 || q1 < q0 || q1 > R.nQ || !std::isfinite(dt)) {
    tc_record_error("tc_rk4_stage_range: bad stage or range");
    return TC_ERR_ARG;
  }
  static const char* const kStageNames[4] = {"tc rk4 stage 1", "tc rk4 stage 2", "tc rk4 stage 3",
                                              "tc rk4 stage 4"};
  TcNvtxRange nvtx_stage(kStageNames[stage]);
  const bool first = stage == 0;
  const double* tx[3] = {first ? R.x0A.as<double>() : R.xiA.as<double>(),
                         first ? R.x0V.as<double>() : R.xiV.as<double>(),
                         first ? R.x0Q.as<double>() : R.xiQ.as<double>()};
  const int range[6] = {a0, a1, v0, v1, q0, q1};
  // FP32C visiting order: computed from the stage-0 positions once per step
  // (targets move by O(dt) within a step) and whenever the ranges change.
  const bool want_order = ctx->precision == TC_FP32C && ctx->target_order == TC_ORDER_HILBERT;
  if (!want_order) {
    R.ordered = false;
  } else if (first || !R.ordered || memcmp(range, R.order_range, sizeof(range)) != 0) {
    tcb::DevBuf* pb[3] = {&R.permA, &R.permV, &R.permQ};
    const int nn[3] = {R.nA, R.nV, R.nQ};
    for (int c = 0; c < 3; ++c) {
      if ((rc = pb[c]->ensure((size_t)std::max(nn[c], 1) * sizeof(int)))) return rc;
      if ((rc = tcb::compute_order(ctx, tx[c], range[2 * c], range[2 * c + 1], pb[c]->as<int>(),
                                   nn[c], nn[c])))
        return rc;
    }
    memcpy(R.order_range, range, sizeof(range));
    R.ordered = true;
  }
  const bool ord = want_order && R.ordered;
  // extents (checked build): the class's stage-input buffer and visiting order
  const tcb::DevBuf* xb[3] = {first ? &R.x0A : &R.xiA, first ? &R.x0V : &R.xiV,
                              first ? &R.x0Q : &R.xiQ};
  const tcb::DevBuf* pbuf[3] = {&R.permA, &R.permV, &R.permQ};
  long long xl[3], pl[3];
  for (int c = 0; c < 3; ++c) {
    xl[c] = (long long)(xb[c]->bytes / (3 * sizeof(double)));
    pl[c] = ord ? (long long)(pbuf[c]->bytes / sizeof(int)) : 0;
  }
  SegDesc segs[3] = {
      {tx[0], ord ? R.permA.as<int>() : nullptr, a0, a1, 0, 0, ctx->delta[0] * ctx->delta[0],
       xl[0], pl[0]},
      {tx[1], ord ? R.permV.as<int>() : nullptr, v0, v1, R.nA, tcb::kNoSelf,
       ctx->delta[1] * ctx->delta[1], xl[1], pl[1]},
      {tx[2], ord ? R.permQ.as<int>() : nullptr, q0, q1, R.nA + R.nV, tcb::kNoSelf,
       ctx->delta[2] * ctx->delta[2], xl[2], pl[2]}};
  int nch = 0;
  const int n_out = R.nA + R.nV + R.nQ;
  if ((rc = tcb::launch_pairs(ctx, segs, 3, R.src.as<double4>(), R.nA,
                              (long long)(R.src.bytes / sizeof(double4)), n_out, &nch)))
    return rc;
  if ((rc = tcb::launch_stage_epilogue(ctx, stage, dt, range, nch, total_ke_device))) return rc;
  if (stage == 3 && R.strat) ++R.step;
  return TC_OK;
}

// Packs the sources of stage 1 from the loaded state (x0A, z0, areaA).
extern "C" int tc_rk4_pack_sources(tc_ctx* ctx) {
  int rc = begin(ctx);
  if (rc) return rc;
  tcb::Rk4State& R = ctx->rk;
  if (!R.ready) return TC_ERR_STATE;
  if (R.strat) return tcb::launch_pack_strat(ctx, R.t0 + (double)R.step * R.strat_dt);
  return tcb::launch_pack(ctx, R.x0A.as<double>(), R.z0.as<double>(), R.areaA.as<double>(), R.nA,
                          R.src.as<double4>(), (long long)(R.src.bytes / sizeof(double4)));
}

extern "C" int tc_rk4_device_buffer(tc_ctx* ctx, int which, void** ptr) {
  if (!ctx || !ptr) return TC_ERR_ARG;
  tcb::Rk4State& R = ctx->rk;
  switch (which) {
    case TC_BUF_SOURCES: *ptr = R.src.ptr; break;
    case TC_BUF_XA: *ptr = R.x0A.ptr; break;
    case TC_BUF_ZETA: *ptr = R.z0.ptr; break;
    case TC_BUF_XV: *ptr = R.x0V.ptr; break;
    case TC_BUF_XQ: *ptr = R.x0Q.ptr; break;
    case TC_BUF_KE: *ptr = R.ke.ptr; break;
    default: return TC_ERR_ARG;
  }
  return R.ready ? TC_OK : TC_ERR_STATE;
}

// Copy rows [row0, row0+nrows) of one RK4 device buffer to (to_buffer = 0)
// or from (to_buffer = 1) memory at `ptr` - device memory or host memory
// (unified addressing tells which) - on the context's stream.
// Row sizes: TC_BUF_SOURCES 4 doubles, TC_BUF_XA/XV/XQ 3, TC_BUF_ZETA/KE 1.
extern "C" int tc_rk4_copy_rows(tc_ctx* ctx, int which, int row0, int nrows, void* ptr,
                                int to_buffer) {
  int rc = begin(ctx);
  if (rc) return rc;
  tcb::Rk4State& R = ctx->rk;
  if (!R.ready) return TC_ERR_STATE;
  void* base = nullptr;
  int width = 0, rows = 0;
  switch (which) {
    case TC_BUF_SOURCES: base = R.src.ptr; width = 4; rows = R.nA; break;
    case TC_BUF_XA: base = R.x0A.ptr; width = 3; rows = R.nA; break;
    case TC_BUF_ZETA: base = R.z0.ptr; width = 1; rows = R.nA; break;
    case TC_BUF_XV: base = R.x0V.ptr; width = 3; rows = R.nV; break;
    case TC_BUF_XQ: base = R.x0Q.ptr; width = 3; rows = R.nQ; break;
    case TC_BUF_KE: base = R.ke.ptr; width = 1; rows = R.nA; break;
    default: return TC_ERR_ARG;
  }
  if (row0 < 0 || nrows < 0 || row0 + nrows > rows || (nrows > 0 && !ptr)) {
    tc_record_error("tc_rk4_copy_rows: rows [%d,%d) outside [0,%d)", row0, row0 + nrows, rows);
    return TC_ERR_ARG;
  }
  if (nrows == 0) return TC_OK;
  char* b = static_cast<char*>(base) + (size_t)row0 * width * sizeof(double);
  size_t bytes = (size_t)nrows * width * sizeof(double);
  TC_CUDA_TRY(cudaMemcpyAsync(to_buffer ? b : ptr, to_buffer ? ptr : b, bytes, cudaMemcpyDefault,
                              ctx->stream));
  return TC_OK;
}

// LoadBalance (PanelVelocityParallel.f90:182-204): contiguous chunks of
// n / num_procs rows, the last rank taking the remainder; 0-based half-open
// [index_start[r], index_end[r]) for rank r.
extern "C" int tc_load_balance(int n, int num_procs, int* index_start, int* index_end) {
  if (n < 0 || num_procs < 1 || !index_start || !index_end) {
    tc_record_error("tc_load_balance: bad arguments (n=%d, num_procs=%d)", n, num_procs);
    return TC_ERR_ARG;
  }
  const int chunk = n / num_procs;
  for (int r = 0; r < num_procs; ++r) {
    index_start[r] = r * chunk;
    index_end[r] = (r + 1) * chunk;
  }
  index_end[num_procs - 1] = n;
  return TC_OK;
}

// Number of visible CUDA devices (ranks map to devices rank % count).
extern "C" int tc_device_count(int* count) {
  if (!count) return TC_ERR_ARG;
  *count = 0;
  cudaError_t e = cudaGetDeviceCount(count);
  if (e != cudaSuccess) {
    *count = 0;
    tc_record_error("cudaGetDeviceCount: %s", cudaGetErrorString(e));
    cudaGetLastError();
    return TC_ERR_CUDA;
  }
  return TC_OK;
}

// Launch-bound small problems: steps 1..nsteps-1 of tc_rk4_advance are
// captured once into a CUDA graph (after step 0 has sized every buffer) and
// replayed as one launch while the shape, the step, the parameters and every
// buffer address stay the same. The graph runs on a private non-blocking
// stream ordered after and before the context's stream by events (the legacy
// NULL stream cannot be captured).
struct tc_advance_graph {
  cudaGraphExec_t exec = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  std::vector<uint64_t> key;  // shape, dt, steps, parameters and buffer addresses at capture
  long long launches = 0, pair_launches = 0, pair_interactions = 0;
  ~tc_advance_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
  }
};

void tc_advance_graph_free(tc_ctx* ctx) {
  delete ctx->agraph;
  ctx->agraph = nullptr;
}

extern "C" int tc_set_rk4_graphs(tc_ctx* ctx, int mode) {
  if (!ctx || mode < 0 || mode > 2) return TC_ERR_ARG;
  ctx->rk4_graphs = mode;
  return TC_OK;
}

namespace {

constexpr int kCaptureFailed = 1;  // advance_graph: no graph, nothing launched

int advance_steps(tc_ctx* ctx, double dt, int first, int last) {
  tcb::Rk4State& R = ctx->rk;
  for (int step = first; step < last; ++step)
    for (int s = 0; s < 4; ++s) {
      int rc = tc_rk4_stage_range(ctx, s, dt, 0, R.nA, 0, R.nV, 0, R.nQ,
                                  s == 0 ? R.totalKE.as<double>() + step : nullptr);
      if (rc) return rc;
    }
  return TC_OK;
}

uint64_t bits(double v) {
  uint64_t u;
  memcpy(&u, &v, sizeof(u));
  return u;
}

std::vector<uint64_t> graph_key(tc_ctx* ctx, double dt, int nsteps) {
  tcb::Rk4State& R = ctx->rk;
  std::vector<uint64_t> k = {(uint64_t)R.nA, (uint64_t)R.nV, (uint64_t)R.nQ, bits(dt),
                             (uint64_t)nsteps, (uint64_t)ctx->precision, (uint64_t)ctx->var64,
                             (uint64_t)ctx->var32, (uint64_t)ctx->auto32, (uint64_t)ctx->auto64,
                             (uint64_t)ctx->target_order,
                             bits(ctx->omega),
                             bits(ctx->delta[0]), bits(ctx->delta[1]), bits(ctx->delta[2])};
  const tcb::DevBuf* bufs[] = {&R.x0A, &R.z0, &R.areaA, &R.x0V, &R.x0Q, &R.xiA, &R.ziA, &R.xiV,
                               &R.xiQ, &R.newA, &R.newZ, &R.newV, &R.newQ, &R.src, &R.ke,
                               &R.keBlocks, &R.totalKE, &R.permA, &R.permV, &R.permQ,
                               &ctx->partial, &ctx->order_buf[0], &ctx->order_buf[1],
                               &ctx->order_buf[2], &ctx->order_buf[3]};
  for (const tcb::DevBuf* b : bufs) k.push_back((uint64_t)(uintptr_t)b->ptr);
  return k;
}

int advance_graph(tc_ctx* ctx, double dt, int nsteps) {
  if (!ctx->agraph) ctx->agraph = new (std::nothrow) tc_advance_graph();
  if (!ctx->agraph) return TC_ERR_NOMEM;
  tc_advance_graph& G = *ctx->agraph;
  if (!G.stream) {
    TC_CUDA_TRY(cudaStreamCreateWithFlags(&G.stream, cudaStreamNonBlocking));
    TC_CUDA_TRY(cudaEventCreateWithFlags(&G.ev[0], cudaEventDisableTiming));
    TC_CUDA_TRY(cudaEventCreateWithFlags(&G.ev[1], cudaEventDisableTiming));
  }
  const std::vector<uint64_t> key = graph_key(ctx, dt, nsteps);
  if (!G.exec || G.key != key) {
    if (G.exec) cudaGraphExecDestroy(G.exec);
    G.exec = nullptr;
    const cudaStream_t user = ctx->stream;
    const long long l0 = ctx->launches, p0 = ctx->pair_launches, i0 = ctx->pair_interactions;
    ctx->stream = G.stream;
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamBeginCapture(G.stream, cudaStreamCaptureModeThreadLocal);
    int rc = ce == cudaSuccess ? advance_steps(ctx, dt, 1, nsteps) : TC_ERR_CUDA;
    if (ce == cudaSuccess) ce = cudaStreamEndCapture(G.stream, &g);
    ctx->stream = user;
    if (rc || ce != cudaSuccess) {
      // capture failed before anything ran: undo the counters and let the caller
      // run the steps without a graph
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      ctx->launches = l0;
      ctx->pair_launches = p0;
      ctx->pair_interactions = i0;
      return kCaptureFailed;
    }
    ce = cudaGraphInstantiate(&G.exec, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
      G.exec = nullptr;
      tc_record_error("RK4 graph instantiation failed: %s", cudaGetErrorString(ce));
      return TC_ERR_CUDA;
    }
    G.key = key;
    G.launches = ctx->launches - l0;
    G.pair_launches = ctx->pair_launches - p0;
    G.pair_interactions = ctx->pair_interactions - i0;
  } else {
    ctx->launches += G.launches;
    ctx->pair_launches += G.pair_launches;
    ctx->pair_interactions += G.pair_interactions;
  }
  TcNvtxRange nvtx_replay("tc rk4 graph replay");
  TC_CUDA_TRY(cudaEventRecord(G.ev[0], ctx->stream));
  TC_CUDA_TRY(cudaStreamWaitEvent(G.stream, G.ev[0], 0));
  TC_CUDA_TRY(cudaGraphLaunch(G.exec, G.stream));
  TC_CUDA_TRY(cudaEventRecord(G.ev[1], G.stream));
  TC_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, G.ev[1], 0));
  return TC_OK;
}

// tc_rk4_advance without the read-back of totalKE: everything is queued on
// the context's stream.
int rk4_advance_enqueue(tc_ctx* ctx, double dt, int nsteps) {
  TcNvtxRange nvtx_advance("tc rk4 advance");
  int rc = begin(ctx);
  if (rc) return rc;
  tcb::Rk4State& R = ctx->rk;
  if (!R.ready) {
    tc_record_error("tc_rk4_advance: no RK4 state loaded");
    return TC_ERR_STATE;
  }
  if (nsteps < 0 || !std::isfinite(dt)) return TC_ERR_ARG;
  if (R.strat && dt != R.strat_dt) {  // forced run continued with another step: rebase its clock
    R.t0 += (double)R.step * R.strat_dt;
    R.step = 0;
    R.strat_dt = dt;
  }
  if ((rc = R.totalKE.ensure((size_t)std::max(nsteps, 1) * sizeof(double)))) return rc;
  if ((rc = tc_rk4_pack_sources(ctx))) return rc;
  // graphs: not for forced runs (their stage times are host arguments of each
  // launch) nor while pair kernels are timed one by one
  const double per_step = 4.0 * ((double)R.nA * R.nA + (double)(R.nV + R.nQ) * R.nA);
  const bool graph = nsteps >= 3 && !R.strat && !ctx->time_pairs &&
                     (ctx->rk4_graphs == 2 || (ctx->rk4_graphs == 1 && per_step <= 4.1e10));
  if (graph) {
    if ((rc = advance_steps(ctx, dt, 0, 1))) return rc;
    rc = advance_graph(ctx, dt, nsteps);
    if (rc == kCaptureFailed) {
      ctx->rk4_graphs = 0;  // this context runs its steps one launch at a time from now on
      rc = advance_steps(ctx, dt, 1, nsteps);
    }
    if (rc) return rc;
  } else if ((rc = advance_steps(ctx, dt, 0, nsteps))) {
    return rc;
  }
  R.steps_total += nsteps;
  return TC_OK;
}

// After the steps of a host-array call: queues the device scans of the new
// positions and (when the caller wants it) vorticity, the read-back of
// totalKE and the state (tc_rk4_store, which synchronises). The caller then
// reads the scans' outcome with scan_results_status(ctx, out, 2).
int rk4_results_to_host(tc_ctx* ctx, double* xA, double* zetaA, double* xV, double* xQ,
                        int nsteps, double* totalKE, double* kineticEnergy, HostArray out[2]) {
  tcb::Rk4State& R = ctx->rk;
  out[0] = HostArray{R.x0A.as<double>(), 3 * (size_t)R.nA, "xA (result)"};
  out[1] = HostArray{zetaA ? R.z0.as<double>() : nullptr, (size_t)R.nA,
                     R.strat ? "relVortA (result)" : "zetaA (result)"};
  int rc = scan_results_device(ctx, out, 2);
  if (rc) return rc;
  if (totalKE && nsteps > 0)
    TC_CUDA_TRY(cudaMemcpyAsync(totalKE, R.totalKE.ptr, (size_t)nsteps * sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->stream));
  return tc_rk4_store(ctx, xA, zetaA, xV, xQ, kineticEnergy, 0);
}

// Error return of a host-array call whose work is queued: waits for it, so
// that no copy still reads the caller's arrays, and drops the loaded state
// when it came from rejected inputs.
int fail_queued(tc_ctx* ctx, int rc, bool drop_state) {
  cudaStreamSynchronize(ctx->stream);
  if (drop_state) ctx->rk.ready = false;
  return rc;
}

}  // namespace

extern "C" int tc_rk4_advance(tc_ctx* ctx, double dt, int nsteps, double* totalKE) {
  int rc = rk4_advance_enqueue(ctx, dt, nsteps);
  if (rc) return rc;
  if (totalKE && nsteps > 0) {
    TC_CUDA_TRY(cudaMemcpyAsync(totalKE, ctx->rk.totalKE.ptr, (size_t)nsteps * sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->stream));
    TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  }
  return TC_OK;
}

// The drop-in BVERK4 call on host arrays: load, nsteps fused steps on the
// device, store back. The host scans the inputs for NaN/Inf while the steps
// run; the results are copied back only after that scan passed.
extern "C" int tc_rk4_step(tc_ctx* ctx, double* xA, double* zetaA, const double* areaA, int nA,
                           double* xV, int nV, double* xQ, int nQ, double dt, int nsteps,
                           double* totalKE, double* kineticEnergy) {
  int rc = rk4_load(ctx, xA, zetaA, areaA, nA, xV, nV, xQ, nQ, 0, false);
  if (rc) return rc;
  if ((rc = rk4_advance_enqueue(ctx, dt, nsteps))) return fail_queued(ctx, rc, false);
  if ((rc = rk4_host_inputs(xA, zetaA, areaA, nA, xV, nV, xQ, nQ)))
    return fail_queued(ctx, rc, true);
  HostArray out[2];
  if ((rc = rk4_results_to_host(ctx, xA, zetaA, xV, xQ, nsteps, totalKE, kineticEnergy, out)))
    return rc;
  return scan_results_status(ctx, out, 2);
}

extern "C" int tc_rk4_step_device(tc_ctx* ctx, double* xA, double* zetaA, const double* areaA,
                                  int nA, double* xV, int nV, double* xQ, int nQ, double dt,
                                  int nsteps, double* totalKE, double* kineticEnergy) {
  int rc = tc_rk4_load(ctx, xA, zetaA, areaA, nA, xV, nV, xQ, nQ, 1);
  if (rc) return rc;
  if ((rc = tc_rk4_advance(ctx, dt, nsteps, totalKE))) return rc;
  return tc_rk4_store(ctx, xA, zetaA, xV, xQ, kineticEnergy, 1);
}

// StratosphereRK4 (PanelVelocityParallel.f90:661-919) on host arrays: nsteps
// forced steps from time t, fused on the device like tc_rk4_step. Each stage's
// source vorticity is absVortA - 2 Omega z - F(x, t_stage) (Juckes forcing F);
// on return relVortA / relVortV (nullable) hold absVort - 2 Omega z - F(x, T),
// T = t + nsteps dt, at the new positions (:908-915), and totalKE[nsteps] the
// stage-1 kinetic energy of each step.
extern "C" int tc_strat_rk4_step(tc_ctx* ctx, double* xA, const double* absVortA,
                                 double* relVortA, const double* areaA, int nA, double* xV,
                                 const double* absVortV, double* relVortV, int nV, double* xQ,
                                 int nQ, double t, double dt, int nsteps, double* totalKE,
                                 double* kineticEnergy) {
  if (!ctx || nsteps < 0 || !std::isfinite(t) || !std::isfinite(dt) || (nA && !absVortA) ||
      (relVortV && nV && !absVortV)) {
    tc_record_error("tc_strat_rk4_step: bad arguments");
    return TC_ERR_ARG;
  }
  int rc = rk4_load(ctx, xA, absVortA, areaA, nA, xV, nV, xQ, nQ, 0, false);
  if (rc) return rc;
  tcb::Rk4State& R = ctx->rk;
  const size_t D = sizeof(double);
  if ((rc = R.absA.ensure((size_t)std::max(nA, 1) * D)) ||
      (rc = R.absV.ensure((size_t)std::max(nV, 1) * D)))
    return rc;
  if (nA) TC_CUDA_TRY(cudaMemcpyAsync(R.absA.ptr, absVortA, nA * D, cudaMemcpyHostToDevice, ctx->stream));
  if (nV && absVortV)
    TC_CUDA_TRY(cudaMemcpyAsync(R.absV.ptr, absVortV, nV * D, cudaMemcpyHostToDevice, ctx->stream));
  R.strat = true;
  R.t0 = t;
  R.step = 0;
  R.strat_dt = dt;
  // (advance packs the stage-1 sources first, which also sets relVortA at t)
  if ((rc = rk4_advance_enqueue(ctx, dt, nsteps))) return fail_queued(ctx, rc, false);
  const HostArray in[2] = {{absVortA, (size_t)nA, "absVortA"},
                           {absVortV, (size_t)nV, "absVortV"}};
  if ((rc = check_finite_host_all(in, 2)) ||
      (rc = rk4_host_inputs(xA, absVortA, areaA, nA, xV, nV, xQ, nQ)))
    return fail_queued(ctx, rc, true);
  HostArray out[2];
  if ((rc = rk4_results_to_host(ctx, xA, relVortA, xV, xQ, nsteps, totalKE, kineticEnergy, out)))
    return rc;
  if (relVortV && nV) {
    tcb::DevBuf rv;
    if ((rc = rv.ensure(nV * D))) return rc;
    if ((rc = tcb::launch_strat_rel_vort(ctx, R.absV.as<double>(), R.x0V.as<double>(), nV,
                                         R.t0 + (double)R.step * dt, rv.as<double>())))
      return rc;
    TC_CUDA_TRY(cudaMemcpyAsync(relVortV, rv.ptr, nV * D, cudaMemcpyDeviceToHost, ctx->stream));
    TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  }
  return scan_results_status(ctx, out, 2);
}

// Pair-kernel variants (the launch shapes the autotuner searches).
extern "C" int tc_pair_variant_count(int precision, int* count) {
  if (!count || (precision != TC_FP64 && precision != TC_FP32C)) return TC_ERR_ARG;
  *count = tcb::variant_count(precision);
  return TC_OK;
}

extern "C" int tc_pair_variant_info(int precision, int id, int* info8) {
  const tcb::PairVariant* v = tcb::variant(precision, id);
  if (!v || !info8) return TC_ERR_ARG;
  int vals[8] = {v->nt, v->tpt, v->ts, v->flush, v->minb, v->unroll, v->nt * v->tpt, v->form};
  for (int j = 0; j < 8; ++j) info8[j] = vals[j];
  return TC_OK;
}

extern "C" int tc_set_pair_variant(tc_ctx* ctx, int precision, int id) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (id == -1 && (precision == TC_FP32C || precision == TC_FP64)) {
    // back to the per-size automatic choice
    if (precision == TC_FP32C) ctx->auto32 = true;
    if (precision == TC_FP64) ctx->auto64 = true;
    return TC_OK;
  }
  if ((rc = tcb::select_variant(ctx, precision, id))) return rc;
  if (precision == TC_FP32C) ctx->auto32 = false;
  if (precision == TC_FP64) ctx->auto64 = false;
  return TC_OK;
}

extern "C" int tc_get_pair_variant(tc_ctx* ctx, int precision, int* id) {
  if (!ctx || !id) return TC_ERR_ARG;
  *id = precision == TC_FP64 ? ctx->var64 : ctx->var32;
  return TC_OK;
}

// Instrumentation: kernels launched by this context, pair-kernel launches and
// pair interactions evaluated since the last reset, and (when enabled) the
// summed CUDA-event time of the pair kernels on the context's stream.
extern "C" int tc_stats_enable_timing(tc_ctx* ctx, int on) {
  if (!ctx) return TC_ERR_ARG;
  ctx->time_pairs = on != 0;
  return TC_OK;
}

extern "C" int tc_stats(tc_ctx* ctx, int reset, long long* launches, long long* pair_launches,
                        long long* pair_interactions, double* pair_ms) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (!ctx->pair_events.empty()) {
    TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (size_t j = 0; j + 1 < ctx->pair_events.size(); j += 2) {
      float ms = 0.f;
      TC_CUDA_TRY(cudaEventElapsedTime(&ms, ctx->pair_events[j], ctx->pair_events[j + 1]));
      ctx->pair_ms += ms;
    }
    for (cudaEvent_t e : ctx->pair_events) cudaEventDestroy(e);
    ctx->pair_events.clear();
  }
  if (launches) *launches = ctx->launches;
  if (pair_launches) *pair_launches = ctx->pair_launches;
  if (pair_interactions) *pair_interactions = ctx->pair_interactions;
  if (pair_ms) *pair_ms = ctx->pair_ms;
  if (reset) {
    ctx->launches = ctx->pair_launches = ctx->pair_interactions = 0;
    ctx->pair_ms = 0.0;
  }
  return TC_OK;
}

// Voronoi BVERK4 (VoronoiVelocityParallel.f90:304-478) on the n used SoA
// generators, areas frozen for the step; the Delaunay/Voronoi rebuild that
// follows in the reference (:480-482) stays with the caller. Unused N_Max
// slots carry zero vorticity and contribute nothing, so they are not passed.
extern "C" int tc_rk4_soa_step(tc_ctx* ctx, double* x, double* y, double* z, double* relVort,
                               const double* area, int n, double dt, int nsteps, double* totalKE,
                               double* kineticEnergy) {
  int rc = begin(ctx);
  if (rc) return rc;
  if (n < 0 || (n > 0 && (!x || !y || !z || !relVort || !area))) {
    tc_record_error("tc_rk4_soa_step: bad arguments");
    return TC_ERR_ARG;
  }
  std::vector<double> xyz(3 * (size_t)n);
  for (int j = 0; j < n; ++j) {
    xyz[3 * (size_t)j] = x[j];
    xyz[3 * (size_t)j + 1] = y[j];
    xyz[3 * (size_t)j + 2] = z[j];
  }
  if ((rc = tc_rk4_step(ctx, xyz.data(), relVort, area, n, nullptr, 0, nullptr, 0, dt, nsteps,
                        totalKE, kineticEnergy)))
    return rc;
  for (int j = 0; j < n; ++j) {
    x[j] = xyz[3 * (size_t)j];
    y[j] = xyz[3 * (size_t)j + 1];
    z[j] = xyz[3 * (size_t)j + 2];
  }
  return TC_OK;
}

extern "C" int tc_reset_rk4(tc_ctx* ctx) {
  int rc = begin(ctx);
  if (rc) return rc;
  cudaStreamSynchronize(ctx->stream);
  tcb::Rk4State& R = ctx->rk;
  DevBuf* bufs[] = {&R.x0A, &R.z0, &R.areaA, &R.x0V, &R.x0Q, &R.xiA, &R.ziA, &R.xiV, &R.xiQ,
                    &R.newA, &R.newZ, &R.newV, &R.newQ, &R.src, &R.ke, &R.keBlocks, &R.totalKE,
                    &R.permA, &R.permV, &R.permQ};
  for (DevBuf* b : bufs) b->release();
  ctx->partial.release();
  tc_advance_graph_free(ctx);
  R.ready = false;
  R.ordered = false;
  R.nA = R.nV = R.nQ = 0;
  return TC_OK;
}
