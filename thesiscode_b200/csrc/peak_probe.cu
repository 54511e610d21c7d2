// CUDA-core throughput probe: the roofline denominators for the Biot-Savart
// kernels. The pair sum runs on the FP32 / FP64 FMA pipes and the MUFU
// reciprocal unit (no tensor cores: an N-body sum is not a contraction), so
// the peaks that bound it are measured here, on the device that runs it,
// with the same launch shape (148 SMs x full occupancy) the kernels use.
//
// Every probe kernel runs a fixed, bounded loop of independent dependency
// chains per thread and writes one value per thread only when `sink` is
// non-null, so the compiler cannot drop the work.
#include <cuda_runtime.h>
#include <cstdint>
#include "tc_internal.h"

namespace {

constexpr int kChains = 8;

__global__ void probe_ffma(int iters, float b, float c, float* sink) {
  float a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = threadIdx.x * 1e-3f + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fmaf(a[k], b, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (sink) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void probe_ffma2(int iters, float b, float c, float* sink) {
  float2 a[kChains];
  const float2 b2 = make_float2(b, b), c2 = make_float2(c, c);
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = make_float2(threadIdx.x * 1e-3f + k, k * 0.5f);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = __ffma2_rn(a[k], b2, c2);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k].x + a[k].y;
  if (sink) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void probe_dfma(int iters, double b, double c, float* sink) {
  double a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = threadIdx.x * 1e-3 + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (sink) sink[blockIdx.x * blockDim.x + threadIdx.x] = (float)s;
}

__device__ __forceinline__ float rcp_approx_f32(float x) {
  float r;
  asm volatile("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ double rcp_approx_f64(double x) {
  double r;
  asm volatile("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  return r;
}

__global__ void probe_rcp32(int iters, float b, float c, float* sink) {
  float a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = 1.0f + threadIdx.x * 1e-3f + k;
  // the add keeps ptxas from folding rcp(rcp(x)); MUFU stays the slower pipe
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = rcp_approx_f32(a[k]) + c;
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (sink) sink[blockIdx.x * blockDim.x + threadIdx.x] = s + b + c;
}

__global__ void probe_rcp64(int iters, double b, double c, float* sink) {
  double a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = 1.0 + threadIdx.x * 1e-3 + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = rcp_approx_f64(a[k]);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (sink) sink[blockIdx.x * blockDim.x + threadIdx.x] = (float)(s + b + c);
}

// FP32 -> FP64 conversions feeding an FP64 add (the flush of FP32 partial
// sums into FP64 accumulators); counts one conversion per op.
__global__ void probe_f2f(int iters, float b, float c, float* sink) {
  double a[kChains];
  float f[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) {
    a[k] = 0.0;
    f[k] = threadIdx.x * 1e-3f + k;
  }
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) {
      a[k] += (double)f[k];
      f[k] = f[k] * b;
    }
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (sink) sink[blockIdx.x * blockDim.x + threadIdx.x] = (float)s + c;
}

// IEEE-rounded FP64 division as the compiler emits it for `a / b`.
__global__ void probe_ddiv(int iters, double b, double c, float* sink) {
  double a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = 1.0 + threadIdx.x * 1e-3 + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = b / a[k] + c;
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (sink) sink[blockIdx.x * blockDim.x + threadIdx.x] = (float)s;
}

}  // namespace

// kind: TC_PROBE_FFMA, TC_PROBE_FFMA2, TC_PROBE_DFMA, TC_PROBE_RCP32,
// TC_PROBE_RCP64, TC_PROBE_DDIV, TC_PROBE_F2F. Returns operations per second (one FMA,
// one reciprocal or one division = 1 op; FFMA2 counts 2) in *ops_per_s.
extern "C" int tc_probe_peak(int device, int kind, int iters, double* ops_per_s) {
  if (!ops_per_s || iters <= 0 || iters > (1 << 22)) return TC_ERR_ARG;
  if (kind < TC_PROBE_FFMA || kind > TC_PROBE_F2F) return TC_ERR_ARG;
  int rc = tc_set_device_checked(device);
  if (rc) return rc;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return TC_ERR_CUDA;
  const int threads = 256;
  const int blocks = prop.multiProcessorCount * (prop.maxThreadsPerMultiProcessor / threads);
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return TC_ERR_CUDA;
  double per_thread_ops = (double)iters * kChains;
  auto launch = [&](int it) {
    switch (kind) {
      case TC_PROBE_FFMA: probe_ffma<<<blocks, threads>>>(it, 0.999999f, 1e-7f, nullptr); break;
      case TC_PROBE_FFMA2: probe_ffma2<<<blocks, threads>>>(it, 0.999999f, 1e-7f, nullptr); break;
      case TC_PROBE_DFMA: probe_dfma<<<blocks, threads>>>(it, 0.999999, 1e-7, nullptr); break;
      case TC_PROBE_RCP32: probe_rcp32<<<blocks, threads>>>(it, 0.f, 1e-7f, nullptr); break;
      case TC_PROBE_RCP64: probe_rcp64<<<blocks, threads>>>(it, 0.0, 0.0, nullptr); break;
      case TC_PROBE_DDIV: probe_ddiv<<<blocks, threads>>>(it, 0.5, 0.75, nullptr); break;
      case TC_PROBE_F2F: probe_f2f<<<blocks, threads>>>(it, 0.999999f, 0.f, nullptr); break;
      default: break;
    }
  };
  if (kind == TC_PROBE_FFMA2) per_thread_ops *= 2.0;
  launch(iters / 8 + 1);  // warm-up
  cudaEventRecord(e0);
  launch(iters);
  cudaEventRecord(e1);
  if (cudaEventSynchronize(e1) != cudaSuccess) return TC_ERR_CUDA;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (cudaGetLastError() != cudaSuccess) return TC_ERR_CUDA;
  *ops_per_s = per_thread_ops * (double)blocks * threads / (ms * 1e-3);
  return TC_OK;
}
