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
#include "bs_core.cuh"
#include "tc_internal.h"

namespace {

constexpr int kChains = 8;

// The far-form pair step of the FP32C kernel itself (tcb::sp_far_run: per
// source pair and target one FADD2, six FFMA2 and two MUFU reciprocals, the
// source pair read from shared memory) with the default variant's shape:
// 128 threads, 3 targets per thread, 6 CTAs per SM, 4 source pairs per
// unrolled body. The 128 source pairs stay resident in shared memory. There
// is no staging, no far test, no flush and no near tile, so its rate
// (pairs/s, one pair = one target x one source) is the ceiling of the pair
// loop's instruction mix on this GPU.
constexpr int kFarT = 3, kFarNT = 128, kFarNP = 128, kFarMinB = 6;

struct FarTile {
  float4 a[kFarNP];
  float4 b[kFarNP];
  float4 c[kFarNP];
  float2 d[kFarNP];
};

__global__ void __launch_bounds__(kFarNT, kFarMinB) probe_far_pairs(int iters, float b, float c,
                                                                    float* sink) {
  __shared__ FarTile tile;
  for (int j = threadIdx.x; j < kFarNP; j += kFarNT) {
    const float s = 1e-3f * (float)(j + 1);
    tile.a[j] = make_float4(s, -s, 0.5f * s, 0.25f * s);         // offsets x, y of two sources
    tile.b[j] = make_float4(-s, s, 1.0f + s, 1.0f + 2.0f * s);   // offsets z; A_k near 1
    tile.c[j] = make_float4(b * s, c * s, s, -s);                // G x', G y'
    tile.d[j] = make_float2(s, 2.0f * s);                        // G z'
  }
  __syncthreads();
  float2 ntx[kFarT], nty[kFarT], ntz[kFarT], bh[kFarT], fx[kFarT], fy[kFarT], fz[kFarT];
#pragma unroll
  for (int t = 0; t < kFarT; ++t) {
    const float u = 1e-4f * (float)(threadIdx.x + 32 * t);
    ntx[t] = make_float2(-u, -u);
    nty[t] = make_float2(u, u);
    ntz[t] = make_float2(-0.5f * u, -0.5f * u);
    bh[t] = make_float2(0.5f + u, 0.5f + u);
    fx[t] = fy[t] = fz[t] = make_float2(0.f, 0.f);
  }
  for (int i = 0; i < iters; ++i)
    tcb::sp_far_run<kFarT, 4>(tile, 0, kFarNP, ntx, nty, ntz, bh, fx, fy, fz);
  float s = 0.f;
#pragma unroll
  for (int t = 0; t < kFarT; ++t) s += fx[t].x + fx[t].y + fy[t].x + fy[t].y + fz[t].x + fz[t].y;
  if (sink) sink[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

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
// TC_PROBE_RCP64, TC_PROBE_DDIV, TC_PROBE_F2F, TC_PROBE_FAR_PAIRS. Returns
// operations per second (one FMA, one reciprocal, one division or one pair = 1
// op; FFMA2 counts 2) in *ops_per_s.
extern "C" int tc_probe_peak(int device, int kind, int iters, double* ops_per_s) {
  if (!ops_per_s || iters <= 0 || iters > (1 << 22)) return TC_ERR_ARG;
  if (kind < TC_PROBE_FFMA || kind > TC_PROBE_FAR_PAIRS) return TC_ERR_ARG;
  int rc = tc_set_device_checked(device);
  if (rc) return rc;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return TC_ERR_CUDA;
  const bool far = kind == TC_PROBE_FAR_PAIRS;
  const int threads = far ? kFarNT : 256;
  const int blocks = far ? prop.multiProcessorCount * kFarMinB
                         : prop.multiProcessorCount * (prop.maxThreadsPerMultiProcessor / threads);
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
      case TC_PROBE_FAR_PAIRS: probe_far_pairs<<<blocks, threads>>>(it, 0.5f, 0.25f, nullptr); break;
      default: break;
    }
  };
  if (kind == TC_PROBE_FFMA2) per_thread_ops *= 2.0;
  if (far) per_thread_ops = (double)iters * kFarNP * 2 * kFarT;  // pairs
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
