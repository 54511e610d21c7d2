// Spatially coherent visiting order of targets for the FP32-compensated pair
// kernel: each target is keyed by its cube face and its position along a 2-D
// Hilbert curve over that face (sphere_order.cuh) and the keys are sorted with
// a stable radix sort, so a CTA's consecutive targets form a compact patch of
// the sphere whatever order the caller stores them in (the reference numbers
// particles in creation order, level by level). The sort is stable and the
// keys are a pure function of the positions, so the order - and with it every
// result - is deterministic.
#include <cub/device/device_radix_sort.cuh>

#include "sphere_order.cuh"
#include "tc_ctx.h"

namespace tcb {
namespace {

__global__ void hilbert_keys_kernel(const double* __restrict__ x, int i0, int n,
                                    unsigned* __restrict__ keys, int* __restrict__ idx) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const size_t b = 3 * (size_t)(i0 + j);
  keys[j] = sphere_key(x[b], x[b + 1], x[b + 2]);
  idx[j] = i0 + j;
}

}  // namespace

// Bytes of sort scratch (CUB's temporary storage) for an order over n targets.
int order_sort_bytes(int n, size_t* bytes) {
  *bytes = 0;
  if (n <= 0) return TC_OK;
  TC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, *bytes, (const unsigned*)nullptr,
                                              (unsigned*)nullptr, (const int*)nullptr, (int*)nullptr,
                                              n, 0, kSphereKeyBits));
  return TC_OK;
}

// perm[i0 .. i1) <- the indices i0..i1-1 sorted by the sphere key of x[i], in
// caller-provided scratch: keys k_in, k_out and indices v_in of i1 - i0 entries
// each, and `temp` of at least order_sort_bytes(i1 - i0) bytes.
int compute_order_into(tc_ctx* ctx, const double* x, int i0, int i1, int* perm, unsigned* k_in,
                       unsigned* k_out, int* v_in, void* temp, size_t temp_bytes) {
  const int n = i1 - i0;
  if (n <= 0) return TC_OK;
  hilbert_keys_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(x, i0, n, k_in, v_in);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  TC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, k_in, k_out, v_in, perm + i0, n, 0,
                                              kSphereKeyBits, ctx->stream));
  return TC_OK;
}

// perm[i0 .. i1) <- the indices i0..i1-1 sorted by the sphere key of x[i].
int compute_order(tc_ctx* ctx, const double* x, int i0, int i1, int* perm) {
  const int n = i1 - i0;
  if (n <= 0) return TC_OK;
  const size_t nb = (size_t)n;
  int rc;
  size_t temp = 0;
  if ((rc = ctx->order_buf[0].ensure(nb * sizeof(unsigned))) ||
      (rc = ctx->order_buf[1].ensure(nb * sizeof(unsigned))) ||
      (rc = ctx->order_buf[2].ensure(nb * sizeof(int))) || (rc = order_sort_bytes(n, &temp)) ||
      (rc = ctx->order_buf[3].ensure(temp)))
    return rc;
  return compute_order_into(ctx, x, i0, i1, perm, ctx->order_buf[0].as<unsigned>(),
                            ctx->order_buf[1].as<unsigned>(), ctx->order_buf[2].as<int>(),
                            ctx->order_buf[3].ptr, temp);
}

}  // namespace tcb
