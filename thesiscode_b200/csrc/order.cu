// Spatially coherent visiting order of targets for the FP32-compensated pair
// kernel: each target is keyed by its cube face and its position along a 2-D
// Hilbert curve over that face (sphere_order.cuh) and the keys are sorted with
// a stable radix sort, so a CTA's consecutive targets form a compact patch of
// the sphere whatever order the caller stores them in (the reference numbers
// particles in creation order, level by level). The sort is stable and the
// keys are a pure function of the positions, so the order - and with it every
// result - is deterministic.
#include <algorithm>

#include <cub/device/device_radix_sort.cuh>

#include "sphere_order.cuh"
#include "tc_ctx.h"

namespace tcb {
namespace {

// Checked build: extents of the key kernel's arrays.
struct KeyBounds {
  BoundsRec* rec;
  long long x_len, key_len;  // points in x; entries in keys and idx
};

__global__ void hilbert_keys_kernel(const double* __restrict__ x, int i0, int n,
                                    unsigned* __restrict__ keys, int* __restrict__ idx,
                                    const KeyBounds kb) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  if (!TC_BC(kb.rec, BC_ORDER_KEYS, j, kb.key_len)) return;
  const size_t b = 3 * (size_t)(i0 + j);
  keys[j] = TC_BC(kb.rec, BC_ORDER_X, i0 + j, kb.x_len) ? sphere_key(x[b], x[b + 1], x[b + 2]) : 0u;
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
                       unsigned* k_out, int* v_in, void* temp, size_t temp_bytes,
                       const OrderExtents& ext) {
  const int n = i1 - i0;
  if (n <= 0) return TC_OK;
  if ((long long)i1 > ext.perm_len || (long long)n > ext.key_len || (long long)i1 > ext.x_len) {
    tc_record_error("visiting order of [%d,%d): %lld points, %lld order entries, %lld keys", i0, i1,
                    ext.x_len, ext.perm_len, ext.key_len);
    return TC_ERR_ARG;
  }
  const KeyBounds kb{ctx->bc_rec, bc_extent(ctx, BC_ORDER_X, ext.x_len),
                     bc_extent(ctx, BC_ORDER_KEYS, ext.key_len)};
  hilbert_keys_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(x, i0, n, k_in, v_in, kb);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  TC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, k_in, k_out, v_in, perm + i0, n, 0,
                                              kSphereKeyBits, ctx->stream));
  return TC_OK;
}

// perm[i0 .. i1) <- the indices i0..i1-1 sorted by the sphere key of x[i].
int compute_order(tc_ctx* ctx, const double* x, int i0, int i1, int* perm, long long x_len,
                  long long perm_len) {
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
  const long long key_len = (long long)std::min(
      {ctx->order_buf[0].bytes / sizeof(unsigned), ctx->order_buf[1].bytes / sizeof(unsigned),
       ctx->order_buf[2].bytes / sizeof(int)});
  return compute_order_into(ctx, x, i0, i1, perm, ctx->order_buf[0].as<unsigned>(),
                            ctx->order_buf[1].as<unsigned>(), ctx->order_buf[2].as<int>(),
                            ctx->order_buf[3].ptr, temp, OrderExtents{x_len, perm_len, key_len});
}

}  // namespace tcb
