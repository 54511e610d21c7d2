// Spatially coherent visiting order of targets for the FP32-compensated pair
// kernel: each target is keyed by its position along a 3-D Hilbert curve
// (10 bits per axis over the cube [-1,1]^3) and the keys are sorted with a
// stable radix sort, so a CTA's consecutive targets form a compact patch of
// the sphere whatever order the caller stores them in (the reference numbers
// particles in creation order, level by level). The sort is stable and the
// keys are a pure function of the positions, so the order - and with it every
// result - is deterministic.
//
// Hilbert index: J. Skilling, "Programming the Hilbert curve", AIP Conf.
// Proc. 707, 381 (2004): the coordinates are transformed in place
// ("axes to transpose") and the transposed bits interleaved.
#include <cub/device/device_radix_sort.cuh>

#include "tc_ctx.h"

namespace tcb {
namespace {

constexpr int kBits = 10;

__device__ __forceinline__ unsigned hilbert_key(double x, double y, double z) {
  const double scale = (double)((1u << kBits) - 1);
  unsigned X[3];
  const double c[3] = {x, y, z};
  for (int i = 0; i < 3; ++i) {
    double q = (c[i] + 1.0) * 0.5 * scale + 0.5;
    q = q < 0.0 ? 0.0 : (q > scale ? scale : q);
    X[i] = (unsigned)q;
  }
  const unsigned M = 1u << (kBits - 1);
  // inverse undo excess work
  for (unsigned Q = M; Q > 1; Q >>= 1) {
    const unsigned P = Q - 1;
    for (int i = 0; i < 3; ++i) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        unsigned t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  // Gray encode
  for (int i = 1; i < 3; ++i) X[i] ^= X[i - 1];
  unsigned t = 0;
  for (unsigned Q = M; Q > 1; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1;
  for (int i = 0; i < 3; ++i) X[i] ^= t;
  // interleave: bit b of X[0], X[1], X[2] from the most significant down
  unsigned key = 0;
  for (int b = kBits - 1; b >= 0; --b)
    for (int i = 0; i < 3; ++i) key = (key << 1) | ((X[i] >> b) & 1u);
  return key;
}

__global__ void hilbert_keys_kernel(const double* __restrict__ x, int i0, int n,
                                    unsigned* __restrict__ keys, int* __restrict__ idx) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const size_t b = 3 * (size_t)(i0 + j);
  keys[j] = hilbert_key(x[b], x[b + 1], x[b + 2]);
  idx[j] = i0 + j;
}

}  // namespace

// perm[i0 .. i1) <- the indices i0..i1-1 sorted by Hilbert key of x[i].
int compute_order(tc_ctx* ctx, const double* x, int i0, int i1, int* perm) {
  const int n = i1 - i0;
  if (n <= 0) return TC_OK;
  const size_t nb = (size_t)n;
  int rc;
  if ((rc = ctx->order_buf[0].ensure(nb * sizeof(unsigned))) ||
      (rc = ctx->order_buf[1].ensure(nb * sizeof(unsigned))) ||
      (rc = ctx->order_buf[2].ensure(nb * sizeof(int))))
    return rc;
  unsigned* k_in = ctx->order_buf[0].as<unsigned>();
  unsigned* k_out = ctx->order_buf[1].as<unsigned>();
  int* v_in = ctx->order_buf[2].as<int>();
  hilbert_keys_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(x, i0, n, k_in, v_in);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  size_t temp = 0;
  TC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp, k_in, k_out, v_in, perm + i0, n, 0,
                                              3 * kBits, ctx->stream));
  if ((rc = ctx->order_buf[3].ensure(temp))) return rc;
  TC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ctx->order_buf[3].ptr, temp, k_in, k_out, v_in,
                                              perm + i0, n, 0, 3 * kBits, ctx->stream));
  return TC_OK;
}

}  // namespace tcb
