// Device side of the direct spherical Biot-Savart sum.
//
// One interaction (target x_i, source x_k with circulation G_k = zeta_k A_k):
//     w_ik = G_k / (1 - x_i.x_k + delta^2)
//     u_i  = -1/(4 pi) * x_i  x  sum_k w_ik (x_k - x_i)
// which equals the reference's sum_k (x_i x x_k) w_ik (BVEActiveRHS,
// PanelVelocityParallel.f90:1316-1333) because x_i x x_i = 0; the cross
// product is taken once per target instead of once per pair.
//
// Work decomposition: blockIdx.x = a tile of TB consecutive targets (one of
// up to three target classes), blockIdx.y = a chunk of consecutive sources.
// Each CTA streams its source chunk through shared memory in tiles of TS and
// writes one FP64 partial sum per target and chunk; the stage epilogue adds
// the chunks in a fixed order, so results are deterministic.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace tcb {

constexpr int kNoSelf = INT32_MIN;

struct TargetSeg {
  const double* x;  // targets, x[3*i + c]
  const int* perm;  // FP32C: target at position p in [i0,i1) is perm[p] (null: p itself)
  int i0, i1;       // target range [i0, i1) computed by this launch
  int out_offset;   // partial row of target i is out_offset + i
  int self_offset;  // source index of target i is i + self_offset (ACTIVE), else kNoSelf
  double d2;        // delta^2 for this class
  int tile_begin;   // first blockIdx.x of this segment
};

struct PairLaunch {
  TargetSeg seg[3];
  int nseg;
  const double4* src;   // packed sources {x, y, z, G}
  int n;                // number of sources
  int chunk_len;        // sources per blockIdx.y chunk (multiple of the tile)
  double* partial;      // partial[(chunk*3 + c)*n_out + row]
  int n_out;
};

// ---------------------------------------------------------------------------
// Reciprocals. The hardware seed (rcp.approx) is refined by Newton-Raphson
// r <- r + r(1 - d r); two steps take an FP64 seed to full precision. This
// replaces the IEEE division of the reference (a ~14-DFMA sequence on this
// GPU) by 4 DFMA; the result is within an ulp of 1/d.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double rcp_seed_f64(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
  return r;
}

__device__ __forceinline__ double rcp_newton2(double d) {
  double r = rcp_seed_f64(d);
  double e = fma(-d, r, 1.0);
  r = fma(r, e, r);
  e = fma(-d, r, 1.0);
  return fma(r, e, r);
}

__device__ __forceinline__ float rcp_approx_f32(float d) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
  return r;
}

__device__ __forceinline__ const TargetSeg& find_seg(const PairLaunch& P, int tile) {
  int s = 0;
  if (P.nseg > 1 && tile >= P.seg[1].tile_begin) s = 1;
  if (P.nseg > 2 && tile >= P.seg[2].tile_begin) s = 2;
  return P.seg[s];
}

// ---------------------------------------------------------------------------
// FP64 pair kernel.
// ---------------------------------------------------------------------------
// FUSED = false: the denominator is rounded exactly like the reference's
// 1.0 - sum(...) (six separately rounded operations). FUSED = true: the
// same expression as 1 - x.y + delta^2 in three fused multiply-adds, one
// rounding instead of six; it differs from the reference's value by the
// reference's own rounding error in the denominator (a few ulps of x.y).
template <bool FUSED>
__device__ __forceinline__ double pair_denominator(const double4& q, const double xi[3], double d2,
                                                   double one_plus_d2) {
  if (FUSED) {
    double s = fma(-q.x, xi[0], one_plus_d2);
    s = fma(-q.y, xi[1], s);
    return fma(-q.z, xi[2], s);
  }
  double s = __dmul_rn(q.x, xi[0]);
  s = __dadd_rn(s, __dmul_rn(q.y, xi[1]));
  s = __dadd_rn(s, __dmul_rn(q.z, xi[2]));
  return __dadd_rn(__dsub_rn(1.0, s), d2);
}

// One work unit: the targets at positions [tile0, min(tile0 + NT*TPT, i_end))
// of x against the sources [c0, c1); FP64 sums written to out[pos],
// out[stride + pos], out[2*stride + pos]. Targets whose source index is
// i + self_offset (self_offset != kNoSelf) skip themselves.
template <int NT, int TPT, int TS, bool FUSED>
__device__ __forceinline__ void fp64_unit(const double* __restrict__ x, int tile0, int i_end,
                                          int self_offset, double d2,
                                          const double4* __restrict__ src, int c0, int c1,
                                          double* __restrict__ out, size_t stride, double4* sm) {
  constexpr int TB = NT * TPT;
  const double one_plus_d2 = 1.0 + d2;
  const bool has_self = self_offset != kNoSelf;

  double xi[TPT][3], acc[TPT][3];
  int self_k[TPT];
#pragma unroll
  for (int t = 0; t < TPT; ++t) {
    int i = tile0 + (int)threadIdx.x + t * NT;
    int ld = i < i_end ? i : tile0;
    xi[t][0] = x[3 * (size_t)ld];
    xi[t][1] = x[3 * (size_t)ld + 1];
    xi[t][2] = x[3 * (size_t)ld + 2];
    acc[t][0] = acc[t][1] = acc[t][2] = 0.0;
    self_k[t] = has_self ? i + self_offset : -1;
  }
  const int self_lo = has_self ? tile0 + self_offset : 0;
  const int self_hi = has_self ? min(tile0 + TB, i_end) + self_offset : 0;

  for (int ts = c0; ts < c1; ts += TS) {
    __syncthreads();
    for (int j = threadIdx.x; j < TS; j += NT) {
      int k = ts + j;
      sm[j] = k < c1 ? src[k] : make_double4(0.0, 0.0, 0.0, 0.0);
    }
    __syncthreads();
    const bool diag = has_self && ts < self_hi && self_lo < ts + TS;
    if (!diag) {
#pragma unroll 2
      for (int j = 0; j < TS; ++j) {
        const double4 q = sm[j];
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
          const double den = pair_denominator<FUSED>(q, xi[t], d2, one_plus_d2);
          const double w = __dmul_rn(q.w, rcp_newton2(den));
          acc[t][0] = fma(w, q.x - xi[t][0], acc[t][0]);
          acc[t][1] = fma(w, q.y - xi[t][1], acc[t][1]);
          acc[t][2] = fma(w, q.z - xi[t][2], acc[t][2]);
        }
      }
    } else {
      for (int j = 0; j < TS; ++j) {
        const double4 q = sm[j];
        const int k = ts + j;
#pragma unroll
        for (int t = 0; t < TPT; ++t) {
          const double den = pair_denominator<FUSED>(q, xi[t], d2, one_plus_d2);
          double w = __dmul_rn(q.w, rcp_newton2(den));
          w = (k == self_k[t]) ? 0.0 : w;
          acc[t][0] = fma(w, q.x - xi[t][0], acc[t][0]);
          acc[t][1] = fma(w, q.y - xi[t][1], acc[t][1]);
          acc[t][2] = fma(w, q.z - xi[t][2], acc[t][2]);
        }
      }
    }
  }
#pragma unroll
  for (int t = 0; t < TPT; ++t) {
    int i = tile0 + (int)threadIdx.x + t * NT;
    if (i < i_end) {
      out[i] = acc[t][0];
      out[stride + i] = acc[t][1];
      out[2 * stride + i] = acc[t][2];
    }
  }
}

template <int NT, int TPT, int TS, int MINB, bool FUSED>
__global__ void __launch_bounds__(NT, MINB) pair_fp64_kernel(const PairLaunch P) {
  __shared__ double4 sm[TS];
  const TargetSeg& G = find_seg(P, blockIdx.x);
  const int tile0 = G.i0 + (int)(blockIdx.x - G.tile_begin) * (NT * TPT);
  const int c0 = (int)blockIdx.y * P.chunk_len;
  const int c1 = min(P.n, c0 + P.chunk_len);
  const size_t stride = (size_t)P.n_out;
  double* out = P.partial + (size_t)blockIdx.y * 3 * stride + G.out_offset;
  fp64_unit<NT, TPT, TS, FUSED>(G.x, tile0, G.i1, G.self_offset, G.d2, P.src, c0, c1, out, stride,
                                sm);
}

// ---------------------------------------------------------------------------
// FP32-compensated pair kernel.
//
// Each CTA takes the position c of the middle target of its tile as origin.
// Sources are converted once per CTA and tile from FP64 to FP32 offsets
// s_k = fl32(x_k - c) (their FP64 difference rounded once), targets likewise
// t_i = fl32(x_i - c). Targets are visited in a spatially coherent order (a
// Hilbert order computed by the library, or the caller's order), so a CTA's
// targets form a compact patch and every nearby pair has small |s_k|, |t_i|:
// d = s_k - t_i carries an absolute error of a few ulps of the patch size
// instead of ulps of 1. The denominator uses the cancellation-free form
//     2(1 - x_i.x_k) + 2 delta^2 = |x_k - x_i|^2 + e_i + e_k,
//     e_i = 1 - |x_i|^2 + 2 delta^2,  e_k = 1 - |x_k|^2
// (evaluated in FP64 once per point, then rounded to FP32), so near pairs
// keep full FP32 relative accuracy. Two targets share each f32x2 instruction
// (FADD2/FFMA2/FMUL2 halve the issue slots; the FP32 pipe stays the bound).
// Per-target FP32 partial sums are added into FP64 accumulators every FLUSH
// sources.
//
// Self pair (TC_ACTIVE, targets are sources): s_k and t_i are rounded from
// the same double, so d = 0 exactly; e_i carries a +1e-30 bias that keeps
// D = e_i + e_k away from 0 and from FP32 subnormals (e is either 0 or at
// least ~1e-17 in magnitude), so w stays finite and w*d adds exactly 0. No
// per-pair mask is needed.
// ---------------------------------------------------------------------------
constexpr float kSelfBias = 1e-30f;

// Far-field form (FM bit 0). For a source tile whose every source lies
// farther than kFarRatio times the CTA's target radius rho (the largest
// |t_i| of the CTA) from the origin, the denominator is expanded as
//     D/2 = A_k + B_i + s_k.nt_i,   A_k = (|s_k|^2 + e_k)/2,
//     B_i = (|t_i|^2 + e_i)/2,      nt_i = -t_i
// (A_k and B_i from FP64, rounded once), and the sum as
//     sum w (s_k - t_i) = sum w s_k + nt_i sum w,
// so the three offset subtractions leave the pair loop: 9 FP32 operations
// per pair instead of 11. With |s| > 3 rho, D >= (|s| - rho)^2 >= 4|s|^2/9,
// so each rounding of the expansion costs at most a few ulps of D, as in the
// near form; the self pair never qualifies (|s_self| = |t_self| <= rho).
// Paired reciprocal (FM bit 1): the two targets of an f32x2 lane pair share
// one MUFU reciprocal q = 1/(D_a D_b): 1/D_a = q D_b, 1/D_b = q D_a.
constexpr float kFarRatio2 = 9.0f;  // kFarRatio = 3

template <bool PR>
__device__ __forceinline__ float2 rcp_pair(float2 D) {
  if (PR) {
    const float q = rcp_approx_f32(__fmul_rn(D.x, D.y));
    return __fmul2_rn(make_float2(q, q), make_float2(D.y, D.x));
  }
  return make_float2(rcp_approx_f32(D.x), rcp_approx_f32(D.y));
}

__device__ __forceinline__ float norm2_f32(float a, float b, float c) {
  return __fmaf_rn(c, c, __fmaf_rn(b, b, __fmul_rn(a, a)));
}

// min (max) of a non-negative float over the CTA: one warp reduction, one
// entry per warp in red[]; the caller synchronises before combine_*.
__device__ __forceinline__ void warp_store_min(float v, unsigned* red) {
  const unsigned m = __reduce_min_sync(0xffffffffu, __float_as_uint(v));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
}
__device__ __forceinline__ void warp_store_max(float v, unsigned* red) {
  const unsigned m = __reduce_max_sync(0xffffffffu, __float_as_uint(v));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
}
template <int NW>
__device__ __forceinline__ float combine_min(const unsigned* red) {
  unsigned m = red[0];
#pragma unroll
  for (int w = 1; w < NW; ++w) m = min(m, red[w]);
  return __uint_as_float(m);
}
template <int NW>
__device__ __forceinline__ float combine_max(const unsigned* red) {
  unsigned m = red[0];
#pragma unroll
  for (int w = 1; w < NW; ++w) m = max(m, red[w]);
  return __uint_as_float(m);
}

// Shared memory of one FP32C unit.
template <int NT, int TS>
struct Fp32cSmem {
  float4 a[TS];           // (sx, sx, sy, sy)
  float4 b[TS];           // (sz, sz, 2G, 2G)
  float2 e[TS];           // near form: (e_k, e_k)
  float2 h[TS];           // far form: (A_k, A_k)
  unsigned tmin[NT / 32]; // per-warp min of |s_k|^2 over the tile
  unsigned rho[NT / 32];  // per-warp max of |t_i|^2 over the CTA's targets
};

// One work unit (targets at visiting positions [tile0, min(tile0 + NT*2*NPAIR,
// i_end)) against sources [c0, c1)).
template <int NT, int NPAIR, int TS, int FLUSH, int UNROLL, int FM>
__device__ __forceinline__ void fp32c_unit(const double* __restrict__ x, const int* __restrict__ perm,
                                           int tile0, int i_end, double d2,
                                           const double4* __restrict__ src, int c0, int c1,
                                           double* __restrict__ out, size_t stride,
                                           Fp32cSmem<NT, TS>& sm) {
  static_assert(TS % FLUSH == 0, "flush interval must divide the tile");
  static_assert(NT % 32 == 0, "whole warps");
  constexpr int TPT = 2 * NPAIR;
  constexpr int TB = NT * TPT;
  constexpr bool FAR = (FM & 1) != 0;
  constexpr bool PR = (FM & 2) != 0;

  const int mid_pos = min(tile0 + TB / 2, i_end - 1);
  const int mid = perm ? perm[mid_pos] : mid_pos;
  const double cx = x[3 * (size_t)mid], cy = x[3 * (size_t)mid + 1], cz = x[3 * (size_t)mid + 2];

  float2 ntx[NPAIR], nty[NPAIR], ntz[NPAIR], ei[NPAIR], bh[NPAIR];
  float2 fx[NPAIR], fy[NPAIR], fz[NPAIR], fw[NPAIR];
  double ax[NPAIR][2], ay[NPAIR][2], az[NPAIR][2], aw[NPAIR][2];
  float rho2 = 0.f;
#pragma unroll
  for (int p = 0; p < NPAIR; ++p) {
    float tv[2][5];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      int pos = tile0 + (int)threadIdx.x + (2 * p + h) * NT;
      int ld = pos < i_end ? (perm ? perm[pos] : pos) : mid;
      double px = x[3 * (size_t)ld], py = x[3 * (size_t)ld + 1], pz = x[3 * (size_t)ld + 2];
      const float tx = (float)(px - cx), ty = (float)(py - cy), tz = (float)(pz - cz);
      const double E = (1.0 - (px * px + py * py + pz * pz)) + 2.0 * d2;
      tv[h][0] = -tx;
      tv[h][1] = -ty;
      tv[h][2] = -tz;
      tv[h][3] = (float)E + kSelfBias;
      const float t2 = norm2_f32(tx, ty, tz);
      tv[h][4] = (float)(0.5 * ((double)t2 + E));
      rho2 = fmaxf(rho2, t2);
      ax[p][h] = ay[p][h] = az[p][h] = aw[p][h] = 0.0;
    }
    ntx[p] = make_float2(tv[0][0], tv[1][0]);
    nty[p] = make_float2(tv[0][1], tv[1][1]);
    ntz[p] = make_float2(tv[0][2], tv[1][2]);
    ei[p] = make_float2(tv[0][3], tv[1][3]);
    bh[p] = make_float2(tv[0][4], tv[1][4]);
    fx[p] = fy[p] = fz[p] = fw[p] = make_float2(0.f, 0.f);
  }
  if (FAR) warp_store_max(rho2, sm.rho);

  for (int ts = c0; ts < c1; ts += TS) {
    __syncthreads();
    float smin = __int_as_float(0x7f800000);  // +inf
    for (int j = threadIdx.x; j < TS; j += NT) {
      int k = ts + j;
      float sx = 0.f, sy = 0.f, sz = 0.f, g = 0.f, e = 1.f, ah = 1.f;
      if (k < c1) {
        const double4 q = src[k];
        sx = (float)(q.x - cx);
        sy = (float)(q.y - cy);
        sz = (float)(q.z - cz);
        g = (float)(2.0 * q.w);
        const double ek = 1.0 - (q.x * q.x + q.y * q.y + q.z * q.z);
        e = (float)ek;
        if (FAR) {
          const float s2 = norm2_f32(sx, sy, sz);
          ah = (float)(0.5 * ((double)s2 + ek));
          smin = fminf(smin, s2);
        }
      }
      sm.a[j] = make_float4(sx, sx, sy, sy);
      sm.b[j] = make_float4(sz, sz, g, g);
      sm.e[j] = make_float2(e, e);
      if (FAR) sm.h[j] = make_float2(ah, ah);
    }
    if (FAR) warp_store_min(smin, sm.tmin);
    __syncthreads();
    // strict: with rho = 0 (one target position) no tile is far
    const bool far = FAR && combine_min<NT / 32>(sm.tmin) > kFarRatio2 * combine_max<NT / 32>(sm.rho);
    if (far) {
      for (int jf = 0; jf < TS; jf += FLUSH) {
#pragma unroll UNROLL
        for (int j = jf; j < jf + FLUSH; ++j) {
          const float4 a = sm.a[j];
          const float4 b = sm.b[j];
          const float2 ah = sm.h[j];
          const float2 sxx = make_float2(a.x, a.y), syy = make_float2(a.z, a.w);
          const float2 szz = make_float2(b.x, b.y), gg = make_float2(b.z, b.w);
#pragma unroll
          for (int p = 0; p < NPAIR; ++p) {
            float2 D = __fadd2_rn(ah, bh[p]);
            D = __ffma2_rn(sxx, ntx[p], D);
            D = __ffma2_rn(syy, nty[p], D);
            D = __ffma2_rn(szz, ntz[p], D);
            const float2 w = __fmul2_rn(gg, rcp_pair<PR>(D));  // 2 w: D/2 above
            fx[p] = __ffma2_rn(w, sxx, fx[p]);
            fy[p] = __ffma2_rn(w, syy, fy[p]);
            fz[p] = __ffma2_rn(w, szz, fz[p]);
            fw[p] = __fadd2_rn(fw[p], w);
          }
        }
#pragma unroll
        for (int p = 0; p < NPAIR; ++p) {
          ax[p][0] = fma(0.5, (double)fx[p].x, ax[p][0]);
          ax[p][1] = fma(0.5, (double)fx[p].y, ax[p][1]);
          ay[p][0] = fma(0.5, (double)fy[p].x, ay[p][0]);
          ay[p][1] = fma(0.5, (double)fy[p].y, ay[p][1]);
          az[p][0] = fma(0.5, (double)fz[p].x, az[p][0]);
          az[p][1] = fma(0.5, (double)fz[p].y, az[p][1]);
          aw[p][0] = fma(0.5, (double)fw[p].x, aw[p][0]);
          aw[p][1] = fma(0.5, (double)fw[p].y, aw[p][1]);
          fx[p] = fy[p] = fz[p] = fw[p] = make_float2(0.f, 0.f);
        }
      }
    } else {
      for (int jf = 0; jf < TS; jf += FLUSH) {
#pragma unroll UNROLL
        for (int j = jf; j < jf + FLUSH; ++j) {
          const float4 a = sm.a[j];
          const float4 b = sm.b[j];
          const float2 ee = sm.e[j];
          const float2 sxx = make_float2(a.x, a.y), syy = make_float2(a.z, a.w);
          const float2 szz = make_float2(b.x, b.y), gg = make_float2(b.z, b.w);
#pragma unroll
          for (int p = 0; p < NPAIR; ++p) {
            const float2 dx = __fadd2_rn(sxx, ntx[p]);
            const float2 dy = __fadd2_rn(syy, nty[p]);
            const float2 dz = __fadd2_rn(szz, ntz[p]);
            float2 D = __fadd2_rn(ee, ei[p]);
            D = __ffma2_rn(dx, dx, D);
            D = __ffma2_rn(dy, dy, D);
            D = __ffma2_rn(dz, dz, D);
            const float2 w = __fmul2_rn(gg, rcp_pair<PR>(D));
            fx[p] = __ffma2_rn(w, dx, fx[p]);
            fy[p] = __ffma2_rn(w, dy, fy[p]);
            fz[p] = __ffma2_rn(w, dz, fz[p]);
          }
        }
#pragma unroll
        for (int p = 0; p < NPAIR; ++p) {
          ax[p][0] += (double)fx[p].x;
          ax[p][1] += (double)fx[p].y;
          ay[p][0] += (double)fy[p].x;
          ay[p][1] += (double)fy[p].y;
          az[p][0] += (double)fz[p].x;
          az[p][1] += (double)fz[p].y;
          fx[p] = fy[p] = fz[p] = make_float2(0.f, 0.f);
        }
      }
    }
  }
  // far tiles: + nt_i sum w; partial rows are indexed by position in the visiting order
#pragma unroll
  for (int p = 0; p < NPAIR; ++p) {
    const float ntxs[2] = {ntx[p].x, ntx[p].y}, ntys[2] = {nty[p].x, nty[p].y},
                ntzs[2] = {ntz[p].x, ntz[p].y};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      int pos = tile0 + (int)threadIdx.x + (2 * p + h) * NT;
      if (FAR) {
        ax[p][h] = fma((double)ntxs[h], aw[p][h], ax[p][h]);
        ay[p][h] = fma((double)ntys[h], aw[p][h], ay[p][h]);
        az[p][h] = fma((double)ntzs[h], aw[p][h], az[p][h]);
      }
      if (pos < i_end) {
        out[pos] = ax[p][h];
        out[stride + pos] = ay[p][h];
        out[2 * stride + pos] = az[p][h];
      }
    }
  }
}


template <int NT, int NPAIR, int TS, int FLUSH, int MINB, int UNROLL, int FM>
__global__ void __launch_bounds__(NT, MINB) pair_fp32c_kernel(const PairLaunch P) {
  __shared__ Fp32cSmem<NT, TS> sm;
  const TargetSeg& G = find_seg(P, blockIdx.x);
  const int tile0 = G.i0 + (int)(blockIdx.x - G.tile_begin) * (NT * 2 * NPAIR);
  const int c0 = (int)blockIdx.y * P.chunk_len;
  const int c1 = min(P.n, c0 + P.chunk_len);
  const size_t stride = (size_t)P.n_out;
  double* out = P.partial + (size_t)blockIdx.y * 3 * stride + G.out_offset;
  fp32c_unit<NT, NPAIR, TS, FLUSH, UNROLL, FM>(G.x, G.perm, tile0, G.i1, G.d2, P.src, c0, c1, out,
                                               stride, sm);
}

// ---------------------------------------------------------------------------
// Batched (ensemble) form: many independent particle sets concatenated in one
// RK4 state. A work item is (target tile of one class of one instance, one
// chunk of that instance's sources); a persistent grid of one wave of CTAs
// takes items from an atomic counter until none is left (no CTA ever waits
// on another). Items are queued longest first, so the uneven instance sizes
// even out across the SMs.
// ---------------------------------------------------------------------------
struct BatchSeg {
  const double* x;   // target positions of the class (concatenated instances)
  const int* perm;   // FP32C visiting order (null: as stored)
  int out_offset;    // partial row of target position p is out_offset + p
  int self_offset;   // TC_ACTIVE: source index of target i is i + self_offset
  double d2;
};

struct BatchItem {
  int seg;           // index into the segment table
  int tile0, i1;     // target positions [tile0, min(tile0 + TB, i1))
  int c0, c1;        // sources [c0, c1) (absolute rows of the packed sources)
  int chunk;         // chunk index within the instance (partial slab)
};

struct BatchLaunch {
  const BatchItem* items;
  int n_items;
  int* counter;      // zeroed before each launch
  const BatchSeg* segs;
  const double4* src;
  double* partial;   // partial[(chunk*3 + c)*stride + row]
  size_t stride;
};

__device__ __forceinline__ int next_item(int* counter, int* slot) {
  __syncthreads();  // every thread is done with the previous item's slot value
  if (threadIdx.x == 0) *slot = atomicAdd(counter, 1);
  __syncthreads();
  return *slot;
}

template <int NT, int NPAIR, int TS, int FLUSH, int MINB, int UNROLL, int FM>
__global__ void __launch_bounds__(NT, MINB) pair_fp32c_batch_kernel(const BatchLaunch B) {
  __shared__ Fp32cSmem<NT, TS> sm;
  __shared__ int slot;
  for (int it = next_item(B.counter, &slot); it < B.n_items; it = next_item(B.counter, &slot)) {
    const BatchItem I = B.items[it];
    const BatchSeg S = B.segs[I.seg];
    double* out = B.partial + (size_t)I.chunk * 3 * B.stride + S.out_offset;
    fp32c_unit<NT, NPAIR, TS, FLUSH, UNROLL, FM>(S.x, S.perm, I.tile0, I.i1, S.d2, B.src, I.c0,
                                                 I.c1, out, B.stride, sm);
  }
}

template <int NT, int TPT, int TS, int MINB, bool FUSED>
__global__ void __launch_bounds__(NT, MINB) pair_fp64_batch_kernel(const BatchLaunch B) {
  __shared__ double4 sm[TS];
  __shared__ int slot;
  for (int it = next_item(B.counter, &slot); it < B.n_items; it = next_item(B.counter, &slot)) {
    const BatchItem I = B.items[it];
    const BatchSeg S = B.segs[I.seg];
    double* out = B.partial + (size_t)I.chunk * 3 * B.stride + S.out_offset;
    fp64_unit<NT, TPT, TS, FUSED>(S.x, I.tile0, I.i1, S.self_offset, S.d2, B.src, I.c0, I.c1, out,
                                  B.stride, sm);
  }
}

}  // namespace tcb
