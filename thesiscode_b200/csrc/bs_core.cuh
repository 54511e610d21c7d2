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

#include "bounds.cuh"

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
  long long x_len;     // checked build: points in x
  long long perm_len;  // checked build: entries in perm
};

struct PairLaunch {
  TargetSeg seg[3];
  int nseg;
  const double4* src;   // packed sources {x, y, z, G}
  int n;                // number of sources
  int chunk_len;        // sources per blockIdx.y chunk (multiple of the tile)
  double* partial;      // partial[(chunk*3 + c)*n_out + row]
  int n_out;
  BoundsRec* bc;        // checked build: violation record (null: release build)
  long long src_len;    // checked build: packed sources in src
  long long partial_len;  // checked build: doubles in partial
};

// Extents a work unit checks its global indices against (checked build).
struct UnitBounds {
  BoundsRec* rec;
  long long x_len, perm_len, src_len;
  long long out_base;  // offset of the unit's out pointer within the partial sums
  long long out_len;   // doubles in the partial sums
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
                                          double* __restrict__ out, size_t stride, double4* sm,
                                          const UnitBounds& ub) {
  constexpr int TB = NT * TPT;
  const double one_plus_d2 = 1.0 + d2;
  const bool has_self = self_offset != kNoSelf;

  double xi[TPT][3], acc[TPT][3];
  int self_k[TPT];
#pragma unroll
  for (int t = 0; t < TPT; ++t) {
    int i = tile0 + (int)threadIdx.x + t * NT;
    int ld = i < i_end ? i : tile0;
    const bool okx = TC_BC(ub.rec, BC_PAIR_X, ld, ub.x_len);
    xi[t][0] = okx ? x[3 * (size_t)ld] : 0.0;
    xi[t][1] = okx ? x[3 * (size_t)ld + 1] : 0.0;
    xi[t][2] = okx ? x[3 * (size_t)ld + 2] : 0.0;
    acc[t][0] = acc[t][1] = acc[t][2] = 0.0;
    self_k[t] = has_self ? i + self_offset : -1;
  }
  const int self_lo = has_self ? tile0 + self_offset : 0;
  const int self_hi = has_self ? min(tile0 + TB, i_end) + self_offset : 0;

  for (int ts = c0; ts < c1; ts += TS) {
    __syncthreads();
    for (int j = threadIdx.x; j < TS; j += NT) {
      int k = ts + j;
      sm[j] = (k < c1 && TC_BC(ub.rec, BC_PAIR_SRC, k, ub.src_len))
                  ? src[k]
                  : make_double4(0.0, 0.0, 0.0, 0.0);
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
      if (TC_BC(ub.rec, BC_PAIR_OUT, ub.out_base + i, ub.out_len)) out[i] = acc[t][0];
      if (TC_BC(ub.rec, BC_PAIR_OUT, ub.out_base + (long long)stride + i, ub.out_len))
        out[stride + i] = acc[t][1];
      if (TC_BC(ub.rec, BC_PAIR_OUT, ub.out_base + 2 * (long long)stride + i, ub.out_len))
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
  const long long base = (long long)blockIdx.y * 3 * (long long)stride + G.out_offset;
  double* out = P.partial + base;
  const UnitBounds ub{P.bc, G.x_len, G.perm_len, P.src_len, base, P.partial_len};
  fp64_unit<NT, TPT, TS, FUSED>(G.x, tile0, G.i1, G.self_offset, G.d2, P.src, c0, c1, out, stride,
                                sm, ub);
}

// ---------------------------------------------------------------------------
// FP32-compensated pair kernel.
//
// Each CTA takes an origin c - the centroid of its targets projected to the
// sphere - and an orthonormal frame R = (e1, e2, e3) with e3 along c. Sources
// are converted once per CTA and tile from FP64 to FP32 offsets
// s_k = fl32(R(x_k - c)) (FP64 difference and rotation, one rounding),
// targets likewise t_i = fl32(R(x_i - c)). Targets are visited in a spatially
// coherent order (the library's cube-face Hilbert order, sphere_order.cuh, or
// the caller's), so a CTA's targets form a compact patch and every nearby pair
// has small |s_k|, |t_i|: d = s_k - t_i carries an absolute error of a few
// ulps of the patch size instead of ulps of 1. Distances and dot products are
// frame-invariant. The denominator uses the cancellation-free form
//     2(1 - x_i.x_k) + 2 delta^2 = |x_k - x_i|^2 + e_i + e_k,
//     e_i = 1 - |x_i|^2 + 2 delta^2,  e_k = 1 - |x_k|^2
// (evaluated in FP64 once per point, then rounded to FP32), so near pairs
// keep full FP32 relative accuracy although RK4 drifts points off the sphere.
//
// Source pairing: the two f32x2 lanes of every FADD2/FFMA2/FMUL2 carry two
// SOURCES (k, k+1) of one target, so a source tile sits in shared memory once
// (no duplicated values): a warp-wide broadcast 128-bit shared load costs two
// wavefronts of the SM-wide shared pipe, and a far source pair costs 7,
// shared by the T targets of a thread.
//
// Two forms of the pair, chosen per 64-source segment (uniform over the CTA):
// * near (11 FP32 operations): d = s_k - t_i, D = |d|^2 + e_i + e_k,
//   T' += (2G_k / D) d;
// * far (7 FP32 operations), for segments whose every source is farther than
//   kFarRatio times the CTA's target radius rho (the largest |t_i|) from the
//   origin: D/2 = A_k + B_i + s_k.(-t_i), A_k = (|s_k|^2 + e_k)/2 and
//   B_i = (|t_i|^2 + e_i)/2 from FP64, and T' += r (G_k x'_k) with
//   x'_k = R x_k (G x'_k from FP64, one rounding). In the rotated frame the
//   first two coordinates of x'_k are small tangential offsets and the third
//   is about 1, so the large common part of the sum (about sum r G) sits in
//   the third coordinate only, and u_i = x_i x R^T T' multiplies it by the
//   target's own small offset. With |s| > 3 rho, D >= (|s| - rho)^2 >=
//   4|s|^2/9, so each rounding of the expansion costs at most a few ulps of D,
//   as in the near form; the self pair never qualifies.
// Near and far sums go into the same accumulators: near sum w (x'_k - x'_i)
// and far sum w x'_k differ by multiples of x'_i, which u = x_i x T ignores.
//
// One MUFU reciprocal (rcp.approx.ftz.f32) per pair. The FP32 partials of the
// two source lanes are added and flushed into FP64 accumulators every FLUSH
// sources in mixed tiles (every FLUSH * FARK sources in tiles whose every
// source is far: far terms are small and smooth, and each flush costs F2F
// conversions on the XU pipe that the reciprocals also need), and rotated
// back to the global frame in FP64 once per target.
//
// Self pair (TC_ACTIVE, targets are sources): s_k and t_i are computed by the
// same explicitly fused FP64 operations from the same double, so d = 0
// exactly; e_i carries a +1e-30 bias that keeps D = e_i + e_k away from 0
// and from FP32 subnormals (e is either 0 or at least ~1e-17 in magnitude),
// so w stays finite and w*d adds exactly 0. No per-pair mask is needed.
//
// Form bits (FM): bit 3 always set (the source-paired form; the bit value
// is part of the variant-info ABI); bit 1 keeps the FP64 accumulators in
// shared memory (one slot per thread, target and coordinate: 6 fewer
// registers per target); bit 2 gives near tiles hi/lo offsets; bits 8-9 hold
// log2 FARK.
// HILO (bit 2): near tiles take d = s - t from hi/lo FP32 splits of both
// offsets, (s_hi - t_hi) + (s_lo - t_lo): the rounding of the offsets to FP32
// (an absolute error of ulps of the patch radius, the dominant FP32C error
// for nearest-neighbour pairs) no longer enters, and d keeps a few ulps of its
// own length. Far tiles are unchanged. Both low parts are needed: for the self
// pair s and t are the same point, so (s_hi - t_hi) and (s_lo - t_lo) are
// both exactly 0 and the pair adds w * 0; correcting one side only would
// leave d = s_lo there, a spurious self term.
// ---------------------------------------------------------------------------
constexpr float kSelfBias = 1e-30f;
constexpr float kFarRatio2 = 9.0f;  // kFarRatio = 3

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

template <int NT, int TS, int T = 1, bool SMACC = false, bool HILO = false>
struct SpSmem {
  float4 a[TS / 2];        // (sx_k, sx_k+1, sy_k, sy_k+1)
  float4 b[TS / 2];        // (sz_k, sz_k+1, A_k, A_k+1)
  float4 c[TS / 2];        // (G x'_k, G x'_k+1, G y'_k, G y'_k+1)
  float2 d[TS / 2];        // (G z'_k, G z'_k+1)
  float4 n[TS / 2];        // near form: (e_k, e_k+1, 2G_k, 2G_k+1)
  double frame[12];        // e1, e2, e3 (rows), origin c
  double csum[3][NT / 32]; // per-warp sums of the target positions
  double acc[SMACC ? 3 * T * NT : 1];  // FP64 accumulators [c][t][thread] (SMACC)
  float4 lo[HILO ? TS / 2 : 1];        // HILO: low parts (slx_k, slx_k+1, sly_k, sly_k+1)
  float2 loz[HILO ? TS / 2 : 1];       // HILO: (slz_k, slz_k+1)
  float tlo[HILO ? 3 * T * NT : 1];    // HILO: -(target low parts) [c][t][thread]
  unsigned tmin[NT / 32];
  unsigned rho[NT / 32];
};

// Orthonormal basis with e3 = c/|c| (Duff, Burgess, Christensen, Hart, Kensler,
// Liani, Pharr, "Building an Orthonormal Basis, Revisited", JCGT 6(1), 2017).
__device__ __forceinline__ void make_frame(double cx, double cy, double cz, double* f) {
  const double inv = rsqrt(fma(cx, cx, fma(cy, cy, cz * cz)));
  const double nx = cx * inv, ny = cy * inv, nz = cz * inv;
  const double sg = copysign(1.0, nz);
  const double a = -1.0 / (sg + nz);
  const double b = nx * ny * a;
  f[0] = 1.0 + sg * nx * nx * a;
  f[1] = sg * b;
  f[2] = -sg * nx;
  f[3] = b;
  f[4] = sg + ny * ny * a;
  f[5] = -ny;
  f[6] = nx;
  f[7] = ny;
  f[8] = nz;
}

// R v with explicitly fused operations, so a target and the same point as a
// source round identically (the self pair then has d = 0 exactly).
__device__ __forceinline__ double frame_dot(const double* e, double vx, double vy, double vz) {
  return fma(e[0], vx, fma(e[1], vy, __dmul_rn(e[2], vz)));
}

__device__ __forceinline__ float2 rcp2(float2 D) {
  return make_float2(rcp_approx_f32(D.x), rcp_approx_f32(D.y));
}

// One far source pair against the thread's T targets.
template <int T>
__device__ __forceinline__ void sp_far_step(const float4 a, const float4 b, const float4 c,
                                            const float2 d, const float2* ntx, const float2* nty,
                                            const float2* ntz, const float2* bh, float2* fx,
                                            float2* fy, float2* fz) {
  const float2 sx = make_float2(a.x, a.y), sy = make_float2(a.z, a.w);
  const float2 sz = make_float2(b.x, b.y), ah = make_float2(b.z, b.w);
  const float2 gx = make_float2(c.x, c.y), gy = make_float2(c.z, c.w);
#pragma unroll
  for (int t = 0; t < T; ++t) {
    float2 D = __fadd2_rn(ah, bh[t]);
    D = __ffma2_rn(sx, ntx[t], D);
    D = __ffma2_rn(sy, nty[t], D);
    D = __ffma2_rn(sz, ntz[t], D);
    const float2 r = rcp2(D);
    fx[t] = __ffma2_rn(r, gx, fx[t]);
    fy[t] = __ffma2_rn(r, gy, fy[t]);
    fz[t] = __ffma2_rn(r, d, fz[t]);
  }
}

// FP64 accumulator of target t, coordinate c: a register, or (SMACC) a
// shared-memory slot of this thread (frees 6 registers per target).
template <int NT, int T, bool SMACC>
struct SpAcc {
  double r[SMACC ? 1 : 3 * T];
  double* sm;
  __device__ __forceinline__ void init(double* base) {
    sm = base + threadIdx.x;
#pragma unroll
    for (int k = 0; k < 3 * T; ++k) {
      if (SMACC)
        sm[k * NT] = 0.0;
      else
        r[k] = 0.0;
    }
  }
  __device__ __forceinline__ void add(int c, int t, double v) {
    if (SMACC)
      sm[(c * T + t) * NT] += v;
    else
      r[c * T + t] += v;
  }
  __device__ __forceinline__ double get(int c, int t) const {
    return SMACC ? sm[(c * T + t) * NT] : r[c * T + t];
  }
};

// Converts the sources of the tile at ts into the CTA's frame: offsets s_k,
// A_k = (|s_k|^2 + e_k)/2, G_k x'_k, e_k, 2G_k (and the hi/lo low parts),
// padding past c1; records each warp's minimum |s_k|^2.
template <int NT, int TS, bool HILO, class Smem>
__device__ __forceinline__ void sp_stage(const double4* __restrict__ src, int ts, int c1,
                                         const double* fr, Smem& sm, const UnitBounds& ub) {
  constexpr int NP = TS / 2;
  float smin = __int_as_float(0x7f800000);  // +inf
  for (int jp = threadIdx.x; jp < NP; jp += NT) {
    float v[2][12];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = ts + 2 * jp + h;
      // padding sources: zero weight, unit denominators
      v[h][0] = v[h][1] = v[h][2] = 0.f;
      v[h][3] = 1.f;
      v[h][4] = v[h][5] = v[h][6] = 0.f;
      v[h][7] = 1.f;
      v[h][8] = 0.f;
      v[h][9] = v[h][10] = v[h][11] = 0.f;
      if (k < c1 && TC_BC(ub.rec, BC_PAIR_SRC, k, ub.src_len)) {
        const double4 q = src[k];
        const double dx = q.x - fr[9], dy = q.y - fr[10], dz = q.z - fr[11];
        const double sxd = frame_dot(fr, dx, dy, dz), syd = frame_dot(fr + 3, dx, dy, dz),
                     szd = frame_dot(fr + 6, dx, dy, dz);
        const float sx = (float)sxd, sy = (float)syd, sz = (float)szd;
        if (HILO) {
          v[h][9] = (float)(sxd - (double)sx);
          v[h][10] = (float)(syd - (double)sy);
          v[h][11] = (float)(szd - (double)sz);
        }
        const double ek = 1.0 - (q.x * q.x + q.y * q.y + q.z * q.z);
        const float s2 = norm2_f32(sx, sy, sz);
        smin = fminf(smin, s2);
        v[h][0] = sx;
        v[h][1] = sy;
        v[h][2] = sz;
        v[h][3] = (float)(0.5 * ((double)s2 + ek));
        v[h][4] = (float)(q.w * frame_dot(fr, q.x, q.y, q.z));
        v[h][5] = (float)(q.w * frame_dot(fr + 3, q.x, q.y, q.z));
        v[h][6] = (float)(q.w * frame_dot(fr + 6, q.x, q.y, q.z));
        v[h][7] = (float)ek;
        v[h][8] = (float)(2.0 * q.w);
      }
    }
    sm.a[jp] = make_float4(v[0][0], v[1][0], v[0][1], v[1][1]);
    sm.b[jp] = make_float4(v[0][2], v[1][2], v[0][3], v[1][3]);
    sm.c[jp] = make_float4(v[0][4], v[1][4], v[0][5], v[1][5]);
    sm.d[jp] = make_float2(v[0][6], v[1][6]);
    sm.n[jp] = make_float4(v[0][7], v[1][7], v[0][8], v[1][8]);
    if (HILO) {
      sm.lo[jp] = make_float4(v[0][9], v[1][9], v[0][10], v[1][10]);
      sm.loz[jp] = make_float2(v[0][11], v[1][11]);
    }
  }
  warp_store_min(smin, sm.tmin);
}

// Far source pairs [j0, j1) of the staged tile against the thread's targets.
template <int T, int UNROLL, class Smem>
__device__ __forceinline__ void sp_far_run(const Smem& sm, int j0, int j1, const float2 (&ntx)[T],
                                           const float2 (&nty)[T], const float2 (&ntz)[T],
                                           const float2 (&bh)[T], float2 (&fx)[T], float2 (&fy)[T],
                                           float2 (&fz)[T]) {
#pragma unroll UNROLL
  for (int j = j0; j < j1; ++j)
    sp_far_step<T>(sm.a[j], sm.b[j], sm.c[j], sm.d[j], ntx, nty, ntz, bh, fx, fy, fz);
}

// Sums the staged tile into the thread's T targets: a tile whose
// every source is far in one tight far loop flushed every FARK segments; else
// per 64-source segment, far or near. With NT = TS/2 source pairs and FP = 32
// every warp staged exactly one segment, so segment g's minimum |s|^2 is warp
// g's and only the segments that hold near sources take the near form;
// otherwise one far test for the whole tile.
template <int NT, int T, int TS, int FLUSH, int UNROLL, bool SMACC, bool HILO, int FARK, class Smem>
__device__ __forceinline__ void sp_sum(const Smem& sm, const float2 (&ntx)[T],
                                       const float2 (&nty)[T], const float2 (&ntz)[T],
                                       const float2 (&bh)[T], const float (&ei)[T],
                                       float2 (&fx)[T], float2 (&fy)[T], float2 (&fz)[T],
                                       SpAcc<NT, T, SMACC>& acc) {
  constexpr int NP = TS / 2;
  constexpr int FP = FLUSH / 2;
  constexpr int FPF = FP * FARK;  // source pairs between flushes in all-far tiles
  constexpr bool PERSEG = (NT == TS / 2) && (FP == 32);
  const float lim = kFarRatio2 * combine_max<NT / 32>(sm.rho);
  const bool tile_far = combine_min<NT / 32>(sm.tmin) > lim;
  if (tile_far) {
    for (int jf = 0; jf < NP; jf += FPF) {
      sp_far_run<T, UNROLL>(sm, jf, jf + FPF, ntx, nty, ntz, bh, fx, fy, fz);
#pragma unroll
      for (int t = 0; t < T; ++t) {
        acc.add(0, t, (double)__fadd_rn(fx[t].x, fx[t].y));
        acc.add(1, t, (double)__fadd_rn(fy[t].x, fy[t].y));
        acc.add(2, t, (double)__fadd_rn(fz[t].x, fz[t].y));
        fx[t] = fy[t] = fz[t] = make_float2(0.f, 0.f);
      }
    }
    return;
  }
  for (int jf = 0; jf < NP; jf += FP) {
    const bool far = PERSEG && __uint_as_float(sm.tmin[jf / FP]) > lim;
    if (far) {
      sp_far_run<T, UNROLL>(sm, jf, jf + FP, ntx, nty, ntz, bh, fx, fy, fz);
    } else {
      // HILO: d = (s_hi - t_hi) + (s_lo - t_lo), accurate to a few ulps of d itself
      float ntl[HILO ? 3 * T : 1];
      if (HILO) {
#pragma unroll
        for (int k = 0; k < 3 * T; ++k) ntl[k] = sm.tlo[k * NT + threadIdx.x];
      }
#pragma unroll 4
      for (int j = jf; j < jf + FP; ++j) {
        const float4 a = sm.a[j];
        const float4 b = sm.b[j];
        const float4 n = sm.n[j];
        const float2 sx = make_float2(a.x, a.y), sy = make_float2(a.z, a.w);
        const float2 sz = make_float2(b.x, b.y);
        const float2 ee = make_float2(n.x, n.y), gg = make_float2(n.z, n.w);
        float4 lo = make_float4(0.f, 0.f, 0.f, 0.f);
        float2 loz = make_float2(0.f, 0.f);
        if (HILO) {
          lo = sm.lo[j];
          loz = sm.loz[j];
        }
#pragma unroll
        for (int t = 0; t < T; ++t) {
          float2 dx = __fadd2_rn(sx, ntx[t]);
          float2 dy = __fadd2_rn(sy, nty[t]);
          float2 dz = __fadd2_rn(sz, ntz[t]);
          if (HILO) {
            dx = __fadd2_rn(dx, __fadd2_rn(make_float2(lo.x, lo.y), make_float2(ntl[t], ntl[t])));
            dy = __fadd2_rn(dy, __fadd2_rn(make_float2(lo.z, lo.w), make_float2(ntl[T + t], ntl[T + t])));
            dz = __fadd2_rn(dz, __fadd2_rn(loz, make_float2(ntl[2 * T + t], ntl[2 * T + t])));
          }
          float2 D = __fadd2_rn(ee, make_float2(ei[t], ei[t]));
          D = __ffma2_rn(dx, dx, D);
          D = __ffma2_rn(dy, dy, D);
          D = __ffma2_rn(dz, dz, D);
          const float2 w = __fmul2_rn(gg, rcp2(D));
          fx[t] = __ffma2_rn(w, dx, fx[t]);
          fy[t] = __ffma2_rn(w, dy, fy[t]);
          fz[t] = __ffma2_rn(w, dz, fz[t]);
        }
      }
    }
#pragma unroll
    for (int t = 0; t < T; ++t) {
      acc.add(0, t, (double)__fadd_rn(fx[t].x, fx[t].y));
      acc.add(1, t, (double)__fadd_rn(fy[t].x, fy[t].y));
      acc.add(2, t, (double)__fadd_rn(fz[t].x, fz[t].y));
      fx[t] = fy[t] = fz[t] = make_float2(0.f, 0.f);
    }
  }
}

// One work unit: targets at visiting positions [tile0, min(tile0 + NT*T,
// i_end)) against sources [c0, c1); FP64 sums in the global frame written to
// out[pos], out[stride + pos], out[2*stride + pos].
template <int NT, int T, int TS, int FLUSH, int UNROLL, bool SMACC, bool HILO, int FARK>
__device__ __forceinline__ void fp32c_sp_unit(const double* __restrict__ x, const int* __restrict__ perm,
                                              int tile0, int i_end, double d2,
                                              const double4* __restrict__ src, int c0, int c1,
                                              double* __restrict__ out, size_t stride,
                                              SpSmem<NT, TS, T, SMACC, HILO>& sm,
                                              const UnitBounds& ub) {
  static_assert(TS % FLUSH == 0 && FLUSH % 2 == 0, "flush interval: even, divides the tile");
  static_assert(NT % 32 == 0, "whole warps");
  static_assert(TS % (FLUSH * FARK) == 0, "far-tile flush interval divides the tile");
  constexpr int TB = NT * T;

  const int mid_pos = min(tile0 + TB / 2, i_end - 1);
  int mid = mid_pos;
  if (perm) mid = TC_BC(ub.rec, BC_PAIR_PERM, mid_pos, ub.perm_len) ? perm[mid_pos] : 0;
  // checked build: an out-of-range target index reads point 0 instead (and is recorded)
  auto target = [&](int p) -> int {
    int ld = p;
    if (perm) ld = TC_BC(ub.rec, BC_PAIR_PERM, p, ub.perm_len) ? perm[p] : 0;
    return TC_BC(ub.rec, BC_PAIR_X, ld, ub.x_len) ? ld : 0;
  };
  // Origin: the CTA's targets' centroid, projected to the sphere (a smaller
  // patch radius than any one target gives: fewer near tiles, smaller FP32
  // offsets); the middle target when the targets surround the centre.
  double px = 0.0, py = 0.0, pz = 0.0;
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const int pos = tile0 + (int)threadIdx.x + t * NT;
    if (pos < i_end) {
      const int ld = target(pos);
      px += x[3 * (size_t)ld];
      py += x[3 * (size_t)ld + 1];
      pz += x[3 * (size_t)ld + 2];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    px += __shfl_xor_sync(0xffffffffu, px, o);
    py += __shfl_xor_sync(0xffffffffu, py, o);
    pz += __shfl_xor_sync(0xffffffffu, pz, o);
  }
  __syncthreads();  // the previous unit (persistent kernel) is done with sm.frame, sm.csum
  if ((threadIdx.x & 31) == 0) {
    sm.csum[0][threadIdx.x >> 5] = px;
    sm.csum[1][threadIdx.x >> 5] = py;
    sm.csum[2][threadIdx.x >> 5] = pz;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int w = 0; w < NT / 32; ++w) {
      sx += sm.csum[0][w];
      sy += sm.csum[1][w];
      sz += sm.csum[2][w];
    }
    const double count = (double)min(TB, i_end - tile0);
    const double n2 = sx * sx + sy * sy + sz * sz;
    double cx, cy, cz;
    if (n2 > 0.25 * count * count) {
      const double inv = 1.0 / sqrt(n2);
      cx = sx * inv;
      cy = sy * inv;
      cz = sz * inv;
    } else {
      const int c = TC_BC(ub.rec, BC_PAIR_X, mid, ub.x_len) ? mid : 0;
      cx = x[3 * (size_t)c];
      cy = x[3 * (size_t)c + 1];
      cz = x[3 * (size_t)c + 2];
    }
    make_frame(cx, cy, cz, sm.frame);
    sm.frame[9] = cx;
    sm.frame[10] = cy;
    sm.frame[11] = cz;
  }
  __syncthreads();
  const double* fr = sm.frame;
  const double cx = fr[9], cy = fr[10], cz = fr[11];

  float2 ntx[T], nty[T], ntz[T], bh[T];
  float ei[T];  // near form only: paired on use
  float2 fx[T], fy[T], fz[T];
  SpAcc<NT, T, SMACC> acc;
  acc.init(sm.acc);
  float rho2 = 0.f;
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const int pos = tile0 + (int)threadIdx.x + t * NT;
    const int ld = pos < i_end ? target(pos) : (TC_BC(ub.rec, BC_PAIR_X, mid, ub.x_len) ? mid : 0);
    const double px = x[3 * (size_t)ld], py = x[3 * (size_t)ld + 1], pz = x[3 * (size_t)ld + 2];
    const double dx = px - cx, dy = py - cy, dz = pz - cz;
    const double txd = frame_dot(fr, dx, dy, dz), tyd = frame_dot(fr + 3, dx, dy, dz),
                 tzd = frame_dot(fr + 6, dx, dy, dz);
    const float tx = (float)txd, ty = (float)tyd, tz = (float)tzd;
    if (HILO) {
      sm.tlo[(0 * T + t) * NT + threadIdx.x] = -(float)(txd - (double)tx);
      sm.tlo[(1 * T + t) * NT + threadIdx.x] = -(float)(tyd - (double)ty);
      sm.tlo[(2 * T + t) * NT + threadIdx.x] = -(float)(tzd - (double)tz);
    }
    const double E = (1.0 - (px * px + py * py + pz * pz)) + 2.0 * d2;
    ntx[t] = make_float2(-tx, -tx);
    nty[t] = make_float2(-ty, -ty);
    ntz[t] = make_float2(-tz, -tz);
    ei[t] = (float)E + kSelfBias;
    const float t2 = norm2_f32(tx, ty, tz);
    const float b = (float)(0.5 * ((double)t2 + E));
    bh[t] = make_float2(b, b);
    rho2 = fmaxf(rho2, t2);
    fx[t] = fy[t] = fz[t] = make_float2(0.f, 0.f);
  }
  warp_store_max(rho2, sm.rho);
  for (int ts = c0; ts < c1; ts += TS) {
    __syncthreads();
    sp_stage<NT, TS, HILO>(src, ts, c1, fr, sm, ub);
    __syncthreads();
    sp_sum<NT, T, TS, FLUSH, UNROLL, SMACC, HILO, FARK>(sm, ntx, nty, ntz, bh, ei, fx, fy, fz, acc);
  }
  // back to the global frame: T = R^T T'
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const int pos = tile0 + (int)threadIdx.x + t * NT;
    if (pos < i_end) {
      const double ax = acc.get(0, t), ay = acc.get(1, t), az = acc.get(2, t);
      if (TC_BC(ub.rec, BC_PAIR_OUT, ub.out_base + pos, ub.out_len))
        out[pos] = fma(fr[0], ax, fma(fr[3], ay, fr[6] * az));
      if (TC_BC(ub.rec, BC_PAIR_OUT, ub.out_base + (long long)stride + pos, ub.out_len))
        out[stride + pos] = fma(fr[1], ax, fma(fr[4], ay, fr[7] * az));
      if (TC_BC(ub.rec, BC_PAIR_OUT, ub.out_base + 2 * (long long)stride + pos, ub.out_len))
        out[2 * stride + pos] = fma(fr[2], ax, fma(fr[5], ay, fr[8] * az));
    }
  }
}

// Template parameters of fp32c_sp_unit from a form bit set FM.
template <int FM>
struct SpForm {
  static constexpr bool smacc = (FM & 2) != 0;
  static constexpr bool hilo = (FM & 4) != 0;
  static constexpr int fark = 1 << ((FM >> 8) & 3);
};

template <int NT, int T, int TS, int FLUSH, int MINB, int UNROLL, int FM>
__global__ void __launch_bounds__(NT, MINB) pair_fp32c_kernel(const PairLaunch P) {
  using F = SpForm<FM>;
  const TargetSeg& G = find_seg(P, blockIdx.x);
  const int tile0 = G.i0 + (int)(blockIdx.x - G.tile_begin) * (NT * T);
  const int c0 = (int)blockIdx.y * P.chunk_len;
  const int c1 = min(P.n, c0 + P.chunk_len);
  const size_t stride = (size_t)P.n_out;
  const long long base = (long long)blockIdx.y * 3 * (long long)stride + G.out_offset;
  double* out = P.partial + base;
  const UnitBounds ub{P.bc, G.x_len, G.perm_len, P.src_len, base, P.partial_len};
  __shared__ SpSmem<NT, TS, T, F::smacc, F::hilo> sm;
  fp32c_sp_unit<NT, T, TS, FLUSH, UNROLL, F::smacc, F::hilo, F::fark>(G.x, G.perm, tile0, G.i1,
                                                                      G.d2, P.src, c0, c1, out,
                                                                      stride, sm, ub);
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
  long long x_len;     // checked build: points in x
  long long perm_len;  // checked build: entries in perm
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
  BoundsRec* bc;          // checked build: violation record (null: release build)
  int n_segs;             // checked build: entries in segs
  long long src_len;      // checked build: packed sources in src
  long long partial_len;  // checked build: doubles in partial
};

__device__ __forceinline__ int next_item(int* counter, int* slot) {
  __syncthreads();  // every thread is done with the previous item's slot value
  if (threadIdx.x == 0) *slot = atomicAdd(counter, 1);
  __syncthreads();
  return *slot;
}

template <int NT, int T, int TS, int FLUSH, int MINB, int UNROLL, int FM>
__global__ void __launch_bounds__(NT, MINB) pair_fp32c_batch_kernel(const BatchLaunch B) {
  using F = SpForm<FM>;
  __shared__ int slot;
  __shared__ SpSmem<NT, TS, T, F::smacc, F::hilo> sm;
  for (int it = next_item(B.counter, &slot); it < B.n_items; it = next_item(B.counter, &slot)) {
    const BatchItem I = B.items[it];
    if (!TC_BC(B.bc, BC_BATCH_SEG, I.seg, B.n_segs)) continue;
    const BatchSeg S = B.segs[I.seg];
    const long long base = (long long)I.chunk * 3 * (long long)B.stride + S.out_offset;
    double* out = B.partial + base;
    const UnitBounds ub{B.bc, S.x_len, S.perm_len, B.src_len, base, B.partial_len};
    fp32c_sp_unit<NT, T, TS, FLUSH, UNROLL, F::smacc, F::hilo, F::fark>(
        S.x, S.perm, I.tile0, I.i1, S.d2, B.src, I.c0, I.c1, out, B.stride, sm, ub);
  }
}

template <int NT, int TPT, int TS, int MINB, bool FUSED>
__global__ void __launch_bounds__(NT, MINB) pair_fp64_batch_kernel(const BatchLaunch B) {
  __shared__ double4 sm[TS];
  __shared__ int slot;
  for (int it = next_item(B.counter, &slot); it < B.n_items; it = next_item(B.counter, &slot)) {
    const BatchItem I = B.items[it];
    if (!TC_BC(B.bc, BC_BATCH_SEG, I.seg, B.n_segs)) continue;
    const BatchSeg S = B.segs[I.seg];
    const long long base = (long long)I.chunk * 3 * (long long)B.stride + S.out_offset;
    double* out = B.partial + base;
    const UnitBounds ub{B.bc, S.x_len, S.perm_len, B.src_len, base, B.partial_len};
    fp64_unit<NT, TPT, TS, FUSED>(S.x, I.tile0, I.i1, S.self_offset, S.d2, B.src, I.c0, I.c1, out,
                                  B.stride, sm, ub);
  }
}

}  // namespace tcb
