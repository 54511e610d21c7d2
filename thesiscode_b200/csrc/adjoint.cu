// Discrete adjoint of the RK4 Biot-Savart step: the gradient of an end-time
// functional J(x(T), zeta(T)) with respect to the initial positions and
// vorticities of the active panels, through nsteps classical RK4 steps
// (the forward map of BVERK4, PanelVelocityParallel.f90:435-658, restricted
// to the active panels, which are the only ones that feed back).
//
// Vector-Jacobian product of one RHS evaluation. With cotangent (mu_x, mu_z)
// on (dx/dt, dzeta/dt) = (u, -2 Omega u_z), the cotangent on u is
// ut_i = mu_x,i + (-2 Omega mu_z,i) z_hat, and for
//     L = sum_i ut_i . u_i,  u_i = -1/(4 pi) sum_{k != i} G_k (x_i x x_k) / D_ik,
//     D_ik = 1 + delta^2 - x_i . x_k,  G_k = zeta_k A_k,
// with v_i = ut_i x x_i and s_ik = x_k . v_i (= ut_i . (x_i x x_k)):
//     dL/dx_i   = -1/(4 pi) [ S1_i x ut_i + S2_i + G_i (P_i + Q_i) ]
//     dL/dzeta_k = -A_k/(4 pi) R_k
//     S1_i = sum_k G_k/D x_k,      S2_i = sum_k G_k s_ik/D^2 x_k     (target side)
//     P_k  = sum_i v_i/D,          Q_k  = sum_i s_ik/D^2 x_i,
//     R_k  = sum_i s_ik/D                                            (source side)
// Both sums are O(N^2) pair loops like the forward one; two kernels compute
// them in FP64 with the forward kernel's tiling (source tiles in shared
// memory, targets in registers, per-chunk partial sums reduced in a fixed
// order). RK4 backward per step, with Y_s the stage inputs and k_s = dt F(Y_s):
//     lk4 = l'/6,               lY4 = dt J(Y4)^T lk4
//     lk3 = l'/3 + lY4,         lY3 = dt J(Y3)^T lk3
//     lk2 = l'/3 + lY3/2,       lY2 = dt J(Y2)^T lk2
//     lk1 = l'/6 + lY2/2,       lY1 = dt J(Y1)^T lk1
//     l   = l' + lY1 + lY2 + lY3 + lY4.
// The state is checkpointed every `ckpt_every` steps on the forward sweep;
// the backward sweep recomputes each segment's stage inputs from its
// checkpoint (one extra forward pass in total).
#include <algorithm>
#include <cmath>
#include <vector>

#include "tc_ctx.h"

namespace tcb {
namespace {

constexpr int kAdjNT = 128;
constexpr int kAdjTS = 128;
constexpr double kInv4Pi = 0.0795774715459476678844418816862571810;  // 1/(4 pi)

struct AdjLaunch {
  const double* x;       // positions x[3i+c] (targets and sources: the same panels)
  const double4* src;    // pass 1: {x, y, z, G}; pass 2: {x, y, z, v_x}
  const double2* src2;   // pass 2: {v_y, v_z}
  const double* v;       // pass 1: v_i per target (3 per row)
  int n;
  int chunk_len;
  double one_plus_d2;
  double* partial;       // [chunk][W][n]
};

__device__ __forceinline__ double adj_rcp(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
  double e = fma(-d, r, 1.0);
  r = fma(r, e, r);
  e = fma(-d, r, 1.0);
  return fma(r, e, r);
}

// Pass 1: per target i, S1 = sum_k G_k/D x_k and S2 = sum_k G_k s_ik/D^2 x_k
// (6 outputs per row).
__global__ void __launch_bounds__(kAdjNT) adj_target_kernel(const AdjLaunch P) {
  __shared__ double4 sm[kAdjTS];
  const int i = blockIdx.x * kAdjNT + threadIdx.x;
  const int ld = i < P.n ? i : P.n - 1;
  const double xi0 = P.x[3 * (size_t)ld], xi1 = P.x[3 * (size_t)ld + 1], xi2 = P.x[3 * (size_t)ld + 2];
  const double v0 = P.v[3 * (size_t)ld], v1 = P.v[3 * (size_t)ld + 1], v2 = P.v[3 * (size_t)ld + 2];
  double a1x = 0, a1y = 0, a1z = 0, a2x = 0, a2y = 0, a2z = 0;
  const int c0 = blockIdx.y * P.chunk_len, c1 = min(P.n, c0 + P.chunk_len);
  for (int ts = c0; ts < c1; ts += kAdjTS) {
    __syncthreads();
    for (int j = threadIdx.x; j < kAdjTS; j += kAdjNT) {
      int k = ts + j;
      sm[j] = k < c1 ? P.src[k] : make_double4(0.0, 0.0, 0.0, 0.0);
    }
    __syncthreads();
    for (int j = 0; j < kAdjTS; ++j) {
      const double4 q = sm[j];
      double D = fma(-q.x, xi0, P.one_plus_d2);
      D = fma(-q.y, xi1, D);
      D = fma(-q.z, xi2, D);
      double r = adj_rcp(D);
      r = (ts + j == i) ? 0.0 : r;  // self pair (D may be 0: r is then NaN before the select)
      const double w1 = q.w * r;
      const double s = fma(q.x, v0, fma(q.y, v1, q.z * v2));  // s_ik = x_k . v_i
      const double w2 = w1 * s * r;
      a1x = fma(w1, q.x, a1x);
      a1y = fma(w1, q.y, a1y);
      a1z = fma(w1, q.z, a1z);
      a2x = fma(w2, q.x, a2x);
      a2y = fma(w2, q.y, a2y);
      a2z = fma(w2, q.z, a2z);
    }
  }
  if (i < P.n) {
    const size_t n = (size_t)P.n;
    double* out = P.partial + (size_t)blockIdx.y * 6 * n + i;
    out[0] = a1x;
    out[n] = a1y;
    out[2 * n] = a1z;
    out[3 * n] = a2x;
    out[4 * n] = a2y;
    out[5 * n] = a2z;
  }
}

// Pass 2: per panel k (as a source of the forward sum), the transposed sums
// over the panels i that it acts on: P_k, Q_k (3 each), R_k (7 outputs).
// Here the thread's row is k and the shared-memory stream is i with {x_i, v_i}.
__global__ void __launch_bounds__(kAdjNT) adj_source_kernel(const AdjLaunch P) {
  __shared__ double4 sa[kAdjTS];
  __shared__ double2 sb[kAdjTS];
  const int k = blockIdx.x * kAdjNT + threadIdx.x;
  const int ld = k < P.n ? k : P.n - 1;
  const double xk0 = P.x[3 * (size_t)ld], xk1 = P.x[3 * (size_t)ld + 1], xk2 = P.x[3 * (size_t)ld + 2];
  double px = 0, py = 0, pz = 0, qx = 0, qy = 0, qz = 0, rr = 0;
  const int c0 = blockIdx.y * P.chunk_len, c1 = min(P.n, c0 + P.chunk_len);
  for (int ts = c0; ts < c1; ts += kAdjTS) {
    __syncthreads();
    for (int j = threadIdx.x; j < kAdjTS; j += kAdjNT) {
      int i = ts + j;
      sa[j] = i < c1 ? P.src[i] : make_double4(0.0, 0.0, 0.0, 0.0);
      sb[j] = i < c1 ? P.src2[i] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int j = 0; j < kAdjTS; ++j) {
      const double4 a = sa[j];
      const double2 b = sb[j];
      double D = fma(-a.x, xk0, P.one_plus_d2);
      D = fma(-a.y, xk1, D);
      D = fma(-a.z, xk2, D);
      double r = adj_rcp(D);
      r = (ts + j == k) ? 0.0 : r;
      // s_ik = x_k . v_i
      const double s = fma(xk0, a.w, fma(xk1, b.x, xk2 * b.y));
      const double sr = s * r;
      const double sr2 = sr * r;
      px = fma(r, a.w, px);
      py = fma(r, b.x, py);
      pz = fma(r, b.y, pz);
      qx = fma(sr2, a.x, qx);
      qy = fma(sr2, a.y, qy);
      qz = fma(sr2, a.z, qz);
      rr += sr;
    }
  }
  if (k < P.n) {
    const size_t n = (size_t)P.n;
    double* out = P.partial + (size_t)blockIdx.y * 7 * n + k;
    out[0] = px;
    out[n] = py;
    out[2 * n] = pz;
    out[3 * n] = qx;
    out[4 * n] = qy;
    out[5 * n] = qz;
    out[6 * n] = rr;
  }
}

// Fused pass: one visit of each pair (i, k) feeds both sides. Rows (targets
// i) keep S1 = sum_k G_k/D x_k and S2 = sum_k G_k s/D^2 x_k in registers;
// columns (sources k) get P, Q, R summed over the CTA's targets: per source,
// across the thread's targets, then the warp (shuffles), then the warps
// (shared memory); one column partial per (target tile, source) goes to
// colpart[(tile*7 + c)*n + k]. Every (tile, k) slot is written exactly once,
// so the combine is a fixed-order sum: deterministic, no atomics.

struct AdjFused {
  const double* x;       // positions of the panels (rows and columns)
  const double4* src;    // {x, y, z, G} per panel
  const double* v;       // v_i per row
  int n;
  int chunk_len;
  double one_plus_d2;
  double* rowpart;       // [chunk][6][n]
  double* colpart;       // [tile][7][n]
};

// LEVELS shuffle steps leave 32 >> LEVELS partial sums per warp and source.
template <int kFNT, int kFTPT, int LEVELS, int kFTS>
__global__ void __launch_bounds__(kFNT) adj_fused_kernel(const AdjFused P) {
  constexpr int kFWARPS = kFNT / 32;
  constexpr int kPARTS = 32 >> LEVELS;
  __shared__ double4 sm[kFTS];
  __shared__ double red[kFWARPS * kPARTS][kFTS][7];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tile0 = blockIdx.x * (kFNT * kFTPT);
  double xi[kFTPT][3], vi[kFTPT][3], s1[kFTPT][3], s2[kFTPT][3];
  int row[kFTPT];
  bool valid[kFTPT];
#pragma unroll
  for (int t = 0; t < kFTPT; ++t) {
    row[t] = tile0 + (int)threadIdx.x + t * kFNT;
    valid[t] = row[t] < P.n;
    const int ld = valid[t] ? row[t] : P.n - 1;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      xi[t][c] = P.x[3 * (size_t)ld + c];
      vi[t][c] = P.v[3 * (size_t)ld + c];
      s1[t][c] = s2[t][c] = 0.0;
    }
  }
  const int c0 = blockIdx.y * P.chunk_len, c1 = min(P.n, c0 + P.chunk_len);
  const size_t N = (size_t)P.n;
  for (int ts = c0; ts < c1; ts += kFTS) {
    __syncthreads();  // previous tile's sm and red are consumed
    for (int j = threadIdx.x; j < kFTS; j += kFNT) {
      int k = ts + j;
      sm[j] = k < c1 ? P.src[k] : make_double4(0.0, 0.0, 0.0, 0.0);
    }
    __syncthreads();
    for (int j = 0; j < kFTS; ++j) {
      const double4 q = sm[j];
      const int k = ts + j;
      double pk[7] = {0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int t = 0; t < kFTPT; ++t) {
        double D = fma(-q.x, xi[t][0], P.one_plus_d2);
        D = fma(-q.y, xi[t][1], D);
        D = fma(-q.z, xi[t][2], D);
        double r = adj_rcp(D);
        r = (valid[t] && k != row[t] && k < c1) ? r : 0.0;  // self pair, padded rows and sources
        const double s = fma(q.x, vi[t][0], fma(q.y, vi[t][1], q.z * vi[t][2]));
        const double w1 = q.w * r;
        const double sr = s * r;
        const double w2 = w1 * sr;
        const double sr2 = sr * r;
        s1[t][0] = fma(w1, q.x, s1[t][0]);
        s1[t][1] = fma(w1, q.y, s1[t][1]);
        s1[t][2] = fma(w1, q.z, s1[t][2]);
        s2[t][0] = fma(w2, q.x, s2[t][0]);
        s2[t][1] = fma(w2, q.y, s2[t][1]);
        s2[t][2] = fma(w2, q.z, s2[t][2]);
        pk[0] = fma(r, vi[t][0], pk[0]);
        pk[1] = fma(r, vi[t][1], pk[1]);
        pk[2] = fma(r, vi[t][2], pk[2]);
        pk[3] = fma(sr2, xi[t][0], pk[3]);
        pk[4] = fma(sr2, xi[t][1], pk[4]);
        pk[5] = fma(sr2, xi[t][2], pk[5]);
        pk[6] += sr;
      }
#pragma unroll
      for (int c = 0; c < 7; ++c) {
#pragma unroll
        for (int o = 16; o >= kPARTS; o >>= 1) pk[c] += __shfl_down_sync(0xffffffffu, pk[c], o);
      }
      if (lane < kPARTS)
#pragma unroll
        for (int c = 0; c < 7; ++c) red[warp * kPARTS + lane][j][c] = pk[c];
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kFTS * 7; idx += kFNT) {
      const int j = idx / 7, c = idx - 7 * j, k = ts + j;
      if (k < c1) {
        double acc = 0.0;
#pragma unroll
        for (int w = 0; w < kFWARPS * kPARTS; ++w) acc += red[w][j][c];
        P.colpart[((size_t)blockIdx.x * 7 + c) * N + k] = acc;
      }
    }
  }
#pragma unroll
  for (int t = 0; t < kFTPT; ++t)
    if (valid[t]) {
      double* out = P.rowpart + (size_t)blockIdx.y * 6 * N + row[t];
      out[0] = s1[t][0];
      out[N] = s1[t][1];
      out[2 * N] = s1[t][2];
      out[3 * N] = s2[t][0];
      out[4 * N] = s2[t][1];
      out[5 * N] = s2[t][2];
    }
}

// Row-major single pass. The source-side sums of panel k are sums over the
// panels j it acts on, for fixed k - row sums like the target side - and
// D_ij = D_ji, so one visit of each ordered pair (i, j) gives row i every sum
// it needs, with s_ij = x_j . v_i and s_ji = x_i . v_j. Q_i enters dL/dx_i only
// as G_i Q_i, next to S2_i, and both weight x_j, so they share one accumulator;
// R_i = sum_j s_ji r = x_i . P_i needs none:
//     S1 += r (G_j x_j),  C += ((G_j x_j).v_i + (G_i x_i).v_j) r^2 x_j  (= S2 + G_i Q),
//     P  += r v_j                                          (r = 1/D_ij)
// 9 accumulators per row and 20 FP64 operations per pair besides the
// reciprocal: rcp.approx.f64 seed + NEWTON Newton-Raphson steps
// r <- r + r (1 - D r) of 2 FMA each (2 steps: full FP64; 1 step: the seed's
// error squared). TPT rows per thread share each source's shared-memory loads.
// No reduction across threads. Rows: partial[(chunk*9 + c)*n + i].
constexpr int kRNT = 128, kRTS = 128, kRowSums = 9;

struct RowLaunch {
  const double4* ra;  // {x, y, z, G x} per panel
  const double4* rb;  // {G y, G z, v_x, v_y}
  const double* rc;   // v_z
  int n;
  int chunk_len;
  double one_plus_d2;
  double* partial;    // [chunk][kRowSums][n]
  BoundsRec* bc;          // checked build: violation record (null: release build)
  long long src_len;      // checked build: entries of ra, rb and rc
  long long partial_len;  // checked build: doubles in partial
};

template <int NEWTON>
__device__ __forceinline__ double adj_rcp_n(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
#pragma unroll
  for (int k = 0; k < NEWTON; ++k) r = fma(r, fma(-d, r, 1.0), r);
  return r;
}

// One source j against the thread's TPT rows. MASK: skip j == row (the
// self term), needed only in the source tile that holds the CTA's own rows.
template <int TPT, int NEWTON, bool MASK>
__device__ __forceinline__ void adj_row_source(const double4 q, const double4 w, const double vz,
                                               int k, const int* row, double one_plus_d2,
                                               const double* x0, const double* x1, const double* x2,
                                               const double* g0, const double* g1, const double* g2,
                                               const double* v0, const double* v1, const double* v2,
                                               double (*a)[kRowSums]) {
#pragma unroll
  for (int t = 0; t < TPT; ++t) {
    double D = fma(-q.x, x0[t], one_plus_d2);
    D = fma(-q.y, x1[t], D);
    D = fma(-q.z, x2[t], D);
    double r = adj_rcp_n<NEWTON>(D);
    if (MASK) r = (k == row[t]) ? 0.0 : r;  // zero-padded sources give r * 0 anyway
    // (G_j x_j).v_i + (G_i x_i).v_j
    double c = q.w * v0[t];
    c = fma(w.x, v1[t], c);
    c = fma(w.y, v2[t], c);
    c = fma(g0[t], w.z, c);
    c = fma(g1[t], w.w, c);
    c = fma(g2[t], vz, c);
    const double cr2 = c * (r * r);
    a[t][0] = fma(r, q.w, a[t][0]);
    a[t][1] = fma(r, w.x, a[t][1]);
    a[t][2] = fma(r, w.y, a[t][2]);
    a[t][3] = fma(cr2, q.x, a[t][3]);
    a[t][4] = fma(cr2, q.y, a[t][4]);
    a[t][5] = fma(cr2, q.z, a[t][5]);
    a[t][6] = fma(r, w.z, a[t][6]);
    a[t][7] = fma(r, w.w, a[t][7]);
    a[t][8] = fma(r, vz, a[t][8]);
  }
}

template <int TPT, int NEWTON, int UNROLL>
__global__ void __launch_bounds__(kRNT) adj_row_kernel(const RowLaunch P) {
  __shared__ double4 sa[kRTS];  // {x_j, G_j x_j}
  __shared__ double4 sb[kRTS];  // {G_j y_j, G_j z_j, v_j,x, v_j,y}
  __shared__ double sc[kRTS];   // v_j,z
  int row[TPT];
  double x0[TPT], x1[TPT], x2[TPT], g0[TPT], g1[TPT], g2[TPT], v0[TPT], v1[TPT], v2[TPT];
  double a[TPT][kRowSums];
#pragma unroll
  for (int t = 0; t < TPT; ++t) {
    row[t] = (blockIdx.x * TPT + t) * kRNT + threadIdx.x;
    int ld = row[t] < P.n ? row[t] : P.n - 1;
    if (!TC_BC(P.bc, BC_ADJ_ROW_IN, ld, P.src_len)) ld = 0;
    const double4 q = P.ra[ld];
    const double4 w = P.rb[ld];
    x0[t] = q.x;
    x1[t] = q.y;
    x2[t] = q.z;
    g0[t] = q.w;
    g1[t] = w.x;
    g2[t] = w.y;
    v0[t] = w.z;
    v1[t] = w.w;
    v2[t] = P.rc[ld];
#pragma unroll
    for (int c = 0; c < kRowSums; ++c) a[t][c] = 0.0;
  }
  // rows of this CTA: [r_lo, r_hi)
  const int r_lo = blockIdx.x * TPT * kRNT, r_hi = r_lo + TPT * kRNT;
  const int c0 = blockIdx.y * P.chunk_len, c1 = min(P.n, c0 + P.chunk_len);
  for (int ts = c0; ts < c1; ts += kRTS) {
    __syncthreads();
    for (int j = threadIdx.x; j < kRTS; j += kRNT) {
      const int k = ts + j;
      const bool in = k < c1 && TC_BC(P.bc, BC_ADJ_ROW_IN, k, P.src_len);
      sa[j] = in ? P.ra[k] : make_double4(0.0, 0.0, 0.0, 0.0);
      sb[j] = in ? P.rb[k] : make_double4(0.0, 0.0, 0.0, 0.0);
      sc[j] = in ? P.rc[k] : 0.0;
    }
    __syncthreads();
    if (ts < r_hi && r_lo < ts + kRTS) {
      for (int j = 0; j < kRTS; ++j)
        adj_row_source<TPT, NEWTON, true>(sa[j], sb[j], sc[j], ts + j, row, P.one_plus_d2, x0, x1,
                                          x2, g0, g1, g2, v0, v1, v2, a);
    } else {
#pragma unroll UNROLL
      for (int j = 0; j < kRTS; ++j)
        adj_row_source<TPT, NEWTON, false>(sa[j], sb[j], sc[j], ts + j, row, P.one_plus_d2, x0,
                                           x1, x2, g0, g1, g2, v0, v1, v2, a);
    }
  }
  const size_t n = (size_t)P.n;
#pragma unroll
  for (int t = 0; t < TPT; ++t) {
    if (row[t] < P.n) {
      const size_t base = (size_t)blockIdx.y * kRowSums * n + row[t];
      double* out = P.partial + base;
#pragma unroll
      for (int c = 0; c < kRowSums; ++c)
        if (TC_BC(P.bc, BC_ADJ_ROW_OUT, base + c * n, P.partial_len)) out[c * n] = a[t][c];
    }
  }
}

// Row-pass combination: g_x = -(S1 x ut + C + G P)/(4 pi), g_zeta = -A (x . P)/(4 pi),
// from `chunks` partial blocks of kRowSums rows each, added in chunk order.
__global__ void adj_combine_row_kernel(const double* __restrict__ x, const double* __restrict__ ut,
                                       const double* __restrict__ zeta,
                                       const double* __restrict__ area, int n,
                                       const double* __restrict__ p, int chunks,
                                       double* __restrict__ out_x, double* __restrict__ out_z,
                                       BoundsRec* bc, long long p_len) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t N = (size_t)n, b = 3 * (size_t)i;
  double s[kRowSums];
#pragma unroll
  for (int w = 0; w < kRowSums; ++w) s[w] = 0.0;
  for (int c = 0; c < chunks; ++c)
#pragma unroll
    for (int w = 0; w < kRowSums; ++w) {
      const size_t j = ((size_t)c * kRowSums + w) * N + i;
      if (TC_BC(bc, BC_ADJ_COMBINE, j, p_len)) s[w] += p[j];
    }
  const double u0 = ut[b], u1 = ut[b + 1], u2 = ut[b + 2];
  const double G = zeta[i] * area[i];
  const double g0 = (s[1] * u2 - s[2] * u1) + s[3] + G * s[6];
  const double g1 = (s[2] * u0 - s[0] * u2) + s[4] + G * s[7];
  const double g2 = (s[0] * u1 - s[1] * u0) + s[5] + G * s[8];
  const double R = x[b] * s[6] + x[b + 1] * s[7] + x[b + 2] * s[8];
  out_x[b] = -kInv4Pi * g0;
  out_x[b + 1] = -kInv4Pi * g1;
  out_x[b + 2] = -kInv4Pi * g2;
  out_z[i] = -kInv4Pi * area[i] * R;
}

// v_i = ut_i x x_i with ut_i = mu_x,i + (-2 Omega mu_z,i) z_hat, mu = dt * l_k.
__global__ void adj_prepare_kernel(const double* __restrict__ x, const double* __restrict__ lkx,
                                   const double* __restrict__ lkz, const double* __restrict__ zeta,
                                   const double* __restrict__ area, int n, double dt, double m2omega,
                                   double* __restrict__ ut, double* __restrict__ v,
                                   double4* __restrict__ src1, double4* __restrict__ src2a,
                                   double2* __restrict__ src2b, double4* __restrict__ ra,
                                   double4* __restrict__ rb, double* __restrict__ rc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t b = 3 * (size_t)i;
  const double u0 = dt * lkx[b], u1 = dt * lkx[b + 1],
               u2 = dt * lkx[b + 2] + m2omega * (dt * lkz[i]);
  const double x0 = x[b], x1 = x[b + 1], x2 = x[b + 2];
  const double v0 = u1 * x2 - u2 * x1, v1 = u2 * x0 - u0 * x2, v2 = u0 * x1 - u1 * x0;
  ut[b] = u0;
  ut[b + 1] = u1;
  ut[b + 2] = u2;
  v[b] = v0;
  v[b + 1] = v1;
  v[b + 2] = v2;
  const double G = zeta[i] * area[i];
  src1[i] = make_double4(x0, x1, x2, G);
  src2a[i] = make_double4(x0, x1, x2, v0);
  src2b[i] = make_double2(v1, v2);
  ra[i] = make_double4(x0, x1, x2, G * x0);
  rb[i] = make_double4(G * x1, G * x2, v0, v1);
  rc[i] = v2;
}

// lY_i = J(Y)^T mu: gx (3 per row) and gz (1 per row), written to out_x/out_z.
// p1: chunks of `st1` rows each, the first 6 = (S1, S2); p2: chunks of `st2`
// rows each, the first 7 = (P, Q, R).
__global__ void adj_combine_kernel(const double* __restrict__ x, const double* __restrict__ ut,
                                   const double* __restrict__ zeta, const double* __restrict__ area,
                                   int n, const double* __restrict__ p1, int ch1, int st1,
                                   const double* __restrict__ p2, int ch2, int st2,
                                   double* __restrict__ out_x, double* __restrict__ out_z) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t N = (size_t)n, b = 3 * (size_t)i;
  double s[6] = {0, 0, 0, 0, 0, 0}, t[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int c = 0; c < ch1; ++c)
    for (int w = 0; w < 6; ++w) s[w] += p1[((size_t)c * st1 + w) * N + i];
  for (int c = 0; c < ch2; ++c)
    for (int w = 0; w < 7; ++w) t[w] += p2[((size_t)c * st2 + w) * N + i];
  const double u0 = ut[b], u1 = ut[b + 1], u2 = ut[b + 2];
  const double G = zeta[i] * area[i];
  // S1 x ut + S2 + G (P + Q)
  const double g0 = (s[1] * u2 - s[2] * u1) + s[3] + G * (t[0] + t[3]);
  const double g1 = (s[2] * u0 - s[0] * u2) + s[4] + G * (t[1] + t[4]);
  const double g2 = (s[0] * u1 - s[1] * u0) + s[5] + G * (t[2] + t[5]);
  out_x[b] = -kInv4Pi * g0;
  out_x[b + 1] = -kInv4Pi * g1;
  out_x[b + 2] = -kInv4Pi * g2;
  out_z[i] = -kInv4Pi * area[i] * t[6];
}

// Linear combinations of adjoint vectors: y = a*x + b*y (in place on y), n4 = 4*nA
// values laid out as [3*nA positions | nA vorticities] in one buffer.
__global__ void axpby_kernel(double a, const double* __restrict__ x, double b, double* __restrict__ y,
                             size_t n) {
  size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (j < n) y[j] = a * x[j] + b * y[j];
}

}  // namespace
}  // namespace tcb

using tcb::DevBuf;

namespace {

struct AdjWork {
  int nA = 0;
  size_t n4 = 0;
  DevBuf ck;        // checkpoints: ncheck x (3nA + nA)
  DevBuf ys;        // stage inputs of one segment: (steps*4) x (3nA + nA)
  DevBuf lam, lk, tmp;  // adjoint state, lk, accumulators (4nA each)
  DevBuf ut, v, s1, s2a, s2b, ra, rb, rc, p1, p2;
};

int adj_stage_vjp(tc_ctx* ctx, AdjWork& W, const double* y, const double* lk, double dt,
                  double* out) {
  // y and lk, out: [3nA | nA] buffers
  const int n = W.nA;
  const double* yx = y;
  const double* yz = y + 3 * (size_t)n;
  const double* area = ctx->rk.areaA.as<double>();
  const int threads = 256, blocks = (n + threads - 1) / threads;
  tcb::adj_prepare_kernel<<<blocks, threads, 0, ctx->stream>>>(
      yx, lk, lk + 3 * (size_t)n, yz, area, n, dt, -2.0 * ctx->omega, W.ut.as<double>(),
      W.v.as<double>(), W.s1.as<double4>(), W.s2a.as<double4>(), W.s2b.as<double2>(),
      W.ra.as<double4>(), W.rb.as<double4>(), W.rc.as<double>());
  TC_CUDA_TRY(cudaGetLastError());
  int rc;
  const double d = ctx->delta[TC_ACTIVE];
  // 3: row-major single pass (default); 0: two passes; 1, 2: fused with column reductions
  const int mode = ctx->adj_mode;
  const int ftb = mode == 1 ? 512 : 512;
  const int ftiles = (n + ftb - 1) / ftb;
  const size_t col_bytes = (size_t)ftiles * 7 * n * sizeof(double);
  int S, S2, st1 = 6, st2 = 7;
  const double* p2ptr = nullptr;
  if (mode >= 3) {
    // row pass: mode 3 one row per thread, 4 two rows per thread (both full FP64
    // reciprocals); 5 and 6 the same with one Newton step; 7 three rows per
    // thread, one Newton step
    const int tpt = mode == 7 ? 3 : (mode == 4 || mode == 6) ? 2 : 1;
    const int newton = mode <= 4 ? 2 : 1;
    const void* fn = tpt == 3   ? (const void*)tcb::adj_row_kernel<3, 1, 1>
                     : tpt == 1 ? (newton == 2 ? (const void*)tcb::adj_row_kernel<1, 2, 2>
                                               : (const void*)tcb::adj_row_kernel<1, 1, 2>)
                                : (newton == 2 ? (const void*)tcb::adj_row_kernel<2, 2, 1>
                                               : (const void*)tcb::adj_row_kernel<2, 1, 1>);
    const int rows_per_cta = tcb::kRNT * tpt;
    const int tiles = (n + rows_per_cta - 1) / rows_per_cta;
    int per_sm = 0;
    TC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, tcb::kRNT, 0));
    const int slots = std::max(1, per_sm) * ctx->num_sms;
    // whole waves: the chunk count that best fills tiles x chunks into the resident slots
    S = 1;
    double best = 0.0;
    for (int c = 1; c <= 32; ++c) {
      if (c > 1 && (n + c - 1) / c < 1024) break;
      const long long items = (long long)tiles * c, waves = (items + slots - 1) / slots;
      const double eff = (double)items / (double)(waves * slots);
      if (eff > best + 0.02) {
        best = eff;
        S = c;
      }
    }
    int chunk = (n + S - 1) / S;
    chunk = (chunk + tcb::kRTS - 1) / tcb::kRTS * tcb::kRTS;
    S = (n + chunk - 1) / chunk;
    if ((rc = W.p1.ensure((size_t)S * tcb::kRowSums * n * sizeof(double)))) return rc;
    const long long src_len = (long long)std::min(
        {W.ra.bytes / sizeof(double4), W.rb.bytes / sizeof(double4), W.rc.bytes / sizeof(double)});
    const long long p1_len = (long long)(W.p1.bytes / sizeof(double));
    tcb::RowLaunch R{W.ra.as<double4>(),
                     W.rb.as<double4>(),
                     W.rc.as<double>(),
                     n,
                     chunk,
                     1.0 + d * d,
                     W.p1.as<double>(),
                     ctx->bc_rec,
                     tcb::bc_extent(ctx, tcb::BC_ADJ_ROW_IN, src_len),
                     tcb::bc_extent(ctx, tcb::BC_ADJ_ROW_OUT, p1_len)};
    const dim3 grid(tiles, S);
    if (tpt == 3)
      tcb::adj_row_kernel<3, 1, 1><<<grid, tcb::kRNT, 0, ctx->stream>>>(R);
    else if (tpt == 1 && newton == 2)
      tcb::adj_row_kernel<1, 2, 2><<<grid, tcb::kRNT, 0, ctx->stream>>>(R);
    else if (tpt == 1)
      tcb::adj_row_kernel<1, 1, 2><<<grid, tcb::kRNT, 0, ctx->stream>>>(R);
    else if (newton == 2)
      tcb::adj_row_kernel<2, 2, 1><<<grid, tcb::kRNT, 0, ctx->stream>>>(R);
    else
      tcb::adj_row_kernel<2, 1, 1><<<grid, tcb::kRNT, 0, ctx->stream>>>(R);
    TC_CUDA_TRY(cudaGetLastError());
    tcb::adj_combine_row_kernel<<<blocks, threads, 0, ctx->stream>>>(
        yx, W.ut.as<double>(), yz, area, n, W.p1.as<double>(), S, out, out + 3 * (size_t)n,
        ctx->bc_rec, tcb::bc_extent(ctx, tcb::BC_ADJ_COMBINE, p1_len));
    TC_CUDA_TRY(cudaGetLastError());
    ctx->launches += 3;
    ctx->pair_launches += 1;
    ctx->pair_interactions += (long long)n * (long long)(n - 1);
    return TC_OK;
  } else if (mode != 0 && col_bytes <= (size_t(16) << 30)) {
    // fused pass: rows and columns from one visit of each pair
    const int slots = 2 * ctx->num_sms;
    S = std::max(1, std::min(16, (2 * slots + ftiles - 1) / ftiles));
    int chunk = (n + S - 1) / S;
    chunk = (chunk + 63) / 64 * 64;  // a multiple of both variants' shared-memory tile
    S = (n + chunk - 1) / chunk;
    S2 = ftiles;
    if ((rc = W.p1.ensure((size_t)S * 6 * n * sizeof(double))) || (rc = W.p2.ensure(col_bytes)))
      return rc;
    tcb::AdjFused F{yx, W.s1.as<double4>(), W.v.as<double>(), n, chunk, 1.0 + d * d,
                    W.p1.as<double>(), W.p2.as<double>()};
    if (mode == 1)
      tcb::adj_fused_kernel<256, 2, 5, 64><<<dim3(ftiles, S), 256, 0, ctx->stream>>>(F);
    else
      tcb::adj_fused_kernel<128, 4, 3, 32><<<dim3(ftiles, S), 128, 0, ctx->stream>>>(F);
    TC_CUDA_TRY(cudaGetLastError());
    ctx->launches += 1;
    ctx->pair_launches += 1;
    ctx->pair_interactions += (long long)n * (long long)(n - 1);
  } else {
    // two passes (target side, then the transposed source side)
    const int tiles = (n + tcb::kAdjNT - 1) / tcb::kAdjNT;
    const int slots = 8 * ctx->num_sms;
    S = std::max(1, std::min(32, (2 * slots + tiles - 1) / tiles));
    int chunk = (n + S - 1) / S;
    chunk = (chunk + tcb::kAdjTS - 1) / tcb::kAdjTS * tcb::kAdjTS;
    S = (n + chunk - 1) / chunk;
    S2 = S;
    if ((rc = W.p1.ensure((size_t)S * 6 * n * sizeof(double))) ||
        (rc = W.p2.ensure((size_t)S * 7 * n * sizeof(double))))
      return rc;
    tcb::AdjLaunch P1{yx, W.s1.as<double4>(), nullptr, W.v.as<double>(), n, chunk, 1.0 + d * d,
                      W.p1.as<double>()};
    tcb::adj_target_kernel<<<dim3(tiles, S), tcb::kAdjNT, 0, ctx->stream>>>(P1);
    TC_CUDA_TRY(cudaGetLastError());
    tcb::AdjLaunch P2{yx, W.s2a.as<double4>(), W.s2b.as<double2>(), nullptr, n, chunk,
                      1.0 + d * d, W.p2.as<double>()};
    tcb::adj_source_kernel<<<dim3(tiles, S), tcb::kAdjNT, 0, ctx->stream>>>(P2);
    TC_CUDA_TRY(cudaGetLastError());
    ctx->launches += 2;
    ctx->pair_launches += 2;
    ctx->pair_interactions += 2LL * n * (long long)(n - 1);
  }
  tcb::adj_combine_kernel<<<blocks, threads, 0, ctx->stream>>>(
      yx, W.ut.as<double>(), yz, area, n, W.p1.as<double>(), S, st1,
      p2ptr ? p2ptr : W.p2.as<double>(), S2, st2, out, out + 3 * (size_t)n);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 2;
  return TC_OK;
}

int axpby(tc_ctx* ctx, double a, const double* x, double b, double* y, size_t n) {
  tcb::axpby_kernel<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(a, x, b, y, n);
  TC_CUDA_TRY(cudaGetLastError());
  ctx->launches += 1;
  return TC_OK;
}

// Copy the RK4 state (x0A, z0) into a [3nA | nA] buffer, or back.
int state_copy(tc_ctx* ctx, double* buf, bool to_state) {
  tcb::Rk4State& R = ctx->rk;
  const size_t b3 = 3 * (size_t)R.nA * sizeof(double), b1 = (size_t)R.nA * sizeof(double);
  if (to_state) {
    TC_CUDA_TRY(cudaMemcpyAsync(R.x0A.ptr, buf, b3, cudaMemcpyDeviceToDevice, ctx->stream));
    TC_CUDA_TRY(cudaMemcpyAsync(R.z0.ptr, buf + 3 * (size_t)R.nA, b1, cudaMemcpyDeviceToDevice,
                                ctx->stream));
  } else {
    TC_CUDA_TRY(cudaMemcpyAsync(buf, R.x0A.ptr, b3, cudaMemcpyDeviceToDevice, ctx->stream));
    TC_CUDA_TRY(cudaMemcpyAsync(buf + 3 * (size_t)R.nA, R.z0.ptr, b1, cudaMemcpyDeviceToDevice,
                                ctx->stream));
  }
  return TC_OK;
}

int stage_input_copy(tc_ctx* ctx, double* buf) {
  tcb::Rk4State& R = ctx->rk;
  const size_t b3 = 3 * (size_t)R.nA * sizeof(double), b1 = (size_t)R.nA * sizeof(double);
  TC_CUDA_TRY(cudaMemcpyAsync(buf, R.xiA.ptr, b3, cudaMemcpyDeviceToDevice, ctx->stream));
  TC_CUDA_TRY(cudaMemcpyAsync(buf + 3 * (size_t)R.nA, R.ziA.ptr, b1, cudaMemcpyDeviceToDevice,
                              ctx->stream));
  return TC_OK;
}

// One forward step of the active panels; when ys != null the four stage
// inputs are stored there ([4][3nA | nA]).
int forward_step(tc_ctx* ctx, double dt, double* ys) {
  tcb::Rk4State& R = ctx->rk;
  const size_t n4 = 4 * (size_t)R.nA;
  int rc;
  if ((rc = tc_rk4_pack_sources(ctx))) return rc;
  if (ys && (rc = state_copy(ctx, ys, false))) return rc;
  for (int s = 0; s < 4; ++s) {
    if ((rc = tc_rk4_stage_range(ctx, s, dt, 0, R.nA, 0, 0, 0, 0, nullptr))) return rc;
    if (ys && s < 3 && (rc = stage_input_copy(ctx, ys + (size_t)(s + 1) * n4))) return rc;
  }
  return TC_OK;
}

__global__ void enstrophy_seed_kernel(const double* __restrict__ z, const double* __restrict__ area,
                                      int n, double* __restrict__ lam, double* __restrict__ jblk) {
  __shared__ double red[256];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double c = 0.0;
  if (i < n) {
    lam[i] = 2.0 * z[i] * area[i];
    c = z[i] * z[i] * area[i];
  }
  red[threadIdx.x] = c;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) jblk[blockIdx.x] = red[0];
}

}  // namespace

// Device time (ms) of the last adjoint call's phases: the forward sweep with
// checkpoints, the recomputation of checkpoint segments, and the backward
// sweep (vector-Jacobian products and combinations).
extern "C" int tc_adjoint_phase_ms(tc_ctx* ctx, double* ms3) {
  if (!ctx || !ms3) return TC_ERR_ARG;
  for (int k = 0; k < 3; ++k) ms3[k] = ctx->adj_ms[k];
  return TC_OK;
}

namespace {

constexpr int kCotangent = -1;  // adjoint_impl: seed with caller-given cotangents

// Gradient of J at time nsteps*dt with respect to the initial active-panel
// state. functional: TC_J_ENSTROPHY (J = sum zeta^2 A), TC_J_PROBE (J = zeta
// of panel `probe` at the end) or kCotangent (J = gT_x . x(T) + gT_zeta . zeta(T),
// a vector-Jacobian product of the whole trajectory). Inputs are host arrays;
// outputs: J (host scalar), g_zeta0 (nA), g_x0 (3*nA), host arrays.
int adjoint_impl(tc_ctx* ctx, const double* xA0, const double* zetaA0, const double* areaA,
                 int nA, double dt, int nsteps, int ckpt_every, int functional, int probe,
                 const double* gT_x, const double* gT_zeta, double* J, double* g_zeta0,
                 double* g_x0) {
  if (ctx->precision != TC_FP64) {
    tc_record_error("tc_rk4_adjoint: the adjoint runs in FP64 (tc_set_precision(ctx, TC_FP64))");
    return TC_ERR_STATE;
  }
  int rc = tc_rk4_load(ctx, xA0, zetaA0, areaA, nA, nullptr, 0, nullptr, 0, 0);
  if (rc) return rc;
  AdjWork W;
  W.nA = nA;
  W.n4 = 4 * (size_t)nA;
  const size_t B = W.n4 * sizeof(double);
  const int ncheck = (nsteps + ckpt_every - 1) / ckpt_every + 1;
  if ((rc = W.ck.ensure((size_t)ncheck * B)) || (rc = W.ys.ensure((size_t)ckpt_every * 4 * B)) ||
      (rc = W.lam.ensure(B)) || (rc = W.lk.ensure(B)) || (rc = W.tmp.ensure(B)) ||
      (rc = W.ut.ensure(3 * (size_t)nA * sizeof(double))) ||
      (rc = W.v.ensure(3 * (size_t)nA * sizeof(double))) ||
      (rc = W.s1.ensure((size_t)nA * sizeof(double4))) ||
      (rc = W.s2a.ensure((size_t)nA * sizeof(double4))) ||
      (rc = W.s2b.ensure((size_t)nA * sizeof(double2))) ||
      (rc = W.ra.ensure((size_t)nA * sizeof(double4))) ||
      (rc = W.rb.ensure((size_t)nA * sizeof(double4))) ||
      (rc = W.rc.ensure((size_t)nA * sizeof(double))))
    return rc;
  double* ck = W.ck.as<double>();
  double* ys = W.ys.as<double>();
  // phase timing: forward sweep, recomputation, backward (CUDA events on the stream)
  cudaEvent_t ev[4];
  for (auto& e : ev) TC_CUDA_TRY(cudaEventCreate(&e));
  struct EvGuard {
    cudaEvent_t* e;
    ~EvGuard() {
      for (int k = 0; k < 4; ++k) cudaEventDestroy(e[k]);
    }
  } ev_guard{ev};
  float recompute_ms = 0.f;
  TC_CUDA_TRY(cudaEventRecord(ev[0], ctx->stream));
  // forward sweep with checkpoints; the last segment's stage inputs are kept
  // as they are computed, so that segment needs no recomputation
  const int last_seg = nsteps > 0 ? (nsteps - 1) / ckpt_every : 0;
  for (int step = 0; step < nsteps; ++step) {
    if (step % ckpt_every == 0 && (rc = state_copy(ctx, ck + (size_t)(step / ckpt_every) * W.n4, false)))
      return rc;
    const int seg = step / ckpt_every;
    double* rec = seg == last_seg ? ys + (size_t)(step - seg * ckpt_every) * 4 * W.n4 : nullptr;
    if ((rc = forward_step(ctx, dt, rec))) return rc;
  }
  TC_CUDA_TRY(cudaEventRecord(ev[1], ctx->stream));
  // seed: l(T) = dJ/dX(T)
  double* lam = W.lam.as<double>();
  TC_CUDA_TRY(cudaMemsetAsync(lam, 0, B, ctx->stream));
  const double* zT = ctx->rk.z0.as<double>();
  if (functional == TC_J_ENSTROPHY) {
    const int blocks = (nA + 255) / 256;
    if ((rc = W.tmp.ensure(std::max(B, (size_t)blocks * sizeof(double))))) return rc;
    enstrophy_seed_kernel<<<blocks, 256, 0, ctx->stream>>>(zT, ctx->rk.areaA.as<double>(), nA,
                                                           lam + 3 * (size_t)nA, W.tmp.as<double>());
    TC_CUDA_TRY(cudaGetLastError());
    std::vector<double> jb(blocks);
    TC_CUDA_TRY(cudaMemcpyAsync(jb.data(), W.tmp.ptr, blocks * sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->stream));
    TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    double acc = 0.0;
    for (double v : jb) acc += v;
    *J = acc;
  } else if (functional == TC_J_PROBE) {
    TC_CUDA_TRY(cudaMemcpyAsync(J, zT + probe, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    const double one = 1.0;
    TC_CUDA_TRY(cudaMemcpyAsync(lam + 3 * (size_t)nA + probe, &one, sizeof(double),
                                cudaMemcpyHostToDevice, ctx->stream));
    TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  } else {
    // the caller's cotangents; J = their dot product with the final state (on the host)
    std::vector<double> xT(3 * (size_t)nA), zTh(nA);
    TC_CUDA_TRY(cudaMemcpyAsync(xT.data(), ctx->rk.x0A.ptr, 3 * (size_t)nA * sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->stream));
    TC_CUDA_TRY(cudaMemcpyAsync(zTh.data(), zT, (size_t)nA * sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->stream));
    if (gT_x)
      TC_CUDA_TRY(cudaMemcpyAsync(lam, gT_x, 3 * (size_t)nA * sizeof(double),
                                  cudaMemcpyHostToDevice, ctx->stream));
    if (gT_zeta)
      TC_CUDA_TRY(cudaMemcpyAsync(lam + 3 * (size_t)nA, gT_zeta, (size_t)nA * sizeof(double),
                                  cudaMemcpyHostToDevice, ctx->stream));
    TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    double acc = 0.0;
    if (gT_x)
      for (size_t k = 0; k < 3 * (size_t)nA; ++k) acc += gT_x[k] * xT[k];
    if (gT_zeta)
      for (int k = 0; k < nA; ++k) acc += gT_zeta[k] * zTh[k];
    *J = acc;
  }
  // backward sweep, one checkpoint segment at a time
  double* lk = W.lk.as<double>();
  double* acc = W.tmp.as<double>();
  double* ly = nullptr;
  DevBuf lyb;
  if ((rc = lyb.ensure(B))) return rc;
  ly = lyb.as<double>();
  for (int seg = (nsteps - 1) / ckpt_every; seg >= 0 && nsteps > 0; --seg) {
    const int s0 = seg * ckpt_every, s1 = std::min(nsteps, s0 + ckpt_every);
    if (seg != last_seg) {
      TC_CUDA_TRY(cudaEventRecord(ev[2], ctx->stream));
      if ((rc = state_copy(ctx, ck + (size_t)seg * W.n4, true))) return rc;
      for (int step = s0; step < s1; ++step)
        if ((rc = forward_step(ctx, dt, ys + (size_t)(step - s0) * 4 * W.n4))) return rc;
      TC_CUDA_TRY(cudaEventRecord(ev[3], ctx->stream));
      TC_CUDA_TRY(cudaEventSynchronize(ev[3]));
      float ms = 0.f;
      TC_CUDA_TRY(cudaEventElapsedTime(&ms, ev[2], ev[3]));
      recompute_ms += ms;
    }
    for (int step = s1 - 1; step >= s0; --step) {
      const double* Y = ys + (size_t)(step - s0) * 4 * W.n4;
      // acc = l' (the identity part); lk for stage 4 = l'/6
      TC_CUDA_TRY(cudaMemcpyAsync(acc, lam, B, cudaMemcpyDeviceToDevice, ctx->stream));
      const double bcoef[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
      const double ccoef[4] = {0.0, 0.5, 0.5, 1.0};  // Y_s = X + c_s k_{s-1}
      // lk_4 = l'/6
      if ((rc = axpby(ctx, bcoef[3], lam, 0.0, lk, W.n4))) return rc;
      for (int s = 3; s >= 0; --s) {
        if ((rc = adj_stage_vjp(ctx, W, Y + (size_t)s * W.n4, lk, dt, ly))) return rc;
        if ((rc = axpby(ctx, 1.0, ly, 1.0, acc, W.n4))) return rc;       // l += lY_s
        if (s > 0) {                                                     // lk_{s-1} = b l' + c_s lY_s
          if ((rc = axpby(ctx, bcoef[s - 1], lam, 0.0, lk, W.n4))) return rc;
          if ((rc = axpby(ctx, ccoef[s], ly, 1.0, lk, W.n4))) return rc;
        }
      }
      TC_CUDA_TRY(cudaMemcpyAsync(lam, acc, B, cudaMemcpyDeviceToDevice, ctx->stream));
    }
  }
  TC_CUDA_TRY(cudaEventRecord(ev[2], ctx->stream));
  TC_CUDA_TRY(cudaEventSynchronize(ev[2]));
  float fwd_ms = 0.f, total_ms = 0.f;
  TC_CUDA_TRY(cudaEventElapsedTime(&fwd_ms, ev[0], ev[1]));
  TC_CUDA_TRY(cudaEventElapsedTime(&total_ms, ev[0], ev[2]));
  ctx->adj_ms[0] = fwd_ms;
  ctx->adj_ms[1] = recompute_ms;
  ctx->adj_ms[2] = total_ms - fwd_ms - recompute_ms;
  TC_CUDA_TRY(cudaMemcpyAsync(g_x0, lam, 3 * (size_t)nA * sizeof(double), cudaMemcpyDeviceToHost,
                              ctx->stream));
  TC_CUDA_TRY(cudaMemcpyAsync(g_zeta0, lam + 3 * (size_t)nA, (size_t)nA * sizeof(double),
                              cudaMemcpyDeviceToHost, ctx->stream));
  TC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return TC_OK;
}

}  // namespace

extern "C" int tc_rk4_adjoint(tc_ctx* ctx, const double* xA0, const double* zetaA0,
                              const double* areaA, int nA, double dt, int nsteps, int ckpt_every,
                              int functional, int probe, double* J, double* g_zeta0, double* g_x0) {
  if (!ctx || nA <= 0 || nsteps < 0 || ckpt_every <= 0 || !xA0 || !zetaA0 || !areaA || !J ||
      !g_zeta0 || !g_x0 || (functional != TC_J_ENSTROPHY && functional != TC_J_PROBE) ||
      (functional == TC_J_PROBE && (probe < 0 || probe >= nA))) {
    tc_record_error("tc_rk4_adjoint: bad arguments");
    return TC_ERR_ARG;
  }
  TcNvtxRange nvtx_adjoint("tc rk4 adjoint");
  return adjoint_impl(ctx, xA0, zetaA0, areaA, nA, dt, nsteps, ckpt_every, functional, probe,
                      nullptr, nullptr, J, g_zeta0, g_x0);
}

extern "C" int tc_rk4_vjp(tc_ctx* ctx, const double* xA0, const double* zetaA0,
                          const double* areaA, int nA, double dt, int nsteps, int ckpt_every,
                          const double* gT_x, const double* gT_zeta, double* J, double* g_zeta0,
                          double* g_x0) {
  if (!ctx || nA <= 0 || nsteps < 0 || ckpt_every <= 0 || !xA0 || !zetaA0 || !areaA || !J ||
      !g_zeta0 || !g_x0 || (!gT_x && !gT_zeta)) {
    tc_record_error("tc_rk4_vjp: bad arguments");
    return TC_ERR_ARG;
  }
  return adjoint_impl(ctx, xA0, zetaA0, areaA, nA, dt, nsteps, ckpt_every, kCotangent, 0, gT_x,
                      gT_zeta, J, g_zeta0, g_x0);
}
