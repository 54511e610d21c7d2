// Icosahedral triangle grid generated on the GPU: the same particles, edges
// and panels, in the same numbering, as the host generator (icos_grid.cpp),
// which restates InitIcosTriGrid / DivideTriPanel / TriPanelArea
// (ParticlesEdgesPanels2.f90:419-645, :760-1090, :1727-1802).
//
// The reference divides the leaf panels of one level in ascending index
// order; a panel's three parent edges are split by whichever adjacent panel
// comes first, i.e. the one with the smaller index (in a uniform refinement
// both panels of a leaf edge are leaves of the same level). Every index the
// sequential loop hands out is therefore a closed form of one prefix sum:
// with f(p) = the number of edges panel p splits first and F(p) the
// exclusive sum of f over the level's leaves before p (i = p - L0),
//     new particle of the r-th edge p splits:  np0 + F(p) + r
//     its child edges:                         ne0 + 2F(p) + 3i + 2r, +1
//     p's interior edges:                      ne0 + 2F(p) + 2f(p) + 3i, +1, +2
//     p's children:                            npan0 + 4i + (0..3)
// Per level: a count kernel (f), a CUB exclusive scan (F), a divide kernel
// (indices, child vertices, edge tables; each panel writes only its own
// side of a shared edge, so no two threads write one location) and a
// geometry kernel (child centres and areas, the parent's centre). Positions
// and centres are computed with explicitly rounded FP64 operations in the
// host generator's operation order, so they equal its values bit for bit;
// areas go through CUDA's atan2/tan and agree to a few ulps.
#include <cub/device/device_scan.cuh>

#include "tc_ctx.h"

// icos_grid.cpp
void tc_icos_root_tables(double px[36], double cx[60], double area[20], int pv[60], int pe[60],
                         int ev[60], int eleft[30], int eright[30]);

namespace tcb {
namespace {

struct GridDev {
  double* px;
  double* px0;  // nullable
  double* cx;
  double* cx0;  // nullable
  double* area;
  int* ev;      // 2 per edge: from, to
  int* eleft;
  int* eright;
  int* echild;  // 2 per edge
  int* pv;      // 3 vertices per panel
  int* pe;      // 3 edges per panel
  int* pchild;  // 4 per panel
  int* nest;
  unsigned char* pdivided;
  unsigned char* edivided;
  int* f;       // per leaf of the level being divided
  int* F;
  int* flag;    // set when a level's particle count differs from the closed form
};

// SphereMidpoint / SphereTriCenter (SphereGeom.f90:91-111) in the host
// generator's operation order, each operation rounded on its own.
__device__ __forceinline__ double3 mid_d(const double* a, const double* b) {
  const double mx = __ddiv_rn(__dadd_rn(a[0], b[0]), 2.0);
  const double my = __ddiv_rn(__dadd_rn(a[1], b[1]), 2.0);
  const double mz = __ddiv_rn(__dadd_rn(a[2], b[2]), 2.0);
  const double n = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(mx, mx), __dmul_rn(my, my)), __dmul_rn(mz, mz)));
  return make_double3(__ddiv_rn(mx, n), __ddiv_rn(my, n), __ddiv_rn(mz, n));
}

__device__ __forceinline__ double3 center_d(const double* a, const double* b, const double* c) {
  const double mx = __ddiv_rn(__dadd_rn(__dadd_rn(a[0], b[0]), c[0]), 3.0);
  const double my = __ddiv_rn(__dadd_rn(__dadd_rn(a[1], b[1]), c[1]), 3.0);
  const double mz = __ddiv_rn(__dadd_rn(__dadd_rn(a[2], b[2]), c[2]), 3.0);
  const double n = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(mx, mx), __dmul_rn(my, my)), __dmul_rn(mz, mz)));
  return make_double3(__ddiv_rn(mx, n), __ddiv_rn(my, n), __ddiv_rn(mz, n));
}

// SphereDistance (SphereGeom.f90:50-65): atan2(|a x b|, a.b).
__device__ __forceinline__ double dist_d(const double* a, const double* b) {
  const double c1 = __dsub_rn(__dmul_rn(a[1], b[2]), __dmul_rn(b[1], a[2]));
  const double c2 = __dsub_rn(__dmul_rn(b[0], a[2]), __dmul_rn(a[0], b[2]));
  const double c3 = __dsub_rn(__dmul_rn(a[0], b[1]), __dmul_rn(b[0], a[1]));
  const double cn = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(c1, c1), __dmul_rn(c2, c2)), __dmul_rn(c3, c3)));
  const double d = __dadd_rn(__dadd_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1])), __dmul_rn(a[2], b[2]));
  return atan2(cn, d);
}

// SphereTriArea by L'Huilier's theorem (SphereGeom.f90:126-145).
__device__ __forceinline__ double tri_area_d(const double* a, const double* b, const double* c) {
  const double s1 = dist_d(a, b), s2 = dist_d(b, c), s3 = dist_d(c, a);
  const double hp = __ddiv_rn(__dadd_rn(__dadd_rn(s1, s2), s3), 2.0);
  const double zz = __dmul_rn(__dmul_rn(__dmul_rn(tan(__ddiv_rn(hp, 2.0)), tan(__ddiv_rn(__dsub_rn(hp, s1), 2.0))),
                                        tan(__ddiv_rn(__dsub_rn(hp, s2), 2.0))),
                              tan(__ddiv_rn(__dsub_rn(hp, s3), 2.0)));
  return __dmul_rn(4.0, atan2(__dsqrt_rn(zz), 1.0));
}

__device__ __forceinline__ bool splits_first(const GridDev& G, int p, int e) {
  return p == min(G.eleft[e], G.eright[e]);
}

__global__ void icos_count_kernel(GridDev G, int L0, int nleaf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nleaf) return;
  const int p = L0 + i;
  int c = 0;
#pragma unroll
  for (int s = 0; s < 3; ++s) c += splits_first(G, p, G.pe[3 * (size_t)p + s]) ? 1 : 0;
  G.f[i] = c;
}

// DivideTriPanel for every leaf p = L0 + i of the level.
__global__ void icos_divide_kernel(GridDev G, int L0, int nleaf, int np0, int ne0, int npan0,
                                   int np_expected) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nleaf) return;
  const int p = L0 + i;
  const int v[3] = {G.pv[3 * (size_t)p], G.pv[3 * (size_t)p + 1], G.pv[3 * (size_t)p + 2]};
  const int c[4] = {npan0 + 4 * i, npan0 + 4 * i + 1, npan0 + 4 * i + 2, npan0 + 4 * i + 3};
  const int Fp = G.F[i];
  if (i == nleaf - 1 && np0 + Fp + G.f[i] != np_expected) atomicExch(G.flag, 1);
  int mids[3];
  int r = 0;  // edges split so far by p
  for (int s = 0; s < 3; ++s) {
    const int e = G.pe[3 * (size_t)p + s];
    const int va = v[s], vb = v[(s + 1) % 3];
    const int first = c[s], second = c[(s + 1) % 3];
    const bool positive = (p == G.eleft[e]);
    const int q = min(G.eleft[e], G.eright[e]);
    int iq, Fq, rank;
    if (q == p) {
      iq = i;
      Fq = Fp;
      rank = r++;
    } else {
      iq = q - L0;
      Fq = G.F[iq];
      rank = 0;
      for (int s2 = 0; s2 < 3; ++s2) {
        const int e2 = G.pe[3 * (size_t)q + s2];
        if (e2 == e) break;
        if (splits_first(G, q, e2)) ++rank;
      }
    }
    const int mid = np0 + Fq + rank;
    const int e1 = ne0 + 2 * Fq + 3 * iq + 2 * rank, e2 = e1 + 1;
    if (q == p) {
      const double3 m = mid_d(G.px + 3 * (size_t)va, G.px + 3 * (size_t)vb);
      G.px[3 * (size_t)mid] = m.x;
      G.px[3 * (size_t)mid + 1] = m.y;
      G.px[3 * (size_t)mid + 2] = m.z;
      if (G.px0) {
        const double3 m0 = mid_d(G.px0 + 3 * (size_t)va, G.px0 + 3 * (size_t)vb);
        G.px0[3 * (size_t)mid] = m0.x;
        G.px0[3 * (size_t)mid + 1] = m0.y;
        G.px0[3 * (size_t)mid + 2] = m0.z;
      }
      G.edivided[e] = 1;
      G.echild[2 * (size_t)e] = e1;
      G.echild[2 * (size_t)e + 1] = e2;
      G.ev[2 * (size_t)e1] = positive ? va : vb;
      G.ev[2 * (size_t)e1 + 1] = mid;
      G.ev[2 * (size_t)e2] = mid;
      G.ev[2 * (size_t)e2 + 1] = positive ? vb : va;
    }
    // own side only: the other panel of e writes the other side
    if (positive) {
      G.eleft[e1] = first;
      G.eleft[e2] = second;
      G.pe[3 * (size_t)first + s] = e1;
      G.pe[3 * (size_t)second + s] = e2;
    } else {
      G.eright[e1] = second;
      G.eright[e2] = first;
      G.pe[3 * (size_t)first + s] = e2;
      G.pe[3 * (size_t)second + s] = e1;
    }
    mids[s] = mid;
  }
  const int m12 = mids[0], m23 = mids[1], m31 = mids[2];
  const int cv[4][3] = {{v[0], m12, m31}, {m12, v[1], m23}, {m31, m23, v[2]}, {m23, m31, m12}};
#pragma unroll
  for (int j = 0; j < 4; ++j) {
#pragma unroll
    for (int s = 0; s < 3; ++s) G.pv[3 * (size_t)c[j] + s] = cv[j][s];
    G.nest[c[j]] = G.nest[p] + 1;
    G.pdivided[c[j]] = 0;
    G.pchild[4 * (size_t)p + j] = c[j];
#pragma unroll
    for (int s = 0; s < 4; ++s) G.pchild[4 * (size_t)c[j] + s] = -1;
  }
  // interior edges: (m23,m31) between c4|c3, (m31,m12) c4|c1, (m12,m23) c4|c2
  const int ia = ne0 + 2 * Fp + 2 * r + 3 * i, ib = ia + 1, ic = ia + 2;
  const int iv[3][2] = {{m23, m31}, {m31, m12}, {m12, m23}};
  const int ir[3] = {c[2], c[0], c[1]};
  const int ie[3] = {ia, ib, ic};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    G.ev[2 * (size_t)ie[k]] = iv[k][0];
    G.ev[2 * (size_t)ie[k] + 1] = iv[k][1];
    G.eleft[ie[k]] = c[3];
    G.eright[ie[k]] = ir[k];
    G.edivided[ie[k]] = 0;
    G.pe[3 * (size_t)c[3] + k] = ie[k];
    G.pe[3 * (size_t)ir[k] + k] = ie[k];
  }
  G.pdivided[p] = 1;
}

// Child centres (SphereTriCenter of its vertices) and areas (TriPanelArea:
// each child's edges are still leaves, so the sum runs over the three
// triangles (edge start, centre, edge end)); the parent takes the centre
// child's position and area 0.
__global__ void icos_geometry_kernel(GridDev G, int L0, int nleaf, int npan0) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 4 * nleaf) return;
  const int q = npan0 + t;
  const int w0 = G.pv[3 * (size_t)q], w1 = G.pv[3 * (size_t)q + 1], w2 = G.pv[3 * (size_t)q + 2];
  const double3 cc = center_d(G.px + 3 * (size_t)w0, G.px + 3 * (size_t)w1, G.px + 3 * (size_t)w2);
  const double cq[3] = {cc.x, cc.y, cc.z};
  double a = 0.0;
  for (int s = 0; s < 3; ++s) {
    const int e = G.pe[3 * (size_t)q + s];
    a = __dadd_rn(a, tri_area_d(G.px + 3 * (size_t)G.ev[2 * (size_t)e], cq,
                                G.px + 3 * (size_t)G.ev[2 * (size_t)e + 1]));
  }
  G.cx[3 * (size_t)q] = cc.x;
  G.cx[3 * (size_t)q + 1] = cc.y;
  G.cx[3 * (size_t)q + 2] = cc.z;
  G.area[q] = a;
  double3 c0 = cc;
  if (G.cx0) {
    c0 = center_d(G.px0 + 3 * (size_t)w0, G.px0 + 3 * (size_t)w1, G.px0 + 3 * (size_t)w2);
    G.cx0[3 * (size_t)q] = c0.x;
    G.cx0[3 * (size_t)q + 1] = c0.y;
    G.cx0[3 * (size_t)q + 2] = c0.z;
  }
  if ((t & 3) == 3) {
    const int p = L0 + (t >> 2);
    G.cx[3 * (size_t)p] = cc.x;
    G.cx[3 * (size_t)p + 1] = cc.y;
    G.cx[3 * (size_t)p + 2] = cc.z;
    if (G.cx0) {
      G.cx0[3 * (size_t)p] = c0.x;
      G.cx0[3 * (size_t)p + 1] = c0.y;
      G.cx0[3 * (size_t)p + 2] = c0.z;
    }
    G.area[p] = 0.0;
  }
}

__global__ void u8_to_int_kernel(const unsigned char* in, int n, int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i];
}

}  // namespace
}  // namespace tcb

// Device-memory outputs on the context's device, written on its stream; the
// call returns when the grid is complete. Array sizes as for tc_icos_grid.
extern "C" int tc_icos_grid_device(tc_ctx* ctx, int level, double* particles_x,
                                   double* particles_x0, double* panels_x, double* panels_x0,
                                   double* panels_area, int* panels_has_children,
                                   int* panels_vertices, int* panels_nest, int* panels_children) {
  if (!ctx) return TC_ERR_ARG;
  int nP, nE, nPan, nAct;
  int rc = tc_icos_grid_sizes(level, &nP, &nE, &nPan, &nAct);
  if (rc) return rc;
  if (!particles_x || !panels_x || !panels_area) {
    tc_record_error("tc_icos_grid_device: particles_x, panels_x and panels_area are required");
    return TC_ERR_ARG;
  }
  TC_CUDA_TRY(cudaSetDevice(ctx->device));
  using tcb::DevBuf;
  DevBuf* B = ctx->grid_buf;
  // 0: ev+echild (4 per edge), 1: eleft+eright (2 per edge), 2: pv+pe+pchild+nest (11 per panel),
  // 3: pdivided+edivided, 4: f+F+flag, 5: CUB scratch
  const size_t nleaf_max = (size_t)nAct / 4 + 1;
  if ((rc = B[0].ensure(4 * (size_t)nE * sizeof(int))) || (rc = B[1].ensure(2 * (size_t)nE * sizeof(int))) ||
      (rc = B[2].ensure(11 * (size_t)nPan * sizeof(int))) || (rc = B[3].ensure((size_t)nPan + nE)) ||
      (rc = B[4].ensure((2 * nleaf_max + 1) * sizeof(int))))
    return rc;
  tcb::GridDev G{};
  G.px = particles_x;
  G.px0 = particles_x0;
  G.cx = panels_x;
  G.cx0 = panels_x0;
  G.area = panels_area;
  G.ev = B[0].as<int>();
  G.echild = G.ev + 2 * (size_t)nE;
  G.eleft = B[1].as<int>();
  G.eright = G.eleft + nE;
  G.pv = B[2].as<int>();
  G.pe = G.pv + 3 * (size_t)nPan;
  G.pchild = G.pe + 3 * (size_t)nPan;
  G.nest = G.pchild + 4 * (size_t)nPan;
  G.pdivided = B[3].as<unsigned char>();
  G.edivided = G.pdivided + nPan;
  G.f = B[4].as<int>();
  G.F = G.f + nleaf_max;
  G.flag = G.F + nleaf_max;
  cudaStream_t st = ctx->stream;

  // level 0 from the host tables
  double px[36], cx[60], area[20];
  int pv[60], pe[60], ev[60], el[30], er[30];
  tc_icos_root_tables(px, cx, area, pv, pe, ev, el, er);
  int pch[80], nest[20];
  for (int j = 0; j < 80; ++j) pch[j] = -1;
  for (int j = 0; j < 20; ++j) nest[j] = 0;
  TC_CUDA_TRY(cudaMemsetAsync(G.pdivided, 0, (size_t)nPan + nE, st));
  TC_CUDA_TRY(cudaMemsetAsync(G.flag, 0, sizeof(int), st));
  TC_CUDA_TRY(cudaMemcpyAsync(G.px, px, sizeof px, cudaMemcpyHostToDevice, st));
  if (G.px0) TC_CUDA_TRY(cudaMemcpyAsync(G.px0, px, sizeof px, cudaMemcpyHostToDevice, st));
  TC_CUDA_TRY(cudaMemcpyAsync(G.cx, cx, sizeof cx, cudaMemcpyHostToDevice, st));
  if (G.cx0) TC_CUDA_TRY(cudaMemcpyAsync(G.cx0, cx, sizeof cx, cudaMemcpyHostToDevice, st));
  TC_CUDA_TRY(cudaMemcpyAsync(G.area, area, sizeof area, cudaMemcpyHostToDevice, st));
  TC_CUDA_TRY(cudaMemcpyAsync(G.pv, pv, sizeof pv, cudaMemcpyHostToDevice, st));
  TC_CUDA_TRY(cudaMemcpyAsync(G.pe, pe, sizeof pe, cudaMemcpyHostToDevice, st));
  TC_CUDA_TRY(cudaMemcpyAsync(G.pchild, pch, sizeof pch, cudaMemcpyHostToDevice, st));
  TC_CUDA_TRY(cudaMemcpyAsync(G.nest, nest, sizeof nest, cudaMemcpyHostToDevice, st));
  TC_CUDA_TRY(cudaMemcpyAsync(G.ev, ev, sizeof ev, cudaMemcpyHostToDevice, st));
  TC_CUDA_TRY(cudaMemcpyAsync(G.eleft, el, sizeof el, cudaMemcpyHostToDevice, st));
  TC_CUDA_TRY(cudaMemcpyAsync(G.eright, er, sizeof er, cudaMemcpyHostToDevice, st));

  int np = 12, ne = 30, npan = 20, L0 = 0;
  for (int k = 1; k <= level; ++k) {
    const int nleaf = npan - L0;  // the leaves: every panel created by the previous level
    const int threads = 256, blocks = (nleaf + threads - 1) / threads;
    tcb::icos_count_kernel<<<blocks, threads, 0, st>>>(G, L0, nleaf);
    TC_CUDA_TRY(cudaGetLastError());
    size_t temp = 0;
    TC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, temp, G.f, G.F, nleaf, st));
    if ((rc = B[5].ensure(temp))) return rc;
    TC_CUDA_TRY(cub::DeviceScan::ExclusiveSum(B[5].ptr, temp, G.f, G.F, nleaf, st));
    // a uniform level-(k-1) grid has 30*4^(k-1) leaf edges: one new particle each
    const int np_next = np + (30 << (2 * (k - 1)));
    tcb::icos_divide_kernel<<<blocks, threads, 0, st>>>(G, L0, nleaf, np, ne, npan, np_next);
    TC_CUDA_TRY(cudaGetLastError());
    const int gblocks = (4 * nleaf + threads - 1) / threads;
    tcb::icos_geometry_kernel<<<gblocks, threads, 0, st>>>(G, L0, nleaf, npan);
    TC_CUDA_TRY(cudaGetLastError());
    ctx->launches += 4;
    np = np_next;
    ne += 2 * (30 << (2 * (k - 1))) + 3 * nleaf;
    L0 = npan;
    npan += 4 * nleaf;
  }
  if (np != nP || ne != nE || npan != nPan) {
    tc_record_error("tc_icos_grid_device: internal size mismatch (%d,%d,%d)", np, ne, npan);
    return TC_ERR_STATE;
  }
  if (panels_vertices)
    TC_CUDA_TRY(cudaMemcpyAsync(panels_vertices, G.pv, 3 * (size_t)nPan * sizeof(int),
                                cudaMemcpyDeviceToDevice, st));
  if (panels_nest)
    TC_CUDA_TRY(cudaMemcpyAsync(panels_nest, G.nest, (size_t)nPan * sizeof(int), cudaMemcpyDeviceToDevice, st));
  if (panels_children)
    TC_CUDA_TRY(cudaMemcpyAsync(panels_children, G.pchild, 4 * (size_t)nPan * sizeof(int),
                                cudaMemcpyDeviceToDevice, st));
  if (panels_has_children) {
    tcb::u8_to_int_kernel<<<(nPan + 255) / 256, 256, 0, st>>>(G.pdivided, nPan, panels_has_children);
    TC_CUDA_TRY(cudaGetLastError());
  }
  int flag = 0;
  TC_CUDA_TRY(cudaMemcpyAsync(&flag, G.flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  TC_CUDA_TRY(cudaStreamSynchronize(st));
  if (flag) {
    tc_record_error("tc_icos_grid_device: a level's particle count differs from 30*4^(level-1)");
    return TC_ERR_STATE;
  }
  return TC_OK;
}
