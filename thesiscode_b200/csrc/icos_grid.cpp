// Icosahedral triangle grid on the unit sphere: the input generator for the
// reference's panel test cases. Host code; it runs once per grid.
//
// Restates, with the same particle / edge / panel numbering:
//   InitIcosTriGrid   ParticlesEdgesPanels2.f90:419-645  (root icosahedron,
//                     level-by-level division of every leaf panel)
//   DivideTriPanel    ParticlesEdgesPanels2.f90:760-1090 (4 children, edge
//                     midpoints shared with an already divided neighbour,
//                     parent takes the centre child's position, area 0)
//   TriPanelArea      ParticlesEdgesPanels2.f90:1727-1802 (sum of spherical
//                     triangles (leaf-edge vertex, centre, next vertex))
//   SphereMidpoint / SphereTriCenter / SphereTriAreaVector / SphereDistance
//                     SphereGeom.f90:50-145
//   PanelMax / ParticleMax / EdgeMax ParticlesEdgesPanels2.f90:2614-2662
// The numbering has to match the reference because the RK4 driver gathers
// leaf panels in index order (GatherPanels, :1556-1619) and the MPI ranks
// split those index ranges (LoadBalance).
#include <cmath>
#include <cstring>
#include <vector>

#include "tc_internal.h"

namespace {

struct V3 {
  double x, y, z;
};

inline V3 sphere_midpoint(const V3& a, const V3& b) {
  V3 m{(a.x + b.x) / 2.0, (a.y + b.y) / 2.0, (a.z + b.z) / 2.0};
  double n = std::sqrt(m.x * m.x + m.y * m.y + m.z * m.z);
  return {m.x / n, m.y / n, m.z / n};
}

inline V3 sphere_tri_center(const V3& a, const V3& b, const V3& c) {
  V3 m{(a.x + b.x + c.x) / 3.0, (a.y + b.y + c.y) / 3.0, (a.z + b.z + c.z) / 3.0};
  double n = std::sqrt(m.x * m.x + m.y * m.y + m.z * m.z);
  return {m.x / n, m.y / n, m.z / n};
}

// Great-circle distance via atan2(|a x b|, a.b) (SphereGeom.f90:50-65).
inline double sphere_distance(const V3& a, const V3& b) {
  double c1 = a.y * b.z - b.y * a.z;
  double c2 = b.x * a.z - a.x * b.z;
  double c3 = a.x * b.y - b.x * a.y;
  double cn = std::sqrt(c1 * c1 + c2 * c2 + c3 * c3);
  double d = a.x * b.x + a.y * b.y + a.z * b.z;
  return std::atan2(cn, d);
}

// L'Huilier's theorem (SphereGeom.f90:126-145).
inline double sphere_tri_area(const V3& a, const V3& b, const V3& c) {
  double s1 = sphere_distance(a, b), s2 = sphere_distance(b, c), s3 = sphere_distance(c, a);
  double hp = (s1 + s2 + s3) / 2.0;
  double zz = std::tan(hp / 2.0) * std::tan((hp - s1) / 2.0) * std::tan((hp - s2) / 2.0) *
              std::tan((hp - s3) / 2.0);
  return 4.0 * std::atan2(std::sqrt(zz), 1.0);
}

struct Grid {
  // particles
  std::vector<V3> px, px0;
  int np = 0;
  // edges (0-based; -1 = none)
  std::vector<int> ev;        // 2 per edge: from, to
  std::vector<int> eleft, eright;
  std::vector<char> edivided;
  std::vector<int> echild;    // 2 per edge
  int ne = 0;
  // panels
  std::vector<V3> cx, cx0;
  std::vector<double> area;
  std::vector<int> pv;        // 3 vertices per panel
  std::vector<int> pe;        // 3 edges per panel
  std::vector<char> pdivided;
  std::vector<int> pchild;    // 4 per panel
  std::vector<int> nest;
  int npan = 0, nactive = 0;

  void reserve(int max_particles, int max_edges, int max_panels) {
    px.assign(max_particles, V3{0, 0, 0});
    px0.assign(max_particles, V3{0, 0, 0});
    ev.assign(2 * (size_t)max_edges, -1);
    eleft.assign(max_edges, -1);
    eright.assign(max_edges, -1);
    edivided.assign(max_edges, 0);
    echild.assign(2 * (size_t)max_edges, -1);
    cx.assign(max_panels, V3{0, 0, 0});
    cx0.assign(max_panels, V3{0, 0, 0});
    area.assign(max_panels, 0.0);
    pv.assign(3 * (size_t)max_panels, -1);
    pe.assign(3 * (size_t)max_panels, -1);
    pdivided.assign(max_panels, 0);
    pchild.assign(4 * (size_t)max_panels, -1);
    nest.assign(max_panels, 0);
  }

  // Leaf edges descending from edge e, first child first (FindLeafEdges,
  // ParticlesEdgesPanels2.f90:2663-2677).
  void leaf_edges(int e, std::vector<int>& out) const {
    if (!edivided[e]) {
      out.push_back(e);
      return;
    }
    leaf_edges(echild[2 * e], out);
    leaf_edges(echild[2 * e + 1], out);
  }

  double tri_panel_area(int p) const {
    const V3& c = cx[p];
    double a = 0.0;
    std::vector<int> leaves;
    for (int s = 0; s < 3; ++s) {
      leaves.clear();
      leaf_edges(pe[3 * p + s], leaves);
      // vertex chain: first vertex of every leaf, then the last leaf's second
      std::vector<int> chain;
      for (int e : leaves) chain.push_back(ev[2 * e]);
      chain.push_back(ev[2 * leaves.back() + 1]);
      for (size_t j = 0; j + 1 < chain.size(); ++j)
        a = a + sphere_tri_area(px[chain[j]], c, px[chain[j + 1]]);
    }
    return a;
  }

  // One parent edge of DivideTriPanel. slot = 0,1,2 for parent edges 1,2,3;
  // (va, vb) = the parent's vertices along that edge in the panel's order;
  // first/second = child panels that touch va and vb. Returns the midpoint.
  int divide_edge(int panel, int slot, int va, int vb, int first, int second) {
    int e = pe[3 * panel + slot];
    bool positive = (panel == eleft[e]);
    int mid;
    if (!edivided[e]) {
      mid = np;
      px[mid] = sphere_midpoint(px[va], px[vb]);
      px0[mid] = sphere_midpoint(px0[va], px0[vb]);
      int e1 = ne, e2 = ne + 1;
      edivided[e] = 1;
      echild[2 * e] = e1;
      echild[2 * e + 1] = e2;
      if (positive) {
        ev[2 * e1] = va; ev[2 * e1 + 1] = mid;
        ev[2 * e2] = mid; ev[2 * e2 + 1] = vb;
        eleft[e1] = first; eleft[e2] = second;
        eright[e1] = eright[e]; eright[e2] = eright[e];
        pe[3 * first + slot] = e1;
        pe[3 * second + slot] = e2;
      } else {
        ev[2 * e1] = vb; ev[2 * e1 + 1] = mid;
        ev[2 * e2] = mid; ev[2 * e2 + 1] = va;
        eleft[e1] = eleft[e]; eleft[e2] = eleft[e];
        eright[e1] = second; eright[e2] = first;
        pe[3 * first + slot] = e2;
        pe[3 * second + slot] = e1;
      }
      np += 1;
      ne += 2;
    } else {
      int c1 = echild[2 * e], c2 = echild[2 * e + 1];
      mid = ev[2 * c1 + 1];
      if (positive) {
        eleft[c1] = first; eleft[c2] = second;
        pe[3 * first + slot] = c1;
        pe[3 * second + slot] = c2;
      } else {
        eright[c1] = second; eright[c2] = first;
        pe[3 * first + slot] = c2;
        pe[3 * second + slot] = c1;
      }
    }
    return mid;
  }

  void divide_tri_panel(int p) {
    int v1 = pv[3 * p], v2 = pv[3 * p + 1], v3 = pv[3 * p + 2];
    int c1 = npan, c2 = npan + 1, c3 = npan + 2, c4 = npan + 3;
    int m12 = divide_edge(p, 0, v1, v2, c1, c2);
    int m23 = divide_edge(p, 1, v2, v3, c2, c3);
    int m31 = divide_edge(p, 2, v3, v1, c3, c1);
    int cv[4][3] = {{v1, m12, m31}, {m12, v2, m23}, {m31, m23, v3}, {m23, m31, m12}};
    for (int j = 0; j < 4; ++j)
      for (int s = 0; s < 3; ++s) pv[3 * (npan + j) + s] = cv[j][s];
    // interior edges: (m23,m31) between c4|c3, (m31,m12) c4|c1, (m12,m23) c4|c2
    int ia = ne, ib = ne + 1, ic = ne + 2;
    ev[2 * ia] = m23; ev[2 * ia + 1] = m31; eleft[ia] = c4; eright[ia] = c3;
    pe[3 * c4 + 0] = ia; pe[3 * c3 + 0] = ia;
    ev[2 * ib] = m31; ev[2 * ib + 1] = m12; eleft[ib] = c4; eright[ib] = c1;
    pe[3 * c4 + 1] = ib; pe[3 * c1 + 1] = ib;
    ev[2 * ic] = m12; ev[2 * ic + 1] = m23; eleft[ic] = c4; eright[ic] = c2;
    pe[3 * c4 + 2] = ic; pe[3 * c2 + 2] = ic;
    ne += 3;
    for (int j = 0; j < 4; ++j) {
      int q = npan + j;
      const int* w = &pv[3 * q];
      cx[q] = sphere_tri_center(px[w[0]], px[w[1]], px[w[2]]);
      cx0[q] = sphere_tri_center(px0[w[0]], px0[w[1]], px0[w[2]]);
      area[q] = tri_panel_area(q);
    }
    cx[p] = cx[c4];
    cx0[p] = cx0[c4];
    area[p] = 0.0;
    pdivided[p] = 1;
    for (int j = 0; j < 4; ++j) {
      nest[npan + j] = nest[p] + 1;
      pchild[4 * p + j] = npan + j;
    }
    npan += 4;
    nactive += 3;
  }

  void init_icosahedron() {
    static const double r[11][3] = {
        {0.0, 0.0, 1.0},
        {0.723606797749978969640917366873, 0.525731112119133606025669084848,
         0.447213595499957939281834733746},
        {-0.276393202250021030359082633126, 0.850650808352039932181540497063,
         0.447213595499957939281834733746},
        {-0.894427190999915878563669467492, 0.0, 0.447213595499957939281834733746},
        {-0.276393202250021030359082633127, -0.850650808352039932181540497063,
         0.447213595499957939281834733746},
        {0.723606797749978969640917366873, -0.525731112119133606025669084848,
         0.447213595499957939281834733746},
        {0.894427190999915878563669467492, 0.0, -0.447213595499957939281834733746},
        {0.276393202250021030359082633127, 0.850650808352039932181540497063,
         -0.447213595499957939281834733746},
        {-0.723606797749978969640917366873, 0.525731112119133606025669084848,
         -0.447213595499957939281834733746},
        {-0.723606797749978969640917366873, -0.525731112119133606025669084848,
         -0.447213595499957939281834733746},
        {0.276393202250021030359082633127, -0.850650808352039932181540497063,
         -0.447213595499957939281834733746}};
    np = 12;
    for (int j = 0; j < 11; ++j) {
      double n = std::sqrt(r[j][0] * r[j][0] + r[j][1] * r[j][1] + r[j][2] * r[j][2]);
      px[j] = V3{r[j][0] / n, r[j][1] / n, r[j][2] / n};
    }
    px[11] = V3{0.0, 0.0, -1.0};
    for (int j = 0; j < 12; ++j) px0[j] = px[j];
    // 30 edges (1-based in the reference, :485-544; stored 0-based here)
    static const int everts[30][2] = {
        {1, 2},  {2, 3},  {3, 1},   {3, 4},   {4, 1},   {4, 5},   {5, 1},   {5, 6},
        {6, 1},  {6, 2},  {2, 8},   {8, 3},   {8, 9},   {9, 3},   {9, 4},   {9, 10},
        {10, 4}, {10, 5}, {10, 11}, {11, 5},  {11, 6},  {11, 7},  {7, 6},   {7, 2},
        {7, 8},  {8, 12}, {12, 9},  {12, 10}, {12, 11}, {12, 7}};
    static const int eleft1[30] = {1,  1,  1,  2,  2,  3,  3,  4,  4,  5,  6,  6,  7,  7,  8,
                                   9,  9,  10, 11, 11, 12, 13, 13, 14, 15, 16, 16, 17, 18, 19};
    static const int eright1[30] = {5,  6,  2,  8,  3,  10, 4,  12, 5,  14, 15, 7,  16, 8,  9,
                                    17, 10, 11, 18, 12, 13, 19, 14, 15, 20, 20, 17, 18, 19, 20};
    ne = 30;
    for (int e = 0; e < 30; ++e) {
      ev[2 * e] = everts[e][0] - 1;
      ev[2 * e + 1] = everts[e][1] - 1;
      eleft[e] = eleft1[e] - 1;
      eright[e] = eright1[e] - 1;
    }
    // 20 panels (:605-644)
    static const int pedges[20][3] = {
        {1, 2, 3},    {3, 4, 5},    {5, 6, 7},    {7, 8, 9},    {9, 10, 1},
        {12, 2, 11},  {12, 13, 14}, {15, 4, 14},  {15, 16, 17}, {18, 6, 17},
        {18, 19, 20}, {21, 8, 20},  {21, 22, 23}, {24, 10, 23}, {24, 25, 11},
        {27, 13, 26}, {28, 16, 27}, {29, 19, 28}, {30, 22, 29}, {26, 25, 30}};
    static const int pverts[20][3] = {
        {1, 2, 3},   {1, 3, 4},   {1, 4, 5},   {1, 5, 6},   {1, 6, 2},
        {8, 3, 2},   {3, 8, 9},   {9, 4, 3},   {4, 9, 10},  {10, 5, 4},
        {5, 10, 11}, {11, 6, 5},  {6, 11, 7},  {7, 2, 6},   {2, 7, 8},
        {12, 9, 8},  {12, 10, 9}, {12, 11, 10}, {12, 7, 11}, {12, 8, 7}};
    npan = 20;
    nactive = 20;
    for (int p = 0; p < 20; ++p)
      for (int s = 0; s < 3; ++s) {
        pe[3 * p + s] = pedges[p][s] - 1;
        pv[3 * p + s] = pverts[p][s] - 1;
      }
    for (int p = 0; p < 20; ++p) {
      const int* w = &pv[3 * p];
      cx[p] = sphere_tri_center(px[w[0]], px[w[1]], px[w[2]]);
      area[p] = tri_panel_area(p);
    }
    for (int p = 0; p < 20; ++p) {
      cx0[p] = cx[p];
      nest[p] = 0;
    }
  }
};

}  // namespace

// The level-0 grid (root icosahedron: 12 particles, 30 edges, 20 panels) in
// the reference's numbering, for the device generator (icos_grid.cu), which
// divides it level by level on the GPU.
void tc_icos_root_tables(double px[36], double cx[60], double area[20], int pv[60], int pe[60],
                         int ev[60], int eleft[30], int eright[30]) {
  Grid g;
  g.reserve(12, 30, 20);
  g.init_icosahedron();
  for (int j = 0; j < 12; ++j) {
    px[3 * j] = g.px[j].x;
    px[3 * j + 1] = g.px[j].y;
    px[3 * j + 2] = g.px[j].z;
  }
  for (int p = 0; p < 20; ++p) {
    cx[3 * p] = g.cx[p].x;
    cx[3 * p + 1] = g.cx[p].y;
    cx[3 * p + 2] = g.cx[p].z;
    area[p] = g.area[p];
    for (int s = 0; s < 3; ++s) {
      pv[3 * p + s] = g.pv[3 * p + s];
      pe[3 * p + s] = g.pe[3 * p + s];
    }
  }
  for (int e = 0; e < 30; ++e) {
    ev[2 * e] = g.ev[2 * e];
    ev[2 * e + 1] = g.ev[2 * e + 1];
    eleft[e] = g.eleft[e];
    eright[e] = g.eright[e];
  }
}

extern "C" int tc_icos_grid_sizes(int level, int* n_particles, int* n_edges, int* n_panels,
                                  int* n_active) {
  if (level < 0 || level > 11) {
    tc_record_error("tc_icos_grid_sizes: level %d outside [0, 11]", level);
    return TC_ERR_ARG;
  }
  long long pan = 0, edg = 0;
  for (int j = 0; j <= level; ++j) {
    pan += 20LL << (2 * j);
    edg += 30LL << (2 * j);
  }
  if (n_particles) *n_particles = (int)(2 + (10LL << (2 * level)));
  if (n_edges) *n_edges = (int)edg;
  if (n_panels) *n_panels = (int)pan;
  if (n_active) *n_active = (int)(20LL << (2 * level));
  return TC_OK;
}

extern "C" int tc_icos_grid(int level, double* particles_x, double* particles_x0,
                            double* panels_x, double* panels_x0, double* panels_area,
                            int* panels_has_children, int* panels_vertices, int* panels_nest,
                            int* panels_children) {
  int nP, nE, nPan, nAct;
  int rc = tc_icos_grid_sizes(level, &nP, &nE, &nPan, &nAct);
  if (rc) return rc;
  if (!particles_x || !panels_x || !panels_area) {
    tc_record_error("tc_icos_grid: particles_x, panels_x and panels_area are required");
    return TC_ERR_ARG;
  }
  Grid g;
  g.reserve(nP, nE, nPan);
  g.init_icosahedron();
  int start = 0;
  for (int k = 1; k <= level; ++k) {
    int n_old = g.npan;
    for (int j = start; j < n_old; ++j)
      if (!g.pdivided[j]) g.divide_tri_panel(j);
    start = n_old - 1;  // the reference restarts at its 1-based nOldPanels
  }
  if (g.np != nP || g.npan != nPan || g.nactive != nAct) {
    tc_record_error("tc_icos_grid: internal size mismatch (%d,%d,%d)", g.np, g.npan, g.nactive);
    return TC_ERR_STATE;
  }
  for (int j = 0; j < nP; ++j) {
    particles_x[3 * (size_t)j] = g.px[j].x;
    particles_x[3 * (size_t)j + 1] = g.px[j].y;
    particles_x[3 * (size_t)j + 2] = g.px[j].z;
    if (particles_x0) {
      particles_x0[3 * (size_t)j] = g.px0[j].x;
      particles_x0[3 * (size_t)j + 1] = g.px0[j].y;
      particles_x0[3 * (size_t)j + 2] = g.px0[j].z;
    }
  }
  for (int p = 0; p < nPan; ++p) {
    panels_x[3 * (size_t)p] = g.cx[p].x;
    panels_x[3 * (size_t)p + 1] = g.cx[p].y;
    panels_x[3 * (size_t)p + 2] = g.cx[p].z;
    if (panels_x0) {
      panels_x0[3 * (size_t)p] = g.cx0[p].x;
      panels_x0[3 * (size_t)p + 1] = g.cx0[p].y;
      panels_x0[3 * (size_t)p + 2] = g.cx0[p].z;
    }
    panels_area[p] = g.area[p];
    if (panels_has_children) panels_has_children[p] = g.pdivided[p] ? 1 : 0;
    if (panels_vertices)
      for (int s = 0; s < 3; ++s) panels_vertices[3 * (size_t)p + s] = g.pv[3 * (size_t)p + s];
    if (panels_nest) panels_nest[p] = g.nest[p];
    if (panels_children)
      for (int s = 0; s < 4; ++s) panels_children[4 * (size_t)p + s] = g.pchild[4 * (size_t)p + s];
  }
  return TC_OK;
}

// GatherPanels index maps (ParticlesEdgesPanels2.f90:1556-1619): leaf panels
// in ascending index order go to active_map, divided panels to passive_map.
extern "C" int tc_gather_maps(int n, const int* has_children, int* active_map, int n_active,
                              int* passive_map, int n_passive) {
  if (n < 0 || !has_children || (n_active && !active_map) || (n_passive && !passive_map)) {
    tc_record_error("tc_gather_maps: bad arguments");
    return TC_ERR_ARG;
  }
  int a = 0, q = 0;
  for (int j = 0; j < n; ++j) {
    if (!has_children[j]) {
      if (a >= n_active) {
        tc_record_error("tc_gather_maps: more leaf panels than n_active=%d", n_active);
        return TC_ERR_ARG;
      }
      active_map[a++] = j;
    } else {
      if (q >= n_passive) {
        tc_record_error("tc_gather_maps: more divided panels than n_passive=%d", n_passive);
        return TC_ERR_ARG;
      }
      passive_map[q++] = j;
    }
  }
  if (a != n_active || q != n_passive) {
    tc_record_error("tc_gather_maps: counted %d active / %d passive, expected %d / %d", a, q,
                    n_active, n_passive);
    return TC_ERR_ARG;
  }
  return TC_OK;
}
