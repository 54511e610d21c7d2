/* CPU restatement of the reference's icosahedral triangle grid generator.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle): it builds the inputs of the CPU
 * baseline and of the benchmark's reference arm without the product library,
 * and the tests compare the product's host and device generators with it bit
 * for bit.
 *
 * Follows, statement for statement and with the reference's 1-based arrays:
 *   InitIcosTriGrid    ParticlesEdgesPanels2.f90:419-645
 *   DivideTriPanel     ParticlesEdgesPanels2.f90:760-1090
 *   TriPanelArea       ParticlesEdgesPanels2.f90:1727-1802
 *   FindLeafEdges      ParticlesEdgesPanels2.f90:2665-2677
 *   PanelMax / ParticleMax / EdgeMax  ParticlesEdgesPanels2.f90:2614-2662
 *   GatherPanels maps  ParticlesEdgesPanels2.f90:1556-1619
 *   SphereDistanceVector, SphereMidpoint, SphereTriCenter,
 *   SphereTriAreaVector SphereGeom.f90:50-65, 91-111, 126-145
 * Fortran's sum(v*v) is evaluated left to right, as gfortran and ifort do
 * without reassociation; built with -ffp-contract=off.
 *
 * The particles' 6-slot edge lists (aParticles%edges) and dual areas are not
 * kept: nothing on the velocity path reads them.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "bve_oracle.h"

/* ---- SphereGeom.f90 ---------------------------------------------------- */

static double sphere_distance(const double *a, const double *b) {
  double c1 = a[1] * b[2] - b[1] * a[2];
  double c2 = b[0] * a[2] - a[0] * b[2];
  double c3 = a[0] * b[1] - b[0] * a[1];
  double cross_norm = sqrt(c1 * c1 + c2 * c2 + c3 * c3);
  double dot = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
  return atan2(cross_norm, dot);
}

static void sphere_midpoint(const double *a, const double *b, double *out) {
  double m[3];
  for (int c = 0; c < 3; ++c) m[c] = (a[c] + b[c]) / 2.0;
  double nrm = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  for (int c = 0; c < 3; ++c) out[c] = m[c] / nrm;
}

static void sphere_tri_center(const double *a, const double *b, const double *c3, double *out) {
  double m[3];
  for (int c = 0; c < 3; ++c) m[c] = (a[c] + b[c] + c3[c]) / 3.0;
  double nrm = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  for (int c = 0; c < 3; ++c) out[c] = m[c] / nrm;
}

static double sphere_tri_area(const double *a, const double *b, const double *c) {
  double s1 = sphere_distance(a, b);
  double s2 = sphere_distance(b, c);
  double s3 = sphere_distance(c, a);
  double hp = (s1 + s2 + s3) / 2.0;
  double zz = tan(hp / 2.0) * tan((hp - s1) / 2.0) * tan((hp - s2) / 2.0) * tan((hp - s3) / 2.0);
  return 4.0 * atan2(sqrt(zz), 1.0);
}

/* ---- grid state, 1-based like the Fortran derived types ----------------- */

typedef struct {
  /* particles */
  int np;
  double *px, *px0; /* x(3, N_Max): px[3*(j-1) + c] */
  /* edges */
  int ne;
  int *everts;      /* verts(2, N): everts[2*(e-1) + s] */
  int *eleft, *eright, *ehas, *echild; /* children(2, N) */
  /* panels */
  int npan, nactive;
  double *cx, *cx0, *area;
  int *pverts, *pedges, *phas, *pchild, *pnest; /* vertices(3,N), edges(3,N), children(4,N) */
} IcosGrid;

#define PX(g, j) (&(g)->px[3 * ((size_t)(j) - 1)])
#define PX0(g, j) (&(g)->px0[3 * ((size_t)(j) - 1)])
#define EV(g, s, e) ((g)->everts[2 * ((size_t)(e) - 1) + (s) - 1])
#define ECH(g, s, e) ((g)->echild[2 * ((size_t)(e) - 1) + (s) - 1])
#define ELEFT(g, e) ((g)->eleft[(size_t)(e) - 1])
#define ERIGHT(g, e) ((g)->eright[(size_t)(e) - 1])
#define EHAS(g, e) ((g)->ehas[(size_t)(e) - 1])
#define PV(g, s, p) ((g)->pverts[3 * ((size_t)(p) - 1) + (s) - 1])
#define PE(g, s, p) ((g)->pedges[3 * ((size_t)(p) - 1) + (s) - 1])
#define PCH(g, s, p) ((g)->pchild[4 * ((size_t)(p) - 1) + (s) - 1])
#define CX(g, p) (&(g)->cx[3 * ((size_t)(p) - 1)])
#define CX0(g, p) (&(g)->cx0[3 * ((size_t)(p) - 1)])

/* FindLeafEdges (:2665-2677): leaf edges below `e`, first child first. */
static void find_leaf_edges(const IcosGrid *g, int e, int *list, int *count) {
  if (!EHAS(g, e)) {
    list[(*count)++] = e;
  } else {
    find_leaf_edges(g, ECH(g, 1, e), list, count);
    find_leaf_edges(g, ECH(g, 2, e), list, count);
  }
}

/* TriPanelArea (:1727-1802): the spherical triangles (leaf-edge vertex j,
 * panel centre, leaf-edge vertex j+1) along the three parent edges. */
static double tri_panel_area(const IcosGrid *g, int p, int *scratch, int scratch_len) {
  const double *center = CX(g, p);
  double a = 0.0;
  for (int s = 1; s <= 3; ++s) {
    int n = 0;
    find_leaf_edges(g, PE(g, s, p), scratch, &n);
    (void)scratch_len;
    /* vertList(j) = verts(1) of leaf j; vertList(n+1) = verts(2) of the last leaf */
    for (int j = 0; j < n; ++j) {
      int va = EV(g, 1, scratch[j]);
      int vb = (j + 1 < n) ? EV(g, 1, scratch[j + 1]) : EV(g, 2, scratch[n - 1]);
      a = a + sphere_tri_area(PX(g, va), center, PX(g, vb));
    }
  }
  return a;
}

/* One parent edge of DivideTriPanel (:790-1004). k = 1, 2, 3 is the parent
 * edge; (va, vb) its end vertices in the panel's order; (ca, cb) the child
 * panels that touch va and vb; mslots lists the three (vertex slot, child)
 * pairs that receive the midpoint. */
static void divide_parent_edge(IcosGrid *g, int panel, int k, int va, int vb, int ca, int cb,
                               const int mslots[3][2], int *n_particles, int *n_edges) {
  int edge = PE(g, k, panel);
  int mid;
  if (!EHAS(g, edge)) {
    mid = *n_particles + 1;
    sphere_midpoint(PX(g, va), PX(g, vb), PX(g, mid));
    sphere_midpoint(PX0(g, va), PX0(g, vb), PX0(g, mid));
    EHAS(g, edge) = 1;
    ECH(g, 1, edge) = *n_edges + 1;
    ECH(g, 2, edge) = *n_edges + 2;
    if (panel == ELEFT(g, edge)) { /* positive orientation */
      EV(g, 1, *n_edges + 1) = va;
      EV(g, 2, *n_edges + 1) = mid;
      EV(g, 1, *n_edges + 2) = mid;
      EV(g, 2, *n_edges + 2) = vb;
      ELEFT(g, *n_edges + 1) = ca;
      ELEFT(g, *n_edges + 2) = cb;
      ERIGHT(g, *n_edges + 1) = ERIGHT(g, edge);
      ERIGHT(g, *n_edges + 2) = ERIGHT(g, edge);
      PE(g, k, ca) = *n_edges + 1;
      PE(g, k, cb) = *n_edges + 2;
    } else { /* negative orientation */
      EV(g, 1, *n_edges + 1) = vb;
      EV(g, 2, *n_edges + 1) = mid;
      EV(g, 1, *n_edges + 2) = mid;
      EV(g, 2, *n_edges + 2) = va;
      ELEFT(g, *n_edges + 1) = ELEFT(g, edge);
      ELEFT(g, *n_edges + 2) = ELEFT(g, edge);
      ERIGHT(g, *n_edges + 1) = cb;
      ERIGHT(g, *n_edges + 2) = ca;
      PE(g, k, ca) = *n_edges + 2;
      PE(g, k, cb) = *n_edges + 1;
    }
    *n_particles += 1;
    *n_edges += 2;
  } else {
    int child1 = ECH(g, 1, edge), child2 = ECH(g, 2, edge);
    mid = EV(g, 2, child1);
    if (panel == ELEFT(g, edge)) {
      ELEFT(g, child1) = ca;
      ELEFT(g, child2) = cb;
      PE(g, k, ca) = child1;
      PE(g, k, cb) = child2;
    } else {
      ERIGHT(g, child1) = cb;
      ERIGHT(g, child2) = ca;
      PE(g, k, ca) = child2;
      PE(g, k, cb) = child1;
    }
  }
  for (int s = 0; s < 3; ++s) PV(g, mslots[s][0], mslots[s][1]) = mid;
}

/* DivideTriPanel (:760-1090). */
static void divide_tri_panel(IcosGrid *g, int panel, int *scratch, int scratch_len) {
  int v1 = PV(g, 1, panel), v2 = PV(g, 2, panel), v3 = PV(g, 3, panel);
  int nest = g->pnest[panel - 1];
  int n_particles = g->np, n_edges = g->ne, n_panels = g->npan;
  PV(g, 1, n_panels + 1) = v1;
  PV(g, 2, n_panels + 2) = v2;
  PV(g, 3, n_panels + 3) = v3;
  /* parent edge 1: midpoint -> vertices(2,+1), (1,+2), (3,+4) */
  const int m1[3][2] = {{2, n_panels + 1}, {1, n_panels + 2}, {3, n_panels + 4}};
  divide_parent_edge(g, panel, 1, v1, v2, n_panels + 1, n_panels + 2, m1, &n_particles, &n_edges);
  /* parent edge 2: midpoint -> vertices(3,+2), (2,+3), (1,+4) */
  const int m2[3][2] = {{3, n_panels + 2}, {2, n_panels + 3}, {1, n_panels + 4}};
  divide_parent_edge(g, panel, 2, v2, v3, n_panels + 2, n_panels + 3, m2, &n_particles, &n_edges);
  /* parent edge 3: midpoint -> vertices(1,+3), (2,+4), (3,+1) */
  const int m3[3][2] = {{1, n_panels + 3}, {2, n_panels + 4}, {3, n_panels + 1}};
  divide_parent_edge(g, panel, 3, v3, v1, n_panels + 3, n_panels + 1, m3, &n_particles, &n_edges);
  /* interior edges (:1007-1057) */
  int c4 = n_panels + 4;
  EV(g, 1, n_edges + 1) = PV(g, 1, c4);
  EV(g, 2, n_edges + 1) = PV(g, 2, c4);
  ELEFT(g, n_edges + 1) = c4;
  ERIGHT(g, n_edges + 1) = n_panels + 3;
  PE(g, 1, c4) = n_edges + 1;
  PE(g, 1, n_panels + 3) = n_edges + 1;
  EV(g, 1, n_edges + 2) = PV(g, 2, c4);
  EV(g, 2, n_edges + 2) = PV(g, 3, c4);
  ELEFT(g, n_edges + 2) = c4;
  ERIGHT(g, n_edges + 2) = n_panels + 1;
  PE(g, 2, c4) = n_edges + 2;
  PE(g, 2, n_panels + 1) = n_edges + 2;
  EV(g, 1, n_edges + 3) = PV(g, 3, c4);
  EV(g, 2, n_edges + 3) = PV(g, 1, c4);
  ELEFT(g, n_edges + 3) = c4;
  ERIGHT(g, n_edges + 3) = n_panels + 2;
  PE(g, 3, c4) = n_edges + 3;
  PE(g, 3, n_panels + 2) = n_edges + 3;
  n_edges += 3;
  /* the new particles and edges exist before the areas walk the leaf edges */
  g->np = n_particles;
  g->ne = n_edges;
  /* subpanel centres and areas (:1061-1069) */
  for (int j = 1; j <= 4; ++j) {
    int q = n_panels + j;
    sphere_tri_center(PX(g, PV(g, 1, q)), PX(g, PV(g, 2, q)), PX(g, PV(g, 3, q)), CX(g, q));
    sphere_tri_center(PX0(g, PV(g, 1, q)), PX0(g, PV(g, 2, q)), PX0(g, PV(g, 3, q)), CX0(g, q));
    g->area[q - 1] = tri_panel_area(g, q, scratch, scratch_len);
  }
  /* centre particle (:1072-1073) and bookkeeping (:1078-1087) */
  memcpy(CX(g, panel), CX(g, c4), 3 * sizeof(double));
  memcpy(CX0(g, panel), CX0(g, c4), 3 * sizeof(double));
  g->area[panel - 1] = 0.0;
  g->phas[panel - 1] = 1;
  for (int j = 1; j <= 4; ++j) {
    g->pnest[n_panels + j - 1] = nest + 1;
    PCH(g, j, panel) = n_panels + j;
  }
  g->npan = n_panels + 4;
  g->nactive += 3;
}

/* PanelMax / ParticleMax / EdgeMax for TRI_PANEL (:2614-2662). */
int or_icos_sizes(int level, int *n_particles, int *n_edges, int *n_panels, int *n_active) {
  if (level < 0 || level > 11) return -1;
  long long pan = 0;
  for (int j = 0; j <= level; ++j) pan += 20LL << (2 * j);
  *n_panels = (int)pan;
  *n_particles = (int)(2 + (10LL << (2 * level)));
  *n_edges = (int)(3 * pan / 2); /* 30 * sum 4^j */
  *n_active = (int)(20LL << (2 * level));
  return 0;
}

static const double kRoot[11][3] = {
    {0.0, 0.0, 1.0},
    {0.723606797749978969640917366873, 0.525731112119133606025669084848, 0.447213595499957939281834733746},
    {-0.276393202250021030359082633126, 0.850650808352039932181540497063, 0.447213595499957939281834733746},
    {-0.894427190999915878563669467492, 0.0, 0.447213595499957939281834733746},
    {-0.276393202250021030359082633127, -0.850650808352039932181540497063, 0.447213595499957939281834733746},
    {0.723606797749978969640917366873, -0.525731112119133606025669084848, 0.447213595499957939281834733746},
    {0.894427190999915878563669467492, 0.0, -0.447213595499957939281834733746},
    {0.276393202250021030359082633127, 0.850650808352039932181540497063, -0.447213595499957939281834733746},
    {-0.723606797749978969640917366873, 0.525731112119133606025669084848, -0.447213595499957939281834733746},
    {-0.723606797749978969640917366873, -0.525731112119133606025669084848, -0.447213595499957939281834733746},
    {0.276393202250021030359082633127, -0.850650808352039932181540497063, -0.447213595499957939281834733746}};

/* edge table (verts, leftPanel, rightPanel) of the icosahedron, :486-576 */
static const int kEdgeVerts[30][2] = {
    {1, 2}, {2, 3}, {3, 1}, {3, 4}, {4, 1}, {4, 5}, {5, 1}, {5, 6}, {6, 1}, {6, 2},
    {2, 8}, {8, 3}, {8, 9}, {9, 3}, {9, 4}, {9, 10}, {10, 4}, {10, 5}, {10, 11}, {11, 5},
    {11, 6}, {11, 7}, {7, 6}, {7, 2}, {7, 8}, {8, 12}, {12, 9}, {12, 10}, {12, 11}, {12, 7}};
static const int kEdgeLeft[30] = {1, 1, 1, 2, 2, 3, 3, 4, 4, 5, 6, 6, 7, 7, 8,
                                  9, 9, 10, 11, 11, 12, 13, 13, 14, 15, 16, 16, 17, 18, 19};
static const int kEdgeRight[30] = {5, 6, 2, 8, 3, 10, 4, 12, 5, 14, 15, 7, 16, 8, 9,
                                   17, 10, 11, 18, 12, 13, 19, 14, 15, 20, 20, 17, 18, 19, 20};
/* panel table (edges, vertices), :580-621 */
static const int kPanelEdges[20][3] = {
    {1, 2, 3}, {3, 4, 5}, {5, 6, 7}, {7, 8, 9}, {9, 10, 1}, {12, 2, 11}, {12, 13, 14},
    {15, 4, 14}, {15, 16, 17}, {18, 6, 17}, {18, 19, 20}, {21, 8, 20}, {21, 22, 23},
    {24, 10, 23}, {24, 25, 11}, {27, 13, 26}, {28, 16, 27}, {29, 19, 28}, {30, 22, 29},
    {26, 25, 30}};
static const int kPanelVerts[20][3] = {
    {1, 2, 3}, {1, 3, 4}, {1, 4, 5}, {1, 5, 6}, {1, 6, 2}, {8, 3, 2}, {3, 8, 9},
    {9, 4, 3}, {4, 9, 10}, {10, 5, 4}, {5, 10, 11}, {11, 6, 5}, {6, 11, 7}, {7, 2, 6},
    {2, 7, 8}, {12, 9, 8}, {12, 10, 9}, {12, 11, 10}, {12, 7, 11}, {12, 8, 7}};

/* NewGrid(TRI_PANEL, initNest = level, AMR = 0) followed by InitIcosTriGrid.
 * Outputs (0-based indices, -1 for "none"; x arrays are (N, 3) row-major =
 * Fortran x(3, N)): particle positions and Lagrangian coordinates, panel
 * centres, Lagrangian centres, areas, hasChildren, vertices, nest, children.
 * Returns 0, or -1 for a level outside [0, 11] or an allocation failure. */
int or_icos_grid(int level, double *particles_x, double *particles_x0, double *panels_x,
                 double *panels_x0, double *panels_area, int *has_children, int *vertices, int *nest,
                 int *children) {
  int nP, nE, nPan, nAct;
  if (or_icos_sizes(level, &nP, &nE, &nPan, &nAct)) return -1;
  IcosGrid g;
  memset(&g, 0, sizeof g);
  g.px = calloc(3 * (size_t)nP, sizeof(double));
  g.px0 = calloc(3 * (size_t)nP, sizeof(double));
  g.everts = calloc(2 * (size_t)nE, sizeof(int));
  g.eleft = calloc((size_t)nE, sizeof(int));
  g.eright = calloc((size_t)nE, sizeof(int));
  g.ehas = calloc((size_t)nE, sizeof(int));
  g.echild = calloc(2 * (size_t)nE, sizeof(int));
  g.cx = calloc(3 * (size_t)nPan, sizeof(double));
  g.cx0 = calloc(3 * (size_t)nPan, sizeof(double));
  g.area = calloc((size_t)nPan, sizeof(double));
  g.pverts = calloc(3 * (size_t)nPan, sizeof(int));
  g.pedges = calloc(3 * (size_t)nPan, sizeof(int));
  g.phas = calloc((size_t)nPan, sizeof(int));
  g.pchild = calloc(4 * (size_t)nPan, sizeof(int));
  g.pnest = calloc((size_t)nPan, sizeof(int));
  /* a leaf edge list is at most 2^level long */
  int scratch_len = (1 << level) + 1;
  int *scratch = malloc((size_t)scratch_len * sizeof(int));
  int rc = 0;
  if (!g.px || !g.px0 || !g.everts || !g.eleft || !g.eright || !g.ehas || !g.echild || !g.cx ||
      !g.cx0 || !g.area || !g.pverts || !g.pedges || !g.phas || !g.pchild || !g.pnest || !scratch) {
    rc = -1;
    goto done;
  }
  /* particles (:431-481) */
  g.np = 12;
  for (int j = 1; j <= 11; ++j) {
    const double *r = kRoot[j - 1];
    double nrm = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    for (int c = 0; c < 3; ++c) PX(&g, j)[c] = r[c] / nrm;
  }
  PX(&g, 12)[0] = 0.0;
  PX(&g, 12)[1] = 0.0;
  PX(&g, 12)[2] = -1.0;
  memcpy(g.px0, g.px, 36 * sizeof(double));
  /* edges */
  g.ne = 30;
  for (int e = 1; e <= 30; ++e) {
    EV(&g, 1, e) = kEdgeVerts[e - 1][0];
    EV(&g, 2, e) = kEdgeVerts[e - 1][1];
    ELEFT(&g, e) = kEdgeLeft[e - 1];
    ERIGHT(&g, e) = kEdgeRight[e - 1];
  }
  /* panels */
  g.npan = 20;
  g.nactive = 20;
  for (int p = 1; p <= 20; ++p)
    for (int s = 1; s <= 3; ++s) {
      PE(&g, s, p) = kPanelEdges[p - 1][s - 1];
      PV(&g, s, p) = kPanelVerts[p - 1][s - 1];
    }
  for (int p = 1; p <= 20; ++p) {
    sphere_tri_center(PX(&g, PV(&g, 1, p)), PX(&g, PV(&g, 2, p)), PX(&g, PV(&g, 3, p)), CX(&g, p));
    g.area[p - 1] = tri_panel_area(&g, p, scratch, scratch_len);
  }
  memcpy(g.cx0, g.cx, 60 * sizeof(double));
  /* recursive division (:630-639): the next level restarts at nOldPanels */
  int start = 1;
  for (int k = 1; k <= level; ++k) {
    int n_old = g.npan;
    for (int j = start; j <= n_old; ++j)
      if (!g.phas[j - 1]) divide_tri_panel(&g, j, scratch, scratch_len);
    start = n_old;
  }
  if (g.np != nP || g.npan != nPan || g.ne != nE || g.nactive != nAct) {
    rc = -1;
    goto done;
  }
  memcpy(particles_x, g.px, 3 * (size_t)nP * sizeof(double));
  if (particles_x0) memcpy(particles_x0, g.px0, 3 * (size_t)nP * sizeof(double));
  memcpy(panels_x, g.cx, 3 * (size_t)nPan * sizeof(double));
  if (panels_x0) memcpy(panels_x0, g.cx0, 3 * (size_t)nPan * sizeof(double));
  memcpy(panels_area, g.area, (size_t)nPan * sizeof(double));
  for (int p = 0; p < nPan; ++p) {
    if (has_children) has_children[p] = g.phas[p];
    if (nest) nest[p] = g.pnest[p];
    if (vertices)
      for (int s = 0; s < 3; ++s) vertices[3 * (size_t)p + s] = g.pverts[3 * (size_t)p + s] - 1;
    if (children)
      for (int s = 0; s < 4; ++s) children[4 * (size_t)p + s] = g.pchild[4 * (size_t)p + s] - 1;
  }
done:
  free(g.px);
  free(g.px0);
  free(g.everts);
  free(g.eleft);
  free(g.eright);
  free(g.ehas);
  free(g.echild);
  free(g.cx);
  free(g.cx0);
  free(g.area);
  free(g.pverts);
  free(g.pedges);
  free(g.phas);
  free(g.pchild);
  free(g.pnest);
  free(scratch);
  return rc;
}

/* GatherPanels (:1556-1619): leaf panels in ascending index order form the
 * active set, divided panels the passive set. Returns 0, or -1 when the counts
 * do not match n_active / n_passive. */
int or_gather_maps(int n, const int *has_children, int *active_map, int n_active, int *passive_map,
                   int n_passive) {
  int a = 0, q = 0;
  for (int j = 0; j < n; ++j) {
    if (has_children[j]) {
      if (q >= n_passive) return -1;
      passive_map[q++] = j;
    } else {
      if (a >= n_active) return -1;
      active_map[a++] = j;
    }
  }
  return (a == n_active && q == n_passive) ? 0 : -1;
}
