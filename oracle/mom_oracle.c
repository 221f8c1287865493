/*
 * CPU oracle for the linear PMCHWT hot path of for90-mom2.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C FP64 restatement of the
 * reference's Fortran routines, used by tests/ (as the checker), by
 * __graft_entry__.smoke() and by the cpu_baseline / reference arm of bench.py.
 * Nothing in the product library links, loads or calls it.
 *
 * Parity status: UNPINNED against reference outputs.  The reference is
 * Fortran 90 and no Fortran compiler exists on either machine, and the
 * reference ships no golden vectors for this path.  The oracle is instead
 * pinned by (a) the closed-form singular integrals checked against adaptive
 * numerical quadrature, (b) the Mie series for the sphere, (c) structural
 * properties (lossless sigma_abs ~ 0, reciprocity).
 *
 * Every routine cites the reference file:line it follows.  The parity quirks
 * are kept on purpose:
 *   - pi is the single-precision literal 3.141592653589 widened to double
 *     (constants.f90:10), and it leaks into mu0, omega, 1/(4 pi), deg->rad;
 *   - the tri_gl13 weights and nodes are single-precision literals
 *     (quad.f90:115-171);
 *   - dotc does not conjugate (linalg.f90:15-21);
 *   - edge / submesh / orientation ordering (mesh.f90:1044-1137, 290-558);
 *   - near pairs use the per-domain average edge length (sysmat.f90:233-260);
 *   - intK4 is zero for the self face (srcint.f90:392-395);
 *   - R = 0 limits of the smoothed Green's functions (green.f90:40-97).
 *
 * Indices are 0-based here; the reference is 1-based.  Only the identity
 * symmetry group and the non-periodic Green's function are restated (the
 * configurations of this path use nothing else).
 */
#include <complex.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* ---- constants.f90:8-14 ------------------------------------------------ */
#define O_PI ((double)3.141592653589f)
#define O_EPS0 8.8541878176e-12
#define O_MU0 (4 * O_PI * 1e-7)
#define O_C0 2.997924580003e8
#define O_ETA0 3.767303134622e2

/* ---- quad.f90:11-171, 277-315: triangle rules -------------------------- */
typedef struct {
  int nq;
  double w[13];
  double nd[13][3]; /* nodes(n,k) of the reference: barycentric factors */
} oquad;

/* quad.f90:115-171 (tri_gl13): default-real literals, i.e. float-rounded. */
static const float gl13_w[13] = {
    -0.149570044467670f, 0.175615257433204f, 0.175615257433204f,
    0.175615257433204f,  0.053347235608839f, 0.053347235608839f,
    0.053347235608839f,  0.077113760890257f, 0.077113760890257f,
    0.077113760890257f,  0.077113760890257f, 0.077113760890257f,
    0.077113760890257f};
static const float gl13_f[3][13] = {
    {0.333333333333333f, 0.479308067841923f, 0.260345966079038f,
     0.260345966079038f, 0.869739794195568f, 0.065130102902216f,
     0.065130102902216f, 0.638444188569809f, 0.638444188569809f,
     0.312865496004875f, 0.312865496004875f, 0.048690315425316f,
     0.048690315425316f},
    {0.333333333333333f, 0.260345966079038f, 0.260345966079038f,
     0.479308067841923f, 0.065130102902216f, 0.065130102902216f,
     0.869739794195568f, 0.048690315425316f, 0.312865496004875f,
     0.048690315425316f, 0.638444188569809f, 0.312865496004875f,
     0.638444188569809f},
    {0.333333333333333f, 0.260345966079038f, 0.479308067841923f,
     0.260345966079038f, 0.065130102902216f, 0.869739794195568f,
     0.065130102902216f, 0.312865496004875f, 0.048690315425316f,
     0.638444188569809f, 0.048690315425316f, 0.638444188569809f,
     0.312865496004875f}};

/* quad.f90:11-27 (tri_gl4), 29-55 (tri_gl7), 89-100 (tri_gl1, tri_gl3):
 * these carry the _dp suffix and are double literals. */
int oracle_tri_rule(const char *name, int *nq, double *w, double *nodes) {
  oquad q;
  memset(&q, 0, sizeof q);
  if (!strcmp(name, "tri_gl13")) {
    q.nq = 13;
    for (int i = 0; i < 13; i++) {
      q.w[i] = (double)gl13_w[i];
      for (int k = 0; k < 3; k++) q.nd[i][k] = (double)gl13_f[k][i];
    }
  } else if (!strcmp(name, "tri_gl1")) {
    q.nq = 1;
    q.w[0] = 1.0;
    for (int k = 0; k < 3; k++) q.nd[0][k] = 0.333333333333333;
  } else if (!strcmp(name, "tri_gl3")) {
    static const double f[3][3] = {{0.666666666666667, 0.166666666666667, 0.166666666666667},
                                   {0.166666666666667, 0.666666666666667, 0.166666666666667},
                                   {0.166666666666667, 0.166666666666667, 0.666666666666667}};
    q.nq = 3;
    for (int i = 0; i < 3; i++) {
      q.w[i] = 0.333333333333333;
      /* quadFactors3 is RESHAPEd column-major into (3,3): element (i,k) = f[k][i]
       * with the listed literals being single precision in the reference
       * (quad.f90:102-113 carry no _dp suffix). */
      for (int k = 0; k < 3; k++) q.nd[i][k] = (double)(float)f[k][i];
    }
  } else if (!strcmp(name, "tri_gl4")) {
    static const double w4[4] = {-0.56250000, 0.52083333, 0.52083333, 0.52083333};
    static const double f4[3][4] = {{1.0 / 3.0, 0.6, 0.2, 0.2},
                                    {1.0 / 3.0, 0.2, 0.6, 0.2},
                                    {1.0 / 3.0, 0.2, 0.2, 0.6}};
    q.nq = 4;
    for (int i = 0; i < 4; i++) {
      q.w[i] = w4[i];
      for (int k = 0; k < 3; k++) q.nd[i][k] = f4[k][i];
    }
  } else if (!strcmp(name, "tri_gl7")) {
    static const double w7[7] = {0.22500000, 0.13239415, 0.13239415, 0.13239415,
                                 0.12593918, 0.12593918, 0.12593918};
    static const double f7[3][7] = {
        {0.33333333, 0.05971587, 0.47014206, 0.47014206, 0.79742698, 0.10128650, 0.10128650},
        {0.33333333, 0.47014206, 0.05971587, 0.47014206, 0.10128650, 0.79742698, 0.10128650},
        {0.33333333, 0.47014206, 0.47014206, 0.05971587, 0.10128650, 0.10128650, 0.79742698}};
    q.nq = 7;
    for (int i = 0; i < 7; i++) {
      q.w[i] = w7[i];
      for (int k = 0; k < 3; k++) q.nd[i][k] = f7[k][i];
    }
  } else {
    return -1; /* quad.f90:312-313 STOPs on an unknown name */
  }
  *nq = q.nq;
  for (int i = 0; i < q.nq; i++) {
    w[i] = q.w[i];
    for (int k = 0; k < 3; k++) nodes[3 * i + k] = q.nd[i][k];
  }
  return 0;
}

/* ---- mesh.f90:27-83 (mesh_container), flattened ----------------------- */
typedef struct {
  int nnodes, nfaces, nedges;
  double *node;      /* [nnodes][3] */
  int *node_parent;  /* [nnodes] */
  int *face_node;    /* [nfaces][3] */
  int *face_edge;    /* [nfaces][3] */
  int *face_id;      /* [nfaces] */
  int *face_parent;  /* [nfaces] */
  double *face_n;    /* [nfaces][3] */
  double *face_cp;   /* [nfaces][3] */
  double *face_s;    /* [nfaces][3 edges][3] : s(:,e) */
  double *face_m;    /* [nfaces][3 edges][3] : m(:,e) */
  double *face_area; /* [nfaces] */
  int *edge_node;    /* [nedges][2] */
  int *edge_bnode;   /* [nedges][2] */
  int *edge_face;    /* [nedges][2] */
  int *edge_parent;  /* [nedges] */
  double *edge_len;  /* [nedges] */
  int *nchild;       /* [nedges] (master only) */
  int *child;        /* [nedges][maxchild][2] (master only) */
  int maxchild;
  double avelen;
} omesh;

/* symmetry.f90:24-40 group_action: point action j (row-major here,
 * j[3 i + k] = J(i, k)), its determinant, a special-action identifier,
 * generator bits and the field actions ef(1:nga) (conjugated representation
 * values). */
#define O_MAXGA 32
enum { O_GID_IDENTITY = 1, O_GID_MXP = 2, O_GID_MYP = 3, O_GID_MZP = 4, O_GID_RZ = 5 };
/* mesh.f90:16-25 boundary types of edges */
enum { O_BND_NONE = 1, O_BND_XPLANE = 2, O_BND_YPLANE = 3, O_BND_ZPLANE = 4, O_BND_RZ1 = 9, O_BND_RZ2 = 10 };
typedef struct {
  double j[9];
  double detj;
  int id, genbits;
  double complex ef[O_MAXGA];
} ogact;

typedef struct {
  omesh master;
  int ndom;
  omesh *dom;
  oquad qd;
  int nga;       /* group of the batch (read_symm); identity unless set */
  ogact *ga;
  int *mbnd;     /* [master nedges] edge boundary type (classify_edges) */
  int **dbnd;    /* per domain [nedges], inherited from the master edge */
} oproblem;

static void *xcalloc(size_t n, size_t s) {
  void *p = calloc(n ? n : 1, s);
  if (!p) abort();
  return p;
}

static void mesh_free(omesh *m) {
  free(m->node); free(m->node_parent); free(m->face_node); free(m->face_edge);
  free(m->face_id); free(m->face_parent); free(m->face_n); free(m->face_cp);
  free(m->face_s); free(m->face_m); free(m->face_area); free(m->edge_node);
  free(m->edge_bnode); free(m->edge_face); free(m->edge_parent); free(m->edge_len);
  free(m->nchild); free(m->child);
  memset(m, 0, sizeof *m);
}

static inline double dotr(const double *a, const double *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static inline double normr(const double *v) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }
static inline void crossr(const double *a, const double *b, double *r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}
static inline void crossc(const cplx *a, const cplx *b, cplx *r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}
static inline int cmp_pairs(const int *a, const int *b) { /* mesh.f90:961-971 */
  return (a[0] == b[0] && a[1] == b[1]) || (a[0] == b[1] && a[1] == b[0]);
}

/* mesh.f90:1265-1322 compute_basis_data */
static void compute_basis_data(omesh *m) {
  m->face_n = xcalloc(3 * m->nfaces, sizeof(double));
  m->face_cp = xcalloc(3 * m->nfaces, sizeof(double));
  m->face_s = xcalloc(9 * m->nfaces, sizeof(double));
  m->face_m = xcalloc(9 * m->nfaces, sizeof(double));
  m->face_area = xcalloc(m->nfaces, sizeof(double));
  m->edge_len = xcalloc(m->nedges, sizeof(double));
  for (int n = 0; n < m->nfaces; n++) {
    const double *p1 = m->node + 3 * m->face_node[3 * n];
    const double *p2 = m->node + 3 * m->face_node[3 * n + 1];
    const double *p3 = m->node + 3 * m->face_node[3 * n + 2];
    double a[3], b[3], c[3], p21[3], p32[3], p13[3];
    for (int i = 0; i < 3; i++) { a[i] = p2[i] - p1[i]; c[i] = p3[i] - p1[i]; }
    crossr(a, c, b);
    double nb = normr(b);
    double *nn = m->face_n + 3 * n;
    for (int i = 0; i < 3; i++) nn[i] = b[i] / nb;
    for (int i = 0; i < 3; i++) { p21[i] = p2[i] - p1[i]; p32[i] = p3[i] - p2[i]; p13[i] = p1[i] - p3[i]; }
    double *s = m->face_s + 9 * n, *mm = m->face_m + 9 * n;
    double l21 = normr(p21), l32 = normr(p32), l13 = normr(p13);
    for (int i = 0; i < 3; i++) { s[i] = p21[i] / l21; s[3 + i] = p32[i] / l32; s[6 + i] = p13[i] / l13; }
    for (int e = 0; e < 3; e++) crossr(s + 3 * e, nn, mm + 3 * e);
    for (int e = 0; e < 3; e++) {
      double l = normr(mm + 3 * e);
      for (int i = 0; i < 3; i++) mm[3 * e + i] = mm[3 * e + i] / l;
    }
    double mp13[3] = {-p13[0], -p13[1], -p13[2]}, cr[3];
    crossr(mp13, p32, cr);
    m->face_area[n] = 0.5 * normr(cr);
    for (int i = 0; i < 3; i++) m->face_cp[3 * n + i] = (p1[i] + p2[i] + p3[i]) / 3.0;
  }
  for (int e = 0; e < m->nedges; e++) {
    const double *a = m->node + 3 * m->edge_node[2 * e], *b = m->node + 3 * m->edge_node[2 * e + 1];
    double d[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
    m->edge_len[e] = normr(d);
  }
}

/* mesh.f90:138-153 average_edge_length */
static double average_edge_length(const omesh *m) {
  double res = 0.0;
  for (int e = 0; e < m->nedges; e++) {
    const double *a = m->node + 3 * m->edge_node[2 * e], *b = m->node + 3 * m->edge_node[2 * e + 1];
    double d[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
    res = res + normr(d);
  }
  return res / m->nedges;
}

/* mesh.f90:1044-1137 build_mesh: unique edges in face order, edge m of a
 * face is (node m, node m+1), the first face to see an edge is its "+" face
 * and bnode(1) is that face's opposite vertex.  The edge search is the
 * reference's linear scan over the edges found so far. */
static void build_mesh(omesh *m, double scale) {
  for (int i = 0; i < 3 * m->nnodes; i++) m->node[i] = m->node[i] * scale; /* mesh.f90:1007 */
  int cap = 3 * m->nfaces;
  int *en = xcalloc(2 * cap, sizeof(int)), *eb = xcalloc(2 * cap, sizeof(int)), *ef = xcalloc(2 * cap, sizeof(int));
  for (int i = 0; i < 2 * cap; i++) en[i] = eb[i] = ef[i] = -1;
  m->face_edge = xcalloc(3 * m->nfaces, sizeof(int));
  int cedge = 0;
  for (int n = 0; n < m->nfaces; n++) {
    for (int k = 0; k < 3; k++) {
      int pair[2] = {m->face_node[3 * n + k], m->face_node[3 * n + (k + 1) % 3]};
      int found = 0;
      for (int l = 0; l < cedge; l++) {
        if (cmp_pairs(en + 2 * l, pair)) {
          found = 1;
          ef[2 * l + 1] = n;
          eb[2 * l + 1] = m->face_node[3 * n + (k + 2) % 3];
          m->face_edge[3 * n + k] = l;
          break;
        }
      }
      if (!found) {
        en[2 * cedge] = pair[0];
        en[2 * cedge + 1] = pair[1];
        ef[2 * cedge] = n;
        eb[2 * cedge] = m->face_node[3 * n + (k + 2) % 3];
        m->face_edge[3 * n + k] = cedge;
        cedge++;
      }
    }
  }
  m->nedges = cedge;
  m->edge_node = xcalloc(2 * cedge, sizeof(int));
  m->edge_bnode = xcalloc(2 * cedge, sizeof(int));
  m->edge_face = xcalloc(2 * cedge, sizeof(int));
  memcpy(m->edge_node, en, 2 * cedge * sizeof(int));
  memcpy(m->edge_bnode, eb, 2 * cedge * sizeof(int));
  memcpy(m->edge_face, ef, 2 * cedge * sizeof(int));
  free(en); free(eb); free(ef);
  m->edge_parent = xcalloc(cedge, sizeof(int));
  for (int e = 0; e < cedge; e++) m->edge_parent[e] = -1;
  m->avelen = average_edge_length(m);
  compute_basis_data(m);
}

/* mesh.f90:290-376 extract_submesh (surface part): faces whose id is in
 * ids, nodes renumbered in master order. */
static void extract_submesh(const omesh *ms, int nids, const int *ids, omesh *sub) {
  memset(sub, 0, sizeof *sub);
  char *nmask = xcalloc(ms->nnodes, 1);
  int nf = 0;
  for (int n = 0; n < ms->nfaces; n++) {
    int hit = 0;
    for (int i = 0; i < nids; i++) hit |= (ids[i] == ms->face_id[n]);
    if (hit) {
      nf++;
      for (int k = 0; k < 3; k++) nmask[ms->face_node[3 * n + k]] = 1;
    }
  }
  int *loc = xcalloc(ms->nnodes, sizeof(int));
  int nn = 0;
  for (int n = 0; n < ms->nnodes; n++) nn += nmask[n];
  sub->nnodes = nn;
  sub->node = xcalloc(3 * nn, sizeof(double));
  sub->node_parent = xcalloc(nn, sizeof(int));
  int c = 0;
  for (int n = 0; n < ms->nnodes; n++) {
    loc[n] = -1;
    if (nmask[n]) {
      memcpy(sub->node + 3 * c, ms->node + 3 * n, 3 * sizeof(double));
      sub->node_parent[c] = n;
      loc[n] = c++;
    }
  }
  sub->nfaces = nf;
  sub->face_node = xcalloc(3 * nf, sizeof(int));
  sub->face_id = xcalloc(nf, sizeof(int));
  sub->face_parent = xcalloc(nf, sizeof(int));
  c = 0;
  for (int n = 0; n < ms->nfaces; n++) {
    int hit = 0;
    for (int i = 0; i < nids; i++) hit |= (ids[i] == ms->face_id[n]);
    if (hit) {
      for (int k = 0; k < 3; k++) sub->face_node[3 * c + k] = loc[ms->face_node[3 * n + k]];
      sub->face_parent[c] = n;
      sub->face_id[c] = ms->face_id[n];
      c++;
    }
  }
  free(nmask);
  free(loc);
}

/* mesh.f90:278-288 invert_faces */
static void invert_faces(omesh *m, int id) {
  for (int n = 0; n < m->nfaces; n++)
    if (m->face_id[n] == id) {
      int t = m->face_node[3 * n];
      m->face_node[3 * n] = m->face_node[3 * n + 2];
      m->face_node[3 * n + 2] = t;
    }
}

/* mesh.f90:378-452 submesh_edge_connectivity (non-periodic part). */
static int submesh_edge_connectivity(omesh *ms, int nsub, omesh *subs) {
  ms->maxchild = nsub;
  ms->nchild = xcalloc(ms->nedges, sizeof(int));
  ms->child = xcalloc((size_t)ms->nedges * nsub * 2, sizeof(int));
  for (int n = 0; n < ms->nedges; n++) {
    for (int s = 0; s < nsub; s++) {
      omesh *sm = subs + s;
      for (int l = 0; l < sm->nedges; l++) {
        int pi[2] = {sm->node_parent[sm->edge_node[2 * l]], sm->node_parent[sm->edge_node[2 * l + 1]]};
        if (cmp_pairs(ms->edge_node + 2 * n, pi)) {
          sm->edge_parent[l] = n;
          int c = ms->nchild[n]++;
          ms->child[((size_t)n * nsub + c) * 2] = s;
          ms->child[((size_t)n * nsub + c) * 2 + 1] = l;
        }
      }
    }
  }
  for (int n = 0; n < ms->nedges; n++)
    if (ms->nchild[n] < 2) return -1; /* mesh.f90:415-418: inconsistent decomposition */
  return 0;
}

static inline void swapi(int *a, int *b) { int t = *a; *a = *b; *b = t; }

/* mesh.f90:454-558 orient_basis (non-periodic part): a child edge's +/-
 * faces are swapped when it shares its + face or its - face (in parent face
 * terms) with an already oriented child. */
static void orient_basis(omesh *ms, omesh *subs) {
  int ns = ms->maxchild;
  char *oriented = xcalloc(ns > 0 ? ns : 1, 1);
  for (int n = 0; n < ms->nedges; n++) {
    int nchild = ms->nchild[n];
    const int *ch = ms->child + (size_t)n * ns * 2;
    memset(oriented, 0, ns);
    oriented[0] = 1;
    for (int mm = 0; mm < nchild; mm++) {
      for (int l = 1; l < nchild; l++) {
        if (oriented[l]) continue;
        for (int k = 0; k < nchild; k++) {
          if (!oriented[k]) continue;
          omesh *sl = subs + ch[2 * l], *sk = subs + ch[2 * k];
          int el = ch[2 * l + 1], ek = ch[2 * k + 1];
          int pf1 = sl->edge_face[2 * el], nf1 = sl->edge_face[2 * el + 1];
          int pf2 = sk->edge_face[2 * ek], nf2 = sk->edge_face[2 * ek + 1];
          if (pf1 != -1) pf1 = sl->face_parent[pf1];
          if (nf1 != -1) nf1 = sl->face_parent[nf1];
          if (pf2 != -1) pf2 = sk->face_parent[pf2];
          if (nf2 != -1) nf2 = sk->face_parent[nf2];
          if (pf1 == pf2 || nf1 == nf2) {
            swapi(sl->edge_face + 2 * el, sl->edge_face + 2 * el + 1);
            swapi(sl->edge_bnode + 2 * el, sl->edge_bnode + 2 * el + 1);
          }
          if (pf1 == pf2 || nf1 == nf2 || pf1 == nf2 || nf1 == pf2) {
            oriented[l] = 1;
            break;
          }
        }
      }
      int cnt = 0;
      for (int i = 0; i < nchild; i++) cnt += oriented[i];
      if (cnt == nchild) break;
    }
  }
  free(oriented);
}

/* interface.f90:357-366 (mesh), 44-105 (sdom), 107-123 (fdom). */
int oracle_problem_create(int nnodes, const double *nodes, int nfaces, const int *faces,
                          const int *face_ids, double scale, int ndom, const int *dom_nsurf,
                          const int *dom_ids, const char *quad_name, void **out) {
  oproblem *P = xcalloc(1, sizeof(oproblem));
  omesh *ms = &P->master;
  ms->nnodes = nnodes;
  ms->nfaces = nfaces;
  ms->node = xcalloc(3 * nnodes, sizeof(double));
  memcpy(ms->node, nodes, 3 * nnodes * sizeof(double));
  ms->face_node = xcalloc(3 * nfaces, sizeof(int));
  memcpy(ms->face_node, faces, 3 * nfaces * sizeof(int));
  ms->face_id = xcalloc(nfaces, sizeof(int));
  memcpy(ms->face_id, face_ids, nfaces * sizeof(int));
  ms->face_parent = xcalloc(nfaces, sizeof(int));
  ms->node_parent = xcalloc(nnodes, sizeof(int));
  for (int i = 0; i < nfaces; i++) ms->face_parent[i] = i;
  for (int i = 0; i < nnodes; i++) ms->node_parent[i] = i;
  build_mesh(ms, scale);
  P->ndom = ndom;
  P->dom = xcalloc(ndom, sizeof(omesh));
  int off = 0;
  for (int d = 0; d < ndom; d++) {
    int ns = dom_nsurf[d];
    int *absid = xcalloc(ns, sizeof(int));
    for (int i = 0; i < ns; i++) absid[i] = abs(dom_ids[off + i]);
    extract_submesh(ms, ns, absid, P->dom + d);
    for (int i = 0; i < ns; i++) {
      if (dom_ids[off + i] == 0) { free(absid); return -2; } /* interface.f90:80-83 */
      if (dom_ids[off + i] < 0) invert_faces(P->dom + d, abs(dom_ids[off + i]));
    }
    build_mesh(P->dom + d, 1.0);
    free(absid);
    off += ns;
  }
  if (submesh_edge_connectivity(ms, ndom, P->dom)) return -3;
  orient_basis(ms, P->dom);
  if (oracle_tri_rule(quad_name, &P->qd.nq, P->qd.w, &P->qd.nd[0][0])) return -4;
  /* batch_defaults / read_symm with no groups: the identity group; no
   * classified boundary edges */
  P->ga = xcalloc(O_MAXGA, sizeof(ogact));
  P->nga = 1;
  P->ga[0].j[0] = P->ga[0].j[4] = P->ga[0].j[8] = 1.0;
  P->ga[0].detj = 1.0;
  P->ga[0].id = O_GID_IDENTITY;
  P->ga[0].genbits = 1 << O_GID_IDENTITY;
  P->ga[0].ef[0] = 1.0;
  P->mbnd = xcalloc(ms->nedges, sizeof(int));
  for (int e = 0; e < ms->nedges; e++) P->mbnd[e] = O_BND_NONE;
  P->dbnd = xcalloc(ndom, sizeof(int *));
  for (int d = 0; d < ndom; d++) {
    P->dbnd[d] = xcalloc(P->dom[d].nedges, sizeof(int));
    for (int e = 0; e < P->dom[d].nedges; e++) P->dbnd[d][e] = O_BND_NONE;
  }
  *out = P;
  return 0;
}

void oracle_problem_free(void *p) {
  oproblem *P = p;
  if (!P) return;
  mesh_free(&P->master);
  for (int d = 0; d < P->ndom; d++) mesh_free(P->dom + d);
  if (P->dbnd)
    for (int d = 0; d < P->ndom; d++) free(P->dbnd[d]);
  free(P->dbnd);
  free(P->mbnd);
  free(P->ga);
  free(P->dom);
  free(P);
}

/* Sizes: [0]=master nedges, then per domain (nnodes, nfaces, nedges). */
void oracle_problem_sizes(void *p, int *out) {
  oproblem *P = p;
  out[0] = P->master.nedges;
  out[1] = P->master.nnodes;
  out[2] = P->master.nfaces;
  for (int d = 0; d < P->ndom; d++) {
    out[3 + 3 * d] = P->dom[d].nnodes;
    out[4 + 3 * d] = P->dom[d].nfaces;
    out[5 + 3 * d] = P->dom[d].nedges;
  }
}

/* Export the topology of domain d (d = -1: master) for comparisons. */
void oracle_problem_export(void *p, int d, double *nodes, int *face_node, int *face_edge,
                           int *edge_node, int *edge_face, int *edge_bnode, int *edge_parent,
                           double *avelen) {
  oproblem *P = p;
  omesh *m = d < 0 ? &P->master : P->dom + d;
  if (nodes) memcpy(nodes, m->node, 3 * m->nnodes * sizeof(double));
  if (face_node) memcpy(face_node, m->face_node, 3 * m->nfaces * sizeof(int));
  if (face_edge) memcpy(face_edge, m->face_edge, 3 * m->nfaces * sizeof(int));
  if (edge_node) memcpy(edge_node, m->edge_node, 2 * m->nedges * sizeof(int));
  if (edge_face) memcpy(edge_face, m->edge_face, 2 * m->nedges * sizeof(int));
  if (edge_bnode) memcpy(edge_bnode, m->edge_bnode, 2 * m->nedges * sizeof(int));
  if (edge_parent) memcpy(edge_parent, m->edge_parent, m->nedges * sizeof(int));
  if (avelen) *avelen = m->avelen;
}

/* ---- mesh.f90:1326-1369 face sign and bnodes --------------------------- */
static inline double get_face_sign(const omesh *m, int f, int e) {
  int ge = m->face_edge[3 * f + e];
  if (f == m->edge_face[2 * ge]) return 1.0;
  if (f == m->edge_face[2 * ge + 1]) return -1.0;
  return 0.0;
}
static inline const double *get_face_bnode(const omesh *m, int f, int e) {
  int ge = m->face_edge[3 * f + e];
  if (m->edge_face[2 * ge] == f) return m->node + 3 * m->edge_bnode[2 * ge];
  return m->node + 3 * m->edge_bnode[2 * ge + 1];
}

/* quad.f90:352-367 quad_tri_points: point = n3 p1 + n1 p2 + n2 p3 */
static void quad_tri_points(const oquad *qd, const omesh *m, int f, double *res /*[nq][3]*/) {
  const double *p1 = m->node + 3 * m->face_node[3 * f];
  const double *p2 = m->node + 3 * m->face_node[3 * f + 1];
  const double *p3 = m->node + 3 * m->face_node[3 * f + 2];
  for (int n = 0; n < qd->nq; n++)
    for (int i = 0; i < 3; i++)
      res[3 * n + i] = qd->nd[n][2] * p1[i] + qd->nd[n][0] * p2[i] + qd->nd[n][1] * p3[i];
}

/* rwgf.f90:13-32 rwg and 54-78 vrwg */
static void rwg(const omesh *m, const double *r, int f, int e, double *res) {
  double L = m->edge_len[m->face_edge[3 * f + e]], A = m->face_area[f];
  double sgn = get_face_sign(m, f, e);
  int ge = m->face_edge[3 * f + e];
  if (sgn > 0) {
    const double *v = m->node + 3 * m->edge_bnode[2 * ge];
    for (int i = 0; i < 3; i++) res[i] = L / (2.0 * A) * (r[i] - v[i]);
  } else {
    const double *v = m->node + 3 * m->edge_bnode[2 * ge + 1];
    for (int i = 0; i < 3; i++) res[i] = L / (2.0 * A) * (v[i] - r[i]);
  }
}

/* rwgf.f90:34-52 rwgDiv */
static inline double rwgDiv(const omesh *m, int f, int e) {
  double sgn = get_face_sign(m, f, e);
  double L = m->edge_len[m->face_edge[3 * f + e]], A = m->face_area[f];
  return sgn * L / A;
}

/* ---- green.f90 --------------------------------------------------------- */
#define OOFPI (1.0 / (4.0 * O_PI))

/* green.f90:110-121 vGf and 40-55 vGs */
static inline cplx Gf_or_s(const double *r0, const double *rp, cplx k, int smooth) {
  double d0 = r0[0] - rp[0], d1 = r0[1] - rp[1], d2 = r0[2] - rp[2];
  double R = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  if (smooth) {
    if (R == 0) return k * (I * OOFPI);
    return OOFPI * ((cexp(I * k * R) - 1.0) / R + 0.5 * (k * k) * R);
  }
  return OOFPI * cexp(I * k * R) / R;
}

/* green.f90:135-151 vgradGf and 74-97 vgradGs */
static inline void gradG_or_s(const double *r0, const double *rp, cplx k, int smooth, cplx *res) {
  double d[3] = {r0[0] - rp[0], r0[1] - rp[1], r0[2] - rp[2]};
  double R = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  cplx ph;
  if (smooth) {
    if (R == 0) { res[0] = res[1] = res[2] = 0; return; }
    double RR = R * R;
    ph = OOFPI * (cexp(I * k * R) * (1.0 / (R * RR) - I * k / RR) - 1.0 / (R * RR) - (k * k) / (2.0 * R));
  } else {
    double RR = R * R;
    ph = OOFPI * cexp(I * k * R) * (1.0 / (R * RR) - I * k / RR);
  }
  for (int i = 0; i < 3; i++) res[i] = ph * d[i];
}

/* ---- int.f90: closed-form singular integrals ---------------------------- */
static inline void edge_pts(const omesh *m, int f, int e, const double **p1, const double **p2) {
  int a = m->face_node[3 * f + e], b = m->face_node[3 * f + (e + 1) % 3];
  *p1 = m->node + 3 * a;
  *p2 = m->node + 3 * b;
}

/* int.f90:15-53 intLm1 */
static double intLm1(const double *r, int f, int e, const omesh *m) {
  const double *p1, *p2;
  edge_pts(m, f, e, &p1, &p2);
  const double *s = m->face_s + 9 * f + 3 * e;
  double a[3], b[3];
  for (int i = 0; i < 3; i++) { a[i] = r[i] - p2[i]; b[i] = r[i] - p1[i]; }
  double Rp = normr(a), Rm = normr(b);
  double c[3], d[3];
  for (int i = 0; i < 3; i++) { c[i] = p2[i] - r[i]; d[i] = p1[i] - r[i]; }
  double sp = dotr(c, s), sm = dotr(d, s);
  double div1 = Rp - sp, div2 = Rm + sm;
  if (fabs(div1) > fabs(div2)) return log((Rm - sm) / div1);
  return log((Rp + sp) / div2);
}

/* int.f90:55-96 intL1 */
static double intL1(const double *r, int f, int e, const omesh *m) {
  const double *p1, *p2;
  edge_pts(m, f, e, &p1, &p2);
  double p[3], rp[3];
  for (int i = 0; i < 3; i++) { p[i] = 0.5 * (p1[i] + p2[i]); rp[i] = r[i] - p[i]; }
  double h = dotr(m->face_n + 3 * f, rp);
  double t = dotr(m->face_m + 9 * f + 3 * e, rp);
  double R02 = t * t + h * h;
  const double *s = m->face_s + 9 * f + 3 * e;
  double a[3], b[3], c[3], d[3];
  for (int i = 0; i < 3; i++) { a[i] = r[i] - p2[i]; b[i] = r[i] - p1[i]; c[i] = p2[i] - r[i]; d[i] = p1[i] - r[i]; }
  double Rp = normr(a), Rm = normr(b), sp = dotr(c, s), sm = dotr(d, s);
  if (R02 == 0) return 0.5 * (sp * Rp - sm * Rm);
  return 0.5 * R02 * intLm1(r, f, e, m) + 0.5 * (sp * Rp - sm * Rm);
}

/* int.f90:98-135 intL3 */
static double intL3(const double *r, int f, int e, const omesh *m) {
  const double *p1, *p2;
  edge_pts(m, f, e, &p1, &p2);
  double p[3], rp[3];
  for (int i = 0; i < 3; i++) { p[i] = 0.5 * (p1[i] + p2[i]); rp[i] = r[i] - p[i]; }
  double h = dotr(m->face_n + 3 * f, rp);
  double t = dotr(m->face_m + 9 * f + 3 * e, rp);
  double R02 = t * t + h * h;
  const double *s = m->face_s + 9 * f + 3 * e;
  double a[3], b[3], c[3], d[3];
  for (int i = 0; i < 3; i++) { a[i] = r[i] - p2[i]; b[i] = r[i] - p1[i]; c[i] = p2[i] - r[i]; d[i] = p1[i] - r[i]; }
  double Rp = normr(a), Rm = normr(b), sp = dotr(c, s), sm = dotr(d, s);
  return 0.75 * R02 * intL1(r, f, e, m) + 0.25 * (sp * (Rp * Rp * Rp) - sm * (Rm * Rm * Rm));
}

/* int.f90:137-162 intSm3h */
static double intSm3h(const double *r, int f, const omesh *m) {
  const double *p1 = m->node + 3 * m->face_node[3 * f];
  const double *p2 = m->node + 3 * m->face_node[3 * f + 1];
  const double *p3 = m->node + 3 * m->face_node[3 * f + 2];
  double a1[3], a2[3], a3[3], t[3];
  for (int i = 0; i < 3; i++) { a1[i] = p1[i] - r[i]; a2[i] = p2[i] - r[i]; a3[i] = p3[i] - r[i]; }
  double n1 = normr(a1), n2 = normr(a2), n3 = normr(a3);
  for (int i = 0; i < 3; i++) { a1[i] /= n1; a2[i] /= n2; a3[i] /= n3; }
  double x = 1.0 + dotr(a1, a2) + dotr(a1, a3) + dotr(a2, a3);
  crossr(a2, a3, t);
  double y = fabs(dotr(a1, t));
  double omega = 2.0 * atan2(y, x);
  double rp1[3] = {r[0] - p1[0], r[1] - p1[1], r[2] - p1[2]};
  if (dotr(m->face_n + 3 * f, rp1) > 0.0) return fabs(omega);
  return -fabs(omega);
}

/* int.f90:181-226 intSm1 */
static double intSm1(const double *r, int f, const omesh *m) {
  const double *p1 = m->node + 3 * m->face_node[3 * f];
  const double *p2 = m->node + 3 * m->face_node[3 * f + 1];
  const double *p3 = m->node + 3 * m->face_node[3 * f + 2];
  double r1[3], r2[3], r3[3];
  for (int i = 0; i < 3; i++) { r1[i] = r[i] - p1[i]; r2[i] = r[i] - p2[i]; r3[i] = r[i] - p3[i]; }
  const double *mm = m->face_m + 9 * f;
  double t1 = dotr(mm, r1), t2 = dotr(mm + 3, r2), t3 = dotr(mm + 6, r3);
  double h = dotr(m->face_n + 3 * f, r1);
  if (h == 0) {
    double e1 = (t1 == 0) ? 0 : intLm1(r, f, 0, m);
    double e2 = (t2 == 0) ? 0 : intLm1(r, f, 1, m);
    double e3 = (t3 == 0) ? 0 : intLm1(r, f, 2, m);
    return -(t1 * e1 + t2 * e2 + t3 * e3);
  }
  return -h * intSm3h(r, f, m) - (t1 * intLm1(r, f, 0, m) + t2 * intLm1(r, f, 1, m) + t3 * intLm1(r, f, 2, m));
}

/* int.f90:228-246 intS1 */
static double intS1(const double *r, int f, const omesh *m) {
  const double *p1 = m->node + 3 * m->face_node[3 * f];
  const double *p2 = m->node + 3 * m->face_node[3 * f + 1];
  const double *p3 = m->node + 3 * m->face_node[3 * f + 2];
  double r1[3], r2[3], r3[3];
  for (int i = 0; i < 3; i++) { r1[i] = r[i] - p1[i]; r2[i] = r[i] - p2[i]; r3[i] = r[i] - p3[i]; }
  const double *mm = m->face_m + 9 * f;
  double t1 = dotr(mm, r1), t2 = dotr(mm + 3, r2), t3 = dotr(mm + 6, r3);
  double h = dotr(m->face_n + 3 * f, r1);
  return (h * h) / 3.0 * intSm1(r, f, m) -
         1.0 / 3.0 * (t1 * intL1(r, f, 0, m) + t2 * intL1(r, f, 1, m) + t3 * intL1(r, f, 2, m));
}

/* int.f90:248-260 intK11, 262-274 intK1m1 */
static double intK11(const double *r, int f, int e, const omesh *m) {
  double sgn = get_face_sign(m, f, e), L = m->edge_len[m->face_edge[3 * f + e]], A = m->face_area[f];
  return sgn * L / A * intS1(r, f, m);
}
static double intK1m1(const double *r, int f, int e, const omesh *m) {
  double sgn = get_face_sign(m, f, e), L = m->edge_len[m->face_edge[3 * f + e]], A = m->face_area[f];
  return sgn * L / A * intSm1(r, f, m);
}

/* int.f90:276-301 intK21, 303-328 intK2m1 */
static void intK2x(const double *r, int f, int e, const omesh *m, int pow_m1, double *res) {
  const double *p1 = m->node + 3 * m->face_node[3 * f];
  double sgn = get_face_sign(m, f, e);
  const double *p = get_face_bnode(m, f, e);
  double rp1[3] = {r[0] - p1[0], r[1] - p1[1], r[2] - p1[2]};
  const double *n = m->face_n + 3 * f;
  double h = dotr(n, rp1);
  double L = m->edge_len[m->face_edge[3 * f + e]], A = m->face_area[f];
  const double *mm = m->face_m + 9 * f;
  double rho[3];
  for (int i = 0; i < 3; i++) rho[i] = r[i] - h * n[i];
  if (!pow_m1) {
    double l1 = intL3(r, f, 0, m), l2 = intL3(r, f, 1, m), l3 = intL3(r, f, 2, m);
    double s1 = intS1(r, f, m);
    for (int i = 0; i < 3; i++)
      res[i] = sgn * L / (2.0 * A) *
               (1.0 / 3.0 * (mm[i] * l1 + mm[3 + i] * l2 + mm[6 + i] * l3) + (rho[i] - p[i]) * s1);
  } else {
    double l1 = intL1(r, f, 0, m), l2 = intL1(r, f, 1, m), l3 = intL1(r, f, 2, m);
    double s1 = intSm1(r, f, m);
    for (int i = 0; i < 3; i++)
      res[i] = sgn * L / (2.0 * A) * (mm[i] * l1 + mm[3 + i] * l2 + mm[6 + i] * l3 + (rho[i] - p[i]) * s1);
  }
}

/* int.f90:330-357 intK31, 359-376 intK3m1 */
static void intK31(const double *r, int f, const omesh *m, double *res) {
  const double *p = m->node + 3 * m->face_node[3 * f];
  const double *n = m->face_n + 3 * f;
  double rp[3] = {r[0] - p[0], r[1] - p[1], r[2] - p[2]};
  double h = dotr(n, rp);
  const double *mm = m->face_m + 9 * f;
  double l1 = intL1(r, f, 0, m), l2 = intL1(r, f, 1, m), l3 = intL1(r, f, 2, m);
  if (h == 0) {
    for (int i = 0; i < 3; i++) res[i] = mm[i] * l1 + mm[3 + i] * l2 + mm[6 + i] * l3;
  } else {
    double sm1 = intSm1(r, f, m);
    for (int i = 0; i < 3; i++) res[i] = mm[i] * l1 + mm[3 + i] * l2 + mm[6 + i] * l3 - h * n[i] * sm1;
  }
}
static void intK3m1(const double *r, int f, const omesh *m, double *res) {
  const double *n = m->face_n + 3 * f;
  const double *mm = m->face_m + 9 * f;
  double l1 = intLm1(r, f, 0, m), l2 = intLm1(r, f, 1, m), l3 = intLm1(r, f, 2, m);
  double sh = intSm3h(r, f, m);
  for (int i = 0; i < 3; i++) res[i] = mm[i] * l1 + mm[3 + i] * l2 + mm[6 + i] * l3 + n[i] * sh;
}

/* int.f90:378-392 intK41, 394-407 intK4m1 */
static void intK4x(const double *r, int f, int e, const omesh *m, int pow_m1, double *res) {
  double sgn = get_face_sign(m, f, e);
  const double *p = get_face_bnode(m, f, e);
  double L = m->edge_len[m->face_edge[3 * f + e]], A = m->face_area[f];
  double k3[3], rp[3] = {r[0] - p[0], r[1] - p[1], r[2] - p[2]}, c[3];
  if (pow_m1) intK3m1(r, f, m, k3); else intK31(r, f, m, k3);
  crossr(rp, k3, c);
  for (int i = 0; i < 3; i++) res[i] = -sgn * L / (2.0 * A) * c[i];
}

/* ---- srcint.f90 (identity group, non-periodic) -------------------------- */

/* srcint.f90:57-118 intK1 with 21-53 intK1singular */
static void intK1(const double *r, int f, const omesh *m, cplx k, int near, const oquad *qd, cplx *res) {
  double qpn[13 * 3];
  double An = m->face_area[f];
  quad_tri_points(qd, m, f, qpn);
  cplx sum = 0;
  for (int t = 0; t < qd->nq; t++) sum += qd->w[t] * Gf_or_s(r, qpn + 3 * t, k, near);
  cplx tmp = An * sum;
  for (int e = 0; e < 3; e++) {
    double divfn = rwgDiv(m, f, e);
    cplx aint = 0;
    if (near) aint = 1.0 / (4.0 * O_PI) * intK1m1(r, f, e, m) - (k * k) / (8.0 * O_PI) * intK11(r, f, e, m);
    res[e] = tmp * divfn + aint;
  }
}

/* srcint.f90:158-224 intK2 with 121-154 intK2singular; res[3 edges][3] */
static void intK2(const double *r, int f, const omesh *m, cplx k, int near, const oquad *qd, cplx *res) {
  double qpn[13 * 3];
  double An = m->face_area[f];
  quad_tri_points(qd, m, f, qpn);
  cplx gv[13];
  for (int t = 0; t < qd->nq; t++) gv[t] = Gf_or_s(r, qpn + 3 * t, k, near) * qd->w[t] * An;
  for (int e = 0; e < 3; e++) {
    cplx acc[3] = {0, 0, 0};
    for (int t = 0; t < qd->nq; t++) {
      double fv[3];
      rwg(m, qpn + 3 * t, f, e, fv);
      for (int i = 0; i < 3; i++) acc[i] += fv[i] * gv[t];
    }
    if (near) {
      double km1[3], k1[3];
      intK2x(r, f, e, m, 1, km1);
      intK2x(r, f, e, m, 0, k1);
      for (int i = 0; i < 3; i++) acc[i] += 1.0 / (4.0 * O_PI) * km1[i] - (k * k) / (8.0 * O_PI) * k1[i];
    }
    for (int i = 0; i < 3; i++) res[3 * e + i] = acc[i];
  }
}

/* srcint.f90:370-448 intK4 with 330-366 intK4singular; res[3 edges][3] */
static void intK4(const double *r, int f, const omesh *m, cplx k, int tface, int near, const oquad *qd,
                  cplx *res) {
  if (f == tface) { /* srcint.f90:392-395 */
    for (int i = 0; i < 9; i++) res[i] = 0;
    return;
  }
  double qpn[13 * 3];
  double An = m->face_area[f];
  quad_tri_points(qd, m, f, qpn);
  cplx ggv[13][3];
  for (int t = 0; t < qd->nq; t++) gradG_or_s(r, qpn + 3 * t, k, near, ggv[t]);
  for (int e = 0; e < 3; e++) {
    cplx acc[3] = {0, 0, 0};
    for (int t = 0; t < qd->nq; t++) {
      double fv[3];
      rwg(m, qpn + 3 * t, f, e, fv);
      cplx fvc[3] = {fv[0], fv[1], fv[2]}, c[3];
      crossc(ggv[t], fvc, c); /* linalg.f90:72-82 vcrosscr */
      for (int i = 0; i < 3; i++) acc[i] += c[i] * qd->w[t];
    }
    for (int i = 0; i < 3; i++) acc[i] = acc[i] * An;
    if (near) {
      double km1[3], k1[3];
      intK4x(r, f, e, m, 1, km1);
      intK4x(r, f, e, m, 0, k1);
      for (int i = 0; i < 3; i++) acc[i] += 1.0 / (4.0 * O_PI) * km1[i] - (k * k) / (8.0 * O_PI) * k1[i];
    }
    for (int i = 0; i < 3; i++) res[3 * e + i] = acc[i];
  }
}

/* sysmat.f90:233-260 near_faces (identity group, no prd) */
static inline int near_faces(const omesh *m, int n, int mm) {
  double threshold = m->avelen * 3;
  double d[3];
  for (int i = 0; i < 3; i++) d[i] = m->face_cp[3 * mm + i] - m->face_cp[3 * n + i];
  double distsq = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  return distsq < threshold * threshold;
}

/* sysmat.f90:272-347 computeD, 359-434 computeH, 446-519 computeK.
 * op: 0 = D, 1 = H, 2 = K.  M is the domain edge matrix (column-major,
 * N_d x N_d), zeroed here.  Test faces [mlo, mhi) only (the full operator
 * when mlo = 0, mhi = nfaces); the OpenMP loop is over source faces, as in
 * the reference. */
static void compute_op(int op, double omega, cplx ri, const omesh *m, const oquad *qd, cplx *M, int mlo,
                       int mhi) {
  int Nd = m->nedges, F = m->nfaces, nq = qd->nq;
  memset(M, 0, sizeof(cplx) * (size_t)Nd * Nd);
  cplx k = ri * omega / O_C0;
  cplx c1 = -I * omega * O_MU0;
  cplx c2 = -1.0 / (I * omega * O_EPS0 * (ri * ri));
  size_t per = (op == 1) ? 3 : 9;
  cplx *intaux = malloc(sizeof(cplx) * per * nq * (size_t)F);
  if (!intaux) abort();
  for (int mm = mlo; mm < mhi; mm++) {
    double qpm[13 * 3], fmv[3][13][3], fmDiv[3];
    quad_tri_points(qd, m, mm, qpm);
    double Am = m->face_area[mm];
    for (int p = 0; p < 3; p++) {
      for (int r = 0; r < nq; r++) rwg(m, qpm + 3 * r, mm, p, fmv[p][r]);
      fmDiv[p] = rwgDiv(m, mm, p);
    }
#pragma omp parallel for schedule(static)
    for (int n = 0; n < F; n++) {
      int near = near_faces(m, n, mm);
      for (int r = 0; r < nq; r++) {
        cplx *dst = intaux + ((size_t)n * nq + r) * per;
        if (op == 0) intK2(qpm + 3 * r, n, m, k, near, qd, dst);
        else if (op == 1) intK1(qpm + 3 * r, n, m, k, near, qd, dst);
        else intK4(qpm + 3 * r, n, m, k, mm, near, qd, dst);
      }
    }
    for (int n = 0; n < F; n++) {
      for (int p = 0; p < 3; p++) {
        for (int q = 0; q < 3; q++) {
          cplx int1 = 0;
          for (int r = 0; r < nq; r++) {
            const cplx *a = intaux + ((size_t)n * nq + r) * per;
            if (op == 1) {
              int1 += qd->w[r] * a[q];
            } else { /* dotc without conjugation, linalg.f90:15-21 */
              cplx dc = fmv[p][r][0] * a[3 * q] + fmv[p][r][1] * a[3 * q + 1] + fmv[p][r][2] * a[3 * q + 2];
              int1 += qd->w[r] * dc;
            }
          }
          if (op == 1) int1 = int1 * Am * fmDiv[p];
          else int1 = int1 * Am;
          int i1 = m->face_edge[3 * mm + p], i2 = m->face_edge[3 * n + q];
          cplx c = (op == 0) ? c1 * int1 : (op == 1) ? c2 * int1 : int1;
          M[i1 + (size_t)i2 * Nd] += c;
        }
      }
    }
  }
  free(intaux);
}

/* sysmat.f90:18-105 sysmat_pmchwt (identity group).  A is 2N x 2N
 * column-major with leading dimension lda; ri holds one complex refractive
 * index per domain.  Test faces [mlo, mhi) of every domain (mhi < 0: all). */
void oracle_sysmat(void *p, double omega, const double *ri_ri, cplx *A, int64_t lda, int mlo, int mhi,
                   int nthreads) {
  oproblem *P = p;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  int N = P->master.nedges;
  for (int64_t j = 0; j < 2 * (int64_t)N; j++) memset(A + j * lda, 0, sizeof(cplx) * 2 * N);
  for (int d = 0; d < P->ndom; d++) {
    omesh *m = P->dom + d;
    cplx ri = ri_ri[2 * d] + I * ri_ri[2 * d + 1];
    cplx Zsi = (ri * ri) / (O_ETA0 * O_ETA0);
    int Nd = m->nedges;
    const int *ind = m->edge_parent;
    int hi = (mhi < 0 || mhi > m->nfaces) ? m->nfaces : mhi;
    int lo = mlo < 0 ? 0 : mlo;
    if (lo > hi) lo = hi;
    cplx *M = malloc(sizeof(cplx) * (size_t)Nd * Nd);
    if (!M) abort();
    for (int op = 0; op < 3; op++) {
      compute_op(op, omega, ri, m, &P->qd, M, lo, hi);
      for (int j = 0; j < Nd; j++)
        for (int i = 0; i < Nd; i++) {
          cplx v = M[i + (size_t)j * Nd];
          int64_t r = ind[i], c = ind[j];
          if (op < 2) {
            A[r + c * lda] += v;
            A[(r + N) + (c + N) * lda] += Zsi * v;
          } else {
            A[(r + N) + c * lda] += v;
            A[r + (c + N) * lda] -= v;
          }
        }
    }
    free(M);
  }
}

/* Bounded CPU sample for timing: the D, H and K rows of test faces
 * [mlo, mhi) of every domain (the same per-pair work as oracle_sysmat, with
 * the rows kept per test face so no 2N x 2N matrix is allocated).  Returns a
 * checksum so the work cannot be elided. */
double oracle_sysmat_sample(void *p, double omega, const double *ri_ri, int mlo, int mhi, int nthreads) {
  oproblem *P = p;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  double chk = 0;
  for (int d = 0; d < P->ndom; d++) {
    omesh *m = P->dom + d;
    cplx ri = ri_ri[2 * d] + I * ri_ri[2 * d + 1];
    int hi = mhi > m->nfaces ? m->nfaces : mhi, lo = mlo < 0 ? 0 : mlo;
    if (lo >= hi) continue;
    /* rows-only variant of compute_op: a face-local row per (test face, p) */
    int Nd = m->nedges, F = m->nfaces, nq = P->qd.nq;
    cplx k = ri * omega / O_C0;
    cplx *rows = calloc((size_t)3 * (hi - lo) * Nd, sizeof(cplx));
    cplx *intaux = malloc(sizeof(cplx) * 9 * nq * (size_t)F);
    if (!rows || !intaux) abort();
    for (int op = 0; op < 3; op++) {
      size_t per = (op == 1) ? 3 : 9;
      for (int mm = lo; mm < hi; mm++) {
        double qpm[13 * 3], fmv[3][13][3];
        quad_tri_points(&P->qd, m, mm, qpm);
        for (int pp = 0; pp < 3; pp++)
          for (int r = 0; r < nq; r++) rwg(m, qpm + 3 * r, mm, pp, fmv[pp][r]);
#pragma omp parallel for schedule(static)
        for (int n = 0; n < F; n++) {
          int near = near_faces(m, n, mm);
          for (int r = 0; r < nq; r++) {
            cplx *dst = intaux + ((size_t)n * nq + r) * per;
            if (op == 0) intK2(qpm + 3 * r, n, m, k, near, &P->qd, dst);
            else if (op == 1) intK1(qpm + 3 * r, n, m, k, near, &P->qd, dst);
            else intK4(qpm + 3 * r, n, m, k, mm, near, &P->qd, dst);
          }
        }
        for (int n = 0; n < F; n++)
          for (int pp = 0; pp < 3; pp++)
            for (int q = 0; q < 3; q++) {
              cplx int1 = 0;
              for (int r = 0; r < nq; r++) {
                const cplx *a = intaux + ((size_t)n * nq + r) * per;
                if (op == 1) int1 += P->qd.w[r] * a[q];
                else int1 += P->qd.w[r] * (fmv[pp][r][0] * a[3 * q] + fmv[pp][r][1] * a[3 * q + 1] + fmv[pp][r][2] * a[3 * q + 2]);
              }
              rows[(size_t)(3 * (mm - lo) + pp) + (size_t)m->face_edge[3 * n + q] * 3 * (hi - lo)] += int1;
            }
      }
    }
    for (size_t i = 0; i < (size_t)3 * (hi - lo) * Nd; i++) chk += cabs(rows[i]);
    free(rows);
    free(intaux);
  }
  return chk;
}

/* One domain operator (D, H or K) for tests: M is N_d x N_d. */
void oracle_operator(void *p, int d, int op, double omega, const double *ri_ri, cplx *M) {
  oproblem *P = p;
  cplx ri = ri_ri[0] + I * ri_ri[1];
  compute_op(op, omega, ri, P->dom + d, &P->qd, M, 0, P->dom[d].nfaces);
}

/* ---- aux.f90:245-261 get_dir / get_pol --------------------------------- */
static void get_dir(double th, double ph, double *d) {
  d[0] = sin(th) * cos(ph);
  d[1] = sin(th) * sin(ph);
  d[2] = cos(th);
}
static void get_pol(double th, double ph, double psi, double *p) {
  p[0] = cos(psi) * sin(ph) - sin(psi) * cos(th) * cos(ph);
  p[1] = -cos(psi) * cos(ph) - sin(psi) * cos(th) * sin(ph);
  p[2] = sin(psi) * sin(th);
}

/* Source description: type 1 = pw (theta, phi, psi in radians), type 10 =
 * pw_elliptic (theta, phi in radians, complex phase).  source.f90:20-58 */
typedef struct {
  int type;
  double theta, phi, psi;
  double phase_re, phase_im;
} osrc;

/* source.f90:63-101 pw_efield / pw_hfield / pw_fields, 103-125 pw_fields_elliptic */
static void src_fields(const osrc *s, double omega, cplx ri, const double *pt, cplx *ef, cplx *hf) {
  double dir[3], pol[3];
  cplx k = ri * omega / O_C0;
  cplx dc[3];
  if (s->type != 1 && s->type != 10) { /* no source (type 0, the SH cross sections): zero fields */
    for (int i = 0; i < 3; i++) ef[i] = hf[i] = 0;
    return;
  }
  get_dir(s->theta, s->phi, dir);
  for (int i = 0; i < 3; i++) dc[i] = dir[i];
  if (s->type == 1) {
    get_pol(s->theta, s->phi, s->psi, pol);
    cplx ph = cexp(I * k * dotr(dir, pt));
    for (int i = 0; i < 3; i++) ef[i] = pol[i] * ph;
    cplx c[3];
    crossc(dc, ef, c);
    for (int i = 0; i < 3; i++) hf[i] = k / (omega * O_MU0) * c[i];
  } else {
    get_pol(s->theta, s->phi, 0.0, pol);
    cplx ph = cexp(I * k * dotr(dir, pt));
    cplx efx[3], efy[3];
    for (int i = 0; i < 3; i++) efx[i] = pol[i] * ph;
    crossc(dc, efx, efy);
    cplx phase = s->phase_re + I * s->phase_im;
    for (int i = 0; i < 3; i++) ef[i] = efx[i] + phase * efy[i];
    /* linalg.f90:37-44 normc */
    double nn = sqrt(creal(conj(ef[0]) * ef[0] + conj(ef[1]) * ef[1] + conj(ef[2]) * ef[2]));
    for (int i = 0; i < 3; i++) ef[i] = ef[i] / nn;
    cplx c[3];
    crossc(dc, ef, c);
    for (int i = 0; i < 3; i++) hf[i] = k / (omega * O_MU0) * c[i];
  }
}

/* source.f90:136-247 srcvec (identity group) on domain d's mesh.  q has 2N
 * entries (N = total edges). */
void oracle_srcvec(void *p, int d, double omega, const double *ri_ri, const osrc *src, cplx *q) {
  oproblem *P = p;
  const omesh *m = P->dom + d;
  const oquad *qd = &P->qd;
  int N = P->master.nedges, nq = qd->nq;
  cplx ri = ri_ri[0] + I * ri_ri[1];
  for (int i = 0; i < 2 * N; i++) q[i] = 0;
  for (int f = 0; f < m->nfaces; f++) {
    double qpm[13 * 3];
    quad_tri_points(qd, m, f, qpm);
    double Am = m->face_area[f];
    cplx ef[13][3], hf[13][3];
    for (int r = 0; r < nq; r++) src_fields(src, omega, ri, qpm + 3 * r, ef[r], hf[r]);
    for (int pp = 0; pp < 3; pp++) {
      cplx Ie = 0, Ih = 0;
      for (int r = 0; r < nq; r++) {
        double fm[3];
        rwg(m, qpm + 3 * r, f, pp, fm);
        Ie += qd->w[r] * (fm[0] * ef[r][0] + fm[1] * ef[r][1] + fm[2] * ef[r][2]);
        Ih += qd->w[r] * (fm[0] * hf[r][0] + fm[1] * hf[r][1] + fm[2] * hf[r][2]);
      }
      int idx = m->edge_parent[m->face_edge[3 * f + pp]];
      q[idx] += Ie * Am;
      q[idx + N] += Ih * Am;
    }
  }
}

/* cs.f90:14-104 cs_prtsrf (identity group) over domain d's mesh. */
void oracle_cs(void *p, int d, double omega, const double *ri_ri, const cplx *x, const osrc *src,
               double *csca, double *cabs) {
  oproblem *P = p;
  const omesh *m = P->dom + d;
  const oquad *qd = &P->qd;
  int N = P->master.nedges, nq = qd->nq;
  cplx ri = ri_ri[0] + I * ri_ri[1];
  double c = 2.0 / (O_EPS0 * O_C0 * creal(ri));
  double sca = 0, abs_ = 0;
  for (int f = 0; f < m->nfaces; f++) {
    double qpn[13 * 3];
    quad_tri_points(qd, m, f, qpn);
    double An = m->face_area[f];
    const double *nor = m->face_n + 3 * f;
    cplx norc[3] = {nor[0], nor[1], nor[2]};
    double int1 = 0, int2 = 0;
    for (int t = 0; t < nq; t++) {
      cplx Et[3] = {0, 0, 0}, Ht[3] = {0, 0, 0};
      for (int pp = 0; pp < 3; pp++) {
        double fr[3], fn[3];
        rwg(m, qpn + 3 * t, f, pp, fr);
        crossr(nor, fr, fn);
        int idx = m->edge_parent[m->face_edge[3 * f + pp]];
        for (int i = 0; i < 3; i++) {
          Ht[i] = Ht[i] - x[idx] * fn[i];
          Et[i] = Et[i] + x[idx + N] * fn[i];
        }
      }
      cplx einc[3], hinc[3], t1[3], Eti[3], Hti[3], Ets[3], Hts[3];
      src_fields(src, omega, ri, qpn + 3 * t, einc, hinc);
      crossc(norc, hinc, t1);
      crossc(t1, norc, Hti);
      crossc(norc, einc, t1);
      crossc(t1, norc, Eti);
      for (int i = 0; i < 3; i++) { Hts[i] = Ht[i] - Hti[i]; Ets[i] = Et[i] - Eti[i]; }
      cplx ch[3] = {conj(Ht[0]), conj(Ht[1]), conj(Ht[2])}, cr[3];
      crossc(Et, ch, cr);
      double Sn = 0.5 * creal(cr[0] * norc[0] + cr[1] * norc[1] + cr[2] * norc[2]);
      int1 += qd->w[t] * Sn;
      cplx chs[3] = {conj(Hts[0]), conj(Hts[1]), conj(Hts[2])};
      crossc(Ets, chs, cr);
      Sn = 0.5 * creal(cr[0] * norc[0] + cr[1] * norc[1] + cr[2] * norc[2]);
      int2 += qd->w[t] * Sn;
    }
    abs_ += int1 * An;
    sca += int2 * An;
  }
  *cabs = -c * abs_;
  *csca = c * sca;
}

/* ffields.f90:16-122 far_fields (identity group) at distance r. */
static void far_fields(const oproblem *P, int d, double omega, cplx ri, const cplx *x, double r, double theta,
                       double phi, cplx *et, cplx *ep) {
  const omesh *m = P->dom + d;
  const oquad *qd = &P->qd;
  int N = P->master.nedges, nq = qd->nq;
  double st = sin(theta), ct = cos(theta), sp = sin(phi), cp = cos(phi);
  cplx k = ri * omega / O_C0;
  cplx Nt = 0, Np = 0, Lt = 0, Lp = 0;
  for (int f = 0; f < m->nfaces; f++) {
    double An = m->face_area[f], qpn[13 * 3];
    quad_tri_points(qd, m, f, qpn);
    for (int q = 0; q < 3; q++) {
      int idx = m->edge_parent[m->face_edge[3 * f + q]];
      cplx q1 = 0, q2 = 0, q3 = 0, q4 = 0;
      for (int t = 0; t < nq; t++) {
        const double *rp = qpn + 3 * t;
        double jg[3];
        rwg(m, rp, f, q, jg);
        cplx jn[3], mn[3];
        for (int i = 0; i < 3; i++) { jn[i] = jg[i] * x[idx]; mn[i] = jg[i] * x[idx + N]; }
        cplx phasor = cexp(-I * k * (rp[0] * st * cp + rp[1] * st * sp + rp[2] * ct));
        q1 += qd->w[t] * (ct * cp * jn[0] + ct * sp * jn[1] - st * jn[2]) * phasor;
        q2 += qd->w[t] * (-sp * jn[0] + cp * jn[1]) * phasor;
        q3 += qd->w[t] * (ct * cp * mn[0] + ct * sp * mn[1] - st * mn[2]) * phasor;
        q4 += qd->w[t] * (-sp * mn[0] + cp * mn[1]) * phasor;
      }
      Nt += q1 * An;
      Np += q2 * An;
      Lt += q3 * An;
      Lp += q4 * An;
    }
  }
  cplx prefix = I * k * cexp(I * k * r) / (4.0 * O_PI * r);
  *et = prefix * (Lp + O_ETA0 / ri * Nt);
  *ep = -prefix * (Lt - O_ETA0 / ri * Np);
}

/* ffields.f90:203-266 rcs_ext / rcs (no polarisation filter).  rcs is
 * ntheta x nphi column-major, as the reference's rcsdata(1:ntheta,1:nphi). */
void oracle_rcs(void *p, int d, double omega, const double *ri_ri, const cplx *x, int ntheta, int nphi,
                double *rcs, int nthreads) {
  oproblem *P = p;
  cplx ri = ri_ri[0] + I * ri_ri[1];
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int n = 0; n < ntheta; n++)
    for (int mm = 0; mm < nphi; mm++) {
      double theta = O_PI * (double)n / (double)(ntheta - 1);
      double phi = 2.0 * O_PI * (double)mm / (double)(nphi - 1);
      cplx et, ep;
      far_fields(P, d, omega, ri, x, 1.0, theta, phi, &et, &ep);
      double a = cabs(et), b = cabs(ep);
      rcs[n + (size_t)mm * ntheta] = a * a + b * b;
    }
}

/* srcint.f90:264-325 intK3 with 227-260 intK3singular (identity group,
 * non-periodic): int_T grad'G div'f_e dS' for the three RWG functions of
 * face f; res[3 edges][3]. */
static void intK3(const double *r, int f, const omesh *m, cplx k, int near, const oquad *qd, cplx *res) {
  double qpn[13 * 3];
  double An = m->face_area[f];
  quad_tri_points(qd, m, f, qpn);
  cplx tmp[3] = {0, 0, 0};
  for (int t = 0; t < qd->nq; t++) {
    cplx g[3];
    gradG_or_s(r, qpn + 3 * t, k, near, g);
    for (int i = 0; i < 3; i++) tmp[i] += g[i] * qd->w[t];
  }
  for (int i = 0; i < 3; i++) tmp[i] *= An;
  cplx sing[3] = {0, 0, 0};
  if (near) {
    double km1[3], k1[3];
    intK3m1(r, f, m, km1);
    intK31(r, f, m, k1);
    for (int i = 0; i < 3; i++) sing[i] = 1.0 / (4.0 * O_PI) * km1[i] - (k * k) / (8.0 * O_PI) * k1[i];
  }
  for (int e = 0; e < 3; e++) {
    double divfn = rwgDiv(m, f, e);
    for (int i = 0; i < 3; i++) res[3 * e + i] = tmp[i] * divfn + sing[i] * divfn;
  }
}

/* Scattered fields of the surface currents of domain d at points
 * (nfields.f90:29-49 scat_fields with 109-197 scat_fields_frags, identity
 * group: one fragment, group factors 1): per face the integrals intK2,
 * intK3, intK4 (no test face), singular parts when the point is within three
 * average edge lengths of the face centroid.  With addsrc the incident field
 * of each source is added (field_plane, nfpost.f90:316-374, does so in the
 * exterior domain).  x: [nsrc][ldx] (J in 0..N-1, M in N..2N-1); pts[npts][3];
 * e, h: [nsrc][npts][3]. */
void oracle_scat_fields(void *p, int d, double omega, const double *ri_ri, int nsrc, const cplx *x, int64_t ldx,
                        const osrc *src, int addsrc, int npts, const double *pts, cplx *e, cplx *h) {
  oproblem *P = p;
  const omesh *m = P->dom + d;
  const oquad *qd = &P->qd;
  const int N = P->master.nedges;
  const cplx ri = ri_ri[0] + I * ri_ri[1];
  const cplx k = ri * omega / O_C0;
  const double thr2 = (m->avelen * 3) * (m->avelen * 3);
  const cplx c1 = I * omega * O_MU0;
  const cplx c2 = 1.0 / (I * omega * O_EPS0 * (ri * ri));
  for (int ip = 0; ip < npts; ip++) {
    const double *r = pts + 3 * ip;
    for (int s = 0; s < nsrc; s++)
      for (int i = 0; i < 3; i++) e[((size_t)s * npts + ip) * 3 + i] = h[((size_t)s * npts + ip) * 3 + i] = 0;
    for (int f = 0; f < m->nfaces; f++) {
      const double *cp = m->face_cp + 3 * f;
      double df[3] = {r[0] - cp[0], r[1] - cp[1], r[2] - cp[2]};
      int near = dotr(df, df) < thr2;
      cplx k2[9], k3[9], k4[9];
      intK2(r, f, m, k, near, qd, k2);
      intK3(r, f, m, k, near, qd, k3);
      intK4(r, f, m, k, -1, near, qd, k4);
      for (int q = 0; q < 3; q++) {
        int idx = m->edge_parent[m->face_edge[3 * f + q]];
        for (int s = 0; s < nsrc; s++) {
          cplx xj = x[(size_t)s * ldx + idx], xm = x[(size_t)s * ldx + idx + N];
          cplx *es = e + ((size_t)s * npts + ip) * 3, *hs = h + ((size_t)s * npts + ip) * 3;
          for (int i = 0; i < 3; i++) {
            es[i] += xj * (c1 * k2[3 * q + i] + c2 * k3[3 * q + i]) + xm * k4[3 * q + i];
            hs[i] += xm * (k2[3 * q + i] / c2 + k3[3 * q + i] / c1) - xj * k4[3 * q + i];
          }
        }
      }
    }
    if (addsrc)
      for (int s = 0; s < nsrc; s++) {
        cplx einc[3], hinc[3];
        src_fields(src + s, omega, ri, r, einc, hinc);
        for (int i = 0; i < 3; i++) {
          e[((size_t)s * npts + ip) * 3 + i] += einc[i];
          h[((size_t)s * npts + ip) * 3 + i] += hinc[i];
        }
      }
  }
}

/* ==== Symmetry groups (symmetry.f90, bc.f90; the nga > 1 parts of
 * sysmat.f90, source.f90 and cs.f90), mirror planes only ==== */

/* symmetry.f90:45-58 group_id, 60-103 group_mp */
static void ga_identity(ogact *g) {
  memset(g, 0, sizeof *g);
  g->j[0] = g->j[4] = g->j[8] = 1.0;
  g->detj = 1.0;
  g->id = O_GID_IDENTITY;
  g->genbits = 1 << O_GID_IDENTITY;
  g->ef[0] = 1.0;
}
static void ga_mirror(int np, ogact *g /* [2] */) {
  ga_identity(g);
  g[0].ef[1] = 1.0;
  memset(g + 1, 0, sizeof *g);
  g[1].j[0] = g[1].j[4] = g[1].j[8] = 1.0;
  g[1].j[4 * (np - 1)] = -1.0;
  g[1].detj = -1.0;
  g[1].ef[0] = 1.0;
  g[1].ef[1] = -1.0;
  g[1].id = np == 1 ? O_GID_MXP : np == 2 ? O_GID_MYP : O_GID_MZP;
  g[1].genbits = 1 << g[1].id;
}

/* symmetry.f90:178-241 product_group: element k = n nb + m is a_n b_m;
 * field actions multiply likewise. */
static int ga_product(ogact *a, int na, const ogact *b, int nb) {
  if (na * nb > O_MAXGA) return -1;
  ogact *t = xcalloc((size_t)na * nb, sizeof(ogact));
  for (int n = 0; n < na; n++)
    for (int m = 0; m < nb; m++) {
      ogact *g = t + n * nb + m;
      for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) {
          double v = 0;
          for (int l = 0; l < 3; l++) v += a[n].j[3 * i + l] * b[m].j[3 * l + k];
          g->j[3 * i + k] = v;
        }
      g->detj = a[n].detj * b[m].detj;
      g->genbits = a[n].genbits | b[m].genbits;
      g->id = 0;
      if (a[n].id == O_GID_IDENTITY && b[m].id == O_GID_IDENTITY) g->id = O_GID_IDENTITY;
      else if (a[n].id != 0 && a[n].id != O_GID_IDENTITY && b[m].id == O_GID_IDENTITY) g->id = a[n].id;
      else if (b[m].id != 0 && b[m].id != O_GID_IDENTITY && a[n].id == O_GID_IDENTITY) g->id = b[m].id;
      for (int n2 = 0; n2 < na; n2++)
        for (int m2 = 0; m2 < nb; m2++) g->ef[n2 * nb + m2] = a[n].ef[n2] * b[m].ef[m2];
    }
  memcpy(a, t, sizeof(ogact) * (size_t)na * nb);
  free(t);
  return na * nb;
}

/* interface.f90:160-210 read_symm: the product of the named groups, starting
 * from the identity.  Names: "id", "mxp", "myp", "mzp" (the rotation groups
 * rN of the reference are not restated).  Returns the group order or < 0. */
int oracle_problem_set_symmetry(void *p, int nnames, const char *const *names) {
  oproblem *P = p;
  ogact *g = P->ga;
  ga_identity(g);
  int n = 1;
  for (int i = 0; i < nnames; i++) {
    ogact two[2];
    if (!strcmp(names[i], "id")) {
      ga_identity(two);
      n = ga_product(g, n, two, 1);
    } else if (!strcmp(names[i], "mxp") || !strcmp(names[i], "myp") || !strcmp(names[i], "mzp")) {
      ga_mirror(names[i][1] - 'w', two);
      n = ga_product(g, n, two, 2);
    } else {
      return -1;
    }
    if (n < 0) return -2;
  }
  P->nga = n;
  return n;
}

/* Group of the problem for tests: j [nga][9] (row-major), detj, ef [nga][nga]
 * (ef[a * nga + r] = field action of element a in representation r). */
void oracle_group_info(void *p, double *j, double *detj, cplx *ef) {
  oproblem *P = p;
  for (int a = 0; a < P->nga; a++) {
    memcpy(j + 9 * a, P->ga[a].j, 9 * sizeof(double));
    detj[a] = P->ga[a].detj;
    for (int r = 0; r < P->nga; r++) ef[a * P->nga + r] = P->ga[a].ef[r];
  }
}

/* mesh.f90:155-175 classify_edges: master edges whose end nodes match a
 * line (0-based master node pair) get boundary type bnd; domain edges take
 * the type of their master edge (mesh.f90:434). */
int oracle_problem_classify_edges(void *p, int nlines, const int *line_nodes, int bnd) {
  oproblem *P = p;
  omesh *ms = &P->master;
  int cnt = 0;
  for (int e = 0; e < ms->nedges; e++)
    for (int l = 0; l < nlines; l++)
      if (cmp_pairs(ms->edge_node + 2 * e, line_nodes + 2 * l)) {
        P->mbnd[e] = bnd;
        cnt++;
      }
  for (int d = 0; d < P->ndom; d++)
    for (int e = 0; e < P->dom[d].nedges; e++) P->dbnd[d][e] = P->mbnd[P->dom[d].edge_parent[e]];
  return cnt;
}

static int has_bnd(const oproblem *P, int d, int bnd) {
  for (int e = 0; e < P->dom[d].nedges; e++)
    if (P->dbnd[d][e] == bnd) return 1;
  return 0;
}

/* bc.f90:237-257 admissible_ga */
static int admissible_ga(const oproblem *P, int d, const ogact *g) {
  if (d == 0) return 1;
  if ((g->genbits >> O_GID_MXP & 1) && !has_bnd(P, d, O_BND_XPLANE)) return 0;
  if ((g->genbits >> O_GID_MYP & 1) && !has_bnd(P, d, O_BND_YPLANE)) return 0;
  if ((g->genbits >> O_GID_MZP & 1) && !has_bnd(P, d, O_BND_ZPLANE)) return 0;
  return 1;
}

/* bc.f90:28-117 edge_bc (mirror planes): for representation nr, id[k] = -1
 * removes coefficient k (J: k < N, M: k >= N) when the field action of a
 * mirror element on a boundary edge of its plane is not -1 (for M the action
 * times det J).  Returns the number of removed coefficients. */
int oracle_edge_bc(void *p, int nr, int *id, cplx *phase) {
  oproblem *P = p;
  int N = P->master.nedges, cnt = 0;
  for (int k = 0; k < 2 * N; k++) {
    id[k] = 0;
    phase[k] = 1.0;
  }
  for (int k = 0; k < N; k++) {
    int bnd = P->mbnd[k];
    for (int n = 0; n < P->nga; n++) {
      const ogact *g = P->ga + n;
      cplx gae = g->ef[nr], gah = g->ef[nr] * g->detj;
      if ((g->id == O_GID_MXP && bnd == O_BND_XPLANE) || (g->id == O_GID_MYP && bnd == O_BND_YPLANE) ||
          (g->id == O_GID_MZP && bnd == O_BND_ZPLANE)) {
        if (creal(-gae) < 0.99) id[k] = -1;
        if (creal(-gah) < 0.99) id[k + N] = -1;
      }
    }
  }
  for (int k = 0; k < 2 * N; k++) cnt += id[k] == -1;
  return cnt;
}

/* J^T r, J v (real) and J v (complex) */
static void jt_vec(const double *j, const double *r, double *o) {
  for (int i = 0; i < 3; i++) o[i] = j[i] * r[0] + j[3 + i] * r[1] + j[6 + i] * r[2];
}
static void j_cvec(const double *j, const cplx *v, cplx *o) {
  for (int i = 0; i < 3; i++) o[i] = j[3 * i] * v[0] + j[3 * i + 1] * v[1] + j[3 * i + 2] * v[2];
}

/* srcint.f90 with a group action g (orthogonal J): the source face mapped by
 * J seen from r equals the face itself seen from J^T r, so
 *   intK1_g(r) = intK1(J^T r),  intK2_g(r) = J intK2(J^T r),
 *   intK4_g(r) = det J  J intK4(J^T r)      ((J a) x (J b) = det J  J (a x b)),
 * the singular parts included (srcint.f90:97-117, 208-223, 418-447). */
static void intK1_g(const double *r, int f, const omesh *m, cplx k, const ogact *g, int near, const oquad *qd,
                    cplx *res) {
  if (g->id == O_GID_IDENTITY) {
    intK1(r, f, m, k, near, qd, res);
    return;
  }
  double rt[3];
  jt_vec(g->j, r, rt);
  intK1(rt, f, m, k, near, qd, res);
}
static void intK2_g(const double *r, int f, const omesh *m, cplx k, const ogact *g, int near, const oquad *qd,
                    cplx *res) {
  if (g->id == O_GID_IDENTITY) {
    intK2(r, f, m, k, near, qd, res);
    return;
  }
  double rt[3];
  cplx t[9];
  jt_vec(g->j, r, rt);
  intK2(rt, f, m, k, near, qd, t);
  for (int e = 0; e < 3; e++) j_cvec(g->j, t + 3 * e, res + 3 * e);
}
static void intK4_g(const double *r, int f, const omesh *m, cplx k, const ogact *g, int tface, int near,
                    const oquad *qd, cplx *res) {
  if (g->id == O_GID_IDENTITY) { /* the self-face shortcut holds for the identity only */
    intK4(r, f, m, k, tface, near, qd, res);
    return;
  }
  double rt[3];
  cplx t[9];
  jt_vec(g->j, r, rt);
  intK4(rt, f, m, k, -1, near, qd, t);
  for (int e = 0; e < 3; e++) {
    j_cvec(g->j, t + 3 * e, res + 3 * e);
    for (int i = 0; i < 3; i++) res[3 * e + i] *= g->detj;
  }
}

/* sysmat.f90:233-260 near_faces: |cp_m - J cp_n| < 3 avelen */
static int near_faces_g(const omesh *m, int n, int mm, const ogact *g) {
  double threshold = m->avelen * 3, jc[3], d[3];
  const double *c = m->face_cp + 3 * n;
  for (int i = 0; i < 3; i++) jc[i] = g->j[3 * i] * c[0] + g->j[3 * i + 1] * c[1] + g->j[3 * i + 2] * c[2];
  for (int i = 0; i < 3; i++) d[i] = m->face_cp[3 * mm + i] - jc[i];
  return d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < threshold * threshold;
}

/* compute_op for one group action (sysmat.f90:272-519 with ga) */
static void compute_op_g(int op, double omega, cplx ri, const omesh *m, const oquad *qd, const ogact *g, cplx *M) {
  int Nd = m->nedges, F = m->nfaces, nq = qd->nq;
  memset(M, 0, sizeof(cplx) * (size_t)Nd * Nd);
  cplx k = ri * omega / O_C0;
  cplx c1 = -I * omega * O_MU0;
  cplx c2 = -1.0 / (I * omega * O_EPS0 * (ri * ri));
  size_t per = (op == 1) ? 3 : 9;
  cplx *intaux = malloc(sizeof(cplx) * per * nq * (size_t)F);
  if (!intaux) abort();
  for (int mm = 0; mm < F; mm++) {
    double qpm[13 * 3], fmv[3][13][3], fmDiv[3];
    quad_tri_points(qd, m, mm, qpm);
    double Am = m->face_area[mm];
    for (int pq = 0; pq < 3; pq++) {
      for (int r = 0; r < nq; r++) rwg(m, qpm + 3 * r, mm, pq, fmv[pq][r]);
      fmDiv[pq] = rwgDiv(m, mm, pq);
    }
#pragma omp parallel for schedule(static)
    for (int n = 0; n < F; n++) {
      int near = near_faces_g(m, n, mm, g);
      for (int r = 0; r < nq; r++) {
        cplx *dst = intaux + ((size_t)n * nq + r) * per;
        if (op == 0) intK2_g(qpm + 3 * r, n, m, k, g, near, qd, dst);
        else if (op == 1) intK1_g(qpm + 3 * r, n, m, k, g, near, qd, dst);
        else intK4_g(qpm + 3 * r, n, m, k, g, mm, near, qd, dst);
      }
    }
    for (int n = 0; n < F; n++)
      for (int pp = 0; pp < 3; pp++)
        for (int q = 0; q < 3; q++) {
          cplx int1 = 0;
          for (int r = 0; r < nq; r++) {
            const cplx *a = intaux + ((size_t)n * nq + r) * per;
            if (op == 1) int1 += qd->w[r] * a[q];
            else int1 += qd->w[r] * (fmv[pp][r][0] * a[3 * q] + fmv[pp][r][1] * a[3 * q + 1] + fmv[pp][r][2] * a[3 * q + 2]);
          }
          int1 = (op == 1) ? int1 * Am * fmDiv[pp] : int1 * Am;
          int i1 = m->face_edge[3 * mm + pp], i2 = m->face_edge[3 * n + q];
          M[i1 + (size_t)i2 * Nd] += (op == 0) ? c1 * int1 : (op == 1) ? c2 * int1 : int1;
        }
  }
  free(intaux);
}

/* sysmat.f90:18-105 sysmat_pmchwt with the problem's group: one 2N x 2N
 * matrix per representation, A[nf] at A + nf (2N)^2 (column-major); the
 * blocks of domain `dom` alone when dom >= 0 (sysmat_pmchwt_nls needs the
 * nonlinear domain's blocks apart, sysmat.f90:112-229). */
void oracle_sysmat_sym_dom(void *p, double omega, const double *ri_ri, cplx *A, int nthreads, int dom) {
  oproblem *P = p;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const int N = P->master.nedges, nga = P->nga;
  const size_t n2 = 2 * (size_t)N;
  memset(A, 0, sizeof(cplx) * n2 * n2 * nga);
  for (int d = 0; d < P->ndom; d++) {
    if (dom >= 0 && d != dom) continue;
    omesh *m = P->dom + d;
    cplx ri = ri_ri[2 * d] + I * ri_ri[2 * d + 1];
    cplx Zsi = (ri * ri) / (O_ETA0 * O_ETA0);
    const int Nd = m->nedges, *ind = m->edge_parent;
    cplx *M = malloc(sizeof(cplx) * (size_t)Nd * Nd);
    if (!M) abort();
    for (int ns = 0; ns < nga; ns++) {
      const ogact *g = P->ga + ns;
      if (!admissible_ga(P, d, g)) continue;
      for (int op = 0; op < 3; op++) {
        compute_op_g(op, omega, ri, m, &P->qd, g, M);
        for (int nf = 0; nf < nga; nf++) {
          cplx gae = g->ef[nf], *Af = A + (size_t)nf * n2 * n2;
          for (int jj = 0; jj < Nd; jj++)
            for (int i = 0; i < Nd; i++) {
              cplx v = gae * M[i + (size_t)jj * Nd];
              size_t r = ind[i], c = ind[jj];
              if (op < 2) {
                Af[r + c * n2] += v;
                Af[(r + N) + (c + N) * n2] += g->detj * Zsi * v;
              } else {
                Af[(r + N) + c * n2] += v;
                Af[r + (c + N) * n2] -= g->detj * v;
              }
            }
        }
      }
    }
    free(M);
  }
}

void oracle_sysmat_sym(void *p, double omega, const double *ri_ri, cplx *A, int nthreads) {
  oracle_sysmat_sym_dom(p, omega, ri_ri, A, nthreads, -1);
}

/* source.f90:250-315 src_field_frags: the source at J^T pt for each element,
 * projected on the representations; ef, hf [nga][3]. */
static void src_field_frags(const oproblem *P, const osrc *s, double omega, cplx ri, const double *pt, cplx *ef,
                            cplx *hf) {
  const int nga = P->nga;
  for (int i = 0; i < 3 * nga; i++) ef[i] = hf[i] = 0;
  for (int na = 0; na < nga; na++) {
    const ogact *g = P->ga + na;
    double pp[3];
    cplx e[3], h[3], je[3], jh[3];
    jt_vec(g->j, pt, pp);
    src_fields(s, omega, ri, pp, e, h);
    j_cvec(g->j, e, je);
    j_cvec(g->j, h, jh);
    for (int nr = 0; nr < nga; nr++)
      for (int i = 0; i < 3; i++) {
        ef[3 * nr + i] += je[i] * g->ef[nr];
        hf[3 * nr + i] += jh[i] * g->ef[nr] * g->detj;
      }
  }
  for (int i = 0; i < 3 * nga; i++) {
    ef[i] /= nga;
    hf[i] /= nga;
  }
}

/* source.f90:136-247 srcvec with the group: q[nr] (2N each) on domain 0. */
void oracle_srcvec_sym(void *p, double omega, const double *ri_ri, const osrc *src, cplx *q) {
  oproblem *P = p;
  const omesh *m = P->dom;
  const oquad *qd = &P->qd;
  const int N = P->master.nedges, nq = qd->nq, nga = P->nga;
  cplx ri = ri_ri[0] + I * ri_ri[1];
  for (size_t i = 0; i < 2 * (size_t)N * nga; i++) q[i] = 0;
  cplx *ef = xcalloc((size_t)3 * nga * nq, sizeof(cplx)), *hf = xcalloc((size_t)3 * nga * nq, sizeof(cplx));
  for (int f = 0; f < m->nfaces; f++) {
    double qpm[13 * 3];
    quad_tri_points(qd, m, f, qpm);
    double Am = m->face_area[f];
    for (int r = 0; r < nq; r++)
      src_field_frags(P, src, omega, ri, qpm + 3 * r, ef + (size_t)3 * nga * r, hf + (size_t)3 * nga * r);
    for (int pp = 0; pp < 3; pp++) {
      int idx = m->edge_parent[m->face_edge[3 * f + pp]];
      for (int nr = 0; nr < nga; nr++) {
        cplx Ie = 0, Ih = 0;
        for (int r = 0; r < nq; r++) {
          double fm[3];
          rwg(m, qpm + 3 * r, f, pp, fm);
          const cplx *e = ef + (size_t)3 * nga * r + 3 * nr, *h = hf + (size_t)3 * nga * r + 3 * nr;
          Ie += qd->w[r] * (fm[0] * e[0] + fm[1] * e[1] + fm[2] * e[2]);
          Ih += qd->w[r] * (fm[0] * h[0] + fm[1] * h[1] + fm[2] * h[2]);
        }
        q[(size_t)nr * 2 * N + idx] += Ie * Am;
        q[(size_t)nr * 2 * N + idx + N] += Ih * Am;
      }
    }
  }
  free(ef);
  free(hf);
}

/* cs.f90:14-104 cs_prtsrf with the group, over domain d's mesh: x holds the
 * solution of every representation for one source, x[nf] at x + nf 2N. */
void oracle_cs_sym(void *p, int d, double omega, const double *ri_ri, const cplx *x, const osrc *src,
                   double *csca, double *cabs) {
  oproblem *P = p;
  const omesh *m = P->dom + d;
  const oquad *qd = &P->qd;
  const int N = P->master.nedges, nq = qd->nq, nga = P->nga;
  cplx ri = ri_ri[0] + I * ri_ri[1];
  double c = 2.0 / (O_EPS0 * O_C0 * creal(ri));
  double sca = 0, abs_ = 0;
  for (int f = 0; f < m->nfaces; f++) {
    double qpn[13 * 3];
    quad_tri_points(qd, m, f, qpn);
    double An = m->face_area[f];
    const double *n0 = m->face_n + 3 * f;
    double int1 = 0, int2 = 0;
    for (int t = 0; t < nq; t++) {
      for (int ns = 0; ns < nga; ns++) {
        const ogact *g = P->ga + ns;
        cplx Et[3] = {0, 0, 0}, Ht[3] = {0, 0, 0};
        double nor[3];
        for (int i = 0; i < 3; i++) nor[i] = g->j[3 * i] * n0[0] + g->j[3 * i + 1] * n0[1] + g->j[3 * i + 2] * n0[2];
        for (int nf = 0; nf < nga; nf++) {
          cplx gae = g->ef[nf];
          for (int pp = 0; pp < 3; pp++) {
            double fr[3], fn0[3], fn[3];
            rwg(m, qpn + 3 * t, f, pp, fr);
            crossr(n0, fr, fn0);
            for (int i = 0; i < 3; i++) fn[i] = g->j[3 * i] * fn0[0] + g->j[3 * i + 1] * fn0[1] + g->j[3 * i + 2] * fn0[2];
            int idx = m->edge_parent[m->face_edge[3 * f + pp]];
            cplx xj = x[(size_t)nf * 2 * N + idx], xm = x[(size_t)nf * 2 * N + idx + N];
            for (int i = 0; i < 3; i++) {
              Ht[i] -= xj * fn[i] * gae * g->detj;
              Et[i] += xm * fn[i] * gae;
            }
          }
        }
        double pt[3];
        for (int i = 0; i < 3; i++)
          pt[i] = g->j[3 * i] * qpn[3 * t] + g->j[3 * i + 1] * qpn[3 * t + 1] + g->j[3 * i + 2] * qpn[3 * t + 2];
        cplx einc[3], hinc[3], norc[3] = {nor[0], nor[1], nor[2]}, t1[3], Eti[3], Hti[3], Ets[3], Hts[3];
        src_fields(src, omega, ri, pt, einc, hinc);
        crossc(norc, hinc, t1);
        crossc(t1, norc, Hti);
        crossc(norc, einc, t1);
        crossc(t1, norc, Eti);
        for (int i = 0; i < 3; i++) {
          Hts[i] = Ht[i] - Hti[i];
          Ets[i] = Et[i] - Eti[i];
        }
        cplx ch[3], cx[3];
        cplx Hc[3] = {conj(Ht[0]), conj(Ht[1]), conj(Ht[2])};
        crossc(Et, Hc, ch);
        int1 += qd->w[t] * 0.5 * creal(ch[0] * nor[0] + ch[1] * nor[1] + ch[2] * nor[2]);
        cplx Hsc[3] = {conj(Hts[0]), conj(Hts[1]), conj(Hts[2])};
        crossc(Ets, Hsc, cx);
        int2 += qd->w[t] * 0.5 * creal(cx[0] * nor[0] + cx[1] * nor[1] + cx[2] * nor[2]);
      }
    }
    abs_ += int1 * An;
    sca += int2 * An;
  }
  *cabs = -c * abs_;
  *csca = c * sca;
}

/* Single-point access to the kernels for unit tests.  which: 1 = intK1,
 * 2 = intK2, 4 = intK4; res holds 3 (intK1) or 9 complex values. */
void oracle_srcint(void *p, int d, int which, const double *r, int f, int tface, const double *k_ri, int near,
                   cplx *res) {
  oproblem *P = p;
  cplx k = k_ri[0] + I * k_ri[1];
  const omesh *m = P->dom + d;
  if (which == 1) intK1(r, f, m, k, near, &P->qd, res);
  else if (which == 2) intK2(r, f, m, k, near, &P->qd, res);
  else intK4(r, f, m, k, tface, near, &P->qd, res);
}

/* The closed-form static integrals over face f of domain d at point r:
 * out[0..2] = intK2m1 (edge e), out[3..5] = intK21, out[6..8] = intK4m1,
 * out[9..11] = intK41, out[12] = intK1m1, out[13] = intK11. */
void oracle_static_integrals(void *p, int d, const double *r, int f, int e, double *out) {
  oproblem *P = p;
  const omesh *m = P->dom + d;
  intK2x(r, f, e, m, 1, out);
  intK2x(r, f, e, m, 0, out + 3);
  intK4x(r, f, e, m, 1, out + 6);
  intK4x(r, f, e, m, 0, out + 9);
  out[12] = intK1m1(r, f, e, m);
  out[13] = intK11(r, f, e, m);
}

/* Quadrature points of face f of domain d (for numerical cross-checks). */
void oracle_face_geometry(void *p, int d, int f, double *nodes9, double *area, int *sign3, double *len3,
                          double *bnode9) {
  oproblem *P = p;
  const omesh *m = P->dom + d;
  for (int k = 0; k < 3; k++) {
    memcpy(nodes9 + 3 * k, m->node + 3 * m->face_node[3 * f + k], 3 * sizeof(double));
    sign3[k] = (int)get_face_sign(m, f, k);
    len3[k] = m->edge_len[m->face_edge[3 * f + k]];
    memcpy(bnode9 + 3 * k, get_face_bnode(m, f, k), 3 * sizeof(double));
  }
  *area = m->face_area[f];
}

double oracle_pi(void) { return O_PI; }
