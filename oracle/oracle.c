/*
 * oracle.c -- CPU restatement of exFEMuS's element assembly + geometric multigrid.
 *
 * TEST INFRASTRUCTURE ONLY: used as the checker by tests/, __graft_entry__.smoke()
 * and the cpu_baseline leg of bench.py.  Never linked into the product library.
 *
 * Every function cites the reference file:line it restates.  Conventions that the
 * reference leaves to libMesh/gencase (node and element order of a structured
 * hierarchy) are fixed here and restated identically by the product's host code:
 *   - lattice: the top level's Q2 nodes sit on an integer lattice (I,J,K);
 *   - node order: class-major (class 0 = level-0 vertices, class l+1 = nodes new on
 *     level l), then K, J, I lexicographic.  This realises the nesting the reference
 *     relies on: level-L Q2 nodes are a prefix, and the Q1 nodes of level L are the
 *     Q2 nodes of level L-1 (src/MGSolverDA.C:895-897);
 *   - element order per level: (ez, ey, ex) lexicographic; element colour
 *     (ex&1)|(ey&1)<<1|(ez&1)<<2;
 *   - local node order: libMesh Quad9/Hex27 (src/MGFE.C:195-370 shape order,
 *     include/MGGeomEl.h surface topology src/MGGeomEl.C:172-177,310-317);
 *   - sparse rows: column-sorted, the order LASPACK's Q_SortEl gives a row before
 *     its first product (contrib/laspack/operats.c:813).
 */
#include "oracle.h"

#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <stdlib.h>
#include <string.h>

#define MAXEN 27
#define MAXVX 8

/* libMesh local-node lattice offsets (a,b,c in half-element units). */
static const int Q9_ABC[9][3] = {{0, 0, 0}, {2, 0, 0}, {2, 2, 0}, {0, 2, 0}, {1, 0, 0},
                                 {2, 1, 0}, {1, 2, 0}, {0, 1, 0}, {1, 1, 0}};
static const int H27_ABC[27][3] = {
    {0, 0, 0}, {2, 0, 0}, {2, 2, 0}, {0, 2, 0}, {0, 0, 2}, {2, 0, 2}, {2, 2, 2}, {0, 2, 2},
    {1, 0, 0}, {2, 1, 0}, {1, 2, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 1}, {2, 2, 1}, {0, 2, 1},
    {1, 0, 2}, {2, 1, 2}, {1, 2, 2}, {0, 1, 2}, {1, 1, 0}, {1, 0, 1}, {2, 1, 1}, {1, 2, 1},
    {0, 1, 1}, {1, 1, 2}, {1, 1, 1}};
/* side -> local nodes; the side's last node is its midpoint/centre
 * (include/MGGeomEl.h:39-51 with src/MGGeomEl.C:172-177 and :310-317). */
static const int Q9_SIDE[4][3] = {{0, 1, 4}, {1, 2, 5}, {2, 3, 6}, {3, 0, 7}};
static const int H27_FACE[6][9] = {{0, 1, 2, 3, 8, 9, 10, 11, 20},  {0, 1, 5, 4, 8, 13, 16, 12, 21},
                                   {1, 2, 6, 5, 9, 14, 17, 13, 22}, {2, 3, 7, 6, 10, 15, 18, 14, 23},
                                   {3, 0, 4, 7, 11, 12, 19, 15, 24}, {4, 5, 6, 7, 16, 17, 18, 19, 25}};
/* neighbour offset and outward normal axis/sign of each side */
static const int Q9_SIDE_DIR[4][3] = {{0, -1, 0}, {1, 0, 0}, {0, 1, 0}, {-1, 0, 0}};
static const int H27_FACE_DIR[6][3] = {{0, 0, -1}, {0, -1, 0}, {1, 0, 0}, {0, 1, 0}, {-1, 0, 0}, {0, 0, 1}};

static const int *local_abc(int dim, int k) { return dim == 2 ? Q9_ABC[k] : H27_ABC[k]; }

/* ====================================================================== mesh */
struct or_mesh {
  int dim, nlev, nen, nvx, nsides, nsn;
  int n0[3];
  int L[3];          /* top lattice extents (2*n_top+1, 1 in z for 2D) */
  int ntop;          /* top nodes */
  int nvert0;
  int *nnodes;       /* [nlev] */
  int *nel;          /* [nlev] */
  int *lat;          /* [ntop*3] */
  double *xyz;       /* [dim*ntop] component-major (reference _xyz layout) */
  int *node_of_lat;  /* lattice index -> node */
  int **conn, **neigh, **ecol; /* per level */
  int **eabc;        /* per level: element lattice index (ex,ey,ez) */
};

static int node_class(const or_mesh *m, const int *p) {
  /* class 0: vertices of level 0; class l+1: first appears on level l. */
  int s0 = 1 << (m->nlev - 1);
  int is_v0 = 1;
  for (int d = 0; d < 3; d++)
    if (p[d] % (2 * s0)) is_v0 = 0;
  if (is_v0) return 0;
  for (int l = 0; l < m->nlev; l++) {
    int s = 1 << (m->nlev - 1 - l), ok = 1;
    for (int d = 0; d < 3; d++)
      if (p[d] % s) ok = 0;
    if (ok) return l + 1;
  }
  return m->nlev;
}

or_mesh *or_mesh_new(int dim, int nlev, const int n0[3], const double box[6]) {
  or_mesh *m = (or_mesh *)calloc(1, sizeof(or_mesh));
  m->dim = dim;
  m->nlev = nlev;
  m->nen = dim == 2 ? 9 : 27;
  m->nvx = dim == 2 ? 4 : 8;
  m->nsides = dim == 2 ? 4 : 6;
  m->nsn = dim == 2 ? 3 : 9;
  int ntop_el[3] = {1, 1, 1};
  for (int d = 0; d < 3; d++) {
    m->n0[d] = d < dim ? n0[d] : 1;
    ntop_el[d] = m->n0[d] << (nlev - 1);
    m->L[d] = d < dim ? 2 * ntop_el[d] + 1 : 1;
  }
  long nlat = (long)m->L[0] * m->L[1] * m->L[2];
  m->ntop = (int)nlat;
  int ncls = nlev + 1;
  int *cnt = (int *)calloc(ncls + 1, sizeof(int));
  for (int K = 0; K < m->L[2]; K++)
    for (int J = 0; J < m->L[1]; J++)
      for (int I = 0; I < m->L[0]; I++) {
        int p[3] = {I, J, K};
        cnt[node_class(m, p) + 1]++;
      }
  for (int c = 0; c < ncls; c++) cnt[c + 1] += cnt[c];
  m->nvert0 = cnt[1];
  m->nnodes = (int *)malloc(nlev * sizeof(int));
  for (int l = 0; l < nlev; l++) m->nnodes[l] = cnt[l + 2];
  m->lat = (int *)malloc(3 * nlat * sizeof(int));
  m->xyz = (double *)malloc(dim * nlat * sizeof(double));
  m->node_of_lat = (int *)malloc(nlat * sizeof(int));
  int *pos = (int *)malloc(ncls * sizeof(int));
  for (int c = 0; c < ncls; c++) pos[c] = cnt[c];
  for (int K = 0; K < m->L[2]; K++)
    for (int J = 0; J < m->L[1]; J++)
      for (int I = 0; I < m->L[0]; I++) {
        int p[3] = {I, J, K};
        int nd = pos[node_class(m, p)]++;
        long li = ((long)K * m->L[1] + J) * m->L[0] + I;
        m->node_of_lat[li] = nd;
        m->lat[3 * nd] = I;
        m->lat[3 * nd + 1] = J;
        m->lat[3 * nd + 2] = K;
        for (int d = 0; d < dim; d++)
          m->xyz[nd + (long)d * nlat] =
              box[2 * d] + (box[2 * d + 1] - box[2 * d]) * ((double)p[d] / (double)(m->L[d] - 1));
      }
  free(pos);
  free(cnt);
  m->nel = (int *)malloc(nlev * sizeof(int));
  m->conn = (int **)malloc(nlev * sizeof(int *));
  m->neigh = (int **)malloc(nlev * sizeof(int *));
  m->ecol = (int **)malloc(nlev * sizeof(int *));
  m->eabc = (int **)malloc(nlev * sizeof(int *));
  for (int l = 0; l < nlev; l++) {
    int ne[3], s = 1 << (nlev - 1 - l);
    for (int d = 0; d < 3; d++) ne[d] = d < dim ? (m->n0[d] << l) : 1;
    int nel = ne[0] * ne[1] * ne[2];
    m->nel[l] = nel;
    m->conn[l] = (int *)malloc((long)nel * m->nen * sizeof(int));
    m->neigh[l] = (int *)malloc((long)nel * m->nsides * sizeof(int));
    m->ecol[l] = (int *)malloc(nel * sizeof(int));
    m->eabc[l] = (int *)malloc(3 * nel * sizeof(int));
    for (int ez = 0; ez < ne[2]; ez++)
      for (int ey = 0; ey < ne[1]; ey++)
        for (int ex = 0; ex < ne[0]; ex++) {
          int e = (ez * ne[1] + ey) * ne[0] + ex;
          int ee[3] = {ex, ey, ez};
          for (int k = 0; k < m->nen; k++) {
            const int *abc = local_abc(dim, k);
            int p[3];
            for (int d = 0; d < 3; d++) p[d] = d < dim ? (2 * ee[d] + abc[d]) * s : 0;
            long li = ((long)p[2] * m->L[1] + p[1]) * m->L[0] + p[0];
            m->conn[l][(long)e * m->nen + k] = m->node_of_lat[li];
          }
          for (int sd = 0; sd < m->nsides; sd++) {
            const int *dir = dim == 2 ? Q9_SIDE_DIR[sd] : H27_FACE_DIR[sd];
            int q[3], ok = 1;
            for (int d = 0; d < 3; d++) {
              q[d] = ee[d] + dir[d];
              if (q[d] < 0 || q[d] >= ne[d]) ok = 0;
            }
            m->neigh[l][(long)e * m->nsides + sd] = ok ? (q[2] * ne[1] + q[1]) * ne[0] + q[0] : -1;
          }
          m->ecol[l][e] = (ex & 1) | ((ey & 1) << 1) | ((ez & 1) << 2);
          m->eabc[l][3 * e] = ex;
          m->eabc[l][3 * e + 1] = ey;
          m->eabc[l][3 * e + 2] = ez;
        }
  }
  return m;
}

void or_mesh_free(or_mesh *m) {
  if (!m) return;
  for (int l = 0; l < m->nlev; l++) {
    free(m->conn[l]);
    free(m->neigh[l]);
    free(m->ecol[l]);
    free(m->eabc[l]);
  }
  free(m->conn);
  free(m->neigh);
  free(m->ecol);
  free(m->eabc);
  free(m->nel);
  free(m->nnodes);
  free(m->lat);
  free(m->xyz);
  free(m->node_of_lat);
  free(m);
}

int or_mesh_nnodes(const or_mesh *m, int lev) { return m->nnodes[lev]; }
int or_mesh_nvert0(const or_mesh *m) { return m->nvert0; }
int or_mesh_nel(const or_mesh *m, int lev) { return m->nel[lev]; }
int or_mesh_nen(const or_mesh *m) { return m->nen; }
void or_mesh_get_xyz(const or_mesh *m, double *xyz) {
  memcpy(xyz, m->xyz, (size_t)m->dim * m->ntop * sizeof(double));
}
void or_mesh_get_lattice(const or_mesh *m, int *lat) { memcpy(lat, m->lat, 3 * (size_t)m->ntop * sizeof(int)); }
void or_mesh_get_conn(const or_mesh *m, int lev, int *conn, int *neigh, int *colour) {
  if (conn) memcpy(conn, m->conn[lev], (size_t)m->nel[lev] * m->nen * sizeof(int));
  if (neigh) memcpy(neigh, m->neigh[lev], (size_t)m->nel[lev] * m->nsides * sizeof(int));
  if (colour) memcpy(colour, m->ecol[lev], (size_t)m->nel[lev] * sizeof(int));
}

/* ============================================================ FE tables */
/* 1D Lagrange basis on {-1,0,+1} (index 0,1,2 = node at -1,0,+1): src/MGFE.C:252-263 */
static double lag1(int a, double x) {
  if (a == 0) return .5 * x * (x - 1.);
  if (a == 2) return .5 * x * (x + 1.);
  return 1. - x * x;
}
static double dlag1(int a, double x) {
  if (a == 0) return x - .5;
  if (a == 2) return x + .5;
  return -2. * x;
}
/* linear basis on the vertices (a = 0 or 2): src/MGFE.C init_lin */
static double lin1(int a, double x) { return a == 0 ? .5 * (1. - x) : .5 * (1. + x); }
static double dlin1(int a, double x) {
  (void)x;
  return a == 0 ? -.5 : .5;
}

typedef struct {
  int dim, ng, nq, nl;
  double w[27];
  double phi[27][27];       /* [qp][shape] */
  double dphi[27][27][3];   /* [qp][shape][dir] reference derivatives */
  double psi[27][8];        /* linear shapes */
  double dpsi[27][8][3];
  /* surface (dim-1) tables on the side's node order */
  int sng, snq;
  double sw[9];
  double sphi[9][9];
  double sdphi[9][9][2];
  double spsi[9][4];        /* linear surface shapes on the side's vertices */
} fe_tab;

/* Gauss points: x-major then y then z (src/MGFE.C:214-227), weights 5/9, 8/9, 5/9. */
static void fe_init(fe_tab *t, int dim) {
  const double g[3] = {-sqrt(3. / 5.), 0., sqrt(3. / 5.)};
  const double gw[3] = {5. / 9., 8. / 9., 5. / 9.};
  memset(t, 0, sizeof(*t));
  t->dim = dim;
  t->ng = dim == 2 ? 9 : 27;
  t->nq = t->ng;
  t->nl = dim == 2 ? 4 : 8;
  for (int q = 0; q < t->ng; q++) {
    int iq[3];
    if (dim == 2) {
      iq[0] = q / 3;
      iq[1] = q % 3;
      iq[2] = 1;
    } else {
      iq[0] = q / 9;
      iq[1] = (q / 3) % 3;
      iq[2] = q % 3;
    }
    double xi[3] = {g[iq[0]], g[iq[1]], dim == 3 ? g[iq[2]] : 0.};
    t->w[q] = gw[iq[0]] * gw[iq[1]] * (dim == 3 ? gw[iq[2]] : 1.);
    for (int s = 0; s < t->nq; s++) {
      const int *abc = local_abc(dim, s);
      double v = 1.;
      for (int d = 0; d < dim; d++) v *= lag1(abc[d], xi[d]);
      t->phi[q][s] = v;
      for (int k = 0; k < dim; k++) {
        double dv = 1.;
        for (int d = 0; d < dim; d++) dv *= (d == k) ? dlag1(abc[d], xi[d]) : lag1(abc[d], xi[d]);
        t->dphi[q][s][k] = dv;
      }
    }
    for (int s = 0; s < t->nl; s++) {
      const int *abc = local_abc(dim, s);
      double v = 1.;
      for (int d = 0; d < dim; d++) v *= lin1(abc[d], xi[d]);
      t->psi[q][s] = v;
      for (int k = 0; k < dim; k++) {
        double dv = 1.;
        for (int d = 0; d < dim; d++) dv *= (d == k) ? dlin1(abc[d], xi[d]) : lin1(abc[d], xi[d]);
        t->dpsi[q][s][k] = dv;
      }
    }
  }
  /* surface element: 1D Edge3 (2D) or Quad9 (3D) on the side's node order */
  int sdim = dim - 1;
  t->sng = sdim == 1 ? 3 : 9;
  t->snq = sdim == 1 ? 3 : 9;
  for (int q = 0; q < t->sng; q++) {
    int iq[2];
    if (sdim == 1) {
      iq[0] = q;
      iq[1] = 1;
    } else {
      iq[0] = q / 3;
      iq[1] = q % 3;
    }
    double xi[2] = {g[iq[0]], g[iq[1]]};
    t->sw[q] = gw[iq[0]] * (sdim == 2 ? gw[iq[1]] : 1.);
    for (int s = 0; s < t->snq; s++) {
      int abc[2];
      if (sdim == 1) {
        abc[0] = s == 0 ? 0 : (s == 1 ? 2 : 1);
        abc[1] = 1;
      } else {
        abc[0] = Q9_ABC[s][0];
        abc[1] = Q9_ABC[s][1];
      }
      double v = 1.;
      for (int d = 0; d < sdim; d++) v *= lag1(abc[d], xi[d]);
      t->sphi[q][s] = v;
      for (int k = 0; k < sdim; k++) {
        double dv = 1.;
        for (int d = 0; d < sdim; d++) dv *= (d == k) ? dlag1(abc[d], xi[d]) : lag1(abc[d], xi[d]);
        t->sdphi[q][s][k] = dv;
      }
      if (s < (sdim == 1 ? 2 : 4)) { /* vertices come first on a side */
        double w = 1.;
        for (int d = 0; d < sdim; d++) w *= lin1(abc[d], xi[d]);
        t->spsi[q][s] = w;
      }
    }
  }
}

void or_side_table(int dim, int *out) {
  int ns = dim == 2 ? 4 : 6, nn = dim == 2 ? 3 : 9;
  for (int s = 0; s < ns; s++)
    for (int k = 0; k < nn; k++) out[s * nn + k] = dim == 2 ? Q9_SIDE[s][k] : H27_FACE[s][k];
}

void or_fe_tables(int dim, double *phi_q, double *dphi_q, double *phi_l, double *w) {
  fe_tab t;
  fe_init(&t, dim);
  for (int q = 0; q < t.ng; q++) {
    if (w) w[q] = t.w[q];
    for (int s = 0; s < t.nq; s++) {
      if (phi_q) phi_q[q * t.nq + s] = t.phi[q][s];
      for (int k = 0; k < dim; k++)
        if (dphi_q) dphi_q[(q * t.nq + s) * dim + k] = t.dphi[q][s][k];
    }
    for (int s = 0; s < t.nl; s++)
      if (phi_l) phi_l[q * t.nl + s] = t.psi[q][s];
  }
}

/* Jacobian + inverse (src/MGFE.C:1066-1170): InvJac[j + i*dim] = d xi_j / d x_i. */
static double jac(const fe_tab *t, int q, const double *xx /* [dim][nen] */, int nen, double *ij) {
  int dim = t->dim;
  double J[3][3] = {{0}};
  for (int s = 0; s < t->nq; s++)
    for (int a = 0; a < dim; a++)
      for (int b = 0; b < dim; b++) J[a][b] += xx[a * nen + s] * t->dphi[q][s][b]; /* dx_a/dxi_b */
  double det;
  if (dim == 2) {
    det = J[0][0] * J[1][1] - J[1][0] * J[0][1];
    double id = 1. / det;
    ij[0] = J[1][1] * id;
    ij[1] = -J[1][0] * id;
    ij[2] = -J[0][1] * id;
    ij[3] = J[0][0] * id;
  } else {
    det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
          J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    double id = 1. / det;
    double inv[3][3]; /* inv = J^{-1}: inv[b][a] = dxi_b/dx_a */
    inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * id;
    inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
    inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
    inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
    inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
    inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
    inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
    inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) ij[j + i * 3] = inv[j][i];
  }
  return det;
}

/* surface Jacobian (src/MGFE.C:1290-1466): |dx/dxi| (edge) or |x_xi x x_eta| (face) */
static double jac_sur(const fe_tab *t, int q, const double *xb /* [dim][nsn] */, int nsn) {
  if (t->dim == 2) {
    double dx = 0, dy = 0;
    for (int s = 0; s < 3; s++) {
      dx += xb[s] * t->sdphi[q][s][0];
      dy += xb[nsn + s] * t->sdphi[q][s][0];
    }
    return sqrt(dx * dx + dy * dy);
  }
  double a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
  for (int s = 0; s < 9; s++)
    for (int d = 0; d < 3; d++) {
      a[d] += xb[d * nsn + s] * t->sdphi[q][s][0];
      b[d] += xb[d * nsn + s] * t->sdphi[q][s][1];
    }
  double c0 = a[1] * b[2] - a[2] * b[1], c1 = a[2] * b[0] - a[0] * b[2], c2 = a[0] * b[1] - a[1] * b[0];
  return sqrt(c0 * c0 + c1 * c1 + c2 * c2);
}

/* ============================================================== system */
typedef struct {
  int n;            /* rows */
  int *ptr, *col;   /* CSR */
  double *val;
} csr;

struct or_sys {
  const or_mesh *m;
  int kind, nv2, nv1, nvars, nlev;
  int *ndof;        /* [nlev] */
  int *nl;          /* Q1 nodes per level */
  int **node_dof;   /* [nlev][nvars*ntop] (reference _node_dof layout) */
  int *bc0, *bc1;   /* top-level DOFs */
  /* node patterns per level */
  int **qq_ptr, **qq_idx, **ql_ptr, **ql_idx;
  csr *A, *P, *R;   /* A[l]; P[l]: l-1 -> l (l>=1); R[l]: l+1 -> l (l<nlev-1) */
  int **diag;       /* diagonal position per row */
  double *rhs;      /* top rhs */
  /* multigrid work */
  double **x, **b, **r;
  double *lu;
  int *piv;
  int lu_ok;
  int **colour;     /* per level item colour */
  int *ncolour;
  int **col_items;  /* per level: items grouped by colour, ascending within a colour */
  int **col_off;    /* per level: [ncolour+1] offsets into col_items */
  const double *turb_k, *turb_w; /* NS: kappa, omega x_old [Ntop] of the turbulence model */
};

static void csr_alloc(csr *c, int n, long nnz) {
  c->n = n;
  c->ptr = (int *)calloc(n + 1, sizeof(int));
  c->col = (int *)malloc((nnz > 0 ? nnz : 1) * sizeof(int));
  c->val = (double *)calloc(nnz > 0 ? nnz : 1, sizeof(double));
}
static void csr_free(csr *c) {
  free(c->ptr);
  free(c->col);
  free(c->val);
}

static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

/* Node pattern of level l = union of the element nodes containing each node
 * (gencase compute_mat_qq, USER_APPL/gencase/src/MGGenCase.C:1781-1862), sorted. */
static void build_node_pattern(or_sys *s, int l) {
  const or_mesh *m = s->m;
  int N = m->nnodes[l], nel = m->nel[l], nen = m->nen, nvx = m->nvx;
  int *ecnt = (int *)calloc(N + 1, sizeof(int));
  for (long k = 0; k < (long)nel * nen; k++) ecnt[m->conn[l][k] + 1]++;
  for (int i = 0; i < N; i++) ecnt[i + 1] += ecnt[i];
  int *elist = (int *)malloc(ecnt[N] * sizeof(int));
  int *fill = (int *)malloc(N * sizeof(int));
  memcpy(fill, ecnt, N * sizeof(int));
  for (int e = 0; e < nel; e++)
    for (int k = 0; k < nen; k++) elist[fill[m->conn[l][(long)e * nen + k]]++] = e;
  s->qq_ptr[l] = (int *)calloc(N + 1, sizeof(int));
  s->ql_ptr[l] = (int *)calloc(N + 1, sizeof(int));
  int cap = 8 * 27;
  int *tq = (int *)malloc(cap * sizeof(int)), *tl = (int *)malloc(cap * sizeof(int));
  /* two passes: count, then fill */
  for (int pass = 0; pass < 2; pass++) {
    for (int n = 0; n < N; n++) {
      int nq = 0, nlv = 0;
      for (int k = ecnt[n]; k < ecnt[n + 1]; k++) {
        const int *c = m->conn[l] + (long)elist[k] * nen;
        for (int j = 0; j < nen; j++) tq[nq++] = c[j];
        for (int j = 0; j < nvx; j++) tl[nlv++] = c[j];
      }
      qsort(tq, nq, sizeof(int), cmp_int);
      qsort(tl, nlv, sizeof(int), cmp_int);
      int uq = 0, ul = 0;
      for (int k = 0; k < nq; k++)
        if (k == 0 || tq[k] != tq[k - 1]) tq[uq++] = tq[k];
      for (int k = 0; k < nlv; k++)
        if (k == 0 || tl[k] != tl[k - 1]) tl[ul++] = tl[k];
      if (pass == 0) {
        s->qq_ptr[l][n + 1] = uq;
        s->ql_ptr[l][n + 1] = ul;
      } else {
        memcpy(s->qq_idx[l] + s->qq_ptr[l][n], tq, uq * sizeof(int));
        memcpy(s->ql_idx[l] + s->ql_ptr[l][n], tl, ul * sizeof(int));
      }
    }
    if (pass == 0) {
      for (int n = 0; n < N; n++) {
        s->qq_ptr[l][n + 1] += s->qq_ptr[l][n];
        s->ql_ptr[l][n + 1] += s->ql_ptr[l][n];
      }
      s->qq_idx[l] = (int *)malloc(s->qq_ptr[l][N] * sizeof(int));
      s->ql_idx[l] = (int *)malloc(s->ql_ptr[l][N] * sizeof(int));
    }
  }
  free(tq);
  free(tl);
  free(fill);
  free(elist);
  free(ecnt);
}

/* DOF-level CSR from the node pattern: blocks qq, ql, lq, ll
 * (src/MGSolverDA.C:1785-2009 reading the four gencase blocks). */
static void build_matrix_pattern(or_sys *s, int l) {
  const or_mesh *m = s->m;
  int N = m->nnodes[l], NL = s->nl[l];
  int n = s->ndof[l];
  csr *A = &s->A[l];
  long nnz = 0;
  for (int v = 0; v < s->nvars; v++) {
    int nn = v < s->nv2 ? N : NL;
    for (int i = 0; i < nn; i++)
      nnz += (long)s->nv2 * (s->qq_ptr[l][i + 1] - s->qq_ptr[l][i]) +
             (long)s->nv1 * (s->ql_ptr[l][i + 1] - s->ql_ptr[l][i]);
  }
  csr_alloc(A, n, nnz);
  long k = 0;
  int row = 0;
  for (int v = 0; v < s->nvars; v++) {
    int nn = v < s->nv2 ? N : NL;
    for (int i = 0; i < nn; i++, row++) {
      A->ptr[row] = (int)k;
      for (int b = 0; b < s->nv2; b++)
        for (int q = s->qq_ptr[l][i]; q < s->qq_ptr[l][i + 1]; q++) A->col[k++] = b * N + s->qq_idx[l][q];
      if (s->nv1)
        for (int q = s->ql_ptr[l][i]; q < s->ql_ptr[l][i + 1]; q++) A->col[k++] = s->nv2 * N + s->ql_idx[l][q];
    }
  }
  A->ptr[n] = (int)k;
  s->diag[l] = (int *)malloc(n * sizeof(int));
  for (int i = 0; i < n; i++) {
    s->diag[l][i] = -1;
    for (int q = A->ptr[i]; q < A->ptr[i + 1]; q++)
      if (A->col[q] == i) s->diag[l][i] = q;
  }
}

/* Prolongation (l-1 -> l): the fine node's row holds the coarse parent's shape
 * functions at the node, |v| > 1e-8 kept (gencase compute_prol_qq,
 * MGGenCase.C:2308-2393, with the embedding matrices of src/MGGeomEl.C:182-600). */
static void build_prol(or_sys *s, int l) {
  const or_mesh *m = s->m;
  int dim = m->dim, nen = m->nen, nvx = m->nvx;
  int Nf = m->nnodes[l], Nc = m->nnodes[l - 1], NLf = s->nl[l], NLc = s->nl[l - 1];
  int s_f = 1 << (m->nlev - 1 - l), s_c = 2 * s_f;
  /* one fine element owning each fine node, one owning each fine vertex */
  int *own = (int *)malloc(Nf * sizeof(int));
  for (int i = 0; i < Nf; i++) own[i] = -1;
  for (int e = 0; e < m->nel[l]; e++)
    for (int k = 0; k < nen; k++) {
      int nd = m->conn[l][(long)e * nen + k];
      if (own[nd] < 0) own[nd] = e;
    }
  int ne_c[3];
  for (int d = 0; d < 3; d++) ne_c[d] = d < dim ? (m->n0[d] << (l - 1)) : 1;
  /* rows: per var block */
  int nrow = s->ndof[l];
  int maxlen = nen;
  csr *P = &s->P[l];
  csr_alloc(P, nrow, (long)nrow * maxlen);
  long k = 0;
  int row = 0;
  for (int v = 0; v < s->nvars; v++) {
    int quad = v < s->nv2;
    int nn = quad ? Nf : NLf;
    for (int i = 0; i < nn; i++, row++) {
      P->ptr[row] = (int)k;
      int e = own[i];
      int ex[3] = {m->eabc[l][3 * e], m->eabc[l][3 * e + 1], m->eabc[l][3 * e + 2]};
      int pe[3] = {ex[0] >> 1, ex[1] >> 1, ex[2] >> 1};
      int pel = (pe[2] * ne_c[1] + pe[1]) * ne_c[0] + pe[0];
      const int *pc = m->conn[l - 1] + (long)pel * nen;
      double xi[3] = {0, 0, 0};
      for (int d = 0; d < dim; d++) {
        int origin = 2 * pe[d] * s_c; /* parent's lattice origin */
        xi[d] = -1. + (double)(m->lat[3 * i + d] - origin) / (double)s_c;
      }
      int ent_c[MAXEN];
      double ent_v[MAXEN];
      int ne = 0;
      int nsh = quad ? nen : nvx;
      for (int kj = 0; kj < nsh; kj++) {
        const int *abc = local_abc(dim, kj);
        double val = 1.;
        for (int d = 0; d < dim; d++) val *= quad ? lag1(abc[d], xi[d]) : lin1(abc[d], xi[d]);
        if (fabs(val) > 1e-8) {
          ent_c[ne] = (quad ? v * Nc : s->nv2 * Nc) + pc[kj];
          ent_v[ne] = val;
          ne++;
        }
      }
      /* sort by column */
      for (int a = 1; a < ne; a++)
        for (int b = a; b > 0 && ent_c[b - 1] > ent_c[b]; b--) {
          int tc = ent_c[b];
          ent_c[b] = ent_c[b - 1];
          ent_c[b - 1] = tc;
          double tv = ent_v[b];
          ent_v[b] = ent_v[b - 1];
          ent_v[b - 1] = tv;
        }
      for (int a = 0; a < ne; a++) {
        P->col[k] = ent_c[a];
        P->val[k] = ent_v[a];
        k++;
      }
    }
  }
  P->ptr[nrow] = (int)k;
  (void)NLc;
  free(own);
}

/* Restriction (l+1 -> l) = transposed embedding, |v| > 1e-6, each row scaled by
 * bc[0][top_dof] % 2 (MGGenCase.C:2452-2569; src/MGSolverDA.C:2406-2428). */
static void build_rest(or_sys *s, int l) {
  csr *P = &s->P[l + 1];
  int nrow = s->ndof[l], ncol = s->ndof[l + 1];
  csr *R = &s->R[l];
  long nnz = 0;
  for (long q = 0; q < P->ptr[ncol]; q++)
    if (fabs(P->val[q]) > 1e-6) nnz++;
  csr_alloc(R, nrow, nnz);
  for (int i = 0; i < ncol; i++)
    for (int q = P->ptr[i]; q < P->ptr[i + 1]; q++)
      if (fabs(P->val[q]) > 1e-6) R->ptr[P->col[q] + 1]++;
  for (int i = 0; i < nrow; i++) R->ptr[i + 1] += R->ptr[i];
  int *fill = (int *)malloc(nrow * sizeof(int));
  memcpy(fill, R->ptr, nrow * sizeof(int));
  for (int i = 0; i < ncol; i++)
    for (int q = P->ptr[i]; q < P->ptr[i + 1]; q++)
      if (fabs(P->val[q]) > 1e-6) {
        int c = P->col[q];
        R->col[fill[c]] = i;
        R->val[fill[c]] = P->val[q];
        fill[c]++;
      }
  free(fill);
  /* Dirichlet mask by the top-level DOF of the same node/variable */
  const or_mesh *m = s->m;
  int top = s->nlev - 1, N = m->nnodes[l], off = m->ntop;
  int row = 0;
  for (int v = 0; v < s->nvars; v++) {
    int nn = v < s->nv2 ? N : s->nl[l];
    for (int i = 0; i < nn; i++, row++) {
      int tdof = s->node_dof[top][i + v * off];
      double mask = (double)(s->bc0[tdof] % 2);
      for (int q = R->ptr[row]; q < R->ptr[row + 1]; q++) R->val[q] *= mask;
    }
  }
}

/* item colours: T -> node (lattice mod 3); NS -> pressure vertex (lattice mod 3) */
static void build_colours(or_sys *s, int l) {
  const or_mesh *m = s->m;
  int sl = 1 << (m->nlev - 1 - l);
  int nitem = s->kind == 0 ? m->nnodes[l] : s->nl[l];
  int step = s->kind == 0 ? sl : 2 * sl;
  s->colour[l] = (int *)malloc(nitem * sizeof(int));
  for (int i = 0; i < nitem; i++) {
    int c = 0, mul = 1;
    for (int d = 0; d < m->dim; d++) {
      c += ((m->lat[3 * i + d] / step) % 3) * mul;
      mul *= 3;
    }
    s->colour[l][i] = c;
  }
  s->ncolour[l] = m->dim == 2 ? 9 : 27;
  int nc = s->ncolour[l];
  s->col_off[l] = (int *)calloc(nc + 1, sizeof(int));
  s->col_items[l] = (int *)malloc((nitem > 0 ? nitem : 1) * sizeof(int));
  for (int i = 0; i < nitem; i++) s->col_off[l][s->colour[l][i] + 1]++;
  for (int c = 0; c < nc; c++) s->col_off[l][c + 1] += s->col_off[l][c];
  int *fill = (int *)malloc((nc + 1) * sizeof(int));
  memcpy(fill, s->col_off[l], (nc + 1) * sizeof(int));
  for (int i = 0; i < nitem; i++) s->col_items[l][fill[s->colour[l][i]]++] = i;
  free(fill);
}

or_sys *or_sys_new(const or_mesh *m, int kind) {
  or_sys *s = (or_sys *)calloc(1, sizeof(or_sys));
  s->m = m;
  s->kind = kind;
  s->nlev = m->nlev;
  s->nv2 = kind == 0 ? 1 : m->dim;
  s->nv1 = kind == 0 ? 0 : 1;
  s->nvars = s->nv2 + s->nv1;
  int L = m->nlev;
  s->ndof = (int *)malloc(L * sizeof(int));
  s->nl = (int *)malloc(L * sizeof(int));
  s->node_dof = (int **)malloc(L * sizeof(int *));
  /* MGSolDA::init_dof (src/MGSolverDA.C:880-951), one subdomain */
  for (int l = 0; l < L; l++) {
    int N = m->nnodes[l];
    int NL = l > 0 ? m->nnodes[l - 1] : m->nvert0;
    s->nl[l] = NL;
    s->ndof[l] = s->nv2 * N + s->nv1 * NL;
    s->node_dof[l] = (int *)malloc((size_t)s->nvars * m->ntop * sizeof(int));
    for (long k = 0; k < (long)s->nvars * m->ntop; k++) s->node_dof[l][k] = -1;
    int cnt = 0;
    for (int v = 0; v < s->nv2; v++)
      for (int k = 0; k < N; k++) s->node_dof[l][k + v * m->ntop] = cnt++;
    for (int v = 0; v < s->nv1; v++)
      for (int k = 0; k < NL; k++) s->node_dof[l][k + (s->nv2 + v) * m->ntop] = cnt++;
  }
  int ntd = s->ndof[L - 1];
  s->bc0 = (int *)malloc(ntd * sizeof(int));
  s->bc1 = (int *)malloc(ntd * sizeof(int));
  for (int i = 0; i < ntd; i++) s->bc0[i] = s->bc1[i] = 1;
  s->qq_ptr = (int **)calloc(L, sizeof(int *));
  s->qq_idx = (int **)calloc(L, sizeof(int *));
  s->ql_ptr = (int **)calloc(L, sizeof(int *));
  s->ql_idx = (int **)calloc(L, sizeof(int *));
  s->A = (csr *)calloc(L, sizeof(csr));
  s->P = (csr *)calloc(L, sizeof(csr));
  s->R = (csr *)calloc(L, sizeof(csr));
  s->diag = (int **)calloc(L, sizeof(int *));
  s->x = (double **)calloc(L, sizeof(double *));
  s->b = (double **)calloc(L, sizeof(double *));
  s->r = (double **)calloc(L, sizeof(double *));
  s->colour = (int **)calloc(L, sizeof(int *));
  s->ncolour = (int *)calloc(L, sizeof(int));
  s->col_items = (int **)calloc(L, sizeof(int *));
  s->col_off = (int **)calloc(L, sizeof(int *));
  for (int l = 0; l < L; l++) {
    build_node_pattern(s, l);
    build_matrix_pattern(s, l);
    build_colours(s, l);
    s->x[l] = (double *)calloc(s->ndof[l], sizeof(double));
    s->b[l] = (double *)calloc(s->ndof[l], sizeof(double));
    s->r[l] = (double *)calloc(s->ndof[l], sizeof(double));
  }
  for (int l = 1; l < L; l++) build_prol(s, l);
  for (int l = 0; l < L - 1; l++) build_rest(s, l);
  s->rhs = (double *)calloc(ntd, sizeof(double));
  return s;
}

void or_sys_free(or_sys *s) {
  if (!s) return;
  for (int l = 0; l < s->nlev; l++) {
    free(s->node_dof[l]);
    free(s->qq_ptr[l]);
    free(s->qq_idx[l]);
    free(s->ql_ptr[l]);
    free(s->ql_idx[l]);
    csr_free(&s->A[l]);
    if (l > 0) csr_free(&s->P[l]);
    if (l < s->nlev - 1) csr_free(&s->R[l]);
    free(s->diag[l]);
    free(s->x[l]);
    free(s->b[l]);
    free(s->r[l]);
    free(s->colour[l]);
    free(s->col_items[l]);
    free(s->col_off[l]);
  }
  free(s->col_items);
  free(s->col_off);
  free(s->node_dof);
  free(s->qq_ptr);
  free(s->qq_idx);
  free(s->ql_ptr);
  free(s->ql_idx);
  free(s->A);
  free(s->P);
  free(s->R);
  free(s->diag);
  free(s->x);
  free(s->b);
  free(s->r);
  free(s->colour);
  free(s->ncolour);
  free(s->ndof);
  free(s->nl);
  free(s->bc0);
  free(s->bc1);
  free(s->rhs);
  free(s->lu);
  free(s->piv);
  free(s);
}

int or_sys_ndof(const or_sys *s, int lev) { return s->ndof[lev]; }
void or_sys_node_dof(const or_sys *s, int lev, int *out) {
  memcpy(out, s->node_dof[lev], (size_t)s->nvars * s->m->ntop * sizeof(int));
}

/* Restated bc_read presets (template_appl/nse/SRC/User_NS.C bc_read; MGSolverDA.C
 * GenBc_loop :781-865): flags depend only on the node coordinates. */
void or_sys_bc_preset(or_sys *s, int preset) {
  const or_mesh *m = s->m;
  int top = s->nlev - 1, off = m->ntop, dim = m->dim;
  int ntd = s->ndof[top];
  for (int i = 0; i < ntd; i++) s->bc0[i] = s->bc1[i] = 1;
  for (int n = 0; n < m->ntop; n++) {
    const int *p = m->lat + 3 * n;
    int lo[3], hi[3], onb = 0;
    for (int d = 0; d < 3; d++) {
      lo[d] = d < dim && p[d] == 0;
      hi[d] = d < dim && p[d] == m->L[d] - 1;
      onb |= lo[d] | hi[d];
    }
    if (!onb) continue;
    for (int v = 0; v < s->nvars; v++) {
      int dof = s->node_dof[top][n + v * off];
      if (dof < 0) continue;
      int b0 = 1, b1 = 0;
      int quad = v < s->nv2;
      switch (preset) {
        case 1: /* heat: T = 0 on every wall */
          b0 = 0;
          b1 = 0;
          break;
        case 2: /* lid-driven cavity: no-slip, u = 1 on the lid interior */
          if (quad) {
            b0 = 0;
            b1 = (v == 0 && hi[1] && !lo[0] && !hi[0]) ? 4 : 0;
          } else if (n == 0) {
            b0 = 0; /* pressure pinned at node 0 */
          }
          break;
        case 3: /* channel: inlet x=0 (u prescribed), walls y,z; outlet natural */
          if (quad) {
            int wall = lo[1] || hi[1] || lo[2] || hi[2];
            if (wall || lo[0]) {
              b0 = 0;
              b1 = (v == 0 && lo[0] && !wall) ? 4 : 0;
            }
          }
          break;
        case 4: /* Boussinesq NS: no-slip on all walls, pressure pinned at node 0 */
          if (quad) {
            b0 = 0;
            b1 = 0;
          } else if (n == 0) {
            b0 = 0;
          }
          break;
        case 5: /* Boussinesq T: x=0 hot (nonhomogeneous), x=1 cold, y walls adiabatic */
          if (lo[0]) {
            b0 = 0;
            b1 = 1;
          } else if (hi[0]) {
            b0 = 0;
            b1 = 0;
          }
          break;
        default:
          break;
      }
      s->bc0[dof] = b0;
      s->bc1[dof] = b1;
    }
  }
  /* re-derive the masked restrictions */
  for (int l = 0; l < s->nlev - 1; l++) {
    csr_free(&s->R[l]);
    build_rest(s, l);
  }
}

void or_sys_set_bc(or_sys *s, const int *bc0, const int *bc1) {
  int ntd = s->ndof[s->nlev - 1];
  memcpy(s->bc0, bc0, ntd * sizeof(int));
  memcpy(s->bc1, bc1, ntd * sizeof(int));
  for (int l = 0; l < s->nlev - 1; l++) {
    csr_free(&s->R[l]);
    build_rest(s, l);
  }
}
void or_sys_get_bc(const or_sys *s, int *bc0, int *bc1) {
  int ntd = s->ndof[s->nlev - 1];
  memcpy(bc0, s->bc0, ntd * sizeof(int));
  memcpy(bc1, s->bc1, ntd * sizeof(int));
}

long or_sys_nnz(const or_sys *s, int lev) { return s->A[lev].ptr[s->A[lev].n]; }
void or_sys_pattern(const or_sys *s, int lev, int *rowptr, int *col) {
  memcpy(rowptr, s->A[lev].ptr, (s->A[lev].n + 1) * sizeof(int));
  memcpy(col, s->A[lev].col, (size_t)or_sys_nnz(s, lev) * sizeof(int));
}
long or_sys_prol_nnz(const or_sys *s, int lev) { return s->P[lev].ptr[s->P[lev].n]; }
void or_sys_prol(const or_sys *s, int lev, int *rowptr, int *col, double *val) {
  const csr *P = &s->P[lev];
  memcpy(rowptr, P->ptr, (P->n + 1) * sizeof(int));
  memcpy(col, P->col, (size_t)P->ptr[P->n] * sizeof(int));
  memcpy(val, P->val, (size_t)P->ptr[P->n] * sizeof(double));
}
long or_sys_rest_nnz(const or_sys *s, int lev) { return s->R[lev].ptr[s->R[lev].n]; }
void or_sys_rest(const or_sys *s, int lev, int *rowptr, int *col, double *val) {
  const csr *R = &s->R[lev];
  memcpy(rowptr, R->ptr, (R->n + 1) * sizeof(int));
  memcpy(col, R->col, (size_t)R->ptr[R->n] * sizeof(int));
  memcpy(val, R->val, (size_t)R->ptr[R->n] * sizeof(double));
}
void or_sys_colours(const or_sys *s, int lev, int *ncol, int *colour_of_item) {
  int nitem = s->kind == 0 ? s->m->nnodes[lev] : s->nl[lev];
  *ncol = s->ncolour[lev];
  memcpy(colour_of_item, s->colour[lev], nitem * sizeof(int));
}

/* ============================================================ assembly */
static int find_col(const csr *A, int row, int col) {
  int lo = A->ptr[row], hi = A->ptr[row + 1] - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    if (A->col[mid] == col) return mid;
    if (A->col[mid] < col) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

/* f_upwind (template_appl/nse/SRC/MGSolverNS.C:336-339; MGSolverT.C upwind block) */
static double upwind_f(double up, double rho, double mod, double h, double diff) {
  double pe = 0.5 * mod * h / diff;
  return up * rho * 0.5 * (1. / tanh(pe) - 1. / pe) * h / mod;
}

/* MGFE::normal_g (src/MGFE.C:1601-1646) on the side's coordinates xb [dim][nsn]: 2D the
 * tangent from side node 0 to 1 turned clockwise, 3D (x1 - x0) x (x3 - x0), normalised */
static void side_normal(int dim, const double *xb, int nsn, double *nrm) {
  double t1[3] = {0, 0, 0}, t3[3] = {0, 0, 0};
  for (int d = 0; d < dim; d++) {
    t1[d] = xb[d * nsn + 1] - xb[d * nsn + 0];
    if (dim == 3) t3[d] = xb[d * nsn + 3] - xb[d * nsn + 0];
  }
  nrm[2] = 0.;
  if (dim == 2) {
    nrm[0] = t1[1];
    nrm[1] = -t1[0];
  } else {
    nrm[0] = t1[1] * t3[2] - t1[2] * t3[1];
    nrm[1] = t1[2] * t3[0] - t1[0] * t3[2];
    nrm[2] = t1[0] * t3[1] - t1[1] * t3[0];
  }
  double mm = 0.;
  for (int d = 0; d < dim; d++) mm += nrm[d] * nrm[d];
  mm = sqrt(mm);
  for (int d = 0; d < dim; d++) nrm[d] /= mm;
}

/* the turbulence template's model constants (template_appl/turb-ckw/DATA/
 * MGSclass_conf.h:296-356: WILCOX, LOWRE) */
#define KW_SIGMA_K 0.6
#define KW_SIGMA_W 0.5
#define KW_BETASTAR 0.09
#define KW_MAX_TAU 100.
#define KW_MU_LOW 1.e-6
#define KW_MU_TOP 1.e+6
#define KW_UP_WIND 1.

/* IRe_eff = IRe (1 + mu_t) of the turbulence template's Navier-Stokes equation
 * (template_appl/turb-ckw/SRC/MGSolverNS.C:256-293) with its kappa-omega f_mu (:685-760:
 * tau = 1/omega, Re_t = kappa tau / IRe, WILCOX with LOWRE: mu_t = alpha* Re_t, capped by
 * nut2 / IRe, clamped to [MU_LOW, MU_TOP]) at one Gauss point; S from the velocity
 * gradients of the NS x_old */
static double ns_eddy_viscosity(const or_sys *s, const or_phys *ph, const int *c, double (*uold)[MAXEN],
                                double (*dphi)[3], const double *phi, int nen, int dim) {
  const double IRe = ph->inv_re;
  double g[9] = {0}, kg = 0., wg = 0.;
  for (int k = 0; k < nen; k++) {
    kg += phi[k] * s->turb_k[c[k]];
    wg += phi[k] * s->turb_w[c[k]];
    for (int a = 0; a < dim; a++)
      for (int d = 0; d < dim; d++) g[a * dim + d] += uold[a][k] * dphi[k][d];
  }
  double sP = 1.e-20;
  for (int a = 0; a < dim; a++)
    for (int b = 0; b < dim; b++) {
      const double sss = g[a + b * dim] + g[b + a * dim];
      sP += sss * sss;
    }
  if (kg < 1.e-20) kg = 1.e-20;
  if (wg < 1.e-20) wg = 1.e-20;
  const double tau_k = 1. / wg;
  const double Re_t = kg * tau_k / IRe;
  double mu_t = Re_t;
  const double alpha_star = (0.024 + 0.166666666667 * Re_t) / (1. + 0.166666666667 * Re_t);
  mu_t *= alpha_star;
  const double nut2 = kg / (7. * sqrt(alpha_star * 0.5 * sP / KW_BETASTAR) / 8.);
  if (mu_t * IRe > nut2) mu_t = nut2 / IRe;
  if (mu_t > KW_MU_TOP) mu_t = KW_MU_TOP;
  if (mu_t < KW_MU_LOW) mu_t = KW_MU_LOW;
  return IRe * (1. + mu_t);
}

void or_sys_set_turb(or_sys *s, const double *kold, const double *wold) {
  s->turb_k = kold;
  s->turb_w = wold;
}

/* One element of MGSolT::GenMatRhs (template_appl/nse/SRC/MGSolverT.C:93-525) or
 * MGSolNS::GenMatRhs (template_appl/nse/SRC/MGSolverNS.C:108-717): local matrix and rhs,
 * boundary sides, scatter into the level matrix (A[Level]->add_matrix) and rhs. */
static void asm_element(or_sys *s, int lev, int mode, const or_phys *ph, const double *xold, const double *vel,
                        const double *temp, const double *qe, const fe_tab *t, int e, double *Ke, double *Fe,
                        double *rhs) {
  const or_mesh *m = s->m;
  int dim = m->dim, nen = m->nen, nvx = m->nvx, top = s->nlev - 1, off = m->ntop;
  csr *A = &s->A[lev];
  int nv2 = s->nv2, nvars = s->nvars;
  int nloc = nv2 * nen + s->nv1 * nvx;
  int dofs[MAXEN * 4];
  int bcv[4][MAXEN], bcb[4][MAXEN];
  double xx[3 * MAXEN];
  double uold[4][MAXEN], vold[3][MAXEN], told[MAXEN];
  double diff_t = ph->inv_prdl * ph->inv_re;
  const int *c = m->conn[lev] + (long)e * nen;
  memset(Ke, 0, (size_t)nloc * nloc * sizeof(double));
  memset(Fe, 0, nloc * sizeof(double));
  /* get_el_dof_bc (src/MGSolverDA.C:987-1041) and get_el_sol (src/MGSolverBase.C:336-354) */
  for (int k = 0; k < nen; k++) {
    for (int d = 0; d < dim; d++) xx[d * nen + k] = m->xyz[c[k] + (long)d * off];
    for (int v = 0; v < nvars; v++) {
      int quad = v < nv2;
      if (!quad && k >= nvx) continue;
      int loc = quad ? v * nen + k : nv2 * nen + k;
      dofs[loc] = s->node_dof[lev][c[k] + v * off];
      int td = s->node_dof[top][c[k] + v * off];
      bcv[v][k] = s->bc0[td];
      bcb[v][k] = s->bc1[td];
      uold[v][k] = xold ? xold[td] : 0.;
    }
    for (int d = 0; d < dim; d++) vold[d][k] = 0.;
    if (s->kind == 0 && vel) {
      /* NS field coupled into T: velocity components are the first dim vars of
       * the NS system on the top level (same node numbering). */
      int Ntop = m->nnodes[top];
      for (int d = 0; d < dim; d++) vold[d][k] = vel[c[k] + d * Ntop];
    }
    if (s->kind == 1)
      for (int d = 0; d < dim; d++) vold[d][k] = uold[d][k];
    told[k] = 0.;
    if (s->kind == 1 && temp) told[k] = temp[c[k]];
    if (s->kind == 0) told[k] = uold[0][k];
  }
  double h[3];
  {
    int v2 = dim == 2 ? 2 : 6, v3 = dim == 2 ? 3 : 7;
    for (int d = 0; d < dim; d++) {
      h[d] = fabs(xx[d * nen + v2] - xx[d * nen + 0]);
      double h1 = fabs(xx[d * nen + v3] - xx[d * nen + 1]);
      if (h[d] < h1) h[d] = h1;
    }
  }
  double q_e = (s->kind == 0 && qe && lev == top) ? qe[e] : 0.;
  for (int q = 0; q < t->ng; q++) {
    double ij[9];
    double det = jac(t, q, xx, nen, ij);
    double JxW = det * t->w[q];
    double dphi[MAXEN][3];
    for (int sh = 0; sh < nen; sh++)
      for (int i = 0; i < dim; i++) {
        double sum = 0.;
        for (int j = 0; j < dim; j++) sum += ij[j + i * dim] * t->dphi[q][sh][j];
        dphi[sh][i] = sum;
      }
    const double *phi = t->phi[q];
    double vg[3] = {0, 0, 0}, mod = 1e-20;
    for (int d = 0; d < dim; d++) {
      for (int k = 0; k < nen; k++) vg[d] += phi[k] * vold[d][k];
      mod += vg[d] * vg[d];
    }
    mod = sqrt(mod);
    if (s->kind == 0) {
      double f[3], tg = 0.;
      for (int d = 0; d < dim; d++) f[d] = (vel ? upwind_f(ph->upwind_t, ph->rhocp, mod, h[d], diff_t) : 0.);
      for (int k = 0; k < nen; k++) tg += phi[k] * told[k];
      for (int i = 0; i < nen; i++) {
        double dt = JxW * bcv[0][i];
        if (mode == 1) Fe[i] += dt * (ph->rhocp * tg * phi[i] * ph->inv_dt + q_e * phi[i]);
        for (int j = 0; j < nen; j++) {
          double adv = 0., lap = 0.;
          for (int d = 0; d < dim; d++) {
            adv += vg[d] * dphi[j][d];
            lap += (diff_t + f[d] * vg[d] * vg[d]) * dphi[j][d] * dphi[i][d];
          }
          Ke[i * nloc + j] += dt * (ph->rhocp * phi[i] * phi[j] * ph->inv_dt + ph->rhocp * adv * phi[i] + lap);
        }
      }
    } else {
      double f[3], tg = 0.;
      for (int d = 0; d < dim; d++) f[d] = upwind_f(ph->upwind_ns, ph->rho, mod, h[d], ph->inv_re);
      for (int k = 0; k < nen; k++) tg += phi[k] * told[k];
      const double *psi = t->psi[q];
      double nu = ph->inv_re, rho = ph->rho;
      if (s->turb_k && s->turb_w) nu = ns_eddy_viscosity(s, ph, c, uold, dphi, phi, nen, dim);
      for (int i = 0; i < nen; i++) {
        for (int a = 0; a < dim; a++) {
          int row = a * nen + i;
          double dt = JxW * bcv[a][i];
          if (mode == 1)
            Fe[row] += dt * (rho * vg[a] * phi[i] * ph->inv_dt + rho * ph->ifr * ph->dirg[a] * phi[i] +
                             ph->buoy * tg * ph->dirg[a] * phi[i]);
          for (int j = 0; j < nen; j++) {
            double adv = 0., lap = 0.;
            for (int d = 0; d < dim; d++) {
              adv += vg[d] * dphi[j][d] * phi[i];
              lap += (nu + f[d] * vg[d] * vg[d]) * dphi[j][d] * dphi[i][d];
            }
            Ke[row * nloc + a * nen + j] +=
                dt * rho *
                (phi[j] * phi[i] * ph->inv_dt + adv + lap + (nu + f[a] * vg[a] * vg[a]) * dphi[j][a] * dphi[i][a]);
            for (int bb = 1; bb < dim; bb++) {
              int b = (a + bb) % dim;
              Ke[row * nloc + b * nen + j] += dt * rho * (nu + f[a] * vg[a] * vg[b]) * dphi[j][a] * dphi[i][b];
            }
          }
          for (int j = 0; j < nvx; j++) Ke[row * nloc + nv2 * nen + j] += dt * (-psi[j] * dphi[i][a]);
        }
      }
      for (int i = 0; i < nvx; i++) {
        int row = nv2 * nen + i;
        for (int j = 0; j < nen; j++)
          for (int b = 0; b < dim; b++) Ke[row * nloc + b * nen + j] += JxW * rho * psi[i] * dphi[j][b];
      }
    }
  }
  /* boundary sides (MGSolverT.C boundary block; MGSolverNS.C:495-687) */
  for (int sd = 0; sd < m->nsides; sd++) {
    if (m->neigh[lev][(long)e * m->nsides + sd] != -1) continue;
    const int *sur = dim == 2 ? Q9_SIDE[sd] : H27_FACE[sd];
    int nsn = m->nsn;
    double xb[3 * 9];
    for (int k = 0; k < nsn; k++)
      for (int d = 0; d < dim; d++) xb[d * nsn + k] = xx[d * nen + sur[k]];
    double nrm[3];
    side_normal(dim, xb, nsn, nrm);
    int last = sur[nsn - 1];
    for (int a = 0; a < nv2; a++) {
      if (bcv[a][last] == 0) {
        double det = jac_sur(t, t->sng - 1, xb, nsn);
        double ipen = det * ph->penalty;
        if (s->kind == 0) {
          int bc_beta = bcb[0][last] % 2;
          for (int k = 0; k < nsn; k++) {
            int lv = sur[k];
            if (mode == 1) Fe[lv] += bc_beta * ipen * uold[0][lv];
            Ke[lv * nloc + lv] += ipen;
          }
        } else {
          for (int k = 0; k < nsn; k++) {
            int lv = sur[k];
            int row = a * nen + lv;
            int bs = bcb[a][lv];
            int bc_rhs = (bs & 4) >> 2, bc_tg = (bs & 2) >> 1, bc_n = bs % 2;
            double vdn = 0.;
            for (int d = 0; d < dim; d++) vdn += nrm[d] * uold[d][lv];
            if (mode == 1)
              Fe[row] += bc_rhs * ipen *
                         ((1 - bc_n) * (1 - bc_tg) * uold[a][lv] + bc_n * vdn * nrm[a] +
                          bc_tg * (uold[a][lv] - vdn * nrm[a]));
            Ke[row * nloc + row] +=
                ((1 - bc_n) * (1 - bc_tg) + bc_tg) * ipen + ipen * nrm[a] * nrm[a] * (bc_n - bc_tg);
            for (int b = a + 1; b < dim; b++)
              Ke[row * nloc + b * nen + lv] += ipen * nrm[b] * nrm[a] * (bc_n - bc_tg);
          }
        }
      } else if (s->kind == 1 && bcb[a][last] != 0) {
        /* Neumann / Robin sides of MGSolNS::GenMatRhs (template_appl/nse/SRC/MGSolverNS.C:
         * 604-681), alpha_t = 1: per surface Gauss point and side node i (row a, i) with
         * flags bit0 normal, bit1 tangential, bit2 rhs, the tangential / normal Robin term
         * lumped on the diagonal, the normal-normal coupling to the later components, and
         * (MESHNUMBER == 1) the pressure traction -n_a p_old phi_i */
        const int nvb = dim == 2 ? 2 : 4;
        for (int q = 0; q < t->sng; q++) {
          double JxW = jac_sur(t, q, xb, nsn) * t->sw[q];
          double pg = 0.;
          for (int k = 0; k < nvb; k++) pg += t->spsi[q][k] * uold[dim][sur[k]];
          for (int i = 0; i < nsn; i++) {
            int lei = sur[i];
            int row = a * nen + lei;
            int bs = bcb[a][lei];
            double dt = JxW * (bcv[a][lei] % 2);
            int bc_rhs = (bs & 4) >> 2, bc_tg = (bs & 2) >> 1, bc_n = bs % 2;
            double phii = t->sphi[q][i];
            if (mode == 1 && ph->traction != 0.) Fe[row] += -1. * bc_rhs * dt * phii * nrm[a] * pg;
            for (int j = 0; j < nsn; j++) {
              double phij = t->sphi[q][j];
              Ke[row * nloc + row] += dt * bc_tg * phij * phii + dt * nrm[a] * nrm[a] * phij * phii * (bc_n - bc_tg);
              for (int b = a + 1; b < dim; b++)
                Ke[row * nloc + b * nen + sur[j]] += dt * nrm[b] * nrm[a] * phij * phii * (bc_n - bc_tg);
            }
          }
        }
      } else if (s->kind == 0 && bcb[0][last] != 0) {
        /* Robin: k dT/dn = -h T (MGSolverT.C Neumann block); constant terms are 0 there */
        for (int q = 0; q < t->sng; q++) {
          double JxW = jac_sur(t, q, xb, nsn) * t->sw[q];
          for (int i = 0; i < nsn; i++) {
            int lei = sur[i];
            int bs = bcb[0][lei];
            double dt = JxW * bcv[0][lei];
            int bc_alpha = (bs & 2) >> 1;
            for (int j = 0; j < nsn; j++)
              Ke[lei * nloc + sur[j]] += dt * bc_alpha * diff_t * t->sphi[q][i] * t->sphi[q][j];
          }
        }
      }
    }
  }
  /* scatter (A[Level]->add_matrix, b[Level]->add_vector) */
  for (int i = 0; i < nloc; i++) {
    int gi = dofs[i];
    if (mode == 1) rhs[gi] += Fe[i];
    for (int j = 0; j < nloc; j++) {
      double v = Ke[i * nloc + j];
      int pos = find_col(A, gi, dofs[j]);
      A->val[pos] += v;
    }
  }
}

/* MGSolT::GenMatRhs (template_appl/nse/SRC/MGSolverT.C:93-525) and
 * MGSolNS::GenMatRhs (template_appl/nse/SRC/MGSolverNS.C:108-717).  Elements are taken
 * colour after colour ((ex&1)|(ey&1)<<1|(ez&1)<<2); elements of one colour share no node,
 * so they scatter into disjoint rows and run in parallel, and every matrix entry receives
 * its element contributions in colour order whatever the thread count. */
void or_sys_assemble(or_sys *s, int lev, int mode, const or_phys *ph, const double *xold, const double *vel,
                     const double *temp, const double *qe) {
  const or_mesh *m = s->m;
  int dim = m->dim, nen = m->nen, nvx = m->nvx, top = s->nlev - 1;
  fe_tab t;
  fe_init(&t, dim);
  csr *A = &s->A[lev];
  memset(A->val, 0, (size_t)A->ptr[A->n] * sizeof(double));
  double *rhs = NULL;
  if (mode == 1) {
    rhs = s->b[lev];
    memset(rhs, 0, s->ndof[lev] * sizeof(double));
  }
  int nloc = s->nv2 * nen + s->nv1 * nvx;
  const int nel = m->nel[lev], ncol = 1 << dim;
  for (int c = 0; c < ncol; c++) {
#pragma omp parallel
    {
      double *Ke = (double *)malloc((size_t)nloc * nloc * sizeof(double));
      double *Fe = (double *)malloc(nloc * sizeof(double));
#pragma omp for schedule(dynamic, 4)
      for (int e = 0; e < nel; e++)
        if (m->ecol[lev][e] == c) asm_element(s, lev, mode, ph, xold, vel, temp, qe, &t, e, Ke, Fe, rhs);
      free(Ke);
      free(Fe);
    }
  }
  if (mode == 1 && lev == top) memcpy(s->rhs, rhs, s->ndof[lev] * sizeof(double));
  if (lev == 0) s->lu_ok = 0;
}

/* ------------------------------------------------------------------ k-omega
 * MGSolTBK::GenMatRhs of the turbulence template (template_appl/turb-ckw/SRC/
 * MGSolverTBKW.C:83-454) with its configuration (template_appl/turb-ckw/DATA/
 * MGSclass_conf.h:276-356, Equations_conf.h:40: TBK_EQUATIONS 5, the coupled kappa-omega
 * system; WILCOX with LOWRE; SIGMA_K 0.6, SIGMA_W 0.5, BETASTAR 0.09, MAX_TAU 100,
 * MU_LOW 1e-6, MU_TOP 1e6, UP_WIND_K 1) and the model of MGSolTBK::f_mu (:484-587).  The
 * coupled system's matrix is block diagonal (no kappa-omega coupling entries), so one
 * variable var (0 kappa, 1 omega) is assembled on a scalar system: its diagonal block and
 * its rhs.  Fields: vel = the Navier-Stokes x_old [dim][Ntop], kold / wold = the kappa and
 * omega x_old [Ntop], dist = the element wall distances of this level (_mgmesh._dist),
 * nu_wall = _muf / _rhof of the omega wall value. */

typedef struct {
  double ire[2], src[2], diss[2], cross;
} kw_coef;

/* MGSolTBK::f_mu, WILCOX + LOWRE (MGSolverTBKW.C:484-587), and the effective
 * viscosities IRe (1 + sigma_v mu_t) (:243-247); kappa is clamped in place */
static void kw_model(double *kg, double wg, double sP, double chi, double IRe, kw_coef *c) {
  if (kg[0] < 1.e-20) kg[0] = 1.e-20;
  double tau_k = 1. / wg;
  if (tau_k > KW_MAX_TAU) tau_k = KW_MAX_TAU;
  double Re_t = kg[0] * tau_k / IRe;
  if (Re_t > KW_MU_TOP) Re_t = KW_MU_TOP;
  if (Re_t < KW_MU_LOW) Re_t = KW_MU_LOW;
  double mu_t = Re_t;
  const double alpha_star = (0.024 + 0.166666666667 * Re_t) / (1. + 0.166666666667 * Re_t);
  mu_t *= alpha_star;
  const double nut2 = kg[0] / (7. * sqrt(alpha_star * 0.5 * sP / KW_BETASTAR) / 8.);
  if (mu_t * IRe < nut2) {
    c->src[0] = 0.5 * mu_t * IRe * sP;
    c->src[1] = 0.5 * 13. * sP / (25.);
  } else {
    c->src[0] = 0.5 * nut2 * sP;
    c->src[1] = 0.5 * 13. * nut2 * sP / (25. * mu_t * IRe);
  }
  c->diss[0] = KW_BETASTAR / tau_k;
  c->diss[1] = 0.0708 / tau_k;
  c->cross = chi > 0 ? chi * tau_k / 8. : 0.;
  const double gamma_star = (0.111111111111 + 0.338983050847 * Re_t) / (1. + 0.338983050847 * Re_t);
  const double beta_star = (0.266666666667 + 0.000244140625 * Re_t * Re_t * Re_t * Re_t) /
                           (1. + 0.000244140625 * Re_t * Re_t * Re_t * Re_t);
  c->diss[0] *= beta_star;
  c->src[1] *= gamma_star;
  c->ire[0] = IRe * (1. + KW_SIGMA_K * alpha_star * mu_t);
  c->ire[1] = IRe * (1. + KW_SIGMA_W * alpha_star * mu_t);
}

static void kw_element(or_sys *s, int lev, int mode, int var, const or_phys *ph, const double *vel,
                       const double *kold, const double *wold, double y, double nu_wall, const fe_tab *t, int e,
                       double *Ke, double *Fe, double *rhs) {
  const or_mesh *m = s->m;
  int dim = m->dim, nen = m->nen, top = s->nlev - 1, off = m->ntop, Ntop = m->nnodes[top];
  csr *A = &s->A[lev];
  int dofs[MAXEN], bcv[MAXEN], bcb[MAXEN];
  double xx[3 * MAXEN], vo[3][MAXEN], ko[MAXEN], wo[MAXEN];
  const double IRe = ph->inv_re, idt = ph->inv_dt;
  const int *c = m->conn[lev] + (long)e * nen;
  memset(Ke, 0, (size_t)nen * nen * sizeof(double));
  memset(Fe, 0, nen * sizeof(double));
  for (int k = 0; k < nen; k++) {
    for (int d = 0; d < dim; d++) xx[d * nen + k] = m->xyz[c[k] + (long)d * off];
    dofs[k] = s->node_dof[lev][c[k]];
    int td = s->node_dof[top][c[k]];
    bcv[k] = s->bc0[td];
    bcb[k] = s->bc1[td];
    for (int d = 0; d < dim; d++) vo[d][k] = vel ? vel[c[k] + d * Ntop] : 0.;
    ko[k] = kold[c[k]];
    wo[k] = wold[c[k]];
  }
  const double *vold = var == 0 ? ko : wo;
  double h[3];
  {
    int v2 = dim == 2 ? 2 : 6, v3 = dim == 2 ? 3 : 7;
    for (int d = 0; d < dim; d++) {
      h[d] = fabs(xx[d * nen + v2] - xx[d * nen + 0]);
      double h1 = fabs(xx[d * nen + v3] - xx[d * nen + 1]);
      if (h[d] < h1) h[d] = h1;
    }
  }
  kw_coef cf = {{IRe, IRe}, {0, 0}, {0, 0}, 0};
  for (int q = 0; q < t->ng; q++) {
    double ij[9];
    double det = jac(t, q, xx, nen, ij);
    double JxW = det * t->w[q];
    double dphi[MAXEN][3];
    for (int sh = 0; sh < nen; sh++)
      for (int i = 0; i < dim; i++) {
        double sum = 0.;
        for (int j = 0; j < dim; j++) sum += ij[j + i * dim] * t->dphi[q][sh][j];
        dphi[sh][i] = sum;
      }
    const double *phi = t->phi[q];
    double vg[3] = {0, 0, 0}, g[9] = {0}, gk[3] = {0, 0, 0}, gw[3] = {0, 0, 0}, kg[2] = {0, 0}, mod = 1e-20;
    for (int k = 0; k < nen; k++) {
      kg[0] += phi[k] * ko[k];
      kg[1] += phi[k] * wo[k];
      for (int d = 0; d < dim; d++) {
        vg[d] += phi[k] * vo[d][k];
        gk[d] += ko[k] * dphi[k][d];
        gw[d] += wo[k] * dphi[k][d];
        for (int a = 0; a < dim; a++) g[a * dim + d] += vo[a][k] * dphi[k][d];
      }
    }
    for (int d = 0; d < dim; d++) mod += vg[d] * vg[d];
    mod = sqrt(mod);
    double sP = 1.e-20, chi = 0., f[3];
    for (int a = 0; a < dim; a++)
      for (int b = 0; b < dim; b++) {
        const double sss = g[a + b * dim] + g[b + a * dim];
        sP += sss * sss;
      }
    for (int d = 0; d < dim; d++) {
      f[d] = upwind_f(KW_UP_WIND, 1., mod, h[d], IRe);
      chi += gk[d] * gw[d];
    }
    kw_model(kg, kg[1], sP, chi, IRe, &cf);
    const double ire = cf.ire[var];
    for (int i = 0; i < nen; i++) {
      const double dt = JxW * bcv[i];
      if (mode == 1) Fe[i] += dt * (kg[var] * phi[i] * idt + cf.src[var] * phi[i] + cf.cross * var * phi[i]);
      for (int j = 0; j < nen; j++) {
        double adv = 0., lap = 0.;
        for (int d = 0; d < dim; d++) {
          adv += vg[d] * dphi[j][d];
          lap += (ire + f[d] * vg[d] * vg[d]) * dphi[j][d] * dphi[i][d];
        }
        Ke[i * nen + j] += dt * (phi[j] * phi[i] * idt + adv * phi[i] + lap + cf.diss[var] * phi[j] * phi[i]);
      }
    }
  }
  /* boundary sides (MGSolverTBKW.C:305-412); IRe_eff is the last Gauss point's */
  for (int sd = 0; sd < m->nsides; sd++) {
    if (m->neigh[lev][(long)e * m->nsides + sd] != -1) continue;
    const int *sur = dim == 2 ? Q9_SIDE[sd] : H27_FACE[sd];
    int nsn = m->nsn;
    double xb[3 * 9];
    for (int k = 0; k < nsn; k++)
      for (int d = 0; d < dim; d++) xb[d * nsn + k] = xx[d * nen + sur[k]];
    int last = sur[nsn - 1];
    if (bcv[last] == 0) {
      const double ipen = jac_sur(t, t->sng - 1, xb, nsn) * idt;
      const double wall = 6. * nu_wall / (KW_BETASTAR * y * y);
      for (int k = 0; k < nsn; k++) {
        int lv = sur[k];
        int bs = bcb[lv], bc_rhs = (bs & 2) >> 1, bc_n = bs % 2;
        double kw = vold[lv] < 1.e-20 ? 1.e-20 : vold[lv];
        if (mode == 1) Fe[lv] += ipen * (bc_n * (1 - bc_rhs) * kw + (1 - bc_n) * bc_rhs * (var * wall));
        Ke[lv * nen + lv] += ipen;
      }
    } else if (bcb[last] != 0) {
      for (int q = 0; q < t->sng; q++) {
        double JxW = jac_sur(t, q, xb, nsn) * t->sw[q];
        for (int i = 0; i < nsn; i++) {
          int lei = sur[i];
          double dt = JxW * (bcv[lei] == 0 ? 0 : 1);
          int bc_n = bcb[lei] % 2;
          for (int j = 0; j < nsn; j++)
            Ke[lei * nen + sur[j]] += 2. * cf.ire[var] * dt * t->sphi[q][j] * t->sphi[q][i] * bc_n / y;
        }
      }
    }
  }
  for (int i = 0; i < nen; i++) {
    int gi = dofs[i];
    if (mode == 1) rhs[gi] += Fe[i];
    for (int j = 0; j < nen; j++) A->val[find_col(A, gi, dofs[j])] += Ke[i * nen + j];
  }
}

/* one level of the variable var of the coupled kappa-omega system on the scalar system
 * s (kind 0): matrix (and, mode 1, rhs) as or_sys_assemble; dist holds this level's
 * element wall distances */
void or_kw_assemble(or_sys *s, int lev, int mode, int var, const or_phys *ph, const double *vel,
                    const double *kold, const double *wold, const double *dist, double nu_wall) {
  const or_mesh *m = s->m;
  int dim = m->dim, nen = m->nen, top = s->nlev - 1;
  fe_tab t;
  fe_init(&t, dim);
  csr *A = &s->A[lev];
  memset(A->val, 0, (size_t)A->ptr[A->n] * sizeof(double));
  double *rhs = NULL;
  if (mode == 1) {
    rhs = s->b[lev];
    memset(rhs, 0, s->ndof[lev] * sizeof(double));
  }
  const int nel = m->nel[lev], ncol = 1 << dim;
  for (int c = 0; c < ncol; c++) {
#pragma omp parallel
    {
      double *Ke = (double *)malloc((size_t)nen * nen * sizeof(double));
      double *Fe = (double *)malloc(nen * sizeof(double));
#pragma omp for schedule(dynamic, 4)
      for (int e = 0; e < nel; e++)
        if (m->ecol[lev][e] == c)
          kw_element(s, lev, mode, var, ph, vel, kold, wold, dist[e], nu_wall, &t, e, Ke, Fe, rhs);
      free(Ke);
      free(Fe);
    }
  }
  if (mode == 1 && lev == top) memcpy(s->rhs, rhs, s->ndof[lev] * sizeof(double));
  if (lev == 0) s->lu_ok = 0;
}

/* MGSolDS::GenMatRhs with ALE_MOVING (template_appl/fsi/SRC/MGSolverDS.C:321-700), one
 * element: fluid (centre bc_vol < 1.5) rows dt JxW (bc_vol_i % 2) fl_int_i (100 Lap_ij) over
 * the Gauss points (:446-480), the boundary penalty det/_dt of sides whose last node has an
 * even bc_vol with the rhs of the x components, fsi_idx and disp_idx without _dir
 * (:600-650); solid rows KeM(i,i) = 1, FeM(i) = u_fsi[_dir] dt + d_old[_dir] (:664-671) */
static void ds_element(or_sys *s, int lev, int mode, int dir, double dt, const double *u, const double *dd,
                       const fe_tab *t, int e, double *Ke, double *Fe, double *rhs) {
  const or_mesh *m = s->m;
  int dim = m->dim, nen = m->nen, top = s->nlev - 1, off = m->ntop, Ntop = m->nnodes[top];
  csr *A = &s->A[lev];
  int dofs[MAXEN], bcv[MAXEN], bcb[MAXEN];
  double xx[3 * MAXEN];
  const int *c = m->conn[lev] + (long)e * nen;
  memset(Ke, 0, (size_t)nen * nen * sizeof(double));
  memset(Fe, 0, nen * sizeof(double));
  for (int k = 0; k < nen; k++) {
    for (int d = 0; d < dim; d++) xx[d * nen + k] = m->xyz[c[k] + (long)d * off];
    dofs[k] = s->node_dof[lev][c[k]];
    int td = s->node_dof[top][c[k]];
    bcv[k] = s->bc0[td];
    bcb[k] = s->bc1[td];
  }
  const int phase = bcv[nen - 1] < 1.5 ? 0 : 1;
  if (phase == 0) {
    for (int q = 0; q < t->ng; q++) {
      double ij[9];
      double det = jac(t, q, xx, nen, ij);
      double JxW = det * t->w[q];
      double dphi[MAXEN][3];
      for (int sh = 0; sh < nen; sh++)
        for (int i = 0; i < dim; i++) {
          double sum = 0.;
          for (int j = 0; j < dim; j++) sum += ij[j + i * dim] * t->dphi[q][sh][j];
          dphi[sh][i] = sum;
        }
      for (int i = 0; i < nen; i++) {
        int fl_int = bcv[i] > 3.5 ? 0 : 1;
        double dtxJxW = JxW * (bcv[i] % 2) * fl_int * dt;
        Fe[i] = 0.;
        for (int j = 0; j < nen; j++) {
          double lap = 0.;
          for (int d = 0; d < dim; d++) lap += dphi[j][d] * dphi[i][d];
          Ke[i * nen + j] += dtxJxW * (100 * lap);
        }
      }
    }
    for (int sd = 0; sd < m->nsides; sd++) {
      if (m->neigh[lev][(long)e * m->nsides + sd] != -1) continue;
      const int *sur = dim == 2 ? Q9_SIDE[sd] : H27_FACE[sd];
      int nsn = m->nsn;
      double xb[3 * 9];
      for (int k = 0; k < nsn; k++)
        for (int d = 0; d < dim; d++) xb[d * nsn + k] = xx[d * nen + sur[k]];
      int last = sur[nsn - 1];
      if (bcv[last] % 2 != 0) continue;
      int bc_var = bcb[last] % 2;
      double ipen = jac_sur(t, t->sng - 1, xb, nsn) / dt;
      for (int k = 0; k < nsn; k++) {
        int lv = sur[k];
        int fl_int = bcv[lv] > 3.5 ? 0 : 1;
        if (mode == 1) Fe[lv] += fl_int * bc_var * ipen * (u[c[lv]] * dt + dd[c[lv]]);
        Ke[lv * nen + lv] += fl_int * ipen;
      }
    }
  } else {
    for (int i = 0; i < nen; i++) {
      Fe[i] = u[c[i] + (long)dir * Ntop] * dt + dd[c[i] + (long)dir * Ntop];
      Ke[i * nen + i] = 1.;
    }
  }
  for (int i = 0; i < nen; i++) {
    int gi = dofs[i];
    if (mode == 1) rhs[gi] += Fe[i];
    for (int j = 0; j < nen; j++) A->val[find_col(A, gi, dofs[j])] += Ke[i * nen + j];
  }
}

/* one level of the displacement direction dir on the scalar system s (kind 0): matrix
 * (and, mode 1, rhs) as or_sys_assemble; u (the FSI velocity) and d (the old
 * displacements) are [dim][ntop] node fields */
void or_ds_assemble(or_sys *s, int lev, int mode, int dir, double dt, const double *u, const double *d) {
  const or_mesh *m = s->m;
  int dim = m->dim, nen = m->nen, top = s->nlev - 1;
  fe_tab t;
  fe_init(&t, dim);
  csr *A = &s->A[lev];
  memset(A->val, 0, (size_t)A->ptr[A->n] * sizeof(double));
  double *rhs = NULL;
  if (mode == 1) {
    rhs = s->b[lev];
    memset(rhs, 0, s->ndof[lev] * sizeof(double));
  }
  const int nel = m->nel[lev], ncol = 1 << dim;
  for (int c = 0; c < ncol; c++) {
#pragma omp parallel
    {
      double *Ke = (double *)malloc((size_t)nen * nen * sizeof(double));
      double *Fe = (double *)malloc(nen * sizeof(double));
#pragma omp for schedule(dynamic, 4)
      for (int e = 0; e < nel; e++)
        if (m->ecol[lev][e] == c) ds_element(s, lev, mode, dir, dt, u, d, &t, e, Ke, Fe, rhs);
      free(Ke);
      free(Fe);
    }
  }
  if (mode == 1 && lev == top) memcpy(s->rhs, rhs, s->ndof[lev] * sizeof(double));
  if (lev == 0) s->lu_ok = 0;
}

void or_sys_get_matrix(const or_sys *s, int lev, double *val) {
  memcpy(val, s->A[lev].val, (size_t)or_sys_nnz(s, lev) * sizeof(double));
}
void or_sys_set_matrix(or_sys *s, int lev, const double *val) {
  memcpy(s->A[lev].val, val, (size_t)or_sys_nnz(s, lev) * sizeof(double));
  if (lev == 0) s->lu_ok = 0;
}
void or_sys_get_rhs(const or_sys *s, double *rhs) { memcpy(rhs, s->rhs, s->ndof[s->nlev - 1] * sizeof(double)); }
void or_sys_set_rhs(or_sys *s, const double *rhs) {
  memcpy(s->rhs, rhs, s->ndof[s->nlev - 1] * sizeof(double));
}

/* A <- A^T on every level (structurally symmetric pattern) */
void or_sys_transpose_all(or_sys *s) {
  for (int l = 0; l < s->nlev; l++) {
    csr *A = &s->A[l];
    long nnz = A->ptr[A->n];
    double *nv = (double *)malloc(nnz * sizeof(double));
    for (int i = 0; i < A->n; i++)
      for (int q = A->ptr[i]; q < A->ptr[i + 1]; q++) nv[find_col(A, A->col[q], i)] = A->val[q];
    memcpy(A->val, nv, nnz * sizeof(double));
    free(nv);
  }
  s->lu_ok = 0;
}

/* ============================================================== threads */
void or_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
int or_get_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ============================================================== solvers */
void or_spmv(const or_sys *s, int lev, const double *x, double *y) {
  const csr *A = &s->A[lev];
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A->n; i++) {
    double sum = 0.;
    for (int q = A->ptr[i]; q < A->ptr[i + 1]; q++) sum += A->val[q] * x[A->col[q]];
    y[i] = sum;
  }
}

/* LaspackVectorM::resid (contrib/matrix/laspack_vectorM.C:147-168) */
static double resid(const or_sys *s, int lev, const double *x, const double *b, double *r) {
  const csr *A = &s->A[lev];
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A->n; i++) {
    double sum = 0.;
    for (int q = A->ptr[i]; q < A->ptr[i + 1]; q++) sum += A->val[q] * x[A->col[q]];
    r[i] = b[i] - sum;
  }
  double nr = 0.; /* in row order, whatever the thread count */
  for (int i = 0; i < A->n; i++) nr += r[i] * r[i];
  return sqrt(nr);
}
static double norm2(const double *v, int n) {
  double s = 0.;
  for (int i = 0; i < n; i++) s += v[i] * v[i];
  return sqrt(s);
}
/* LaspackVectorM::matrix_mult (laspack_vectorM.C:170-189) */
static void matmul(const csr *M, const double *x, double *y) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < M->n; i++) {
    double sum = 0.;
    for (int q = M->ptr[i]; q < M->ptr[i + 1]; q++) sum += M->val[q] * x[M->col[q]];
    y[i] = sum;
  }
}

/* multi-colour Gauss-Seidel (the parallel ordering of SORForwIter at omega=1,
 * contrib/laspack/itersolv.c:850-894); rows of one colour are not coupled, so each
 * colour's rows are updated in parallel exactly as in sequence */
static void gs_sweep(or_sys *s, int lev, double *x, const double *b, int reverse) {
  const csr *A = &s->A[lev];
  int nc = s->ncolour[lev];
  for (int cc = 0; cc < nc; cc++) {
    int c = reverse ? nc - 1 - cc : cc;
    const int t0 = s->col_off[lev][c], t1 = s->col_off[lev][c + 1];
#pragma omp parallel for schedule(static)
    for (int t = t0; t < t1; t++) {
      const int i = s->col_items[lev][t];
      double sum = b[i], d = 0.;
      for (int q = A->ptr[i]; q < A->ptr[i + 1]; q++) {
        if (A->col[q] == i) d = A->val[q];
        else sum -= A->val[q] * x[A->col[q]];
      }
      x[i] = sum / d;
    }
  }
}

/* multi-colour pressure-node Vanka with a diagonal velocity block: the restated
 * VankaNSIterD (contrib/laspack/itersolv.c:156-275) with the pressure-row residual,
 * the pressure-pressure entry and a damping omega.  Within one colour every patch's
 * correction is computed from the iterate at the start of the colour and then all
 * corrections are applied (patches of one colour are disjoint), so the result does not
 * depend on the order of patches inside a colour, and a colour's patches run in
 * parallel; colours run in sequence. */
#define OR_MAXSTAR (3 * 125 + 8)
static void vanka_sweep(or_sys *s, int lev, double *x, const double *b, double omega, int reverse, int l1) {
  const csr *A = &s->A[lev];
  int N = s->m->nnodes[lev], nv2 = s->nv2;
  int nc = s->ncolour[lev];
  int pbase = nv2 * N;
  int n = s->ndof[lev];
  double *dx = (double *)calloc(n, sizeof(double));
  char *touched = (char *)calloc(n, 1);
  for (int cc = 0; cc < nc; cc++) {
    int c = reverse ? nc - 1 - cc : cc;
    const int t0 = s->col_off[lev][c], t1 = s->col_off[lev][c + 1];
#pragma omp parallel
    {
      /* per star DOF of the patch: its diagonal (l1-modified) and its B^T coupling */
      double sa[OR_MAXSTAR], sg[OR_MAXSTAR];
#pragma omp for schedule(dynamic, 8)
      for (int t = t0; t < t1; t++) {
        const int mnode = s->col_items[lev][t];
        int pi = pbase + mnode;
        double rp = b[pi], cpp = 0.;
        double S = 0., T = 0.;
        for (int q = A->ptr[pi]; q < A->ptr[pi + 1]; q++) {
          int j = A->col[q];
          rp -= A->val[q] * x[j];
          if (j == pi) cpp = A->val[q];
        }
        /* pass 1: Schur sums */
        int ns = 0;
        for (int q = A->ptr[pi]; q < A->ptr[pi + 1]; q++) {
          int j = A->col[q];
          if (j >= pbase) continue;
          double r = b[j], a = 0., g = 0., al1 = 0.;
          for (int qq = A->ptr[j]; qq < A->ptr[j + 1]; qq++) {
            int cj = A->col[qq];
            r -= A->val[qq] * x[cj];
            if (cj == j) a = A->val[qq];
            if (cj == pi) g = A->val[qq];
            if (cj < pbase && cj != j) al1 += fabs(A->val[qq]);
          }
          if (l1) a = (a >= 0 ? a + 0.5 * al1 : a - 0.5 * al1);
          S += A->val[q] * g / a;
          T += A->val[q] * r / a;
          dx[j] = r; /* keep the residual for pass 2 */
          touched[j] = 1;
          sa[ns] = a;
          sg[ns] = g;
          ns++;
        }
        S -= cpp;
        T -= rp;
        double dp = (fabs(S) > 1e-300) ? T / S : 0.;
        /* pass 2: velocity corrections */
        ns = 0;
        for (int q = A->ptr[pi]; q < A->ptr[pi + 1]; q++) {
          int j = A->col[q];
          if (j >= pbase) continue;
          dx[j] = omega * (dx[j] - sg[ns] * dp) / sa[ns];
          ns++;
        }
        dx[pi] = omega * dp;
        touched[pi] = 1;
      }
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++)
      if (touched[i]) {
        x[i] += dx[i];
        dx[i] = 0.;
        touched[i] = 0;
      }
  }
  free(dx);
  free(touched);
}

/* full-block Vanka: exact solve of each pressure-node patch (velocity DOFs of the
 * pressure row + the pressure DOF) with a dense LU; reference analogue VankaNSIter
 * (contrib/laspack/itersolv.c:277-426), which approximates the same local system. */
static void dense_solve(double *a, double *r, int n) {
  for (int k = 0; k < n; k++) {
    int p = k;
    for (int i = k + 1; i < n; i++)
      if (fabs(a[i * n + k]) > fabs(a[p * n + k])) p = i;
    if (p != k) {
      for (int j = 0; j < n; j++) {
        double t = a[k * n + j];
        a[k * n + j] = a[p * n + j];
        a[p * n + j] = t;
      }
      double t = r[k];
      r[k] = r[p];
      r[p] = t;
    }
    double d = a[k * n + k];
    if (d == 0.) continue;
    for (int i = k + 1; i < n; i++) {
      double l = a[i * n + k] / d;
      if (l == 0.) continue;
      for (int j = k; j < n; j++) a[i * n + j] -= l * a[k * n + j];
      r[i] -= l * r[k];
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    double sum = r[i];
    for (int j = i + 1; j < n; j++) sum -= a[i * n + j] * r[j];
    r[i] = a[i * n + i] != 0. ? sum / a[i * n + i] : 0.;
  }
}
static void vanka_full_sweep(or_sys *s, int lev, double *x, const double *b, double omega, int reverse) {
  const csr *A = &s->A[lev];
  int N = s->m->nnodes[lev], nv2 = s->nv2, NL = s->nl[lev], nc = s->ncolour[lev];
  int pbase = nv2 * N;
  int maxp = 3 * 125 + 8;
  int *jj = (int *)malloc(maxp * sizeof(int));
  int *loc = (int *)malloc(s->ndof[lev] * sizeof(int));
  for (int i = 0; i < s->ndof[lev]; i++) loc[i] = -1;
  double *a = (double *)malloc((size_t)maxp * maxp * sizeof(double)), *r = (double *)malloc(maxp * sizeof(double));
  for (int cc = 0; cc < nc; cc++) {
    int c = reverse ? nc - 1 - cc : cc;
    for (int mnode = 0; mnode < NL; mnode++) {
      if (s->colour[lev][mnode] != c) continue;
      int pi = pbase + mnode, np = 0;
      for (int q = A->ptr[pi]; q < A->ptr[pi + 1]; q++)
        if (A->col[q] < pbase) jj[np++] = A->col[q];
      jj[np++] = pi;
      for (int k = 0; k < np; k++) loc[jj[k]] = k;
      memset(a, 0, (size_t)np * np * sizeof(double));
      for (int k = 0; k < np; k++) {
        int j = jj[k];
        double rr = b[j];
        for (int q = A->ptr[j]; q < A->ptr[j + 1]; q++) {
          rr -= A->val[q] * x[A->col[q]];
          int lc = loc[A->col[q]];
          if (lc >= 0) a[k * np + lc] = A->val[q];
        }
        r[k] = rr;
      }
      dense_solve(a, r, np);
      for (int k = 0; k < np; k++) {
        x[jj[k]] += omega * r[k];
        loc[jj[k]] = -1;
      }
    }
  }
  free(jj);
  free(loc);
  free(a);
  free(r);
}

void or_smooth(or_sys *s, int lev, const or_mg_params *p, int nsweeps, double *x, const double *b) {
  for (int it = 0; it < nsweeps; it++) {
    if (p->smoother == 0) gs_sweep(s, lev, x, b, p->reverse_colours);
    else if (p->smoother == 1) vanka_sweep(s, lev, x, b, p->omega, p->reverse_colours, 0);
    else if (p->smoother == 3) vanka_sweep(s, lev, x, b, p->omega, p->reverse_colours, 1);
    else vanka_full_sweep(s, lev, x, b, p->omega, p->reverse_colours);
  }
}

/* pressure gauge DOF: a pressure DOF flagged bc0 == 0.  The reference has no pressure
 * Dirichlet condition (pressure rows are never bc-scaled, MGSolverNS.C:458-489); the
 * enclosed-flow pressure level is fixed here by projection, p -= p[gauge], after each
 * cycle, and by an identity row in the coarsest direct solve only. */
static int is_gauge(const or_sys *s, int lev, int dof) {
  if (s->kind != 1) return 0;
  int N = s->m->nnodes[lev], base = s->nv2 * N;
  if (dof < base) return 0;
  int node = dof - base;
  int td = s->node_dof[s->nlev - 1][node + s->nv2 * s->m->ntop];
  return s->bc0[td] == 0;
}
static void gauge_shift(const or_sys *s, double *x) {
  if (s->kind != 1) return;
  int top = s->nlev - 1, N = s->m->nnodes[top], base = s->nv2 * N;
  for (int i = 0; i < s->nl[top]; i++)
    if (is_gauge(s, top, base + i)) {
      double p0 = x[base + i];
      for (int k = 0; k < s->nl[top]; k++) x[base + k] -= p0;
      return;
    }
}

/* dense LU with partial pivoting of the coarsest matrix (replaces the coarse
 * _solver[0]->solve(..., 60) of src/MGSolverBase.C:223 with a direct solve) */
static int coarse_factor(or_sys *s) {
  const csr *A = &s->A[0];
  int n = A->n;
  free(s->lu);
  free(s->piv);
  s->lu = (double *)calloc((size_t)n * n, sizeof(double));
  s->piv = (int *)malloc(n * sizeof(int));
  for (int i = 0; i < n; i++)
    for (int q = A->ptr[i]; q < A->ptr[i + 1]; q++) s->lu[(size_t)i * n + A->col[q]] = A->val[q];
  /* pressure gauge: the gauge DOF's row becomes the identity in the coarse factor only */
  for (int i = 0; i < n; i++)
    if (is_gauge(s, 0, i)) {
      for (int j = 0; j < n; j++) s->lu[(size_t)i * n + j] = 0.;
      s->lu[(size_t)i * n + i] = 1.;
    }
  double *a = s->lu;
  for (int k = 0; k < n; k++) {
    int p = k;
    double mx = fabs(a[(size_t)k * n + k]);
    for (int i = k + 1; i < n; i++)
      if (fabs(a[(size_t)i * n + k]) > mx) {
        mx = fabs(a[(size_t)i * n + k]);
        p = i;
      }
    s->piv[k] = p;
    if (mx == 0.) return -1;
    if (p != k)
      for (int j = 0; j < n; j++) {
        double t = a[(size_t)k * n + j];
        a[(size_t)k * n + j] = a[(size_t)p * n + j];
        a[(size_t)p * n + j] = t;
      }
    double inv = 1. / a[(size_t)k * n + k];
#pragma omp parallel for schedule(static) if (n - k > 64)
    for (int i = k + 1; i < n; i++) {
      double l = a[(size_t)i * n + k] * inv;
      a[(size_t)i * n + k] = l;
      if (l != 0.)
        for (int j = k + 1; j < n; j++) a[(size_t)i * n + j] -= l * a[(size_t)k * n + j];
    }
  }
  s->lu_ok = 1;
  return 0;
}

int or_coarse_solve(or_sys *s, const double *b, double *x) {
  if (!s->lu_ok && coarse_factor(s) != 0) return -1;
  int n = s->A[0].n;
  const double *a = s->lu;
  for (int i = 0; i < n; i++) x[i] = is_gauge(s, 0, i) ? 0. : b[i];
  for (int k = 0; k < n; k++) {
    int p = s->piv[k];
    if (p != k) {
      double t = x[k];
      x[k] = x[p];
      x[p] = t;
    }
  }
  for (int i = 0; i < n; i++) {
    double sum = x[i];
    for (int j = 0; j < i; j++) sum -= a[(size_t)i * n + j] * x[j];
    x[i] = sum;
  }
  for (int i = n - 1; i >= 0; i--) {
    double sum = x[i];
    for (int j = i + 1; j < n; j++) sum -= a[(size_t)i * n + j] * x[j];
    x[i] = sum / a[(size_t)i * n + i];
  }
  return 0;
}

/* One smoothing call of nsweeps sweeps that also returns the accuracy the reference's
 * level solver reports (LaspackLinearSolverM::solve returns GetLastAccuracy(),
 * contrib/matrix/laspack_linear_solverM.C:123-125): RTCResult stores ||r||/||b||
 * (contrib/laspack/rtc.c:48-70), and the stationary iterations evaluate it on a residual
 * they refresh only while Iter < MaxIter (SORForwIter, contrib/laspack/itersolv.c:850-894),
 * so after nsweeps >= 1 sweeps it is the relative residual of the iterate before the last
 * sweep; with no sweep, that of the iterate as given. */
static double smooth_acc(or_sys *s, int L, const or_mg_params *p, int nsweeps, double *x, const double *b,
                         double bn) {
  if (nsweeps > 0) or_smooth(s, L, p, nsweeps - 1, x, b);
  double acc = resid(s, L, x, b, s->r[L]) / bn;
  if (nsweeps > 0) or_smooth(s, L, p, 1, x, b);
  return acc;
}

/* MGSolBase::MGStep (src/MGSolverBase.C:212-289).  Returns the level's accuracy in the
 * reference's sense (smooth_acc of the post-smoothing call; after the coarse solve, its
 * relative residual), leaves r[L] = b - A x of the final iterate. */
static double mg_step(or_sys *s, int L, const or_mg_params *p) {
  int top = s->nlev - 1;
  double *x = s->x[L], *b = s->b[L], *r = s->r[L];
  double bn = norm2(b, s->ndof[L]);
  if (bn == 0.) bn = 1.;
  if (L == 0) {
    or_coarse_solve(s, b, x);
    return resid(s, 0, x, b, r) / bn;
  }
  int mul = (p->double_below_top && L < top) ? 2 : 1;
  double rest = smooth_acc(s, L, p, p->nu_pre * mul, x, b, bn);
  resid(s, L, x, b, r);
  matmul(&s->R[L - 1], r, s->b[L - 1]);
  memset(s->x[L - 1], 0, s->ndof[L - 1] * sizeof(double));
  double crest = 0.;
  for (int g = 0; g < p->gamma; g++) crest = mg_step(s, L - 1, p);
  matmul(&s->P[L], s->x[L - 1], r);
  if (!p->cond_corr || crest < rest) /* the conditional correction of :262-263 */
    for (int i = 0; i < s->ndof[L]; i++) x[i] += p->corr_damp * r[i];
  rest = smooth_acc(s, L, p, p->nu_post * mul, x, b, bn);
  resid(s, L, x, b, r);
  return rest;
}

/* MGSolBase::MGSolve (src/MGSolverBase.C:163-208): V-cycles until the relative
 * residual ||b-Ax||/||b|| reaches eps (stop_test 0, the workloads' stated test), or
 * until the top level's accuracy in the reference's sense falls below eps*(1+||b||)
 * (stop_test 1, the exit test of :201).  hist holds the relative residual. */
int or_mg_solve(or_sys *s, const or_mg_params *p, double *x, or_mg_stats *st) {
  int top = s->nlev - 1, n = s->ndof[top];
  memcpy(s->b[top], s->rhs, n * sizeof(double));
  memcpy(s->x[top], x, n * sizeof(double));
  double bn = norm2(s->b[top], n);
  st->bnorm = bn;
  st->converged = 0;
  st->cycles = 0;
  st->last_acc = 0.;
  double rel = resid(s, top, s->x[top], s->b[top], s->r[top]) / (bn > 0 ? bn : 1.);
  st->rel_res = rel;
  if (p->stop_test == 0 && rel <= p->eps) st->converged = 1;
  while (!st->converged && st->cycles < p->max_cycles) {
    double acc = mg_step(s, top, p);
    rel = norm2(s->r[top], n) / (bn > 0 ? bn : 1.);
    gauge_shift(s, s->x[top]);
    if (st->cycles < 256) st->hist[st->cycles] = rel;
    st->cycles++;
    st->rel_res = rel;
    st->last_acc = acc;
    if (!(rel == rel)) break;
    if (p->stop_test == 1 ? acc < p->eps * (1. + bn) : rel <= p->eps) st->converged = 1;
  }
  memcpy(x, s->x[top], n * sizeof(double));
  return st->converged ? 0 : 1;
}
