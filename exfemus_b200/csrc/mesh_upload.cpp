// mesh_upload.cpp -- a multilevel quad9/hex27 hierarchy from host arrays: the state that
// MGMesh::read_c (src/MGMesh.C:493-908) holds after reading gencase's mesh file, for one
// subdomain (the LASPACK path is single-process, src/MGSolverBase.C:51-55).
//
// Node numbering is taken as given; it must be level-nested as MGSolDA::init_dof
// (src/MGSolverDA.C:880-951) assumes for one subdomain: the nodes of level L are the top
// nodes 0..nnodes[L]-1, the element vertices of level L are nodes of level L-1 (the Q1
// nodes of L), and those of level 0 are the first nvert0 nodes.  Element connectivity is
// in top node numbers (get_el_nod_conn, src/MGMesh.C:190-211), neighbours level-local.
//
// Element colours: greedy first fit in (z, y, x) order of the element centroids, an
// element taking the smallest colour no element sharing a node with it has.  On the
// structured boxes of exf_mesh_create this reproduces (ex&1)|(ey&1)<<1|(ez&1)<<2.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "exf_internal.h"
#include "fe_topology.h"

namespace exf {

// indices 0..n-1 ordered by the key (z, y, x) of points p(i) (stable: ties keep index order)
template <class P>
static std::vector<int> zyx_order(int n, int dim, P p) {
  std::vector<int> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
    for (int d = dim - 1; d >= 0; d--) {
      const double xa = p(a, d), xb = p(b, d);
      if (xa != xb) return xa < xb;
    }
    return false;
  });
  return ord;
}

// first-fit colouring of items in `order`: conflicts(i, visit) calls visit(j) for every item
// j that may not share i's colour
template <class F>
static int greedy_colour(int n, const std::vector<int> &order, F conflicts, std::vector<int> &colour) {
  colour.assign(n, -1);
  std::vector<int> stamp(64, -1);
  int ncol = 0;
  for (int i : order) {
    conflicts(i, [&](int j) {
      const int c = colour[j];
      if (c >= 0) {
        if (c >= (int)stamp.size()) stamp.resize(2 * c + 2, -1);
        stamp[c] = i;
      }
    });
    int c = 0;
    while (c < (int)stamp.size() && stamp[c] == i) c++;
    colour[i] = c;
    ncol = std::max(ncol, c + 1);
  }
  return ncol;
}

static void colour_elements(const exf_mesh *m, MeshLevel &ml) {
  const int nen = m->nen, nvx = m->nvx, dim = m->dim;
  // elements of every node
  std::vector<int> ptr(ml.nnodes + 1, 0), lst;
  for (size_t k = 0; k < ml.conn.size(); k++) ptr[ml.conn[k] + 1]++;
  for (int i = 0; i < ml.nnodes; i++) ptr[i + 1] += ptr[i];
  lst.resize(ptr[ml.nnodes]);
  std::vector<int> fill(ptr.begin(), ptr.end() - 1);
  for (int e = 0; e < ml.nel; e++)
    for (int k = 0; k < nen; k++) lst[fill[ml.conn[(size_t)e * nen + k]]++] = e;
  std::vector<double> cen((size_t)ml.nel * 3, 0.);
  for (int e = 0; e < ml.nel; e++)
    for (int d = 0; d < dim; d++) {
      double s = 0.;
      for (int k = 0; k < nvx; k++) s += m->xyz[(size_t)ml.conn[(size_t)e * nen + k] + (size_t)d * m->ntop];
      cen[3 * (size_t)e + d] = s / nvx;
    }
  const std::vector<int> ord = zyx_order(ml.nel, dim, [&](int e, int d) { return cen[3 * (size_t)e + d]; });
  greedy_colour(ml.nel, ord,
                [&](int e, auto visit) {
                  for (int k = 0; k < nen; k++) {
                    const int n = ml.conn[(size_t)e * nen + k];
                    for (int q = ptr[n]; q < ptr[n + 1]; q++)
                      if (lst[q] != e) visit(lst[q]);
                  }
                },
                ml.colour);
}

// node order used by the smoother colourings and sweep orders of uploaded meshes
std::vector<int> node_zyx_order(const exf_mesh *m, int n) {
  return zyx_order(n, m->dim, [&](int i, int d) { return m->xyz[(size_t)i + (size_t)d * m->ntop]; });
}

// smoother colouring of uploaded meshes: items ordered by node coordinates, first fit
int colour_items_greedy(const exf_mesh *m, int nitem, const std::vector<int> &order,
                        const std::vector<int> &cptr, const std::vector<int> &cidx, std::vector<int> &colour) {
  (void)m;
  return greedy_colour(nitem, order,
                       [&](int i, auto visit) {
                         for (int q = cptr[i]; q < cptr[i + 1]; q++)
                           if (cidx[q] != i) visit(cidx[q]);
                       },
                       colour);
}

}  // namespace exf

using namespace exf;

extern "C" int exf_mesh_upload(const exf_mesh_data *d, exf_mesh **out) {
  if (!d || !out || (d->dim != 2 && d->dim != 3) || d->nlev < 1 || d->nlev > 12 || !d->nnodes || !d->xyz ||
      !d->nel || !d->conn || !d->neigh) {
    set_error("exf_mesh_upload: bad descriptor");
    return EXF_ERR_ARG;
  }
  const int dim = d->dim, nlev = d->nlev;
  for (int l = 0; l < nlev; l++)
    if (d->nel[l] < 1 || d->nnodes[l] < 1 || (l > 0 && d->nnodes[l] < d->nnodes[l - 1])) {
      set_error("exf_mesh_upload: level %d has %d nodes and %d elements", l, d->nnodes[l], d->nel[l]);
      return EXF_ERR_ARG;
    }
  if (d->nvert0 < 1 || d->nvert0 > d->nnodes[0]) {
    set_error("exf_mesh_upload: nvert0 %d outside 1..%d", d->nvert0, d->nnodes[0]);
    return EXF_ERR_ARG;
  }
  EXF_CUDA(cudaSetDevice(d->device));
  exf_mesh *m = new exf_mesh();
  m->dim = dim;
  m->nlev = nlev;
  m->device = d->device;
  m->lattice = false;
  m->has_parent = d->parent != nullptr;
  m->nen = dim == 2 ? 9 : 27;
  m->nvx = dim == 2 ? 4 : 8;
  m->nsides = dim == 2 ? 4 : 6;
  m->nsn = dim == 2 ? 3 : 9;
  m->ntop = d->nnodes[nlev - 1];
  m->nvert0 = d->nvert0;
  m->xyz.assign(d->xyz, d->xyz + (size_t)dim * m->ntop);
  for (int k = 0; k < dim; k++) {
    double lo = m->xyz[(size_t)k * m->ntop], hi = lo;
    for (int i = 0; i < m->ntop; i++) {
      lo = std::min(lo, m->xyz[(size_t)i + (size_t)k * m->ntop]);
      hi = std::max(hi, m->xyz[(size_t)i + (size_t)k * m->ntop]);
    }
    m->box[2 * k] = lo;
    m->box[2 * k + 1] = hi;
  }
  auto fail = [&](const char *what, int l, long i) {
    set_error("exf_mesh_upload: %s (level %d, entry %ld)", what, l, i);
    delete m;
    return EXF_ERR_ARG;
  };
  m->lev.resize(nlev);
  long eoff = 0, poff = 0;
  for (int l = 0; l < nlev; l++) {
    MeshLevel &ml = m->lev[l];
    ml.nnodes = d->nnodes[l];
    ml.nel = d->nel[l];
    ml.ne[0] = ml.nel;
    const int nvl = l > 0 ? d->nnodes[l - 1] : d->nvert0;  // Q1 nodes of level l
    ml.conn.assign(d->conn + eoff * m->nen, d->conn + (eoff + ml.nel) * m->nen);
    ml.neigh.assign(d->neigh + eoff * m->nsides, d->neigh + (eoff + ml.nel) * m->nsides);
    for (long k = 0; k < (long)ml.conn.size(); k++) {
      const int n = ml.conn[k];
      if (n < 0 || n >= ml.nnodes) return fail("element node outside the level's nodes", l, k);
      if (k % m->nen < m->nvx && n >= nvl) return fail("element vertex is not a Q1 node of the level", l, k);
    }
    for (long k = 0; k < (long)ml.neigh.size(); k++)
      if (ml.neigh[k] < -1 || ml.neigh[k] >= ml.nel) return fail("neighbour outside the level's elements", l, k);
    if (m->has_parent && l > 0) {
      ml.parent.assign(d->parent + poff, d->parent + poff + ml.nel);
      for (int e = 0; e < ml.nel; e++)
        if (ml.parent[e] < 0 || ml.parent[e] >= d->nel[l - 1]) return fail("parent outside the coarser level", l, e);
      poff += ml.nel;
    }
    eoff += ml.nel;
    colour_elements(m, ml);
  }
  int rc = mesh_finish_levels(m);
  if (rc == EXF_OK) rc = upload_fe_table(m);
  if (rc != EXF_OK) {
    delete m;
    return rc;
  }
  *out = m;
  return EXF_OK;
}
