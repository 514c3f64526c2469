// mesh_refine.cpp -- a multilevel quad9 / hex27 hierarchy by uniform refinement of a coarse
// mesh, the role gencase plays upstream of the solver: libMesh's uniformly_refine(nlev - 1)
// on the coarse mesh and printMesh's level-nested node numbering
// (USER_APPL/gencase/src/MGGenCase.C:176-181, 234-...).
//
// Each element of level L has 2^dim children, the sub-cells of its reference element with
// its own orientation: child c = (cx, cy, cz) in {0, 1}^dim takes the points 2c + abc_k of
// the parent's 5^dim lattice (abc_k the local node's offset in half-element units,
// fe_topology.h), so its local node order is the libMesh one.  A lattice point with every
// coordinate even is a parent node; any other point is the centre of the sub-edge,
// sub-face or sub-cell spanned by the parent nodes at its neighbouring even points and is
// identified by that sorted set of parent nodes, so elements that share an edge or face
// create its new points once.  New points get the coordinates of the parent's
// triquadratic (biquadratic) map at the point's reference coordinates, so curved elements
// stay curved; a point keeps the coordinates of the first element that creates it.
//
// Numbering is level-nested as MGSolDA::init_dof requires (src/MGSolverDA.C:880-951):
// level L+1 keeps the nodes of level L with their numbers and appends its new points in
// the order the elements (and their local nodes) create them.  Element neighbours are
// found by matching side vertex sets; the parent of child e*2^dim + c is e.
#include <algorithm>
#include <array>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "exf_internal.h"
#include "fe_topology.h"

namespace exf {

namespace {

struct Hierarchy {
  int dim = 0, nlev = 0, nvert0 = 0;
  std::vector<int> nnodes, nel;
  std::vector<double> xyz;  // [dim][nnodes.back()] after finish
  std::vector<std::vector<double>> pts;  // per node, during refinement
  std::vector<int> conn, neigh, parent;  // all levels, level after level
};

// 1D quadratic Lagrange basis on the nodes -1, 0, 1 (offsets 0, 1, 2)
inline double lag(int a, double s) {
  if (a == 0) return 0.5 * s * (s - 1.);
  if (a == 1) return 1. - s * s;
  return 0.5 * s * (s + 1.);
}

template <int DIM>
int refine_dim(const exf_mesh_coarse *c, Hierarchy &H) {
  constexpr int NEN = DIM == 2 ? 9 : 27, NS = DIM == 2 ? 4 : 6, NSV = DIM == 2 ? 2 : 4;
  constexpr int NCH = 1 << DIM, NL = DIM == 2 ? 5 : 5;
  const int(*ABC)[3] = DIM == 2 ? Q9_ABC : H27_ABC;
  auto side_node = [](int s, int k) { return DIM == 2 ? Q9_SIDE[s][k] : H27_FACE[s][k]; };
  // local node at each point of the 3^dim element lattice
  int loc[3][3][3];
  for (int k = 0; k < NEN; k++) loc[ABC[k][0]][ABC[k][1]][DIM == 3 ? ABC[k][2] : 0] = k;

  H.dim = DIM;
  H.nlev = c->nlev;
  H.nvert0 = c->nvert0;
  H.nnodes.assign(1, c->nnode0);
  H.nel.assign(1, c->nel0);
  H.pts.assign(c->nnode0, std::vector<double>(DIM));
  for (int n = 0; n < c->nnode0; n++)
    for (int d = 0; d < DIM; d++) H.pts[n][d] = c->xyz0[(size_t)d * c->nnode0 + n];
  std::vector<int> cur(c->conn0, c->conn0 + (size_t)c->nel0 * NEN);
  for (int e = 0; e < c->nel0; e++)
    for (int k = 0; k < NEN; k++) {
      const int n = cur[(size_t)e * NEN + k];
      if (n < 0 || n >= c->nnode0 || (k < NCH) != (n < c->nvert0)) {
        set_error("exf_mesh_refine: element %d local node %d is node %d (nodes 0..%d are the %d vertices, "
                  "vertices first in each element)", e, k, n, c->nnode0 - 1, c->nvert0);
        return EXF_ERR_ARG;
      }
    }

  auto neighbours = [&](const std::vector<int> &cn, int nel, std::vector<int> &nb) {
    std::map<std::array<int, 4>, std::pair<int, int>> open;
    nb.assign((size_t)nel * NS, -1);
    for (int e = 0; e < nel; e++)
      for (int s = 0; s < NS; s++) {
        std::array<int, 4> key = {-1, -1, -1, -1};
        for (int k = 0; k < NSV; k++) key[k] = cn[(size_t)e * NEN + side_node(s, k)];
        std::sort(key.begin(), key.begin() + NSV);
        auto it = open.find(key);
        if (it == open.end()) {
          open.emplace(key, std::make_pair(e, s));
        } else {
          nb[(size_t)e * NS + s] = it->second.first;
          nb[(size_t)it->second.first * NS + it->second.second] = e;
          open.erase(it);
        }
      }
  };

  std::vector<int> nb;
  neighbours(cur, c->nel0, nb);
  H.conn = cur;
  H.neigh = nb;
  for (int l = 1; l < c->nlev; l++) {
    const int nel = H.nel.back();
    if ((long)nel * NCH > (1L << 30)) {
      set_error("exf_mesh_refine: level %d would have more than 2^30 elements", l);
      return EXF_ERR_ARG;
    }
    std::vector<int> next((size_t)nel * NCH * NEN);
    std::map<std::array<int, 8>, int> made;  // corner parent nodes of a new point -> node
    int nn = H.nnodes.back();
    for (int e = 0; e < nel; e++) {
      const int *pc = &cur[(size_t)e * NEN];
      int id[NL][NL][DIM == 3 ? NL : 1];
      const int nz = DIM == 3 ? NL : 1;
      for (int pz = 0; pz < nz; pz++)
        for (int py = 0; py < NL; py++)
          for (int px = 0; px < NL; px++) {
            const int p[3] = {px, py, pz};
            bool even = true;
            for (int d = 0; d < DIM; d++) even &= (p[d] % 2) == 0;
            if (even) {
              id[px][py][pz] = pc[loc[px / 2][py / 2][DIM == 3 ? pz / 2 : 0]];
              continue;
            }
            // the parent nodes at the even points around p
            std::array<int, 8> key;
            key.fill(-1);
            int nk = 0;
            for (int cz = 0; cz < (DIM == 3 ? 2 : 1); cz++)
              for (int cy = 0; cy < 2; cy++)
                for (int cx = 0; cx < 2; cx++) {
                  const int q[3] = {cx, cy, cz};
                  int a[3] = {0, 0, 0};
                  bool skip = false;
                  for (int d = 0; d < 3; d++) {
                    if (d >= DIM) break;
                    if (p[d] % 2 == 0) {
                      if (q[d]) skip = true;  // an even axis takes one corner
                      a[d] = p[d] / 2;
                    } else {
                      a[d] = (p[d] - 1) / 2 + q[d];
                    }
                  }
                  if (!skip) key[nk++] = pc[loc[a[0]][a[1]][a[2]]];
                }
            std::sort(key.begin(), key.begin() + nk);
            auto it = made.find(key);
            if (it != made.end()) {
              id[px][py][pz] = it->second;
              continue;
            }
            // a new point: the parent's map at reference coordinates p / 2 - 1
            std::vector<double> x(DIM, 0.);
            for (int k = 0; k < NEN; k++) {
              double w = 1.;
              for (int d = 0; d < DIM; d++) w *= lag(ABC[k][d], 0.5 * p[d] - 1.);
              for (int d = 0; d < DIM; d++) x[d] += w * H.pts[pc[k]][d];
            }
            H.pts.push_back(x);
            made.emplace(key, nn);
            id[px][py][pz] = nn++;
          }
      for (int ch = 0; ch < NCH; ch++) {
        const int cc[3] = {ch & 1, (ch >> 1) & 1, (ch >> 2) & 1};
        int *out = &next[((size_t)e * NCH + ch) * NEN];
        for (int k = 0; k < NEN; k++) {
          const int px = 2 * cc[0] + ABC[k][0], py = 2 * cc[1] + ABC[k][1];
          const int pz = DIM == 3 ? 2 * cc[2] + ABC[k][2] : 0;
          out[k] = id[px][py][pz];
        }
        H.parent.push_back(e);
      }
    }
    neighbours(next, nel * NCH, nb);
    H.nnodes.push_back(nn);
    H.nel.push_back(nel * NCH);
    H.conn.insert(H.conn.end(), next.begin(), next.end());
    H.neigh.insert(H.neigh.end(), nb.begin(), nb.end());
    cur.swap(next);
  }
  const int ntop = H.nnodes.back();
  H.xyz.assign((size_t)DIM * ntop, 0.);
  for (int n = 0; n < ntop; n++)
    for (int d = 0; d < DIM; d++) H.xyz[(size_t)d * ntop + n] = H.pts[n][d];
  H.pts.clear();
  return EXF_OK;
}

template <class T>
T *dup(const std::vector<T> &v) {
  T *p = static_cast<T *>(std::malloc(std::max<size_t>(1, v.size()) * sizeof(T)));
  if (p && !v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
  return p;
}

}  // namespace

}  // namespace exf

using namespace exf;

int exf_mesh_refine_arrays(const exf_mesh_coarse *c, exf_mesh_data *out) {
  if (!c || !out || (c->dim != 2 && c->dim != 3) || c->nlev < 1 || c->nlev > 12 || c->nnode0 < 1 || c->nel0 < 1 ||
      c->nvert0 < 1 || c->nvert0 > c->nnode0 || !c->xyz0 || !c->conn0) {
    set_error("exf_mesh_refine: bad argument");
    return EXF_ERR_ARG;
  }
  Hierarchy H;
  int rc;
  try {
    rc = c->dim == 2 ? refine_dim<2>(c, H) : refine_dim<3>(c, H);
  } catch (const std::bad_alloc &) {
    set_error("exf_mesh_refine: out of host memory");
    return EXF_ERR_NOMEM;
  }
  if (rc != EXF_OK) return rc;
  memset(out, 0, sizeof(*out));
  out->dim = c->dim;
  out->nlev = c->nlev;
  out->device = c->device;
  out->nvert0 = c->nvert0;
  out->nnodes = dup(H.nnodes);
  out->nel = dup(H.nel);
  out->xyz = dup(H.xyz);
  out->conn = dup(H.conn);
  out->neigh = dup(H.neigh);
  out->parent = c->nlev > 1 ? dup(H.parent) : nullptr;
  if (!out->nnodes || !out->nel || !out->xyz || !out->conn || !out->neigh || (c->nlev > 1 && !out->parent)) {
    exf_mesh_data_free(out);
    set_error("exf_mesh_refine: out of host memory");
    return EXF_ERR_NOMEM;
  }
  return EXF_OK;
}

void exf_mesh_data_free(exf_mesh_data *d) {
  if (!d) return;
  std::free(const_cast<int *>(d->nnodes));
  std::free(const_cast<double *>(d->xyz));
  std::free(const_cast<int *>(d->nel));
  std::free(const_cast<int *>(d->conn));
  std::free(const_cast<int *>(d->neigh));
  std::free(const_cast<int *>(d->parent));
  memset(d, 0, sizeof(*d));
}

int exf_mesh_refine(const exf_mesh_coarse *c, exf_mesh **out) {
  if (!out) return EXF_ERR_ARG;
  exf_mesh_data d;
  EXF_TRY(exf_mesh_refine_arrays(c, &d));
  const int rc = exf_mesh_upload(&d, out);
  exf_mesh_data_free(&d);
  return rc;
}
