// mesh_host.cpp -- structured multilevel quad9/hex27 hierarchy on the host.
//
// The reference reads this hierarchy from gencase's HDF5 output (MGMesh::read_c,
// src/MGMesh.C:493-908); gencase itself (USER_APPL/gencase/src/MGGenCase.C:63-232)
// needs libMesh.  Meshing stays on the host here too; the generator fixes the ordering
// rules gencase leaves to libMesh:
//   * the top level's Q2 nodes sit on an integer lattice (I,J,K);
//   * nodes are numbered class-major (class 0 = level-0 vertices, class l+1 = nodes that
//     first appear on level l), then K, J, I -- so level-L nodes are a prefix and the Q1
//     nodes of level L are the Q2 nodes of level L-1 (src/MGSolverDA.C:895-897);
//   * elements per level in (ez, ey, ex) order, colour (ex&1)|(ey&1)<<1|(ez&1)<<2;
//   * local node order of libMesh Quad9/Hex27 (fe_topology.h).
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>

#include "exf_internal.h"
#include "fe_topology.h"

namespace exf {

static int node_class(const exf_mesh *m, const int *p) {
  int s0 = 1 << (m->nlev - 1);
  bool v0 = true;
  for (int d = 0; d < 3; d++)
    if (p[d] % (2 * s0)) v0 = false;
  if (v0) return 0;
  for (int l = 0; l < m->nlev; l++) {
    int s = 1 << (m->nlev - 1 - l);
    bool ok = true;
    for (int d = 0; d < 3; d++)
      if (p[d] % s) ok = false;
    if (ok) return l + 1;
  }
  return m->nlev;
}

int build_mesh_host(exf_mesh *m) {
  const int dim = m->dim, nlev = m->nlev;
  m->nen = dim == 2 ? 9 : 27;
  m->nvx = dim == 2 ? 4 : 8;
  m->nsides = dim == 2 ? 4 : 6;
  m->nsn = dim == 2 ? 3 : 9;
  for (int d = 0; d < 3; d++) {
    if (d >= dim) m->n0[d] = 1;
    int nt = m->n0[d] << (nlev - 1);
    m->L[d] = d < dim ? 2 * nt + 1 : 1;
  }
  long nlat = (long)m->L[0] * m->L[1] * m->L[2];
  if (nlat > (1L << 30)) {
    set_error("mesh too large: %ld lattice nodes", nlat);
    return EXF_ERR_ARG;
  }
  m->ntop = (int)nlat;
  const int ncls = nlev + 1;
  std::vector<int> cnt(ncls + 1, 0);
  std::vector<int> cls(nlat);
  for (int K = 0; K < m->L[2]; K++)
    for (int J = 0; J < m->L[1]; J++)
      for (int I = 0; I < m->L[0]; I++) {
        int p[3] = {I, J, K};
        long li = ((long)K * m->L[1] + J) * m->L[0] + I;
        cls[li] = node_class(m, p);
        cnt[cls[li] + 1]++;
      }
  for (int c = 0; c < ncls; c++) cnt[c + 1] += cnt[c];
  m->nvert0 = cnt[1];
  m->lat.assign(3 * nlat, 0);
  m->xyz.assign((size_t)dim * nlat, 0.);
  std::vector<int> node_of_lat(nlat);
  std::vector<int> pos(cnt.begin(), cnt.end() - 1);
  for (int K = 0; K < m->L[2]; K++)
    for (int J = 0; J < m->L[1]; J++)
      for (int I = 0; I < m->L[0]; I++) {
        int p[3] = {I, J, K};
        long li = ((long)K * m->L[1] + J) * m->L[0] + I;
        int nd = pos[cls[li]]++;
        node_of_lat[li] = nd;
        for (int d = 0; d < 3; d++) m->lat[3 * nd + d] = p[d];
        for (int d = 0; d < dim; d++)
          m->xyz[nd + (size_t)d * nlat] =
              m->box[2 * d] + (m->box[2 * d + 1] - m->box[2 * d]) * ((double)p[d] / (double)(m->L[d] - 1));
      }
  m->lev.clear();
  m->lev.resize(nlev);
  for (int l = 0; l < nlev; l++) {
    MeshLevel &ml = m->lev[l];
    ml.nnodes = cnt[l + 2];
    int s = 1 << (nlev - 1 - l);
    for (int d = 0; d < 3; d++) ml.ne[d] = d < dim ? (m->n0[d] << l) : 1;
    ml.nel = ml.ne[0] * ml.ne[1] * ml.ne[2];
    ml.conn.assign((size_t)ml.nel * m->nen, 0);
    ml.neigh.assign((size_t)ml.nel * m->nsides, -1);
    ml.colour.assign(ml.nel, 0);
    for (int ez = 0; ez < ml.ne[2]; ez++)
      for (int ey = 0; ey < ml.ne[1]; ey++)
        for (int ex = 0; ex < ml.ne[0]; ex++) {
          int e = (ez * ml.ne[1] + ey) * ml.ne[0] + ex;
          int ee[3] = {ex, ey, ez};
          for (int k = 0; k < m->nen; k++) {
            const int *abc = dim == 2 ? Q9_ABC[k] : H27_ABC[k];
            int p[3];
            for (int d = 0; d < 3; d++) p[d] = d < dim ? (2 * ee[d] + abc[d]) * s : 0;
            long li = ((long)p[2] * m->L[1] + p[1]) * m->L[0] + p[0];
            ml.conn[(size_t)e * m->nen + k] = node_of_lat[li];
          }
          for (int sd = 0; sd < m->nsides; sd++) {
            const int *dir = dim == 2 ? Q9_SIDE_DIR[sd] : H27_FACE_DIR[sd];
            int q[3];
            bool ok = true;
            for (int d = 0; d < 3; d++) {
              q[d] = ee[d] + dir[d];
              if (q[d] < 0 || q[d] >= ml.ne[d]) ok = false;
            }
            ml.neigh[(size_t)e * m->nsides + sd] = ok ? (q[2] * ml.ne[1] + q[1]) * ml.ne[0] + q[0] : -1;
          }
          ml.colour[e] = (ex & 1) | ((ey & 1) << 1) | ((ez & 1) << 2);
        }
  }
  EXF_TRY(m->d_lat.alloc(m->lat.size()));
  EXF_CUDA(cudaMemcpy(m->d_lat.p, m->lat.data(), m->lat.size() * sizeof(int), cudaMemcpyHostToDevice));
  return mesh_finish_levels(m);
}

// Element lists grouped by colour (stable in element order) and the device copies of
// the connectivity, neighbours and coordinates.  Elements of one colour share no node, so
// one assembly launch per colour scatters into disjoint rows.
int mesh_finish_levels(exf_mesh *m) {
  for (int l = 0; l < m->nlev; l++) {
    MeshLevel &ml = m->lev[l];
    int ncol = 0;
    for (int e = 0; e < ml.nel; e++) ncol = std::max(ncol, ml.colour[e] + 1);
    std::vector<int> elist;
    elist.reserve(ml.nel);
    ml.ecol_off.assign(ncol + 1, 0);
    for (int c = 0; c < ncol; c++) {
      ml.ecol_off[c] = (int)elist.size();
      for (int e = 0; e < ml.nel; e++)
        if (ml.colour[e] == c) elist.push_back(e);
    }
    ml.ecol_off[ncol] = (int)elist.size();
    EXF_TRY(ml.d_conn.alloc(ml.conn.size()));
    EXF_TRY(ml.d_neigh.alloc(ml.neigh.size()));
    EXF_TRY(ml.d_elist.alloc(elist.size()));
    EXF_CUDA(cudaMemcpy(ml.d_conn.p, ml.conn.data(), ml.conn.size() * sizeof(int), cudaMemcpyHostToDevice));
    EXF_CUDA(cudaMemcpy(ml.d_neigh.p, ml.neigh.data(), ml.neigh.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (!elist.empty())
      EXF_CUDA(cudaMemcpy(ml.d_elist.p, elist.data(), elist.size() * sizeof(int), cudaMemcpyHostToDevice));
  }
  EXF_TRY(m->d_xyz.alloc(m->xyz.size()));
  EXF_CUDA(cudaMemcpy(m->d_xyz.p, m->xyz.data(), m->xyz.size() * sizeof(double), cudaMemcpyHostToDevice));
  return EXF_OK;
}

}  // namespace exf
