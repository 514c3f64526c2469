// soln_out.cpp -- solution output as XDMF over raw binary datasets: the role of
// MGEquationsSystem::print_soln (src/MGEquationsSystem.C:606-721) with HDF5 replaced by
// files that the XDMF text addresses by byte offset.
//
// What is written follows the reference's datasets one for one:
//  * MSH0CONN (MGMesh::print_conn_lin_hf5, src/MGMesh.C:1074-1195): every quad9 / hex27
//    element as its 2^dim linear sub-cells.  A sub-cell spans one cell of the element's
//    3^dim node lattice; its corners are listed in the element's own vertex order (the
//    lattice offsets of vertices 0..2^dim-1, halved), so each sub-cell has the element's
//    orientation.  Sub-cells come in the reference's order: in 2D the order of the vertex
//    each one holds (counter-clockwise), in 3D x fastest, then y, then z.
//  * X1, X2, X3 (MGMesh::print_mesh_h5, src/MGMesh.C:976-1015): node coordinates, X3 = 0
//    in 2D.
//  * one node dataset per variable (MGSolDA::print_u, src/MGSolverDA.C:1219-1290):
//    quadratic variables node by node; linear ones from the element's vertex values times
//    the linear basis at each node (the element Prol of MGGeomEl), so vertices keep their
//    values and the other nodes get averages of the vertices of the edge, face or cell
//    they sit in, summed in vertex order as the reference's row-by-vertex product does.
//  * the XDMF file (print_soln_xmf; MGMesh::print_xmf_topology / print_xmf_geometry,
//    src/MGMesh.C:439-477; MGSolDA::print_xml_attrib, src/MGSolverDA.C:1184-1214): Grid
//    "Mesh" with Time, Topology, Geometry X_Y_Z and one node Attribute per variable, each
//    DataItem Format="Binary" with Endian and Seek instead of an HDF path.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "exf_internal.h"
#include "fe_topology.h"

namespace exf {

namespace {

// corners (local node numbers) of the 2^dim linear sub-cells of a quad9 / hex27 element
template <int DIM>
std::vector<int> sub_cells() {
  constexpr int NEN = DIM == 2 ? 9 : 27, NVX = 1 << DIM;
  const int(*ABC)[3] = DIM == 2 ? Q9_ABC : H27_ABC;
  int loc[3][3][3];
  for (int k = 0; k < NEN; k++) loc[ABC[k][0]][ABC[k][1]][ABC[k][2]] = k;
  std::vector<int> sc;
  for (int s = 0; s < NVX; s++) {
    int o[3] = {0, 0, 0};
    for (int d = 0; d < DIM; d++) o[d] = DIM == 2 ? ABC[s][d] / 2 : (s >> d) & 1;
    for (int v = 0; v < NVX; v++) {
      int p[3] = {0, 0, 0};
      for (int d = 0; d < DIM; d++) p[d] = o[d] + ABC[v][d] / 2;
      sc.push_back(loc[p[0]][p[1]][p[2]]);
    }
  }
  return sc;
}

// value at every node of a linear variable given at the vertices, element by element
template <int DIM>
void linear_to_nodes(const exf_node_fields *f, const double *v, double *out) {
  constexpr int NEN = DIM == 2 ? 9 : 27, NVX = 1 << DIM;
  const int(*ABC)[3] = DIM == 2 ? Q9_ABC : H27_ABC;
  // w[k][j]: the linear basis of vertex j at node k (products of 0, 1/2, 1: exact)
  double w[NEN][NVX];
  for (int k = 0; k < NEN; k++)
    for (int j = 0; j < NVX; j++) {
      double x = 1.;
      for (int d = 0; d < DIM; d++) {
        const int a = ABC[k][d], b = ABC[j][d] / 2;  // node offset 0..2, vertex side 0..1
        x *= a == 1 ? 0.5 : (a / 2 == b ? 1. : 0.);
      }
      w[k][j] = x;
    }
  for (int e = 0; e < f->nel; e++) {
    const int *c = f->conn + (size_t)e * NEN;
    double vc[NVX];
    for (int j = 0; j < NVX; j++) vc[j] = v[c[j]];
    for (int k = 0; k < NEN; k++) {
      double s = 0.;
      for (int j = 0; j < NVX; j++) s += w[k][j] * vc[j];
      out[c[k]] = s;
    }
  }
}

std::string join(const char *dir, const std::string &name) {
  if (!dir || !*dir) return name;
  std::string d(dir);
  if (d.back() != '/') d += '/';
  return d + name;
}

std::string step_str(int t_step, int ndigits) {
  char b[32];
  snprintf(b, sizeof(b), "%0*d", ndigits, t_step);
  return b;
}

int write_file(const std::string &path, const std::vector<const void *> &parts, const std::vector<size_t> &bytes) {
  FILE *fp = fopen(path.c_str(), "wb");
  if (!fp) {
    set_error("exf_write_xdmf: cannot open %s for writing", path.c_str());
    return EXF_ERR_IO;
  }
  bool ok = true;
  for (size_t i = 0; i < parts.size() && ok; i++)
    if (bytes[i]) ok = fwrite(parts[i], 1, bytes[i], fp) == bytes[i];
  ok = (fclose(fp) == 0) && ok;
  if (!ok) {
    set_error("exf_write_xdmf: writing %s failed", path.c_str());
    return EXF_ERR_IO;
  }
  return EXF_OK;
}

}  // namespace

}  // namespace exf

using namespace exf;

namespace {

// a displacement system's variable name (MGSolDS: dx, dy, dz)
const char *ds_name(const exf_sys *s) { return s->ds_dir == 1 ? "dy" : s->ds_dir == 2 ? "dz" : "dx"; }

// one XDMF step (case_file: MGEquationsSystem::print_case_xmf, src/MGEquationsSystem.C:
// 872-935: no <Time>, the coordinates of the base mesh file <basemesh>.bin)
int write_xdmf_step(const exf_node_fields *f, const exf_soln_out *o, bool case_file) {
  if (!f || !o || (f->dim != 2 && f->dim != 3) || f->nnodes < 1 || f->nel < 1 || !f->xyz || !f->conn ||
      f->nvars < 0 || (f->nvars > 0 && (!f->names || !f->order || !f->vals)) || !o->basesol || !o->basemesh ||
      !o->connlin || o->ndigits < 1 || o->ndigits > 9 || o->t_step < 0) {
    set_error(case_file ? "exf_write_xdmf_case: bad argument" : "exf_write_xdmf: bad argument");
    return EXF_ERR_ARG;
  }
  const int dim = f->dim, nen = dim == 2 ? 9 : 27, nvx = 1 << dim, nsub = 1 << dim;
  const size_t nn = (size_t)f->nnodes;
  for (size_t i = 0; i < (size_t)f->nel * nen; i++)
    if (f->conn[i] < 0 || f->conn[i] >= f->nnodes) {
      set_error("exf_write_xdmf: element %zu local node %zu is node %d (of %d)", i / nen, i % nen, f->conn[i],
                f->nnodes);
      return EXF_ERR_ARG;
    }
  for (int v = 0; v < f->nvars; v++) {
    if (!f->names[v] || !*f->names[v] || (f->order[v] != 1 && f->order[v] != 2)) {
      set_error("exf_write_xdmf: variable %d needs a name and order 1 or 2", v);
      return EXF_ERR_ARG;
    }
    for (const char *c = f->names[v]; *c; c++)
      if (*c == '"' || *c == '<' || *c == '>' || *c == '&') {
        set_error("exf_write_xdmf: variable name %s is not plain XML text", f->names[v]);
        return EXF_ERR_ARG;
      }
  }
  const std::string step = step_str(o->t_step, o->ndigits);
  const std::string conn_name = std::string(o->basemesh) + o->connlin + ".bin";
  const std::string coord_name = std::string(o->basemesh) + (case_file ? "" : "." + step) + ".bin";
  const std::string sol_name = std::string(o->basesol) + "." + step + ".bin";
  const std::string xmf_name = std::string(o->basesol) + "." + step + ".xmf";

  // MSH0CONN
  const std::vector<int> sc = dim == 2 ? sub_cells<2>() : sub_cells<3>();
  const size_t nsc = (size_t)f->nel * nsub;
  std::vector<int32_t> conn_lin(nsc * nvx);
  for (int e = 0; e < f->nel; e++)
    for (int k = 0; k < nsub * nvx; k++) conn_lin[(size_t)e * nsub * nvx + k] = f->conn[(size_t)e * nen + sc[k]];
  EXF_TRY(write_file(join(o->dir, conn_name), {conn_lin.data()}, {conn_lin.size() * sizeof(int32_t)}));

  // X1, X2, X3
  std::vector<double> zero(dim == 2 ? nn : 0, 0.);
  std::vector<const void *> cp;
  std::vector<size_t> cb;
  for (int d = 0; d < 3; d++) {
    cp.push_back(d < dim ? (const void *)(f->xyz + d * nn) : (const void *)zero.data());
    cb.push_back(nn * sizeof(double));
  }
  EXF_TRY(write_file(join(o->dir, coord_name), cp, cb));

  // node datasets
  std::vector<double> sol((size_t)f->nvars * nn, 0.);
  for (int v = 0; v < f->nvars; v++) {
    const double *in = f->vals + (size_t)v * nn;
    double *out = sol.data() + (size_t)v * nn;
    if (f->order[v] == 2) {
      memcpy(out, in, nn * sizeof(double));
    } else if (dim == 2) {
      linear_to_nodes<2>(f, in, out);
    } else {
      linear_to_nodes<3>(f, in, out);
    }
  }
  EXF_TRY(write_file(join(o->dir, sol_name), {sol.data()}, {sol.size() * sizeof(double)}));

  // the XDMF text
  const uint16_t probe = 1;
  const char *endian = *(const unsigned char *)&probe ? "Little" : "Big";
  std::string x;
  char b[512];
  auto item = [&](const char *tag, const char *type, int prec, size_t rows, int cols, size_t seek,
                  const std::string &file) {
    snprintf(b, sizeof(b),
             "<%s DataType=\"%s\" Precision=\"%d\" Dimensions=\"%zu  %d\" Format=\"Binary\" Endian=\"%s\" "
             "Seek=\"%zu\">\n",
             tag, type, prec, rows, cols, endian, seek);
    x += b;
    x += file + "\n</" + tag + ">\n";
  };
  x += "<?xml version=\"1.0\" ?>\n<Xdmf>\n<Domain>\n<Grid Name=\"Mesh\">\n";
  if (!case_file) {
    snprintf(b, sizeof(b), "<Time Value=\"%.17g\" />\n", o->time);
    x += b;
  }
  snprintf(b, sizeof(b), "<Topology Type=\"%s\" Dimensions=\"%zu\">\n", dim == 2 ? "Quadrilateral" : "Hexahedron",
           nsc);
  x += b;
  item("DataStructure", "Int", 4, nsc, nvx, 0, conn_name);
  x += "</Topology>\n<Geometry Type=\"X_Y_Z\">\n";
  for (int d = 0; d < 3; d++) item("DataStructure", "Float", 8, nn, 1, d * nn * sizeof(double), coord_name);
  x += "</Geometry>\n";
  for (int v = 0; v < f->nvars; v++) {
    snprintf(b, sizeof(b), "<Attribute Name=\"%s\" AttributeType=\"Scalar\" Center=\"Node\">\n", f->names[v]);
    x += b;
    item("DataItem", "Float", 8, nn, 1, v * nn * sizeof(double), sol_name);
    x += "</Attribute>\n";
  }
  x += "</Grid>\n</Domain>\n</Xdmf>\n";
  return write_file(join(o->dir, xmf_name), {x.data()}, {x.size()});
}

}  // namespace

int exf_write_xdmf(const exf_node_fields *f, const exf_soln_out *o) { return write_xdmf_step(f, o, false); }
int exf_write_xdmf_case(const exf_node_fields *f, const exf_soln_out *o) { return write_xdmf_step(f, o, true); }

int exf_print_soln(exf_sys *const *sys, int nsys, const char *const *names, const double *refvalue,
                   const exf_soln_out *o) {
  if (!sys || nsys < 1 || !o) {
    set_error("exf_print_soln: bad argument");
    return EXF_ERR_ARG;
  }
  const exf_mesh *m = nullptr;
  for (int k = 0; k < nsys; k++) {
    CHECK_SYS(sys[k]);
    if (!m) m = sys[k]->mesh;
    if (sys[k]->mesh != m) {
      set_error("exf_print_soln: system %d lives on another mesh", k);
      return EXF_ERR_ARG;
    }
  }
  EXF_TRY(mesh_pull_xyz(const_cast<exf_mesh *>(m)));  // coordinates after mesh motion
  const size_t nn = (size_t)m->ntop;
  std::vector<std::string> nm;
  std::vector<int> order;
  std::vector<double> vals;
  int var = 0;
  for (int k = 0; k < nsys; k++) {
    exf_sys *s = sys[k];
    std::vector<double> x(s->L[s->nlev - 1].ndof);
    EXF_TRY(exf_sys_get_x(s, x.data()));
    const std::vector<int> &nd = s->node_dof[s->nlev - 1];
    for (int v = 0; v < s->nvars; v++, var++) {
      static const char *ns_names[4] = {"u", "v", "w", "p"};
      if (names) {
        nm.push_back(names[var] ? names[var] : "");
      } else if (s->kind == EXF_KIND_NS) {
        nm.push_back(v < s->nv2 ? ns_names[v] : "p");
      } else {
        nm.push_back(s->kind == EXF_KIND_K ? "kt" : s->kind == EXF_KIND_W ? "wt" : s->kind == EXF_KIND_DS ? ds_name(s) : "T");
      }
      order.push_back(v < s->nv2 ? 2 : 1);
      const double ref = refvalue ? refvalue[var] : 1.;
      const size_t base = vals.size();
      vals.resize(base + nn, 0.);
      for (size_t i = 0; i < nn; i++) {
        const int d = nd[i + (size_t)v * nn];
        if (d >= 0) vals[base + i] = x[d] * ref;
      }
    }
  }
  std::vector<const char *> np;
  for (const std::string &n : nm) np.push_back(n.c_str());
  const exf::MeshLevel &T = m->lev[m->nlev - 1];
  exf_node_fields f;
  f.dim = m->dim;
  f.nnodes = m->ntop;
  f.xyz = m->xyz.data();
  f.nel = T.nel;
  f.conn = T.conn.data();
  f.nvars = var;
  f.names = np.data();
  f.order = order.data();
  f.vals = vals.data();
  return exf_write_xdmf(&f, o);
}

// MGEquationsSystem::print_case (src/MGEquationsSystem.C:814-935): the initial state of
// every variable (x_old, MGSolDA::print_u) with its boundary flags (MGSolDA::print_bc,
// src/MGSolverDA.C:1418-1520): <name>bd = bc[1] and <name>vl = bc[0] at every node; for a
// linear variable the vertex flags are carried to the other nodes by the element's linear
// map and stored as integers (truncated), as print_bc's int buffer does.
int exf_print_case(exf_sys *const *sys, int nsys, const char *const *names, const double *refvalue,
                   const exf_soln_out *o) {
  if (!sys || nsys < 1 || !o) {
    set_error("exf_print_case: bad argument");
    return EXF_ERR_ARG;
  }
  const exf_mesh *m = nullptr;
  for (int k = 0; k < nsys; k++) {
    CHECK_SYS(sys[k]);
    if (!m) m = sys[k]->mesh;
    if (sys[k]->mesh != m) {
      set_error("exf_print_case: system %d lives on another mesh", k);
      return EXF_ERR_ARG;
    }
  }
  EXF_TRY(mesh_pull_xyz(const_cast<exf_mesh *>(m)));  // coordinates after mesh motion
  const size_t nn = (size_t)m->ntop;
  const exf::MeshLevel &T = m->lev[m->nlev - 1];
  const int nen = m->nen, nvx = m->nvx;
  const int(*ABC)[3] = m->dim == 2 ? Q9_ABC : H27_ABC;
  // linear basis of vertex j at node k (0, 1/2, 1 products), as linear_to_nodes
  std::vector<double> w((size_t)nen * nvx);
  for (int k = 0; k < nen; k++)
    for (int j = 0; j < nvx; j++) {
      double x = 1.;
      for (int d = 0; d < m->dim; d++) {
        const int a = ABC[k][d], b = ABC[j][d] / 2;
        x *= a == 1 ? 0.5 : (a / 2 == b ? 1. : 0.);
      }
      w[(size_t)k * nvx + j] = x;
    }
  std::vector<std::string> nm;
  std::vector<int> order;
  std::vector<double> vals;
  int var = 0;
  for (int k = 0; k < nsys; k++) {
    exf_sys *s = sys[k];
    std::vector<double> xo(s->L[s->nlev - 1].ndof);
    EXF_TRY(exf_sys_get_xold(s, xo.data()));
    const std::vector<int> &nd = s->node_dof[s->nlev - 1];
    for (int v = 0; v < s->nvars; v++, var++) {
      static const char *ns_names[4] = {"u", "v", "w", "p"};
      std::string name;
      if (names) name = names[var] ? names[var] : "";
      else if (s->kind == EXF_KIND_NS) name = v < s->nv2 ? ns_names[v] : "p";
      else name = s->kind == EXF_KIND_K ? "kt" : s->kind == EXF_KIND_W ? "wt" : s->kind == EXF_KIND_DS ? ds_name(s) : "T";
      const bool quad = v < s->nv2;
      const double ref = refvalue ? refvalue[var] : 1.;
      std::vector<double> val(nn, 0.), bd(nn, 0.), vl(nn, 0.);
      for (size_t i = 0; i < nn; i++) {
        const int d = nd[i + (size_t)v * nn];
        if (d < 0) continue;
        val[i] = xo[d] * ref;
        bd[i] = s->bc1[d];
        vl[i] = s->bc0[d];
      }
      if (!quad)  // the flags of the other nodes from the vertices, truncated to integers
        for (int e = 0; e < T.nel; e++) {
          const int *c = &T.conn[(size_t)e * nen];
          for (double *f : {bd.data(), vl.data()}) {
            double fc[8];
            for (int j = 0; j < nvx; j++) fc[j] = f[c[j]];
            for (int kk = 0; kk < nen; kk++) {
              double sum = 0.;
              for (int j = 0; j < nvx; j++) sum += w[(size_t)kk * nvx + j] * fc[j];
              f[c[kk]] = (double)(int)sum;
            }
          }
        }
      const std::string names3[3] = {name, name + "bd", name + "vl"};
      const std::vector<double> *data3[3] = {&val, &bd, &vl};
      for (int q = 0; q < 3; q++) {
        nm.push_back(names3[q]);
        order.push_back(q == 0 && !quad ? 1 : 2);
        vals.insert(vals.end(), data3[q]->begin(), data3[q]->end());
      }
    }
  }
  std::vector<const char *> np;
  for (const std::string &n : nm) np.push_back(n.c_str());
  exf_node_fields f;
  f.dim = m->dim;
  f.nnodes = m->ntop;
  f.xyz = m->xyz.data();
  f.nel = T.nel;
  f.conn = T.conn.data();
  f.nvars = (int)nm.size();
  f.names = np.data();
  f.order = order.data();
  f.vals = vals.data();
  return exf_write_xdmf_case(&f, o);
}
