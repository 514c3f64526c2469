// mgsol_cuda_adapter.cpp -- the C++ adapter a maintainer adds to exFEMuS to run an
// equation's GenMatRhs / MGSolve / MGTimeStep through the B200 library, compiled against
// include/exfemus_b200.h and run as a test program.
//
// MGSolBase below is a stand-in for the reference's base class (include/MGSolverBase.h:
// 118-361): the same virtual methods with the same parameters, so the adapter's overrides
// are the ones MGSolNS / MGSolT would inherit.  The boundary flags come from a user
// bc_read(x, bc0, bc1) per top node, the role of MGSolNS::bc_read
// (template_appl/nse/SRC/User_NS.C) in GenBc (src/MGSolverDA.C:696-865), and reach the
// device through exf_sys_set_bc.  Errors abort with the library's message, as the
// reference's solvers do (contrib/matrix/laspack_linear_solverM.C:108-122).
//
// Run: a lid-driven cavity (Q2-Q1, 16x16, 3 levels, Re 400) for three Picard steps
// (MGTimeStep: x_old -> GenMatRhs on every level -> MGSolve -> x_old update), FP64 and then
// mixed precision; prints one line per step and exits 0 when every solve converged.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "exfemus_b200.h"

// ---------------------------------------------------------------- stand-in interface
class MGSolBase {
 public:
  virtual ~MGSolBase() {}
  virtual void MGDofBcOp() = 0;
  virtual void GenMatRhs(const double time, const int Level, const int mode) = 0;
  virtual void MGSolve(double Eps, int MaxIter, const int Gamma = 1, const int Nc_pre = 8,
                       const int Nc_coarse = 40, const int Nc_post = 8) = 0;
  virtual void MGTimeStep(const double time, const int delta_t_step_in) = 0;
};

// ---------------------------------------------------------------------- the adapter
class MGSolCuda : public MGSolBase {
 public:
  MGSolCuda(exf_mesh *mesh, int kind, int dim) : _mesh(mesh), _kind(kind), _dim(dim) {}
  ~MGSolCuda() override { exf_sys_destroy(_sys); }

  // init_dof + pattern + transfers, then GenBc from the user's bc_read
  void MGDofBcOp() override {
    check(exf_sys_create(_mesh, _kind, &_sys));
    int ntop = 0;
    int nlev = 0;
    while (exf_mesh_info(_mesh, nlev, nullptr, nullptr, nullptr) == EXF_OK) nlev++;
    _nlev = nlev;
    check(exf_mesh_info(_mesh, nlev - 1, &ntop, nullptr, nullptr));
    _ntop = ntop;
    int ndof = 0;
    check(exf_sys_ndof(_sys, nlev - 1, &ndof));
    _ndof = ndof;
    _xyz.resize((size_t)_dim * ntop);
    check(exf_mesh_get_xyz(_mesh, _xyz.data()));
    GenBc();
  }
  void GenMatRhs(const double /*time*/, const int Level, const int mode) override {
    check(exf_gen_mat_rhs(_sys, &_phys, Level, mode));
  }
  void MGSolve(double Eps, int MaxIter, const int Gamma = 1, const int Nc_pre = 8, const int /*Nc_coarse*/ = 40,
               const int Nc_post = 8) override {
    exf_mg_params p = _mg;
    p.eps = Eps;
    p.max_cycles = MaxIter;
    p.gamma = Gamma;
    p.nu_pre = Nc_pre;
    p.nu_post = Nc_post;
    const int rc = exf_mg_solve(_sys, &p, &_last);
    if (rc != EXF_OK && rc != EXF_ERR_NOT_CONVERGED) check(rc);
  }
  void MGTimeStep(const double time, const int) override {
    for (int l = _nlev - 1; l >= 0; l--) GenMatRhs(time, l, l == _nlev - 1 ? 1 : 0);
    MGSolve(1.e-10, 100, 1, 3, 40, 3);
    check(exf_sys_xold_update(_sys));
  }

  void set_xold(const std::vector<double> &x) { check(exf_sys_set_xold(_sys, x.data())); }
  std::vector<double> x() {
    std::vector<double> v(_ndof);
    check(exf_sys_get_x(_sys, v.data()));
    return v;
  }
  exf_phys _phys{};
  exf_mg_params _mg{};
  exf_solve_stats _last{};
  int _ndof = 0, _ntop = 0;

 protected:
  // the user's boundary rule for one node: bc0 = 1 natural / 0 Dirichlet per variable,
  // bc1 the variable's boundary-type flag
  virtual void bc_read(const double *xp, int *bc0, int *bc1) = 0;
  void GenBc() {
    std::vector<int> b0(_ndof, 1), b1(_ndof, 1);
    const int nv2 = _kind == EXF_KIND_NS ? _dim : 1;
    int NL = 0;  // pressure nodes of the top level: the Q2 nodes of the level below
    if (_nlev >= 2) check(exf_mesh_info(_mesh, _nlev - 2, &NL, nullptr, nullptr));
    else check(exf_mesh_info(_mesh, 0, nullptr, nullptr, &NL));
    for (int n = 0; n < _ntop; n++) {
      double xp[3] = {0, 0, 0};
      for (int d = 0; d < _dim; d++) xp[d] = _xyz[(size_t)n + (size_t)d * _ntop];
      int f0[4] = {1, 1, 1, 1}, f1[4] = {1, 1, 1, 1};
      bc_read(xp, f0, f1);
      for (int v = 0; v < nv2; v++) {
        b0[(size_t)v * _ntop + n] = f0[v];
        b1[(size_t)v * _ntop + n] = f1[v];
      }
      if (_kind == EXF_KIND_NS && n < NL) {
        b0[(size_t)nv2 * _ntop + n] = f0[nv2];
        b1[(size_t)nv2 * _ntop + n] = f1[nv2];
      }
    }
    check(exf_sys_set_bc(_sys, b0.data(), b1.data()));
  }
  static void check(int rc) {
    if (rc != EXF_OK) {
      std::fprintf(stderr, "exfemus_b200: %s\n", exf_last_error());
      std::abort();
    }
  }
  exf_mesh *_mesh;
  exf_sys *_sys = nullptr;
  int _kind, _dim, _nlev = 0;
  std::vector<double> _xyz;
};

// ------------------------------------------------------------ a user equation class
// lid-driven cavity: no-slip walls, u = 1 on the lid interior, the pressure fixed at the
// corner (0, 0)
class CavityNS : public MGSolCuda {
 public:
  explicit CavityNS(exf_mesh *m) : MGSolCuda(m, EXF_KIND_NS, 2) {}

 protected:
  void bc_read(const double *xp, int *bc0, int *bc1) override {
    const double eps = 1e-12;
    const bool wall = xp[0] < eps || xp[0] > 1 - eps || xp[1] < eps || xp[1] > 1 - eps;
    if (wall) {
      bc0[0] = bc0[1] = 0;
      bc1[0] = bc1[1] = 0;
      if (xp[1] > 1 - eps && xp[0] > eps && xp[0] < 1 - eps) bc1[0] = 4;  // nonhomogeneous: data in x_old
    }
    if (xp[0] < eps && xp[1] < eps) bc0[2] = 0;  // pressure gauge
  }
};

int main() {
  exf_mesh_desc d{};
  d.dim = 2;
  d.nlev = 3;
  d.n0[0] = d.n0[1] = 4;
  d.n0[2] = 1;
  d.box[1] = d.box[3] = 1.0;
  exf_mesh *mesh = nullptr;
  if (exf_mesh_create(&d, &mesh) != EXF_OK) {
    std::fprintf(stderr, "mesh: %s\n", exf_last_error());
    return 2;
  }
  int ok = 1;
  for (int prec = EXF_PREC_FP64; prec <= EXF_PREC_MIXED; prec++) {
    CavityNS ns(mesh);
    ns.MGDofBcOp();
    ns._phys.inv_re = 1.0 / 400.0;
    ns._phys.inv_prdl = ns._phys.rho = ns._phys.rhocp = ns._phys.penalty = 1.0;
    ns._phys.upwind_ns = 0.1;
    ns._phys.upwind_t = 1.0;
    ns._mg.double_below_top = 1;
    ns._mg.smoother = EXF_SMOOTH_VANKA;
    ns._mg.omega = 0.4;
    ns._mg.corr_damp = 0.95;
    ns._mg.precision = prec;
    ns._mg.use_graph = 1;
    // x_old carries the lid velocity at the nonhomogeneous Dirichlet nodes
    std::vector<double> xyz(2 * (size_t)ns._ntop), x0(ns._ndof, 0.0);
    exf_mesh_get_xyz(mesh, xyz.data());
    for (int n = 0; n < ns._ntop; n++)
      if (xyz[(size_t)ns._ntop + n] > 1 - 1e-12 && xyz[n] > 1e-12 && xyz[n] < 1 - 1e-12) x0[n] = 1.0;
    ns.set_xold(x0);
    for (int step = 0; step < 3; step++) {
      ns.MGTimeStep(0.0, 1);
      std::printf("precision %d step %d: cycles %d rel_res %.3e converged %d\n", prec, step, ns._last.cycles,
                  ns._last.rel_res, ns._last.converged);
      ok &= ns._last.converged && ns._last.rel_res <= 1e-10;
    }
    const std::vector<double> x = ns.x();
    double umax = 0.0;
    for (int n = 0; n < ns._ntop; n++) umax = std::fmax(umax, std::fabs(x[n]));
    std::printf("precision %d: max |u| %.6f\n", prec, umax);
    ok &= std::fabs(umax - 1.0) < 1e-8;  // the lid speed, reached on the lid
  }
  exf_mesh_destroy(mesh);
  std::printf(ok ? "adapter ok\n" : "adapter FAILED\n");
  return ok ? 0 : 1;
}
