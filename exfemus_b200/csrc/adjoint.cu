// adjoint.cu -- discrete adjoint of the temperature solve.
//
// With the advecting velocity frozen, the assembled heat system A T = b(q, g) is linear
// in the per-element sources q_e (rhs term bc_vol * q_e * int phi_i, MGSolverT.C volume
// rhs) and in the Dirichlet data g held in x_old at Dirichlet DOFs (rhs term
// bc_beta * Ipenalty * T_old, MGSolverT.C Dirichlet block).  For J = w^T T:
//   A^T lambda = w,   dJ/dq_e = sum_i lambda_i bc_vol_i int_e phi_i,   dJ/dg_i = lambda_i W_ii
// where W = d b / d x_old is diagonal (sum of the Dirichlet penalties of the sides that
// carry node i).  A^T is solved with the same multigrid on the transposed level
// matrices, colours swept in reverse order (the adjoint of a forward multi-colour sweep).
// Semantics follow LinearSolverM::adjoint_solve (contrib/matrix/linear_solverM.C) and
// KSPSolveTranspose (contrib/matrix/petsc_linear_solverM.C:691-732); the LASPACK backend
// aborts there (LaspackMatrixM::get_transpose, contrib/matrix/laspack_matrixM.C:97-99).
#include <cmath>
#include <vector>

#include "exf_internal.h"
#include "fe_topology.h"

namespace exf {

static double lag1h(int a, double x) {
  if (a == 0) return .5 * x * (x - 1.);
  if (a == 2) return .5 * x * (x + 1.);
  return 1. - x * x;
}
static double dlag1h(int a, double x) {
  if (a == 0) return x - .5;
  if (a == 2) return x + .5;
  return -2. * x;
}

template <int DIM>
struct SrcTab {
  static constexpr int NEN = DIM == 2 ? 9 : 27;
  double w[NEN];
  double phi[NEN][NEN];        // [qp][shape]
  double dphi[NEN][NEN][DIM];  // [qp][shape][dir]
};

template <int DIM>
__global__ void k_source_grad(SrcTab<DIM> tab, const int *conn, int nel, const double *xyz, int ntop,
                              const int *bc0, const double *lambda, double *djdq) {
  constexpr int NEN = SrcTab<DIM>::NEN;
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  const int *c = conn + (long)e * NEN;
  double acc = 0.;
  for (int q = 0; q < NEN; q++) {
    double J[DIM][DIM];
    for (int a = 0; a < DIM; a++)
      for (int b = 0; b < DIM; b++) {
        double s = 0.;
        for (int k = 0; k < NEN; k++) s += xyz[c[k] + (long)a * ntop] * tab.dphi[q][k][b];
        J[a][b] = s;
      }
    double det;
    if (DIM == 2) {
      det = J[0][0] * J[1][1] - J[1][0] * J[0][1];
    } else {
      const int o = DIM - 1;
      det = J[0][0] * (J[1][1] * J[o][o] - J[1][o] * J[o][1]) - J[0][1] * (J[1][0] * J[o][o] - J[1][o] * J[o][0]) +
            J[0][o] * (J[1][0] * J[o][1] - J[1][1] * J[o][0]);
    }
    const double JxW = det * tab.w[q];
    double s = 0.;
    for (int i = 0; i < NEN; i++) s += lambda[c[i]] * (double)bc0[c[i]] * tab.phi[q][i];
    acc += JxW * s;
  }
  djdq[e] = acc;
}

template <int DIM>
static int source_grad(exf_sys *s, const double *d_lambda, double *d_djdq) {
  SrcTab<DIM> t;
  const double g[3] = {-sqrt(3. / 5.), 0., sqrt(3. / 5.)};
  const double gw[3] = {5. / 9., 8. / 9., 5. / 9.};
  constexpr int NEN = SrcTab<DIM>::NEN;
  for (int q = 0; q < NEN; q++) {
    int iq[3] = {DIM == 2 ? q / 3 : q / 9, DIM == 2 ? q % 3 : (q / 3) % 3, DIM == 2 ? 1 : q % 3};
    double xi[3] = {g[iq[0]], g[iq[1]], g[iq[2]]};
    t.w[q] = gw[iq[0]] * gw[iq[1]] * (DIM == 3 ? gw[iq[2]] : 1.);
    for (int sh = 0; sh < NEN; sh++) {
      const int *abc = DIM == 2 ? Q9_ABC[sh] : H27_ABC[sh];
      double v = 1.;
      for (int d = 0; d < DIM; d++) v *= lag1h(abc[d], xi[d]);
      t.phi[q][sh] = v;
      for (int k = 0; k < DIM; k++) {
        double dv = 1.;
        for (int d = 0; d < DIM; d++) dv *= d == k ? dlag1h(abc[d], xi[d]) : lag1h(abc[d], xi[d]);
        t.dphi[q][sh][k] = dv;
      }
    }
  }
  exf_mesh *m = s->mesh;
  const MeshLevel &ml = m->lev[s->nlev - 1];
  k_source_grad<DIM><<<(ml.nel + 127) / 128, 128, 0, s->stream>>>(t, ml.d_conn.p, ml.nel, m->d_xyz.p, m->ntop,
                                                                  s->d_bc0.p, d_lambda, d_djdq);
  EXF_LAUNCH_CHECK();
  return EXF_OK;
}

__global__ void k_mul(const double *a, const double *b, double *c, long n) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) c[i] = a[i] * b[i];
}
__global__ void k_fill(double *a, double v, long n) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

}  // namespace exf

using namespace exf;

extern "C" {

int exf_adjoint_forward(exf_sys *s, const exf_phys *ph, const exf_mg_params *p, exf_solve_stats *st) {
  CHECK_SYS(s);
  if (!ph || !p || !st) return EXF_ERR_ARG;
  if (s->kind != EXF_KIND_T) {
    set_error("the adjoint entry points take the temperature system");
    return EXF_ERR_ARG;
  }
  if (s->transposed) EXF_TRY(exf_sys_transpose(s));
  EXF_TRY(exf_assemble_all(s, ph));
  return exf_mg_solve(s, p, st);
}

int exf_adjoint_backward(exf_sys *s, const exf_phys *ph, const exf_mg_params *p, const double *djdx, double *djdq,
                         double *djdg, exf_solve_stats *st) {
  CHECK_SYS(s);
  if (!ph || !p || !djdx || !st) return EXF_ERR_ARG;
  if (s->kind != EXF_KIND_T || !s->assembled) {
    set_error("exf_adjoint_backward needs an assembled temperature system (call exf_adjoint_forward)");
    return EXF_ERR_STATE;
  }
  const int top = s->nlev - 1;
  SysLevel &T = s->L[top];
  const long n = T.ndof;
  const long nel = s->mesh->lev[top].nel;
  cudaStream_t stm = s->stream;
  DBuf<double> &x_fwd = s->adj_x, &b_fwd = s->adj_b, &xold_sav = s->adj_xold, &qe_sav = s->adj_qe,
                &wdiag = s->adj_w, &lam = s->adj_lam, &gq = s->adj_gq;
  EXF_TRY(x_fwd.ensure(n));
  EXF_TRY(b_fwd.ensure(n));
  EXF_TRY(xold_sav.ensure(n));
  EXF_TRY(qe_sav.ensure(nel));
  EXF_TRY(wdiag.ensure(n));
  EXF_TRY(lam.ensure(n));
  EXF_TRY(gq.ensure(nel));
  EXF_CUDA(cudaMemcpyAsync(x_fwd.p, T.x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, stm));
  EXF_CUDA(cudaMemcpyAsync(b_fwd.p, T.b.p, n * sizeof(double), cudaMemcpyDeviceToDevice, stm));
  EXF_CUDA(cudaMemcpyAsync(xold_sav.p, s->xold.p, n * sizeof(double), cudaMemcpyDeviceToDevice, stm));
  EXF_CUDA(cudaMemcpyAsync(qe_sav.p, s->src_qe.p, nel * sizeof(double), cudaMemcpyDeviceToDevice, stm));
  // W = d b / d x_old (diagonal): rhs with x_old = 1, q = 0, no mass term
  exf_phys phw = *ph;
  phw.inv_dt = 0.;
  k_fill<<<(n + 255) / 256, 256, 0, stm>>>(s->xold.p, 1.0, n);
  EXF_CUDA(cudaMemsetAsync(s->src_qe.p, 0, nel * sizeof(double), stm));
  EXF_LAUNCH_CHECK();
  EXF_TRY(assemble_level(s, &phw, top, 1));
  EXF_CUDA(cudaMemcpyAsync(wdiag.p, T.b.p, n * sizeof(double), cudaMemcpyDeviceToDevice, stm));
  EXF_CUDA(cudaMemcpyAsync(s->xold.p, xold_sav.p, n * sizeof(double), cudaMemcpyDeviceToDevice, stm));
  EXF_CUDA(cudaMemcpyAsync(s->src_qe.p, qe_sav.p, nel * sizeof(double), cudaMemcpyDeviceToDevice, stm));
  EXF_TRY(assemble_level(s, ph, top, 1));  // restores the forward top matrix and rhs
  EXF_TRY(sync_fp32(s, top));
  // A^T lambda = dJ/dT with colours reversed
  EXF_TRY(exf_sys_transpose(s));
  EXF_CUDA(cudaMemcpyAsync(T.b.p, djdx, n * sizeof(double), cudaMemcpyHostToDevice, stm));
  EXF_CUDA(cudaMemsetAsync(T.x.p, 0, n * sizeof(double), stm));
  exf_mg_params pa = *p;
  pa.reverse_colours = !p->reverse_colours;
  int rc = exf_mg_solve(s, &pa, st);
  if (rc != EXF_OK && rc != EXF_ERR_NOT_CONVERGED) return rc;
  EXF_CUDA(cudaMemcpyAsync(lam.p, T.x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, stm));
  if (djdq) {
    EXF_TRY(s->dim == 2 ? source_grad<2>(s, lam.p, gq.p) : source_grad<3>(s, lam.p, gq.p));
    EXF_CUDA(cudaMemcpyAsync(djdq, gq.p, nel * sizeof(double), cudaMemcpyDeviceToHost, stm));
  }
  if (djdg) {
    k_mul<<<(n + 255) / 256, 256, 0, stm>>>(lam.p, wdiag.p, T.r.p, n);
    EXF_LAUNCH_CHECK();
    EXF_CUDA(cudaMemcpyAsync(djdg, T.r.p, n * sizeof(double), cudaMemcpyDeviceToHost, stm));
  }
  // restore the forward state
  EXF_TRY(exf_sys_transpose(s));
  EXF_CUDA(cudaMemcpyAsync(T.x.p, x_fwd.p, n * sizeof(double), cudaMemcpyDeviceToDevice, stm));
  EXF_CUDA(cudaMemcpyAsync(T.b.p, b_fwd.p, n * sizeof(double), cudaMemcpyDeviceToDevice, stm));
  EXF_CUDA(cudaStreamSynchronize(stm));
  return rc;
}

}  // extern "C"
