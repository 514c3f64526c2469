// assemble.cu -- element-batched Q2 (heat) and Q2-Q1 Taylor-Hood (Navier-Stokes)
// assembly into the node-block matrix (GenMatRhs).
//
// One CTA per element of the current colour; elements of one colour share no node,
// so every matrix/rhs entry they touch is written by exactly one CTA: the scatter is a
// plain read-add-write, needs no atomics, and the summation order is fixed by the
// colour order (results are deterministic).  Geometry, shape tables and per-Gauss-point
// coefficients live in shared memory; each thread owns (i,j) node pairs and integrates
// every variable block of that pair over the Gauss points.
//
// Restates MGSolT::GenMatRhs (template_appl/nse/SRC/MGSolverT.C:93-525) and
// MGSolNS::GenMatRhs (template_appl/nse/SRC/MGSolverNS.C:108-717), NS_EQUATIONS==1:
//   velocity blocks  (MGSolverNS.C:401-433), B^T (:438-452), B (:458-489),
//   upwind f = UP*rho*0.5*(coth Pe - 1/Pe)*h/|v| (:336-339),
//   rhs (:381-388), Dirichlet penalty Ipenalty = det_side*penalty (:531-601),
//   heat: MGSolverT.C volume block and Dirichlet/Robin boundary blocks.
#include <cmath>
#include <vector>

#include "exf_internal.h"
#include "fe_topology.h"

namespace exf {

template <int DIM>
struct FE {
  static constexpr int NEN = DIM == 2 ? 9 : 27;
  static constexpr int NVX = DIM == 2 ? 4 : 8;
  static constexpr int NQ = DIM == 2 ? 9 : 27;
  static constexpr int NSIDE = DIM == 2 ? 4 : 6;
  static constexpr int NSN = DIM == 2 ? 3 : 9;
  static constexpr int NSQ = DIM == 2 ? 3 : 9;
};

// reference-element tables, built once on the host (src/MGFE.C:195-945)
template <int DIM>
struct FETab {
  double w[FE<DIM>::NQ];
  double phi[FE<DIM>::NQ][FE<DIM>::NEN];
  double dphi[FE<DIM>::NQ][FE<DIM>::NEN][DIM];
  double psi[FE<DIM>::NQ][FE<DIM>::NVX];
  double sw[FE<DIM>::NSQ];
  double sphi[FE<DIM>::NSQ][FE<DIM>::NSN];
  double sdphi[FE<DIM>::NSQ][FE<DIM>::NSN][DIM - 1];
  double spsi[FE<DIM>::NSQ][DIM == 2 ? 2 : 4];  // linear shapes on the side's vertices
};

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
static double lin1(int a, double x) { return a == 0 ? .5 * (1. - x) : .5 * (1. + x); }

template <int DIM>
static void fill_tab(FETab<DIM> &t) {
  const double g[3] = {-sqrt(3. / 5.), 0., sqrt(3. / 5.)};
  const double gw[3] = {5. / 9., 8. / 9., 5. / 9.};
  using F = FE<DIM>;
  for (int q = 0; q < F::NQ; q++) {
    int iq[3];
    if (DIM == 2) {
      iq[0] = q / 3;
      iq[1] = q % 3;
      iq[2] = 1;
    } else {
      iq[0] = q / 9;
      iq[1] = (q / 3) % 3;
      iq[2] = q % 3;
    }
    double xi[3] = {g[iq[0]], g[iq[1]], DIM == 3 ? g[iq[2]] : 0.};
    t.w[q] = gw[iq[0]] * gw[iq[1]] * (DIM == 3 ? gw[iq[2]] : 1.);
    for (int s = 0; s < F::NEN; s++) {
      const int *abc = DIM == 2 ? Q9_ABC[s] : H27_ABC[s];
      double v = 1.;
      for (int d = 0; d < DIM; d++) v *= lag1(abc[d], xi[d]);
      t.phi[q][s] = v;
      for (int k = 0; k < DIM; k++) {
        double dv = 1.;
        for (int d = 0; d < DIM; d++) dv *= (d == k) ? dlag1(abc[d], xi[d]) : lag1(abc[d], xi[d]);
        t.dphi[q][s][k] = dv;
      }
    }
    for (int s = 0; s < F::NVX; s++) {
      const int *abc = DIM == 2 ? Q9_ABC[s] : H27_ABC[s];
      double v = 1.;
      for (int d = 0; d < DIM; d++) v *= lin1(abc[d], xi[d]);
      t.psi[q][s] = v;
    }
  }
  const int sdim = DIM - 1;
  for (int q = 0; q < F::NSQ; q++) {
    int iq[2];
    if (sdim == 1) {
      iq[0] = q;
      iq[1] = 1;
    } else {
      iq[0] = q / 3;
      iq[1] = q % 3;
    }
    double xi[2] = {g[iq[0]], g[iq[1]]};
    t.sw[q] = gw[iq[0]] * (sdim == 2 ? gw[iq[1]] : 1.);
    for (int s = 0; s < F::NSN; s++) {
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
      t.sphi[q][s] = v;
      for (int k = 0; k < sdim; k++) {
        double dv = 1.;
        for (int d = 0; d < sdim; d++) dv *= (d == k) ? dlag1(abc[d], xi[d]) : lag1(abc[d], xi[d]);
        t.sdphi[q][s][k] = dv;
      }
      if (s < (sdim == 1 ? 2 : 4)) {  // vertices come first on a side
        double w = 1.;
        for (int d = 0; d < sdim; d++) w *= lin1(abc[d], xi[d]);
        t.spsi[q][s] = w;
      }
    }
  }
}

struct SideTab {
  int nodes[6][9];
  int dir[6][3];
};

template <int DIM>
struct AsmArgs {
  const FETab<DIM> *tab;
  SideTab side;
  const int *elist;      // elements of this colour
  int nel_c;
  const int *conn, *neigh;
  const double *xyz;     // [dim][ntop]
  int ntop;
  int N, NL, Ntop;       // level Q2 nodes, level Q1 nodes, top Q2 nodes
  const int *bc0, *bc1;  // top-level flags
  const double *xold;    // own x_old (top)
  const double *vel;     // coupled NS x_old (top) for T, or null
  int vel_Ntop;
  const double *temp;    // coupled T x_old (top) for NS buoyancy, or null
  const double *kold, *wold;  // NS: kappa, omega x_old (top) of the eddy viscosity, or null
  const double *qe;      // per top element source (T), or null
  const int *qq_ptr, *ql_ptr;
  const uint8_t *pos_qq, *pos_ql;
  long nqq, nql, nqqL;
  double *vv, *vp, *pv, *pp;
  double *rhs;           // level rhs or null (mode 0)
  exf_phys ph;
  int kind;
};

template <int DIM>
__device__ double jac_sur(const FETab<DIM> *t, int q, const double (*xx)[FE<DIM>::NEN], const int *sur) {
  // side coordinates read from the element's coordinates in shared memory (xx[d][sur[s]])
  if (DIM == 2) {
    double dx = 0, dy = 0;
    for (int s = 0; s < 3; s++) {
      dx += xx[0][sur[s]] * t->sdphi[q][s][0];
      dy += xx[1][sur[s]] * t->sdphi[q][s][0];
    }
    return sqrt(dx * dx + dy * dy);
  } else {
    double a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
#pragma unroll 1
    for (int s = 0; s < 9; s++)
      for (int d = 0; d < 3; d++) {
        a[d] += xx[d][sur[s]] * t->sdphi[q][s][0];
        b[d] += xx[d][sur[s]] * t->sdphi[q][s][DIM - 2];
      }
    double c0 = a[1] * b[2] - a[2] * b[1], c1 = a[2] * b[0] - a[0] * b[2], c2 = a[0] * b[1] - a[1] * b[0];
    return sqrt(c0 * c0 + c1 * c1 + c2 * c2);
  }
}

// 3D: register cap for 4 CTAs per SM (64 registers, no spills; measured fastest)
#ifndef EXF_ASM_MINB3
#define EXF_ASM_MINB3 4
#endif
#ifndef EXF_ASM_MINB2
#define EXF_ASM_MINB2 1
#endif
// One element of one level (a CTA): element data, Gauss-point fields and coefficients,
// the volume integrals of every node pair, B / B^T, the rhs (mode 1) and the boundary
// sides, each added to the level's matrix in place (elements of one colour share no node).
template <int DIM, int NT>
__device__ __forceinline__ void assemble_element(const AsmArgs<DIM> &A, const int e, const int mode) {
  using F = FE<DIM>;
  constexpr int NEN = F::NEN, NVX = F::NVX, NQ = F::NQ;
  const int tid = threadIdx.x;
  const bool ns = A.kind == EXF_KIND_NS;
  const int nv2 = ns ? DIM : 1;

  __shared__ int s_conn[NEN];
  __shared__ double s_xx[DIM][NEN];
  __shared__ int s_bcv[DIM + 1][NEN];
  __shared__ int s_bcb[DIM + 1][NEN];
  __shared__ double s_uold[DIM + 1][NEN];
  __shared__ double s_vold[DIM][NEN];
  __shared__ double s_told[NEN];
  __shared__ double s_phi[NQ][NEN];
  __shared__ double s_dphi[NQ][NEN][DIM];
  __shared__ double s_psi[NQ][NVX];
  __shared__ double s_ij[NQ][DIM * DIM];
  __shared__ double s_JxW[NQ];
  __shared__ double s_cM[NQ];          // JxW*rho*inv_dt (NS) or JxW*rhocp*inv_dt (T)
  __shared__ double s_cA[NQ][DIM];     // JxW*rho*v_k
  __shared__ double s_cL[NQ][DIM];     // JxW*rho*(nu + f_k v_k^2)
  __shared__ double s_cT[NQ][DIM * DIM];  // JxW*rho*(nu + f_a v_a v_b)
  __shared__ double s_cR[NQ][DIM];     // rhs coefficient per component
  __shared__ double s_h[DIM];
  __shared__ double s_J[NQ][DIM * DIM];  // Jacobian entries per Gauss point
  __shared__ double s_vg[NQ][DIM + 1];   // velocity (and temperature) at each Gauss point
  __shared__ double s_kt[NEN], s_wt[NEN];  // NS with the eddy viscosity: kappa, omega

  const FETab<DIM> *t = A.tab;
  // ---- element data (get_el_dof_bc, get_el_sol)
  for (int k = tid; k < NEN; k += NT) {
    int nd = A.conn[(long)e * NEN + k];
    s_conn[k] = nd;
    for (int d = 0; d < DIM; d++) s_xx[d][k] = A.xyz[nd + (long)d * A.ntop];
    for (int v = 0; v < nv2; v++) {
      long td = (long)v * A.Ntop + nd;
      s_bcv[v][k] = A.bc0[td];
      s_bcb[v][k] = A.bc1[td];
      s_uold[v][k] = A.xold ? A.xold[td] : 0.;
    }
    if (ns && k < NVX) {
      long td = (long)nv2 * A.Ntop + nd;
      s_bcv[DIM][k] = A.bc0[td];
      s_bcb[DIM][k] = A.bc1[td];
      s_uold[DIM][k] = A.xold ? A.xold[td] : 0.;
    }
    for (int d = 0; d < DIM; d++) {
      if (ns) s_vold[d][k] = s_uold[d][k];
      else s_vold[d][k] = A.vel ? A.vel[nd + (long)d * A.vel_Ntop] : 0.;
    }
    if (ns) s_told[k] = A.temp ? A.temp[nd] : 0.;
    else s_told[k] = s_uold[0][k];
    if (ns && A.kold) {
      s_kt[k] = A.kold[nd];
      s_wt[k] = A.wold[nd];
    }
  }
  for (int i = tid; i < NQ * NEN; i += NT) (&s_phi[0][0])[i] = (&t->phi[0][0])[i];
  for (int i = tid; i < NQ * NVX; i += NT) (&s_psi[0][0])[i] = (&t->psi[0][0])[i];
  __syncthreads();
  if (tid < DIM) {
    const int v2 = DIM == 2 ? 2 : 6, v3 = DIM == 2 ? 3 : 7;
    double h = fabs(s_xx[tid][v2] - s_xx[tid][0]);
    double h1 = fabs(s_xx[tid][v3] - s_xx[tid][1]);
    s_h[tid] = h < h1 ? h1 : h;
  }
  __syncthreads();
  // ---- per Gauss point: Jacobian (src/MGFE.C:1066-1170), fields, coefficients
  const exf_phys &ph = A.ph;
  const double diff_t = ph.inv_prdl * ph.inv_re;
  const double q_e = (!ns && A.qe) ? A.qe[e] : 0.;
  // the 27-term sums of every Gauss point first, one per thread (Jacobian entries, then
  // the interpolated velocity and temperature), each in node order
  constexpr int NSUM = DIM * DIM + DIM + 1;
  for (int p = tid; p < NQ * NSUM; p += NT) {
    const int q = p / NSUM, c = p % NSUM;
    double sum = 0.;
    if (c < DIM * DIM) {
      const int a = c / DIM, b = c % DIM;
#pragma unroll 1
      for (int s = 0; s < NEN; s++) sum += s_xx[a][s] * t->dphi[q][s][b];
      s_J[q][c] = sum;
    } else if (c < DIM * DIM + DIM) {
      const int d = c - DIM * DIM;
#pragma unroll 1
      for (int k = 0; k < NEN; k++) sum += s_phi[q][k] * s_vold[d][k];
      s_vg[q][d] = sum;
    } else {
#pragma unroll 1
      for (int k = 0; k < NEN; k++) sum += s_phi[q][k] * s_told[k];
      s_vg[q][DIM] = sum;
    }
  }
  __syncthreads();
  // then per (Gauss point, component d): the inverse Jacobian (each of the DIM threads of a
  // point computes it, the d = 0 one stores it) and row d of the coefficients
  for (int pq = tid; pq < NQ * DIM; pq += NT) {
    const int q = pq / DIM, dd = pq % DIM;
    double J[DIM][DIM];
    for (int a = 0; a < DIM; a++)
      for (int b = 0; b < DIM; b++) J[a][b] = s_J[q][a * DIM + b];
    double det, inv[DIM][DIM];  // inv[b][a] = dxi_b/dx_a
    if (DIM == 2) {
      det = J[0][0] * J[1][1] - J[1][0] * J[0][1];
      double id = 1. / det;
      inv[0][0] = J[1][1] * id;
      inv[0][1] = -J[0][1] * id;
      inv[1][0] = -J[1][0] * id;
      inv[1][1] = J[0][0] * id;
    } else {
      const int o = DIM - 1;  // keeps indices in range for DIM==2 instantiations
      det = J[0][0] * (J[1][1] * J[o][o] - J[1][o] * J[o][1]) - J[0][1] * (J[1][0] * J[o][o] - J[1][o] * J[o][0]) +
            J[0][o] * (J[1][0] * J[o][1] - J[1][1] * J[o][0]);
      double id = 1. / det;
      inv[0][0] = (J[1][1] * J[o][o] - J[1][o] * J[o][1]) * id;
      inv[0][1] = (J[0][o] * J[o][1] - J[0][1] * J[o][o]) * id;
      inv[0][o] = (J[0][1] * J[1][o] - J[0][o] * J[1][1]) * id;
      inv[1][0] = (J[1][o] * J[o][0] - J[1][0] * J[o][o]) * id;
      inv[1][1] = (J[0][0] * J[o][o] - J[0][o] * J[o][0]) * id;
      inv[1][o] = (J[0][o] * J[1][0] - J[0][0] * J[1][o]) * id;
      inv[o][0] = (J[1][0] * J[o][1] - J[1][1] * J[o][0]) * id;
      inv[o][1] = (J[0][1] * J[o][0] - J[0][0] * J[o][1]) * id;
      inv[o][o] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
    }
    const double JxW = det * t->w[q];
    double vg[DIM], mod = 1e-20;
    for (int d = 0; d < DIM; d++) {
      vg[d] = s_vg[q][d];
      mod += vg[d] * vg[d];
    }
    const double tg = s_vg[q][DIM];
    mod = sqrt(mod);
    if (dd == 0) {
      for (int i = 0; i < DIM; i++)
        for (int j = 0; j < DIM; j++) s_ij[q][j + i * DIM] = inv[j][i];
      s_JxW[q] = JxW;
      s_cM[q] = JxW * (ns ? ph.rho : ph.rhocp) * ph.inv_dt;
    }
    const int a = dd;
    if (ns) {
      const double pe = 0.5 * mod * s_h[a] / ph.inv_re;
      const double fa = ph.upwind_ns * ph.rho * 0.5 * (1. / tanh(pe) - 1. / pe) * s_h[a] / mod;
      s_cA[q][a] = JxW * ph.rho * vg[a];
      s_cL[q][a] = JxW * ph.rho * (ph.inv_re + fa * vg[a] * vg[a]);
      for (int b = 0; b < DIM; b++) s_cT[q][a * DIM + b] = JxW * ph.rho * (ph.inv_re + fa * vg[a] * vg[b]);
      s_cR[q][a] = JxW * (ph.rho * vg[a] * ph.inv_dt + ph.rho * ph.ifr * ph.dirg[a] + ph.buoy * tg * ph.dirg[a]);
    } else {
      double fa = 0.;
      if (A.vel) {
        const double pe = 0.5 * mod * s_h[a] / diff_t;
        fa = ph.upwind_t * ph.rhocp * 0.5 * (1. / tanh(pe) - 1. / pe) * s_h[a] / mod;
      }
      s_cA[q][a] = JxW * ph.rhocp * vg[a];
      s_cL[q][a] = JxW * (diff_t + fa * vg[a] * vg[a]);
      if (a == 0) s_cR[q][0] = JxW * (ph.rhocp * tg * ph.inv_dt + q_e);
    }
  }
  __syncthreads();
  // global shape derivatives (get_dphi_gl_g, src/MGFE.C:1496-1520)
  for (int p = tid; p < NQ * NEN; p += NT) {
    int q = p / NEN, s = p % NEN;
    for (int i = 0; i < DIM; i++) {
      double sum = 0.;
      for (int j = 0; j < DIM; j++) sum += s_ij[q][j + i * DIM] * t->dphi[q][s][j];
      s_dphi[q][s][i] = sum;
    }
  }
  __syncthreads();
  if (ns && A.kold) {
    // the turbulence template's momentum equation (template_appl/turb-ckw/SRC/
    // MGSolverNS.C:256-293, f_mu :685-760): IRe_eff = IRe (1 + mu_t) in the viscous terms,
    // the upwind Peclet number keeps IRe; kappa-omega, WILCOX and LOWRE: tau = 1/omega,
    // Re_t = kappa tau / IRe, mu_t = alpha* Re_t capped by nut2 / IRe, then clamped
    for (int q = tid; q < NQ; q += NT) {
      double g[DIM][DIM], kg = 0., wg = 0.;
      for (int a = 0; a < DIM; a++)
        for (int d = 0; d < DIM; d++) g[a][d] = 0.;
      for (int k = 0; k < NEN; k++) {
        kg += s_phi[q][k] * s_kt[k];
        wg += s_phi[q][k] * s_wt[k];
        for (int a = 0; a < DIM; a++)
          for (int d = 0; d < DIM; d++) g[a][d] += s_uold[a][k] * s_dphi[q][k][d];
      }
      double sP = 1.e-20;
      for (int a = 0; a < DIM; a++)
        for (int b = 0; b < DIM; b++) {
          const double sss = g[a][b] + g[b][a];
          sP += sss * sss;
        }
      if (kg < 1.e-20) kg = 1.e-20;
      if (wg < 1.e-20) wg = 1.e-20;
      const double IRe = ph.inv_re, Re_t = kg * (1. / wg) / IRe;
      const double astar = (0.024 + 0.166666666667 * Re_t) / (1. + 0.166666666667 * Re_t);
      double mu_t = Re_t * astar;
      const double nut2 = kg / (7. * sqrt(astar * 0.5 * sP / 0.09) / 8.);
      if (mu_t * IRe > nut2) mu_t = nut2 / IRe;
      mu_t = fmin(fmax(mu_t, 1.e-6), 1.e+6);
      const double add = s_JxW[q] * ph.rho * IRe * mu_t;
      for (int a = 0; a < DIM; a++) {
        s_cL[q][a] += add;
        for (int b = 0; b < DIM; b++) s_cT[q][a * DIM + b] += add;
      }
    }
    __syncthreads();
  }

  // ---- volume integrals, node pairs (i,j)
  const int *qq_ptr = A.qq_ptr;
  for (int p = tid; p < NEN * NEN; p += NT) {
    const int i = p / NEN, j = p % NEN;
    const int ni = s_conn[i];
    const long blk = qq_ptr[ni] + A.pos_qq[((long)e * NEN + i) * NEN + j];
    if (!ns) {
      const double old = A.vv[blk];  // loaded before the Gauss-point loop hides its latency
      double K = 0.;
#pragma unroll 1
      for (int q = 0; q < NQ; q++) {
        const double pi = s_phi[q][i], pj = s_phi[q][j];
        double adv = 0., lap = 0.;
        for (int k = 0; k < DIM; k++) {
          const double gj = s_dphi[q][j][k];
          adv += s_cA[q][k] * gj;
          lap += s_cL[q][k] * gj * s_dphi[q][i][k];
        }
        K += pi * (s_cM[q] * pj + adv) + lap;
      }
      A.vv[blk] = old + s_bcv[0][i] * K;
    } else {
      double old[DIM * DIM];  // the pair's entries, loaded before the Gauss-point loop
      for (int c = 0; c < DIM * DIM; c++) old[c] = A.vv[(long)c * A.nqq + blk];
      double M = 0., T[DIM * DIM];
      for (int k = 0; k < DIM * DIM; k++) T[k] = 0.;
#pragma unroll 1
      for (int q = 0; q < NQ; q++) {
        const double pi = s_phi[q][i], pj = s_phi[q][j];
        double gj[DIM], gi[DIM], adv = 0., lap = 0.;
        for (int k = 0; k < DIM; k++) {
          gj[k] = s_dphi[q][j][k];
          gi[k] = s_dphi[q][i][k];
          adv += s_cA[q][k] * gj[k];
          lap += s_cL[q][k] * gj[k] * gi[k];
        }
        M += pi * (s_cM[q] * pj + adv) + lap;
        for (int a = 0; a < DIM; a++) {
          const double ga = s_dphi[q][j][a];
          for (int b = 0; b < DIM; b++) T[a * DIM + b] += s_cT[q][a * DIM + b] * ga * gi[b];
        }
      }
      for (int a = 0; a < DIM; a++) {
        const double bcv = s_bcv[a][i];
        for (int b = 0; b < DIM; b++) {
          double v = T[a * DIM + b] + (a == b ? M : 0.);
          A.vv[(long)(a * DIM + b) * A.nqq + blk] = old[a * DIM + b] + bcv * v;
        }
      }
    }
  }
  if (ns) {
    // E_b(iv, j) = sum_q JxW psi_iv d_b phi_j : B^T (velocity rows) and B (pressure rows)
    for (int p = tid; p < NVX * NEN; p += NT) {
      const int iv = p / NEN, j = p % NEN;
      // B^T: row (a, node j), column pressure vertex iv; B: pressure row iv, column (b,
      // node j); the entries are loaded before the Gauss-point loop
      const int nj = s_conn[j];
      const long kq = A.ql_ptr[nj] + A.pos_ql[((long)e * NEN + j) * NVX + iv];
      const int niv = s_conn[iv];
      const long kp = qq_ptr[niv] + A.pos_qq[((long)e * NEN + iv) * NEN + j];
      double oq[DIM], op[DIM];
      for (int a = 0; a < DIM; a++) {
        oq[a] = A.vp[(long)a * A.nql + kq];
        op[a] = A.pv[(long)a * A.nqqL + kp];
      }
      double E[DIM];
      for (int b = 0; b < DIM; b++) E[b] = 0.;
      for (int q = 0; q < NQ; q++) {
        const double w = s_JxW[q] * s_psi[q][iv];
        for (int b = 0; b < DIM; b++) E[b] += w * s_dphi[q][j][b];
      }
      for (int a = 0; a < DIM; a++) A.vp[(long)a * A.nql + kq] = oq[a] + s_bcv[a][j] * (-E[a]);
      for (int b = 0; b < DIM; b++) A.pv[(long)b * A.nqqL + kp] = op[b] + ph.rho * E[b];
    }
  }
  // rhs
  if (mode == 1) {
    for (int p = tid; p < nv2 * NEN; p += NT) {
      const int a = p / NEN, i = p % NEN;
      double &r = A.rhs[(long)a * A.N + s_conn[i]];
      const double old = r;
      double F = 0.;
      for (int q = 0; q < NQ; q++) F += s_phi[q][i] * s_cR[q][a];
      r = old + s_bcv[a][i] * F;
    }
  }
  __syncthreads();

  // ---- boundary sides: Dirichlet penalty (and Robin for T), one side at a time
  for (int sd = 0; sd < F::NSIDE; sd++) {
    if (A.neigh[(long)e * F::NSIDE + sd] != -1) continue;
    const int *sur = A.side.nodes[sd];
    const int last = sur[F::NSN - 1];
    const double det = jac_sur<DIM>(t, F::NSQ - 1, s_xx, sur);
    const double ipen = det * ph.penalty;
    // MGFE::normal_g (src/MGFE.C:1601-1646): 2D the tangent from side node 0 to 1 turned
    // clockwise, 3D (x1 - x0) x (x3 - x0), normalised
    double nrm[3] = {0., 0., 0.};
    {
      double t1[3] = {0., 0., 0.}, t3[3] = {0., 0., 0.};
      for (int d = 0; d < DIM; d++) {
        t1[d] = s_xx[d][sur[1]] - s_xx[d][sur[0]];
        if (DIM == 3) t3[d] = s_xx[d][sur[3]] - s_xx[d][sur[0]];
      }
      if (DIM == 2) {
        nrm[0] = t1[1];
        nrm[1] = -t1[0];
      } else {
        nrm[0] = t1[1] * t3[2] - t1[2] * t3[1];
        nrm[1] = t1[2] * t3[0] - t1[0] * t3[2];
        nrm[2] = t1[0] * t3[1] - t1[1] * t3[0];
      }
      double mm = 0.;
      for (int d = 0; d < DIM; d++) mm += nrm[d] * nrm[d];
      mm = sqrt(mm);
      for (int d = 0; d < DIM; d++) nrm[d] /= mm;
    }
    for (int p = tid; p < nv2 * F::NSN; p += NT) {
      const int a = p / F::NSN, k = p % F::NSN;
      const int lv = sur[k];
      const int nlv = s_conn[lv];
      const long blk = qq_ptr[nlv] + A.pos_qq[((long)e * NEN + lv) * NEN + lv];
      if (s_bcv[a][last] == 0) {
        if (!ns) {
          const int bc_beta = s_bcb[0][last] % 2;
          A.vv[blk] += ipen;
          if (mode == 1) A.rhs[nlv] += bc_beta * ipen * s_uold[0][lv];
        } else {
          const int bs = s_bcb[a][lv];
          const int bc_rhs = (bs & 4) >> 2, bc_tg = (bs & 2) >> 1, bc_n = bs % 2;
          double vdn = 0.;
          for (int d = 0; d < DIM; d++) vdn += nrm[d] * s_uold[d][lv];
          A.vv[(long)(a * DIM + a) * A.nqq + blk] +=
              ((1 - bc_n) * (1 - bc_tg) + bc_tg) * ipen + ipen * nrm[a] * nrm[a] * (bc_n - bc_tg);
          for (int b = a + 1; b < DIM; b++)
            A.vv[(long)(a * DIM + b) * A.nqq + blk] += ipen * nrm[b] * nrm[a] * (bc_n - bc_tg);
          if (mode == 1)
            A.rhs[(long)a * A.N + nlv] +=
                bc_rhs * ipen *
                ((1 - bc_n) * (1 - bc_tg) * s_uold[a][lv] + bc_n * vdn * nrm[a] +
                 bc_tg * (s_uold[a][lv] - vdn * nrm[a]));
        }
      } else if (ns && s_bcb[a][last] != 0) {
        // Neumann / Robin sides (template_appl/nse/SRC/MGSolverNS.C:604-681), alpha_t = 1:
        // row (a, lv) takes, per surface Gauss point, the tangential / normal Robin term
        // lumped on its diagonal, the normal-normal coupling to the later components and,
        // with phys.traction (the reference's MESHNUMBER == 1), the pressure traction
        // -n_a p_old phi
        constexpr int NVB = DIM == 2 ? 2 : 4;
        const int bs = s_bcb[a][lv];
        const int bc_rhs = (bs & 4) >> 2, bc_tg = (bs & 2) >> 1, bc_n = bs % 2;
        const int bcv2 = s_bcv[a][lv] % 2;
        double diag = 0., fr = 0.;
        for (int q = 0; q < F::NSQ; q++) {
          const double dt = jac_sur<DIM>(t, q, s_xx, sur) * t->sw[q] * bcv2;
          const double phii = t->sphi[q][k];
          double pg = 0.;
          for (int kv = 0; kv < NVB; kv++) pg += t->spsi[q][kv] * s_uold[DIM][sur[kv]];
          fr += -1. * bc_rhs * dt * phii * nrm[a] * pg;
          for (int j = 0; j < F::NSN; j++) {
            const double phij = t->sphi[q][j];
            diag += dt * bc_tg * phij * phii + dt * nrm[a] * nrm[a] * phij * phii * (bc_n - bc_tg);
          }
        }
        A.vv[(long)(a * DIM + a) * A.nqq + blk] += diag;
        for (int b = a + 1; b < DIM; b++)  // normal-normal coupling, one column node at a time
          for (int j = 0; j < F::NSN; j++) {
            double o = 0.;
            for (int q = 0; q < F::NSQ; q++)
              o += jac_sur<DIM>(t, q, s_xx, sur) * t->sw[q] * bcv2 * nrm[b] * nrm[a] * t->sphi[q][j] *
                   t->sphi[q][k] * (bc_n - bc_tg);
            const long bj = qq_ptr[nlv] + A.pos_qq[((long)e * NEN + lv) * NEN + sur[j]];
            A.vv[(long)(a * DIM + b) * A.nqq + bj] += o;
          }
        if (mode == 1 && ph.traction != 0.) A.rhs[(long)a * A.N + nlv] += fr;
      } else if (!ns && s_bcb[0][last] != 0) {
        // Robin: k dT/dn = -h T; the constant terms of the reference are zero
        const int bs = s_bcb[0][lv];
        const int bc_alpha = (bs & 2) >> 1;
        const double bv = s_bcv[0][lv];
        for (int j = 0; j < F::NSN; j++) {
          double v = 0.;
          for (int q = 0; q < F::NSQ; q++) v += jac_sur<DIM>(t, q, s_xx, sur) * t->sw[q] * t->sphi[q][k] * t->sphi[q][j];
          const long bj = qq_ptr[nlv] + A.pos_qq[((long)e * NEN + lv) * NEN + sur[j]];
          A.vv[bj] += bv * bc_alpha * diff_t * v;
        }
      }
    }
    __syncthreads();
  }
}

template <int DIM, int NT>
__global__ void __launch_bounds__(NT, DIM == 3 ? EXF_ASM_MINB3 : EXF_ASM_MINB2) k_assemble(AsmArgs<DIM> A, int mode) {
  assemble_element<DIM, NT>(A, A.elist[blockIdx.x], mode);
}

// One colour of every level in one launch: work item {level, element}, the level's
// arguments copied to shared memory (levels write separate matrices, so their elements of
// one colour run together; each entry still receives its elements in colour order)
template <int DIM, int NT>
__global__ void __launch_bounds__(NT, DIM == 3 ? EXF_ASM_MINB3 : EXF_ASM_MINB2)
    k_assemble_levels(const AsmArgs<DIM> *__restrict__ args, const int2 *__restrict__ work) {
  __shared__ AsmArgs<DIM> sA;
  static_assert(sizeof(AsmArgs<DIM>) % 4 == 0, "argument block copied in words");
  const int2 w = work[blockIdx.x];
  const int *src = reinterpret_cast<const int *>(args + w.x);
  int *dst = reinterpret_cast<int *>(&sA);
  for (int k = threadIdx.x; k < (int)(sizeof(AsmArgs<DIM>) / 4); k += NT) dst[k] = src[k];
  __syncthreads();
  assemble_element<DIM, NT>(sA, w.y, sA.rhs ? 1 : 0);
}

template <int DIM>
static int upload_tab(exf_mesh *m) {
  FETab<DIM> h;
  fill_tab<DIM>(h);
  EXF_TRY(m->d_fetab.alloc(sizeof(FETab<DIM>)));
  EXF_CUDA(cudaMemcpy(m->d_fetab.p, &h, sizeof(FETab<DIM>), cudaMemcpyHostToDevice));
  return EXF_OK;
}

// the mesh owns its element type's FE tables on its own device, so systems on different
// devices (driven from different threads) never share or replace them
int upload_fe_table(exf_mesh *m) { return m->dim == 2 ? upload_tab<2>(m) : upload_tab<3>(m); }

// the arguments of level lev's assembly, its matrix (and rhs for mode 1) zeroed on the stream
template <int DIM>
static int level_args(exf_sys *s, const exf_phys *ph, int lev, int mode, AsmArgs<DIM> &a) {
  exf_mesh *m = s->mesh;
  if (!m->d_fetab.p || m->d_fetab.n != sizeof(FETab<DIM>)) {
    set_error("assembly: the mesh has no FE tables of dimension %d", DIM);
    return EXF_ERR_STATE;
  }
  SysLevel &L = s->L[lev];
  const MeshLevel &ml = m->lev[lev];
  const int top = s->nlev - 1;
  cudaStream_t st = s->stream;
  memset(&a, 0, sizeof(a));
  a.tab = reinterpret_cast<const FETab<DIM> *>(m->d_fetab.p);
  for (int sd = 0; sd < FE<DIM>::NSIDE; sd++) {
    for (int k = 0; k < FE<DIM>::NSN; k++) a.side.nodes[sd][k] = DIM == 2 ? Q9_SIDE[sd][k] : H27_FACE[sd][k];
    for (int d = 0; d < 3; d++) a.side.dir[sd][d] = DIM == 2 ? Q9_SIDE_DIR[sd][d] : H27_FACE_DIR[sd][d];
  }
  a.conn = ml.d_conn.p;
  a.neigh = ml.d_neigh.p;
  a.xyz = m->d_xyz.p;
  a.ntop = m->ntop;
  a.N = L.N;
  a.NL = L.NL;
  a.Ntop = s->L[top].N;
  a.bc0 = s->d_bc0.p;
  a.bc1 = s->d_bc1.p;
  a.xold = s->xold.p;
  a.vel = nullptr;
  a.temp = nullptr;
  a.vel_Ntop = s->L[top].N;
  if (s->other && s->kind == EXF_KIND_T && s->other->kind == EXF_KIND_NS) {
    a.vel = s->other->xold.p;
    a.vel_Ntop = s->other->L[top].N;
  }
  if (s->other && s->kind == EXF_KIND_NS && s->other->kind == EXF_KIND_T) a.temp = s->other->xold.p;
  a.kold = a.wold = nullptr;
  if (s->kind == EXF_KIND_NS && s->ns_k && s->ns_w) {
    a.kold = s->ns_k->xold.p;
    a.wold = s->ns_w->xold.p;
  }
  a.qe = (lev == top && s->kind == EXF_KIND_T) ? s->src_qe.p : nullptr;
  a.qq_ptr = L.qq_ptr.p;
  a.ql_ptr = L.ql_ptr.p;
  a.pos_qq = L.pos_qq.p;
  a.pos_ql = L.pos_ql.p;
  a.nqq = L.nqq;
  a.nql = L.nql;
  a.nqqL = L.nqqL;
  a.vv = L.A.vv.p;
  a.vp = L.A.vp.p;
  a.pv = L.A.pv.p;
  a.pp = L.A.pp.p;
  a.rhs = mode == 1 ? L.b.p : nullptr;
  a.ph = *ph;
  a.kind = s->kind;
  EXF_TRY(L.A.vv.zero(st));
  if (s->nv1) {
    EXF_TRY(L.A.vp.zero(st));
    EXF_TRY(L.A.pv.zero(st));
    EXF_TRY(L.A.pp.zero(st));
  }
  if (mode == 1) EXF_TRY(L.b.zero(st));
  return EXF_OK;
}

template <int DIM>
static int assemble_dim(exf_sys *s, const exf_phys *ph, int lev, int mode) {
  AsmArgs<DIM> a;
  EXF_TRY(level_args<DIM>(s, ph, lev, mode, a));
  const MeshLevel &ml = s->mesh->lev[lev];
  constexpr int NT = DIM == 2 ? 128 : 256;
  for (int c = 0; c + 1 < (int)ml.ecol_off.size(); c++) {
    int n = ml.ecol_off[c + 1] - ml.ecol_off[c];
    if (n == 0) continue;
    a.elist = ml.d_elist.p + ml.ecol_off[c];
    a.nel_c = n;
    k_assemble<DIM, NT><<<n, NT, 0, s->stream>>>(a, mode);
    EXF_LAUNCH_CHECK();
    EXF_COUNT(1);
  }
  return EXF_OK;
}

// every level (the top one with its rhs) in one launch per colour: the work list of
// colour c is {level, element} for every level's elements of colour c, top level first,
// built once per system
template <int DIM>
static int assemble_all_dim(exf_sys *s, const exf_phys *ph) {
  const int nl = s->nlev, top = nl - 1;
  exf_mesh *m = s->mesh;
  if (s->asm_work_off.empty()) {
    int ncol = 0;
    for (int l = 0; l < nl; l++) ncol = std::max(ncol, (int)m->lev[l].ecol_off.size() - 1);
    std::vector<int2> work;
    std::vector<int> off(1, 0);
    for (int c = 0; c < ncol; c++) {
      for (int l = top; l >= 0; l--) {
        const MeshLevel &ml = m->lev[l];
        if (c + 1 >= (int)ml.ecol_off.size()) continue;
        std::vector<int> el(ml.ecol_off[c + 1] - ml.ecol_off[c]);
        if (!el.empty())
          EXF_CUDA(cudaMemcpy(el.data(), ml.d_elist.p + ml.ecol_off[c], el.size() * sizeof(int),
                              cudaMemcpyDeviceToHost));
        for (int e : el) work.push_back(make_int2(l, e));
      }
      off.push_back((int)work.size());
    }
    EXF_TRY(s->asm_work.alloc(std::max<size_t>(1, work.size()) * sizeof(int2)));
    if (!work.empty())
      EXF_CUDA(cudaMemcpy(s->asm_work.p, work.data(), work.size() * sizeof(int2), cudaMemcpyHostToDevice));
    s->asm_work_off = off;
  }
  std::vector<AsmArgs<DIM>> args(nl);
  for (int l = 0; l < nl; l++) EXF_TRY(level_args<DIM>(s, ph, l, l == top ? 1 : 0, args[l]));
  EXF_TRY(s->asm_args.ensure(nl * sizeof(AsmArgs<DIM>)));
  EXF_CUDA(cudaMemcpyAsync(s->asm_args.p, args.data(), nl * sizeof(AsmArgs<DIM>), cudaMemcpyHostToDevice, s->stream));
  constexpr int NT = DIM == 2 ? 128 : 256;
  const AsmArgs<DIM> *d_args = reinterpret_cast<const AsmArgs<DIM> *>(s->asm_args.p);
  const int2 *d_work = reinterpret_cast<const int2 *>(s->asm_work.p);
  for (int c = 0; c + 1 < (int)s->asm_work_off.size(); c++) {
    const int n = s->asm_work_off[c + 1] - s->asm_work_off[c];
    if (n == 0) continue;
    k_assemble_levels<DIM, NT><<<n, NT, 0, s->stream>>>(d_args, d_work + s->asm_work_off[c]);
    EXF_LAUNCH_CHECK();
    EXF_COUNT(1);
  }
  // `args` is pageable host memory: the asynchronous copy has staged it by the time the
  // call returned, so it may go out of scope while the launches read the device copy
  return EXF_OK;
}

int assemble_all_levels(exf_sys *s, const exf_phys *ph) {
  if (s->mesh->dim == 2) return assemble_all_dim<2>(s, ph);
  return assemble_all_dim<3>(s, ph);
}

int assemble_level(exf_sys *s, const exf_phys *ph, int lev, int mode) {
  if (s->mesh->dim == 2) return assemble_dim<2>(s, ph, lev, mode);
  return assemble_dim<3>(s, ph, lev, mode);
}

// ---------------------------------------------------------------- kappa-omega
// One variable (var 0 kappa, 1 omega) of MGSolTBK::GenMatRhs, the turbulence template's
// coupled kappa-omega system (template_appl/turb-ckw/SRC/MGSolverTBKW.C:83-454; its
// matrix has no kappa-omega blocks, so each variable is its own scalar system), with the
// template's model (MGSolTBK::f_mu, :484-587, WILCOX and LOWRE, constants of
// template_appl/turb-ckw/DATA/MGSclass_conf.h:296-356).  Per Gauss point, with the
// Navier-Stokes velocity v and the kappa, omega fields interpolated from the nodes:
//   tau = min(1/omega, MAX_TAU), Re_t = clamp(kappa tau / IRe, MU_LOW, MU_TOP),
//   alpha* = (0.024 + Re_t/6) / (1 + Re_t/6), mu_t = alpha* Re_t,
//   S = 1e-20 + sum_ij (dv_i/dx_j + dv_j/dx_i)^2, nut2 = kappa / (7 sqrt(alpha* S / 2 / beta*) / 8),
//   sources and dissipations of the 2006 model with the low-Re factors gamma*, beta*,
//   cross = max(grad kappa . grad omega, 0) tau / 8, IRe_eff = IRe (1 + sigma alpha* mu_t),
// then the reference's volume terms (time, advection, upwinded diffusion, dissipation;
// rhs: x_old / dt, source, cross for omega), its Dirichlet sides (penalty det / dt, the
// omega wall value 6 nu / (beta* y^2) where the flags ask for it) and its Neumann sides
// (2 IRe_eff / y with the last Gauss point's IRe_eff, as the reference leaves it).
constexpr double kKwSigmaK = 0.6, kKwSigmaW = 0.5, kKwBetaStar = 0.09, kKwMaxTau = 100., kKwMuLow = 1.e-6,
                 kKwMuTop = 1.e+6, kKwUpwind = 1.;

template <int DIM>
struct KwArgs {
  const FETab<DIM> *tab;
  const int *conn, *neigh, *elist;
  const double *xyz;
  int ntop, Ntop;
  const int *bc0, *bc1;
  const double *kold, *wold, *vel, *dist;
  const int *qq_ptr;
  const uint8_t *pos_qq;
  double *vv, *rhs;
  double ire, idt, nu_wall;
  int var;
  int sides[FE<DIM>::NSIDE][FE<DIM>::NSN];
};

template <int DIM, int NT>
__global__ void __launch_bounds__(NT) k_assemble_kw(KwArgs<DIM> A, int mode) {
  using F = FE<DIM>;
  constexpr int NEN = F::NEN, NQ = F::NQ;
  const int tid = threadIdx.x, e = A.elist[blockIdx.x];
  __shared__ int s_conn[NEN], s_bcv[NEN], s_bcb[NEN];
  __shared__ double s_xx[DIM][NEN];
  __shared__ double s_v[DIM][NEN], s_k[NEN], s_w[NEN];
  __shared__ double s_dphi[NQ][NEN][DIM];
  __shared__ double s_cM[NQ], s_cA[NQ][DIM], s_cL[NQ][DIM], s_cR[NQ];
  __shared__ double s_h[DIM], s_ire_last;
  const FETab<DIM> *t = A.tab;
  for (int k = tid; k < NEN; k += NT) {
    const int nd = A.conn[(long)e * NEN + k];
    s_conn[k] = nd;
    for (int d = 0; d < DIM; d++) {
      s_xx[d][k] = A.xyz[nd + (long)d * A.ntop];
      s_v[d][k] = A.vel ? A.vel[nd + (long)d * A.Ntop] : 0.;
    }
    s_bcv[k] = A.bc0[nd];
    s_bcb[k] = A.bc1[nd];
    s_k[k] = A.kold[nd];
    s_w[k] = A.wold[nd];
  }
  __syncthreads();
  if (tid < DIM) {
    const int v2 = DIM == 2 ? 2 : 6, v3 = DIM == 2 ? 3 : 7;
    const double h = fabs(s_xx[tid][v2] - s_xx[tid][0]), h1 = fabs(s_xx[tid][v3] - s_xx[tid][1]);
    s_h[tid] = h < h1 ? h1 : h;
  }
  __syncthreads();
  const int var = A.var;
  const double IRe = A.ire, idt = A.idt;
  for (int q = tid; q < NQ; q += NT) {  // one thread per Gauss point
    double J[DIM][DIM];
    for (int a = 0; a < DIM; a++)
      for (int b = 0; b < DIM; b++) {
        double sum = 0.;
        for (int k = 0; k < NEN; k++) sum += s_xx[a][k] * t->dphi[q][k][b];
        J[a][b] = sum;
      }
    double det, inv[DIM][DIM];  // inv[b][a] = dxi_b / dx_a
    if constexpr (DIM == 2) {
      det = J[0][0] * J[1][1] - J[1][0] * J[0][1];
      const double id = 1. / det;
      inv[0][0] = J[1][1] * id;
      inv[0][1] = -J[0][1] * id;
      inv[1][0] = -J[1][0] * id;
      inv[1][1] = J[0][0] * id;
    } else {
      const int o = DIM - 1;
      det = J[0][0] * (J[1][1] * J[o][o] - J[1][o] * J[o][1]) - J[0][1] * (J[1][0] * J[o][o] - J[1][o] * J[o][0]) +
            J[0][o] * (J[1][0] * J[o][1] - J[1][1] * J[o][0]);
      const double id = 1. / det;
      inv[0][0] = (J[1][1] * J[o][o] - J[1][o] * J[o][1]) * id;
      inv[0][1] = (J[0][o] * J[o][1] - J[0][1] * J[o][o]) * id;
      inv[0][o] = (J[0][1] * J[1][o] - J[0][o] * J[1][1]) * id;
      inv[1][0] = (J[1][o] * J[o][0] - J[1][0] * J[o][o]) * id;
      inv[1][1] = (J[0][0] * J[o][o] - J[0][o] * J[o][0]) * id;
      inv[1][o] = (J[0][o] * J[1][0] - J[0][0] * J[1][o]) * id;
      inv[o][0] = (J[1][0] * J[o][1] - J[1][1] * J[o][0]) * id;
      inv[o][1] = (J[0][1] * J[o][0] - J[0][0] * J[o][1]) * id;
      inv[o][o] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
    }
    const double JxW = det * t->w[q];
    double vg[DIM], g[DIM][DIM], gk[DIM], gw[DIM], kg = 0., wg = 0.;
    for (int d = 0; d < DIM; d++) {
      vg[d] = gk[d] = gw[d] = 0.;
      for (int a = 0; a < DIM; a++) g[a][d] = 0.;
    }
    for (int k = 0; k < NEN; k++) {
      const double ph = t->phi[q][k];
      kg += ph * s_k[k];
      wg += ph * s_w[k];
      for (int d = 0; d < DIM; d++) {
        double dp = 0.;
        for (int b = 0; b < DIM; b++) dp += inv[b][d] * t->dphi[q][k][b];
        s_dphi[q][k][d] = dp;
        vg[d] += ph * s_v[d][k];
        gk[d] += s_k[k] * dp;
        gw[d] += s_w[k] * dp;
        for (int a = 0; a < DIM; a++) g[a][d] += s_v[a][k] * dp;
      }
    }
    double mod = 1e-20, sP = 1.e-20, chi = 0.;
    for (int d = 0; d < DIM; d++) mod += vg[d] * vg[d];
    mod = sqrt(mod);
    for (int a = 0; a < DIM; a++)
      for (int b = 0; b < DIM; b++) {
        const double sss = g[a][b] + g[b][a];
        sP += sss * sss;
      }
    for (int d = 0; d < DIM; d++) chi += gk[d] * gw[d];
    // f_mu (WILCOX, LOWRE)
    if (kg < 1.e-20) kg = 1.e-20;
    double tau = 1. / wg;
    if (tau > kKwMaxTau) tau = kKwMaxTau;
    double Re_t = kg * tau / IRe;
    if (Re_t > kKwMuTop) Re_t = kKwMuTop;
    if (Re_t < kKwMuLow) Re_t = kKwMuLow;
    const double astar = (0.024 + 0.166666666667 * Re_t) / (1. + 0.166666666667 * Re_t);
    const double mu_t = Re_t * astar;
    const double nut2 = kg / (7. * sqrt(astar * 0.5 * sP / kKwBetaStar) / 8.);
    double src0, src1;
    if (mu_t * IRe < nut2) {
      src0 = 0.5 * mu_t * IRe * sP;
      src1 = 0.5 * 13. * sP / 25.;
    } else {
      src0 = 0.5 * nut2 * sP;
      src1 = 0.5 * 13. * nut2 * sP / (25. * mu_t * IRe);
    }
    const double gstar = (0.111111111111 + 0.338983050847 * Re_t) / (1. + 0.338983050847 * Re_t);
    const double r4 = Re_t * Re_t * Re_t * Re_t;
    const double bstar = (0.266666666667 + 0.000244140625 * r4) / (1. + 0.000244140625 * r4);
    const double diss = var == 0 ? kKwBetaStar / tau * bstar : 0.0708 / tau;
    const double src = var == 0 ? src0 : src1 * gstar;
    const double cross = chi > 0 ? chi * tau / 8. : 0.;
    const double ire = IRe * (1. + (var == 0 ? kKwSigmaK : kKwSigmaW) * astar * mu_t);
    s_cM[q] = JxW * (idt + diss);
    s_cR[q] = JxW * ((var == 0 ? kg : wg) * idt + src + cross * var);
    for (int d = 0; d < DIM; d++) {
      const double pe = 0.5 * mod * s_h[d] / IRe;
      const double fu = kKwUpwind * 0.5 * (1. / tanh(pe) - 1. / pe) * s_h[d] / mod;
      s_cA[q][d] = JxW * vg[d];
      s_cL[q][d] = JxW * (ire + fu * vg[d] * vg[d]);
    }
    if (q == NQ - 1) s_ire_last = ire;
  }
  __syncthreads();
  // volume integrals of the node pairs and the rhs
  for (int p = tid; p < NEN * NEN; p += NT) {
    const int i = p / NEN, j = p % NEN;
    const long blk = A.qq_ptr[s_conn[i]] + A.pos_qq[((long)e * NEN + i) * NEN + j];
    const double old = A.vv[blk];
    double K = 0.;
    for (int q = 0; q < NQ; q++) {
      const double pi = t->phi[q][i], pj = t->phi[q][j];
      double adv = 0., lap = 0.;
      for (int d = 0; d < DIM; d++) {
        adv += s_cA[q][d] * s_dphi[q][j][d];
        lap += s_cL[q][d] * s_dphi[q][j][d] * s_dphi[q][i][d];
      }
      K += pi * (s_cM[q] * pj + adv) + lap;
    }
    A.vv[blk] = old + s_bcv[i] * K;
  }
  if (mode == 1)
    for (int i = tid; i < NEN; i += NT) {
      double f = 0.;
      for (int q = 0; q < NQ; q++) f += s_cR[q] * t->phi[q][i];
      A.rhs[s_conn[i]] += s_bcv[i] * f;
    }
  __syncthreads();
  // boundary sides, one after the other (a node may lie on two of them)
  const double y = A.dist[e];
  for (int sd = 0; sd < F::NSIDE; sd++) {
    if (A.neigh[(long)e * F::NSIDE + sd] != -1) continue;
    const int *sur = A.sides[sd];
    const int last = sur[F::NSN - 1];
    for (int k = tid; k < F::NSN; k += NT) {
      const int lv = sur[k];
      const long dblk = A.qq_ptr[s_conn[lv]] + A.pos_qq[((long)e * NEN + lv) * NEN + lv];
      if (s_bcv[last] == 0) {
        const double ipen = jac_sur<DIM>(t, F::NSQ - 1, s_xx, sur) * idt;
        const int bs = s_bcb[lv], bc_rhs = (bs & 2) >> 1, bc_n = bs % 2;
        const double xo = var == 0 ? s_k[lv] : s_w[lv];
        const double kw = xo < 1.e-20 ? 1.e-20 : xo;
        const double wall = 6. * A.nu_wall / (kKwBetaStar * y * y);
        A.vv[dblk] += ipen;
        if (mode == 1) A.rhs[s_conn[lv]] += ipen * (bc_n * (1 - bc_rhs) * kw + (1 - bc_n) * bc_rhs * (var * wall));
      } else if (s_bcb[last] != 0) {
        const double fac = 2. * s_ire_last * (s_bcv[lv] == 0 ? 0. : 1.) * (s_bcb[lv] % 2) / y;
        for (int j = 0; j < F::NSN; j++) {
          double v = 0.;
          for (int q = 0; q < F::NSQ; q++) v += jac_sur<DIM>(t, q, s_xx, sur) * t->sw[q] * t->sphi[q][j] * t->sphi[q][k];
          const long bj = A.qq_ptr[s_conn[lv]] + A.pos_qq[((long)e * NEN + lv) * NEN + sur[j]];
          A.vv[bj] += fac * v;
        }
      }
    }
    __syncthreads();
  }
}

template <int DIM>
static int assemble_kw_dim(exf_sys *s, const exf_phys *ph, int lev, int mode) {
  const exf_mesh *m = s->mesh;
  const int top = s->nlev - 1;
  SysLevel &L = s->L[lev];
  const MeshLevel &ml = m->lev[lev];
  if (!s->turb || s->wall_off.empty() || !(ph->inv_dt > 0.)) {
    set_error("kappa-omega assembly needs the partner system (exf_sys_couple), the wall distances "
              "(exf_sys_set_wall) and a time step (phys.inv_dt > 0)");
    return EXF_ERR_STATE;
  }
  KwArgs<DIM> a;
  memset(&a, 0, sizeof(a));
  a.tab = reinterpret_cast<const FETab<DIM> *>(m->d_fetab.p);
  for (int sd = 0; sd < FE<DIM>::NSIDE; sd++)
    for (int k = 0; k < FE<DIM>::NSN; k++) a.sides[sd][k] = DIM == 2 ? Q9_SIDE[sd][k] : H27_FACE[sd][k];
  a.conn = ml.d_conn.p;
  a.neigh = ml.d_neigh.p;
  a.xyz = m->d_xyz.p;
  a.ntop = m->ntop;
  a.Ntop = s->L[top].N;
  a.bc0 = s->d_bc0.p;
  a.bc1 = s->d_bc1.p;
  const exf_sys *kk = s->kind == EXF_KIND_K ? s : s->turb, *ww = s->kind == EXF_KIND_W ? s : s->turb;
  a.kold = kk->xold.p;
  a.wold = ww->xold.p;
  a.vel = (s->other && s->other->kind == EXF_KIND_NS) ? s->other->xold.p : nullptr;
  a.dist = s->wall_dist.p + s->wall_off[lev];
  a.qq_ptr = L.qq_ptr.p;
  a.pos_qq = L.pos_qq.p;
  a.vv = L.A.vv.p;
  a.rhs = mode == 1 ? L.b.p : nullptr;
  a.ire = ph->inv_re;
  a.idt = ph->inv_dt;
  a.nu_wall = s->nu_wall;
  a.var = s->kind == EXF_KIND_K ? 0 : 1;
  EXF_TRY(L.A.vv.zero(s->stream));
  if (mode == 1) EXF_TRY(L.b.zero(s->stream));
  constexpr int NT = DIM == 2 ? 64 : 128;
  for (int c = 0; c + 1 < (int)ml.ecol_off.size(); c++) {
    const int n = ml.ecol_off[c + 1] - ml.ecol_off[c];
    if (n == 0) continue;
    a.elist = ml.d_elist.p + ml.ecol_off[c];
    k_assemble_kw<DIM, NT><<<n, NT, 0, s->stream>>>(a, mode);
    EXF_LAUNCH_CHECK();
    EXF_COUNT(1);
  }
  return EXF_OK;
}

int assemble_kw_level(exf_sys *s, const exf_phys *ph, int lev, int mode) {
  if (s->mesh->dim == 2) return assemble_kw_dim<2>(s, ph, lev, mode);
  return assemble_kw_dim<3>(s, ph, lev, mode);
}

// ---- the fluid-structure template's mesh displacement, one direction ------------------
// MGSolDS::GenMatRhs (template_appl/fsi/SRC/MGSolverDS.C:321-700, ALE_MOVING): phase from
// the element centre's bc0 (< 2 fluid); fluid rows K_ij = sum_q JxW (bc0_i % 2) fl_i dt
// (100 grad phi_j . grad phi_i), fl_i = 0 on interface nodes (bc0 > 3), rhs 0; boundary
// sides whose last node has an even bc0: K_ii += fl_i det_side(last Gauss point) / dt,
// rhs fl_i (bc1_last % 2) det/dt (u_fsi_x dt + d_old_x); solid rows K_ii = 1, rhs
// u_fsi_dir dt + d_old_dir.  One CTA per element, the elements of one colour per launch.
template <int DIM>
struct DsArgs {
  const FETab<DIM> *tab;
  const int *conn, *neigh, *elist;
  const double *xyz;
  int ntop, Ntop;
  const int *bc0, *bc1;
  const double *ux, *ud, *dx, *dd;  // [Ntop]: u_fsi and d_old, direction 0 and direction dir
  const int *qq_ptr;
  const uint8_t *pos_qq;
  double *vv, *rhs;
  double dt;
  int sides[FE<DIM>::NSIDE][FE<DIM>::NSN];
};

template <int DIM, int NT>
__global__ void __launch_bounds__(NT) k_assemble_ds(DsArgs<DIM> A, int mode) {
  using F = FE<DIM>;
  constexpr int NEN = F::NEN, NQ = F::NQ;
  const int tid = threadIdx.x, e = A.elist[blockIdx.x];
  __shared__ int s_conn[NEN], s_bcv[NEN];
  __shared__ double s_xx[DIM][NEN];
  __shared__ double s_dphi[NQ][NEN][DIM];
  __shared__ double s_jxw[NQ];
  const FETab<DIM> *t = A.tab;
  for (int k = tid; k < NEN; k += NT) {
    const int nd = A.conn[(long)e * NEN + k];
    s_conn[k] = nd;
    for (int d = 0; d < DIM; d++) s_xx[d][k] = A.xyz[nd + (long)d * A.ntop];
    s_bcv[k] = A.bc0[nd];
  }
  __syncthreads();
  const double dt = A.dt;
  if (s_bcv[NEN - 1] >= 2) {  // solid: the displacement follows the FSI velocity
    for (int i = tid; i < NEN; i += NT) {
      const int nd = s_conn[i];
      A.vv[A.qq_ptr[nd] + A.pos_qq[((long)e * NEN + i) * NEN + i]] += 1.;
      if (mode == 1) A.rhs[nd] += A.ud[nd] * dt + A.dd[nd];
    }
    return;
  }
  for (int q = tid; q < NQ; q += NT) {  // one thread per Gauss point
    double J[DIM][DIM];
    for (int a = 0; a < DIM; a++)
      for (int b = 0; b < DIM; b++) {
        double sum = 0.;
        for (int k = 0; k < NEN; k++) sum += s_xx[a][k] * t->dphi[q][k][b];
        J[a][b] = sum;
      }
    double det, inv[DIM][DIM];  // inv[b][a] = dxi_b / dx_a
    if constexpr (DIM == 2) {
      det = J[0][0] * J[1][1] - J[1][0] * J[0][1];
      const double id = 1. / det;
      inv[0][0] = J[1][1] * id;
      inv[0][1] = -J[0][1] * id;
      inv[1][0] = -J[1][0] * id;
      inv[1][1] = J[0][0] * id;
    } else {
      const int o = DIM - 1;
      det = J[0][0] * (J[1][1] * J[o][o] - J[1][o] * J[o][1]) - J[0][1] * (J[1][0] * J[o][o] - J[1][o] * J[o][0]) +
            J[0][o] * (J[1][0] * J[o][1] - J[1][1] * J[o][0]);
      const double id = 1. / det;
      inv[0][0] = (J[1][1] * J[o][o] - J[1][o] * J[o][1]) * id;
      inv[0][1] = (J[0][o] * J[o][1] - J[0][1] * J[o][o]) * id;
      inv[0][o] = (J[0][1] * J[1][o] - J[0][o] * J[1][1]) * id;
      inv[1][0] = (J[1][o] * J[o][0] - J[1][0] * J[o][o]) * id;
      inv[1][1] = (J[0][0] * J[o][o] - J[0][o] * J[o][0]) * id;
      inv[1][o] = (J[0][o] * J[1][0] - J[0][0] * J[1][o]) * id;
      inv[o][0] = (J[1][0] * J[o][1] - J[1][1] * J[o][0]) * id;
      inv[o][1] = (J[0][1] * J[o][0] - J[0][0] * J[o][1]) * id;
      inv[o][o] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
    }
    s_jxw[q] = det * t->w[q];
    for (int k = 0; k < NEN; k++)
      for (int d = 0; d < DIM; d++) {
        double dp = 0.;
        for (int b = 0; b < DIM; b++) dp += inv[b][d] * t->dphi[q][k][b];
        s_dphi[q][k][d] = dp;
      }
  }
  __syncthreads();
  for (int p = tid; p < NEN * NEN; p += NT) {
    const int i = p / NEN, j = p % NEN;
    const int bv = s_bcv[i];
    if (bv % 2 == 0 || bv > 3) continue;  // a zero row factor
    double K = 0.;
    for (int q = 0; q < NQ; q++) {
      double lap = 0.;
      for (int d = 0; d < DIM; d++) lap += s_dphi[q][j][d] * s_dphi[q][i][d];
      K += s_jxw[q] * dt * (100. * lap);
    }
    A.vv[A.qq_ptr[s_conn[i]] + A.pos_qq[((long)e * NEN + i) * NEN + j]] += K;
  }
  __syncthreads();
  // boundary sides, one after the other (a node may lie on two of them)
  for (int sd = 0; sd < F::NSIDE; sd++) {
    if (A.neigh[(long)e * F::NSIDE + sd] != -1) continue;
    const int *sur = A.sides[sd];
    const int last = sur[F::NSN - 1];
    if (s_bcv[last] % 2 != 0) continue;
    const int bc_var = A.bc1[s_conn[last]] % 2;
    for (int k = tid; k < F::NSN; k += NT) {
      const int lv = sur[k], nd = s_conn[lv];
      if (s_bcv[lv] > 3) continue;  // interface node
      const double ipen = jac_sur<DIM>(t, F::NSQ - 1, s_xx, sur) / dt;
      A.vv[A.qq_ptr[nd] + A.pos_qq[((long)e * NEN + lv) * NEN + lv]] += ipen;
      if (mode == 1 && bc_var) A.rhs[nd] += ipen * (A.ux[nd] * dt + A.dx[nd]);
    }
    __syncthreads();
  }
}

template <int DIM>
static int assemble_ds_dim(exf_sys *s, int lev, int mode) {
  const exf_mesh *m = s->mesh;
  SysLevel &L = s->L[lev];
  const MeshLevel &ml = m->lev[lev];
  if (s->ds_dir < 0) {
    set_error("displacement assembly needs its direction, dt and fields (exf_sys_set_ds)");
    return EXF_ERR_STATE;
  }
  DsArgs<DIM> a;
  memset(&a, 0, sizeof(a));
  a.tab = reinterpret_cast<const FETab<DIM> *>(m->d_fetab.p);
  for (int sd = 0; sd < FE<DIM>::NSIDE; sd++)
    for (int k = 0; k < FE<DIM>::NSN; k++) a.sides[sd][k] = DIM == 2 ? Q9_SIDE[sd][k] : H27_FACE[sd][k];
  a.conn = ml.d_conn.p;
  a.neigh = ml.d_neigh.p;
  a.xyz = m->d_xyz.p;
  a.ntop = m->ntop;
  a.Ntop = m->ntop;
  a.bc0 = s->d_bc0.p;
  a.bc1 = s->d_bc1.p;
  const long off = (long)s->ds_dir * m->ntop;
  if (s->ds_host) {  // the [dim][ntop] fields of exf_sys_set_ds
    a.ux = s->ds_u.p;
    a.ud = s->ds_u.p + off;
    a.dx = s->ds_d.p;
    a.dd = s->ds_d.p + off;
  } else {  // coupled: the velocity system's x_old ([dim][ntop] first), the DS systems' x_old
    const exf_sys *v = s->other, *x0 = s->ds_dir == 0 ? s : s->ds_x;
    if (!v || v->kind != EXF_KIND_NS || !x0 || x0->kind != EXF_KIND_DS || x0->ds_dir != 0) {
      set_error("a coupled displacement system needs the velocity system and the dx system (exf_sys_couple)");
      return EXF_ERR_STATE;
    }
    a.ux = v->xold.p;
    a.ud = v->xold.p + off;
    a.dx = x0->xold.p;
    a.dd = s->xold.p;
  }
  a.qq_ptr = L.qq_ptr.p;
  a.pos_qq = L.pos_qq.p;
  a.vv = L.A.vv.p;
  a.rhs = mode == 1 ? L.b.p : nullptr;
  a.dt = s->ds_dt;
  EXF_TRY(L.A.vv.zero(s->stream));
  if (mode == 1) EXF_TRY(L.b.zero(s->stream));
  constexpr int NT = DIM == 2 ? 64 : 128;
  for (int c = 0; c + 1 < (int)ml.ecol_off.size(); c++) {
    const int n = ml.ecol_off[c + 1] - ml.ecol_off[c];
    if (n == 0) continue;
    a.elist = ml.d_elist.p + ml.ecol_off[c];
    k_assemble_ds<DIM, NT><<<n, NT, 0, s->stream>>>(a, mode);
    EXF_LAUNCH_CHECK();
    EXF_COUNT(1);
  }
  return EXF_OK;
}

int assemble_ds_level(exf_sys *s, int lev, int mode) {
  if (s->mesh->dim == 2) return assemble_ds_dim<2>(s, lev, mode);
  return assemble_ds_dim<3>(s, lev, mode);
}

// MGSolDS::MGTimeStep with moving_mesh and FINE_MOVEMENT (MGSolverDS.C:724-744): the node
// coordinates of the direction move by the step's displacement increment
__global__ void k_ds_move(double *xyz, const double *x, const double *xold, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) xyz[i] += x[i] - xold[i];
}

int ds_move_mesh(exf_sys *s) {
  exf_mesh *m = s->mesh;
  const int n = m->ntop;
  if (s->ds_dir < 0 || s->L[s->nlev - 1].ndof != n) {
    set_error("mesh motion needs the displacement system's direction (exf_sys_set_ds)");
    return EXF_ERR_STATE;
  }
  const int nb = (n + 255) / 256 < 148 * 8 ? (n + 255) / 256 : 148 * 8;
  k_ds_move<<<nb, 256, 0, s->stream>>>(m->d_xyz.p + (long)s->ds_dir * n, s->L[s->nlev - 1].x.p, s->xold.p, n);
  EXF_LAUNCH_CHECK();
  EXF_COUNT(1);
  m->xyz_moved = true;
  return EXF_OK;
}

int mesh_pull_xyz(exf_mesh *m) {
  if (!m->xyz_moved) return EXF_OK;
  EXF_CUDA(cudaSetDevice(m->device));
  EXF_CUDA(cudaDeviceSynchronize());
  EXF_CUDA(cudaMemcpy(m->xyz.data(), m->d_xyz.p, m->xyz.size() * sizeof(double), cudaMemcpyDeviceToHost));
  m->xyz_moved = false;
  return EXF_OK;
}

}  // namespace exf
