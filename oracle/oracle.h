/*
 * oracle.h -- CPU restatement of exFEMuS's assembly + geometric-multigrid path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links or calls this
 * code; it is the checker used by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline leg of bench.py.  All arithmetic is FP64.  The reference's LASPACK path
 * is single-process (src/MGSolverBase.C:51-55); here the independent items of one colour
 * may run on several threads (or_set_threads) without changing any result.
 *
 * Parity anchors: the reference ships no golden vectors or asserting tests.  The
 * restatement is pinned (a) against the reference's own embedding tables and
 * surface topology (tests/golden fixtures generated from src/MGGeomEl.C), (b) by
 * the analytic known answers the reference's discretisation must satisfy, and (c)
 * by the vendored LASPACK C library compiled from the reference sources
 * (oracle/_ref), whose Mul_QV / GMRESIter / SORForwIter / Transp_Q are run on the
 * restated matrices.
 */
#ifndef EXF_ORACLE_H
#define EXF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Physics parameters (same meaning as the product's exf_phys). */
typedef struct {
  double inv_re;     /* _IRe: kinematic viscosity (nondimensional 1/Re)          */
  double inv_prdl;   /* _IPrdl: 1/Pr; heat diffusivity = inv_prdl*inv_re          */
  double rho;        /* density factor (1)                                        */
  double rhocp;      /* rho*cp (1)                                                */
  double inv_dt;     /* 1/dt of the mass (time) term; 0 = steady                  */
  double penalty;    /* Dirichlet penalty scale: Ipenalty = det_side*penalty      */
  double upwind_ns;  /* UP_WIND_NS (0.1)                                          */
  double upwind_t;   /* UP_WIND_T (1.0)                                           */
  double ifr;        /* _IFr gravity factor                                       */
  double dirg[3];    /* _dirg gravity direction                                   */
  double buoy;       /* Boussinesq source: f += buoy*T*dirg                       */
  double traction;   /* 1: natural NS sides with bc1 bit 2 get the pressure traction */
                     /* rhs -n_a p_old phi_i (the reference's MESHNUMBER == 1)      */
} or_phys;

typedef struct {
  double eps;        /* stop: ||b-Ax||/||b|| <= eps                               */
  int max_cycles;
  int gamma;         /* 1 = V-cycle                                               */
  int nu_pre, nu_post;
  int double_below_top; /* MGStep doubles the sweeps below the top (1 = as ref)   */
  int smoother;      /* 0 = multi-colour Gauss-Seidel, 1 = multi-colour Vanka     */
  double omega;      /* Vanka damping                                             */
  double corr_damp;  /* coarse-correction factor (0.95 in the reference)          */
  int cond_corr;     /* 1 = reference's conditional correction                    */
  int reverse_colours; /* 1 = sweep colours in reverse order (adjoint)            */
  int stop_test;     /* 0: ||b-Ax||/||b|| <= eps; 1: reference accuracy < eps(1+||b||) */
} or_mg_params;

typedef struct {
  int cycles;
  int converged;
  double rel_res;
  double bnorm;
  double hist[256];
  double last_acc;   /* top-level accuracy of the last cycle in the reference's sense */
} or_mg_stats;

/* ------------------------------------------------------------------ mesh */
typedef struct or_mesh or_mesh;
or_mesh *or_mesh_new(int dim, int nlev, const int n0[3], const double box[6]);
void or_mesh_free(or_mesh *m);
int or_mesh_nnodes(const or_mesh *m, int lev);   /* Q2 nodes of level lev      */
int or_mesh_nvert0(const or_mesh *m);            /* Q1 nodes of level 0        */
int or_mesh_nel(const or_mesh *m, int lev);
int or_mesh_nen(const or_mesh *m);
void or_mesh_get_xyz(const or_mesh *m, double *xyz);       /* [dim][ntop]      */
void or_mesh_get_lattice(const or_mesh *m, int *lat);      /* [ntop][3]        */
void or_mesh_get_conn(const or_mesh *m, int lev, int *conn, int *neigh, int *colour);

/* ---------------------------------------------------------------- system */
typedef struct or_sys or_sys;
/* kind: 0 = temperature (1 quadratic var), 1 = coupled Navier-Stokes (dim quadratic + 1 linear) */
or_sys *or_sys_new(const or_mesh *m, int kind);
void or_sys_free(or_sys *s);
int or_sys_ndof(const or_sys *s, int lev);
void or_sys_node_dof(const or_sys *s, int lev, int *out);  /* [nvars*ntop]      */
/* bc preset ids: 1 heat all-Dirichlet, 2 cavity, 3 channel, 4 Boussinesq NS, 5 Boussinesq T */
void or_sys_bc_preset(or_sys *s, int preset);
void or_sys_set_bc(or_sys *s, const int *bc0, const int *bc1);
void or_sys_get_bc(const or_sys *s, int *bc0, int *bc1);
long or_sys_nnz(const or_sys *s, int lev);
void or_sys_pattern(const or_sys *s, int lev, int *rowptr, int *col);
long or_sys_prol_nnz(const or_sys *s, int lev);
void or_sys_prol(const or_sys *s, int lev, int *rowptr, int *col, double *val);
long or_sys_rest_nnz(const or_sys *s, int lev);
void or_sys_rest(const or_sys *s, int lev, int *rowptr, int *col, double *val);
void or_sys_colours(const or_sys *s, int lev, int *ncol, int *colour_of_item);

/* ------------------------------------------------------------- assembly */
/* xold: top-level solution of this system; vel: top-level NS solution (T only,
 * may be NULL); temp: top-level T solution (NS buoyancy, may be NULL); qe: per
 * top-level element source (T only, may be NULL).  mode 1 = matrix+rhs, 0 = matrix. */
void or_sys_assemble(or_sys *s, int lev, int mode, const or_phys *ph,
                     const double *xold, const double *vel, const double *temp,
                     const double *qe);
/* Navier-Stokes systems: kappa and omega x_old [Ntop] of the turbulence model, whose eddy
 * viscosity then enters the momentum equation (NULL: laminar) */
void or_sys_set_turb(or_sys *s, const double *kold, const double *wold);
/* one level of variable var (0 kappa, 1 omega) of the coupled kappa-omega system of the
 * turbulence template on a scalar system (MGSolTBK::GenMatRhs) */
void or_kw_assemble(or_sys *s, int lev, int mode, int var, const or_phys *ph, const double *vel,
                    const double *kold, const double *wold, const double *dist, double nu_wall);
void or_ds_assemble(or_sys *s, int lev, int mode, int dir, double dt, const double *u, const double *d);
void or_sys_get_matrix(const or_sys *s, int lev, double *val);
void or_sys_set_matrix(or_sys *s, int lev, const double *val);
void or_sys_get_rhs(const or_sys *s, double *rhs);
void or_sys_set_rhs(or_sys *s, const double *rhs);
void or_sys_transpose_all(or_sys *s);

/* -------------------------------------------------------------- threads */
/* Loops over independent items of one colour (Vanka patches, Gauss-Seidel rows, assembly
 * elements) and over matrix rows run on this many threads (OpenMP builds; 1 otherwise).
 * Every item is computed by one thread in a fixed order and every reduction runs in row
 * order, so results do not depend on the thread count. */
void or_set_threads(int n);
int or_get_threads(void);

/* -------------------------------------------------------------- solvers */
void or_spmv(const or_sys *s, int lev, const double *x, double *y);
int or_mg_solve(or_sys *s, const or_mg_params *p, double *x, or_mg_stats *st);
int or_coarse_solve(or_sys *s, const double *b, double *x);
/* one smoothing call on level lev (for per-iterate parity tests) */
void or_smooth(or_sys *s, int lev, const or_mg_params *p, int nsweeps, double *x, const double *b);

/* FE tables (for golden checks): Q2/Q1 shape values at the Gauss points. */
void or_fe_tables(int dim, double *phi_q, double *dphi_q, double *phi_l, double *w);
/* side -> local node table (the restated _surf_top) */
void or_side_table(int dim, int *out);

#ifdef __cplusplus
}
#endif
#endif
