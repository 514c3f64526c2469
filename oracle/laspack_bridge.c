/*
 * laspack_bridge.c -- CSR entry points into the vendored LASPACK C library, compiled
 * from the reference sources (contrib/laspack/*.c) by oracle/Makefile into
 * oracle/_ref/liblaspack_ref.so.
 *
 * TEST INFRASTRUCTURE ONLY (the reference's own CPU solver kernels, used as an
 * independent check of the restated oracle and as the CPU baseline).  The QMatrix is
 * filled row by row with 1-based positions as LaspackMatrixM does
 * (contrib/matrix/laspack_matrixM.C:43-56); solvers are called as
 * LaspackLinearSolverM::solve does (contrib/matrix/laspack_linear_solverM.C:38-126).
 */
#include <stdlib.h>

#include "errhandl.h"
#include "itersolv.h"
#include "operats.h"
#include "precond.h"
#include "qmatrix.h"
#include "qvector.h"
#include "rtc.h"

static void fill_q(QMatrix *Q, int n, const int *ptr, const int *col, const double *val) {
  Q_Constr(Q, "A", (size_t)n, _LPFalse, Rowws, Normal, _LPTrue);
  for (int i = 0; i < n; i++) {
    int len = ptr[i + 1] - ptr[i];
    Q_SetLen(Q, (size_t)(i + 1), (size_t)len);
    for (int k = 0; k < len; k++)
      Q_SetEntry(Q, (size_t)(i + 1), (size_t)k, (size_t)(col[ptr[i] + k] + 1), val[ptr[i] + k]);
  }
}
static void fill_v(QVector *V, const char *name, int n, const double *x) {
  V_Constr(V, (char *)name, (size_t)n, Normal, _LPTrue);
  for (int i = 0; i < n; i++) V_SetCmp(V, (size_t)(i + 1), x ? x[i] : 0.);
}
static void get_v(QVector *V, int n, double *x) {
  for (int i = 0; i < n; i++) x[i] = V_GetCmp(V, (size_t)(i + 1));
}

/* y = A x through Mul_QV (contrib/laspack/operats.c:782) */
int lpb_spmv(int n, const int *ptr, const int *col, const double *val, const double *x, double *y) {
  QMatrix A;
  QVector X, Y;
  fill_q(&A, n, ptr, col, val);
  fill_v(&X, "x", n, x);
  fill_v(&Y, "y", n, NULL);
  Asgn_VV(&Y, Mul_QV(&A, &X));
  get_v(&Y, n, y);
  int rc = LASResult() == LASOK ? 0 : 1;
  V_Destr(&X);
  V_Destr(&Y);
  Q_Destr(&A);
  return rc;
}

/* y = A^T x through Transp_Q (operats.c:1325) and Mul_QV */
int lpb_spmv_t(int n, const int *ptr, const int *col, const double *val, const double *x, double *y) {
  QMatrix A;
  QVector X, Y;
  fill_q(&A, n, ptr, col, val);
  fill_v(&X, "x", n, x);
  fill_v(&Y, "y", n, NULL);
  Asgn_VV(&Y, Mul_QV(Transp_Q(&A), &X));
  get_v(&Y, n, y);
  int rc = LASResult() == LASOK ? 0 : 1;
  V_Destr(&X);
  V_Destr(&Y);
  Q_Destr(&A);
  return rc;
}

/* GMRES(restart) to relative accuracy tol (itersolv.c:1341), unpreconditioned
 * (precond 0) or with LASPACK's ILU(0) (precond 1, ILUPrecond, precond.c; the default
 * level solver of the reference's LASPACK backend is GMRES + ILU,
 * contrib/matrix/linear_solverM.h:200-205); transpose != 0 solves A^T x = b through
 * Transp_Q (operats.c:1325). */
int lpb_gmres_pc(int n, const int *ptr, const int *col, const double *val, const double *b, double *x, double tol,
                 int maxit, int restart, int transpose, int precond, int *iters, double *acc) {
  QMatrix A;
  QVector X, B;
  fill_q(&A, n, ptr, col, val);
  fill_v(&X, "x", n, x);
  fill_v(&B, "b", n, b);
  SetRTCAccuracy(tol);
  SetGMRESRestart(restart);
  PrecondProcType pc = precond == 1 ? ILUPrecond : NULL;
  if (transpose) {
    QMatrix *At = Transp_Q(&A);
    GMRESIter(At, &X, &B, maxit, pc, 1.);
  } else {
    GMRESIter(&A, &X, &B, maxit, pc, 1.);
  }
  get_v(&X, n, x);
  *iters = GetLastNoIter();
  *acc = GetLastAccuracy();
  int rc = LASResult() == LASOK ? 0 : 1;
  V_Destr(&X);
  V_Destr(&B);
  Q_Destr(&A);
  return rc;
}

int lpb_gmres(int n, const int *ptr, const int *col, const double *val, const double *b, double *x, double tol,
              int maxit, int restart, int transpose, int *iters, double *acc) {
  return lpb_gmres_pc(n, ptr, col, val, b, x, tol, maxit, restart, transpose, 0, iters, acc);
}

/* forward SOR sweeps (itersolv.c:850-894), omega = 1 is lexicographic Gauss-Seidel */
int lpb_sorforw(int n, const int *ptr, const int *col, const double *val, const double *b, double *x, int nsweeps,
                double omega, double *acc) {
  QMatrix A;
  QVector X, B;
  fill_q(&A, n, ptr, col, val);
  fill_v(&X, "x", n, x);
  fill_v(&B, "b", n, b);
  SetRTCAccuracy(1e-30);
  SORForwIter(&A, &X, &B, nsweeps, NULL, omega);
  get_v(&X, n, x);
  *acc = GetLastAccuracy();
  int rc = LASResult() == LASOK ? 0 : 1;
  V_Destr(&X);
  V_Destr(&B);
  Q_Destr(&A);
  return rc;
}

/* y = ILUPrecond(c) (precond.c:75-110) with the ILU(0) factor of A (factor.c:25-320) */
int lpb_ilu_apply(int n, const int *ptr, const int *col, const double *val, const double *c, double *y) {
  QMatrix A;
  QVector C, Y;
  fill_q(&A, n, ptr, col, val);
  fill_v(&C, "c", n, c);
  fill_v(&Y, "y", n, NULL);
  ILUPrecond(&A, &Y, &C, 1.);
  get_v(&Y, n, y);
  int rc = LASResult() == LASOK ? 0 : 1;
  V_Destr(&C);
  V_Destr(&Y);
  Q_Destr(&A);
  return rc;
}
