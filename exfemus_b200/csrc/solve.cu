// solve.cu -- multigrid building blocks on the node-block matrix:
//   residual / SpMV (LaspackVectorM::resid, contrib/matrix/laspack_vectorM.C:147-168),
//   restriction / prolongation (LaspackVectorM::matrix_mult, :170-189),
//   multi-colour Gauss-Seidel (SORForwIter at omega=1, contrib/laspack/itersolv.c:850-894),
//   multi-colour pressure-node Vanka (VankaNSIterD, itersolv.c:156-275, restated with the
//   pressure-row residual and damping), coarsest-level direct solve, vector helpers.
//
// All kernels are templated on the value type: FP64 for the plain path and the outer
// defect correction, FP32 (storage and accumulation) for the mixed-precision V-cycle.
// Reductions are two-stage with a fixed order, so every result is bitwise reproducible.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "exf_internal.h"

namespace exf {

static inline unsigned nblk(long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

template <class T>
struct VT;
template <>
struct VT<double> {
  static const double *vv(const SysLevel &L) { return L.A.vv.p; }
  static const double *vp(const SysLevel &L) { return L.A.vp.p; }
  static const double *pv(const SysLevel &L) { return L.A.pv.p; }
  static const double *pp(const SysLevel &L) { return L.A.pp.p; }
  static const double *pq(const Transfer &t) { return t.val.p; }
  static double *x(SysLevel &L) { return L.x.p; }
  static double *b(SysLevel &L) { return L.b.p; }
  static double *r(SysLevel &L) { return L.r.p; }
  static double *dx(SysLevel &L) { return L.dx.p; }
};
template <>
struct VT<float> {
  static const float *vv(const SysLevel &L) { return L.A32.vv.p; }
  static const float *vp(const SysLevel &L) { return L.A32.vp.p; }
  static const float *pv(const SysLevel &L) { return L.A32.pv.p; }
  static const float *pp(const SysLevel &L) { return L.A32.pp.p; }
  static const float *pq(const Transfer &t) { return t.val32.p; }
  static float *x(SysLevel &L) { return L.x32.p; }
  static float *b(SysLevel &L) { return L.b32.p; }
  static float *r(SysLevel &L) { return L.r32.p; }
  static float *dx(SysLevel &L) { return L.dx32.p; }
};

// ------------------------------------------------------------ reductions
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.;
  if (threadIdx.x == 0)
    for (int k = 0; k < NT / 32; k++) r += sh[k];
  __syncthreads();
  return r;
}
__global__ void k_reduce_partials(const double *part, int n, double *out) {
  EXF_PDL_WAIT();
  __shared__ double sh[32];
  double v = 0.;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += part[i];
  v = block_sum<1024>(v, sh);
  if (threadIdx.x == 0) *out = v;
}

static int ensure_partials(exf_sys *s, int nblk_needed) {
  if (s->red.nblk < nblk_needed) {
    EXF_TRY(s->red.part.alloc(nblk_needed));
    s->red.nblk = nblk_needed;
    s->buf_epoch++;
  }
  if (!s->red.out.p) EXF_TRY(s->red.out.alloc(16));
  return EXF_OK;
}

// acc[a] += sum over the node row n of the d x d blocks times x (and B^T times p);
// two blocks per lane in flight
template <class T, int D, int LPR, bool PRESSURE>
__device__ __forceinline__ void node_row_dot(int n, int lane, int N, const int *__restrict__ qq_ptr,
                                             const int *__restrict__ qq_col, const int *__restrict__ ql_ptr,
                                             const int *__restrict__ ql_col, long nqq, long nql,
                                             const T *__restrict__ vv, const T *__restrict__ vp,
                                             const T *__restrict__ x, T acc[D]) {
  const int k0 = qq_ptr[n], k1 = qq_ptr[n + 1];
  int k = k0 + lane;
  for (; k + LPR < k1; k += 2 * LPR) {
    const int c0 = qq_col[k], c1 = qq_col[k + LPR];
    T v0[D * D], v1[D * D], x0[D], x1[D];
#pragma unroll
    for (int q = 0; q < D * D; q++) {
      v0[q] = vv[(long)q * nqq + k];
      v1[q] = vv[(long)q * nqq + k + LPR];
    }
#pragma unroll
    for (int bb = 0; bb < D; bb++) {
      x0[bb] = x[(long)bb * N + c0];
      x1[bb] = x[(long)bb * N + c1];
    }
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int bb = 0; bb < D; bb++) acc[a] += v0[a * D + bb] * x0[bb] + v1[a * D + bb] * x1[bb];
  }
  if (k < k1) {
    const int c0 = qq_col[k];
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int bb = 0; bb < D; bb++) acc[a] += vv[(long)(a * D + bb) * nqq + k] * x[(long)bb * N + c0];
  }
  if (PRESSURE) {
    for (int kp = ql_ptr[n] + lane; kp < ql_ptr[n + 1]; kp += LPR) {
      const T p = x[(long)D * N + ql_col[kp]];
#pragma unroll
      for (int a = 0; a < D; a++) acc[a] += vp[(long)a * nql + kp] * p;
    }
  }
}

// ------------------------------------------------------------------ SpMV
// row groups: g < N -> Q2 node g (d outputs), g >= N -> Q1 node g-N (1 output).
// LPR lanes per row group; the node-block index k is shared by the d*d planes.
template <class T, int D, int LPR, bool NS, int NT>
__global__ void __launch_bounds__(NT)
    k_spmv_resid(int N, int NL, const int *__restrict__ qq_ptr, const int *__restrict__ qq_col,
                 const int *__restrict__ ql_ptr, const int *__restrict__ ql_col, long nqq, long nql, long nqqL,
                 const T *__restrict__ vv, const T *__restrict__ vp, const T *__restrict__ pv,
                 const T *__restrict__ pp, const T *__restrict__ x, const T *__restrict__ b, T *__restrict__ r,
                 double *__restrict__ part) {
  EXF_PDL_WAIT();
  __shared__ double sh[32];
  const int lane = threadIdx.x % LPR;
  const long g = ((long)blockIdx.x * NT + threadIdx.x) / LPR;
  const long ngroups = (long)N + (NS ? NL : 0);
  // every lane takes part in the shuffles below; only loads and stores are guarded
  const bool vel = g < N;
  const bool prs = NS && g >= N && g < ngroups;
  T acc[D];
#pragma unroll
  for (int a = 0; a < D; a++) acc[a] = T(0);
  if (vel) {
    node_row_dot<T, D, LPR, NS>((int)g, lane, N, qq_ptr, qq_col, ql_ptr, ql_col, nqq, nql, vv, vp, x, acc);
  } else if (prs) {
    const int m = (int)(g - N);
    const int k0 = qq_ptr[m], k1 = qq_ptr[m + 1];
    for (int k = k0 + lane; k < k1; k += LPR) {
      const int nn = qq_col[k];
#pragma unroll
      for (int bb = 0; bb < D; bb++) acc[0] += pv[(long)bb * nqqL + k] * x[(long)bb * N + nn];
    }
    const int l0 = ql_ptr[m], l1 = ql_ptr[m + 1];
    for (int k = l0 + lane; k < l1; k += LPR) acc[0] += pp[k] * x[(long)D * N + ql_col[k]];
  }
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) acc[a] += __shfl_down_sync(0xffffffffu, acc[a], o, LPR);
  double nrm = 0.;
  if (lane == 0) {
    if (vel) {
#pragma unroll
      for (int a = 0; a < D; a++) {
        const long row = (long)a * N + g;
        T rv = b ? b[row] - acc[a] : acc[a];
        r[row] = rv;
        nrm += (double)rv * (double)rv;
      }
    } else if (prs) {
      const long row = (long)D * N + (g - N);
      T rv = b ? b[row] - acc[0] : acc[0];
      r[row] = rv;
      nrm += (double)rv * (double)rv;
    }
  }
  if (part) {
    double tot = block_sum<NT>(nrm, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
  }
}

template <class T, int D, bool NS>
static int launch_spmv(exf_sys *s, int lev, const T *x, const T *b, T *r, double *d_norm2) {
  SysLevel &L = s->L[lev];
  constexpr int NT = 256;
  constexpr int LPR = D == 3 ? 32 : (NS ? 16 : 8);
  long ngroups = (long)L.N + (NS ? L.NL : 0);
  unsigned grid = nblk(ngroups * LPR, NT);
  if (d_norm2) EXF_TRY(ensure_partials(s, grid));
  EXF_CUDA(launch_pdl(k_spmv_resid<T, D, LPR, NS, NT>, dim3(grid), dim3(NT), 0, s->stream, L.N, L.NL, L.qq_ptr.p,
                      L.qq_col.p, L.ql_ptr.p, L.ql_col.p, L.nqq, L.nql, L.nqqL, VT<T>::vv(L), VT<T>::vp(L),
                      VT<T>::pv(L), VT<T>::pp(L), x, b, r, d_norm2 ? s->red.part.p : nullptr));
  EXF_COUNT(1);
  if (d_norm2) {
    EXF_CUDA(launch_pdl(k_reduce_partials, dim3(1), dim3(1024), 0, s->stream, s->red.part.p, (int)grid, d_norm2));
    EXF_COUNT(1);
  }
  return EXF_OK;
}

template <class T>
int spmv_resid(exf_sys *s, int lev, const T *x, const T *b, T *r, double *d_norm2) {
  const bool ns = s->kind == EXF_KIND_NS;
  if (s->dim == 2) return ns ? launch_spmv<T, 2, true>(s, lev, x, b, r, d_norm2)
                             : launch_spmv<T, 1, false>(s, lev, x, b, r, d_norm2);
  return ns ? launch_spmv<T, 3, true>(s, lev, x, b, r, d_norm2) : launch_spmv<T, 1, false>(s, lev, x, b, r, d_norm2);
}
template int spmv_resid<double>(exf_sys *, int, const double *, const double *, double *, double *);
template int spmv_resid<float>(exf_sys *, int, const float *, const float *, float *, double *);

// ------------------------------------------------------------ transfers
// b_c[(a,c)] = mask[(a,c)] * sum_f R[c,f] r_f[(a,f)]   (restriction, rows = coarse DOFs)
template <class T>
__global__ void k_restrict(int nv2, int nv1, int Nc, int NLc, int Nf, const int *__restrict__ rq_ptr,
                           const int *__restrict__ rq_col, const T *__restrict__ rq_val,
                           const int *__restrict__ rl_ptr, const int *__restrict__ rl_col,
                           const T *__restrict__ rl_val, const double *__restrict__ mask, const T *__restrict__ rf,
                           T *__restrict__ bc) {
  EXF_PDL_WAIT();
  long row = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long nq = (long)nv2 * Nc;
  if (row >= nq + (long)nv1 * NLc) return;
  T acc = T(0);
  if (row < nq) {
    int a = (int)(row / Nc), c = (int)(row % Nc);
    const T *src = rf + (long)a * Nf;
    for (int k = rq_ptr[c]; k < rq_ptr[c + 1]; k++) acc += rq_val[k] * src[rq_col[k]];
  } else {
    int c = (int)(row - nq);
    const T *src = rf + (long)nv2 * Nf;
    for (int k = rl_ptr[c]; k < rl_ptr[c + 1]; k++) acc += rl_val[k] * src[rl_col[k]];
  }
  bc[row] = (T)mask[row] * acc;
}

template <class T>
int restrict_op(exf_sys *s, int lev_c, const T *r_f, T *b_c) {
  SysLevel &C = s->L[lev_c];
  SysLevel &F = s->L[lev_c + 1];
  long nrow = C.ndof;
  EXF_CUDA(launch_pdl(k_restrict<T>, dim3(nblk(nrow, 256)), dim3(256), 0, s->stream, s->nv2, s->nv1, C.N, C.NL, F.N,
                      C.Rq.ptr.p, C.Rq.col.p, VT<T>::pq(C.Rq), s->nv1 ? C.Rl.ptr.p : nullptr,
                      s->nv1 ? C.Rl.col.p : nullptr, s->nv1 ? VT<T>::pq(C.Rl) : nullptr, C.rmask.p, r_f, b_c));
  EXF_COUNT(1);
  return EXF_OK;
}
template int restrict_op<double>(exf_sys *, int, const double *, double *);
template int restrict_op<float>(exf_sys *, int, const float *, float *);

// x_f[(a,f)] += damp * sum_c P[f,c] x_c[(a,c)]   (damp = 0 -> y = P x overwrite mode)
template <class T>
__global__ void k_prolong(int nv2, int nv1, int Nf, int NLf, int Nc, const int *__restrict__ pq_ptr,
                          const int *__restrict__ pq_col, const T *__restrict__ pq_val,
                          const int *__restrict__ pl_ptr, const int *__restrict__ pl_col,
                          const T *__restrict__ pl_val, const T *__restrict__ xc, T *__restrict__ xf, T damp,
                          int overwrite, const double *cond_rest) {
  EXF_PDL_WAIT();
  if (cond_rest && !(cond_rest[1] < cond_rest[0])) return;
  long row = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long nq = (long)nv2 * Nf;
  if (row >= nq + (long)nv1 * NLf) return;
  T acc = T(0);
  if (row < nq) {
    int a = (int)(row / Nf), f = (int)(row % Nf);
    const T *src = xc + (long)a * Nc;
    for (int k = pq_ptr[f]; k < pq_ptr[f + 1]; k++) acc += pq_val[k] * src[pq_col[k]];
  } else {
    int f = (int)(row - nq);
    const T *src = xc + (long)nv2 * Nc;
    for (int k = pl_ptr[f]; k < pl_ptr[f + 1]; k++) acc += pl_val[k] * src[pl_col[k]];
  }
  if (overwrite) xf[row] = acc;
  else xf[row] += damp * acc;
}

template <class T>
static int prolong_impl(exf_sys *s, int lev_f, const T *x_c, T *x_f, double damp, int overwrite,
                        const double *cond) {
  SysLevel &F = s->L[lev_f];
  SysLevel &C = s->L[lev_f - 1];
  long nrow = F.ndof;
  EXF_CUDA(launch_pdl(k_prolong<T>, dim3(nblk(nrow, 256)), dim3(256), 0, s->stream, s->nv2, s->nv1, F.N, F.NL, C.N,
                      F.Pq.ptr.p, F.Pq.col.p, VT<T>::pq(F.Pq), s->nv1 ? F.Pl.ptr.p : nullptr,
                      s->nv1 ? F.Pl.col.p : nullptr, s->nv1 ? VT<T>::pq(F.Pl) : nullptr, x_c, x_f, (T)damp, overwrite,
                      cond));
  EXF_COUNT(1);
  return EXF_OK;
}
template <class T>
int prolong_add(exf_sys *s, int lev_f, const T *x_c, T *x_f, double damp) {
  if (damp == 0.) return prolong_impl<T>(s, lev_f, x_c, x_f, 0., 1, nullptr);
  return prolong_impl<T>(s, lev_f, x_c, x_f, damp, 0, nullptr);
}
template int prolong_add<double>(exf_sys *, int, const double *, double *, double);
template int prolong_add<float>(exf_sys *, int, const float *, float *, double);
template <class T>
int prolong_cond(exf_sys *s, int lev_f, const T *x_c, T *x_f, double damp, const double *cond) {
  return prolong_impl<T>(s, lev_f, x_c, x_f, damp, 0, cond);
}
template int prolong_cond<double>(exf_sys *, int, const double *, double *, double, const double *);
template int prolong_cond<float>(exf_sys *, int, const float *, float *, double, const double *);

// ------------------------------------------------------ Gauss-Seidel (scalar)
// one colour: nodes of one colour never share an element, so they are not coupled and
// the colour is updated in parallel exactly as a sequential sweep would.
template <class T, int LPR>
__global__ void k_gs_colour(const int *__restrict__ items, int nitems, const int *__restrict__ qq_ptr,
                            const int *__restrict__ qq_col, const int *__restrict__ diag_pos,
                            const T *__restrict__ vv, const T *__restrict__ b, T *x) {
  EXF_PDL_WAIT();
  const int lane = threadIdx.x % LPR;
  const long g = ((long)blockIdx.x * blockDim.x + threadIdx.x) / LPR;
  const bool valid = g < nitems;  // all lanes reach the shuffles
  const int n = valid ? items[g] : 0;
  const int dp = valid ? diag_pos[n] : 0;
  T acc[1] = {T(0)};
  if (valid) node_row_dot<T, 1, LPR, false>(n, lane, 0, qq_ptr, qq_col, nullptr, nullptr, 0, 0, vv, nullptr, x, acc);
#pragma unroll
  for (int o = LPR / 2; o > 0; o >>= 1) acc[0] += __shfl_down_sync(0xffffffffu, acc[0], o, LPR);
  // the row product included the diagonal term; remove it (x[n] is not updated yet)
  if (valid && lane == 0) x[n] = (b[n] - (acc[0] - vv[dp] * x[n])) / vv[dp];
}

// --------------------------------------------------------------- Vanka
// Patch of pressure node m: the velocity DOFs of pressure row m (all Q2 nodes of the
// elements around vertex m, every component) plus p_m.  With the velocity block
// approximated by its diagonal the local saddle system is solved in closed form:
//   dp = (sum_j D_mj r_j/a_jj - r_m) / (sum_j D_mj G_jm/a_jj - c_mm)
//   du_j = (r_j - G_jm dp)/a_jj ;  x += omega*(du, dp)
// After every assembly k_vanka_prep stores, per (patch, star DOF), {1/a_jj, D_mj/a_jj,
// G_jm/a_jj} contiguously in patch order, and per patch the Schur denominator.
// Per colour: (1) k_vanka_rows computes the residual of every velocity row in the
// colour's stars and of the patches' pressure rows from the iterate at the start of the
// colour (a masked SpMV over disjoint stars, fully parallel, residuals written in patch
// order); (2) k_vanka_solve, one CTA per patch, reduces the Schur numerator with warp
// shuffles in a fixed order and writes its own star.  Stars of one colour are disjoint,
// so the sweep is deterministic and independent of scheduling.

template <class T, int D, int LPR, int NT>
__global__ void __launch_bounds__(NT)
    k_vanka_rows(const int *__restrict__ rows, int nrows, int gbase, const int *__restrict__ items, int npatch,
                 int N, const int *__restrict__ qq_ptr, const int *__restrict__ qq_col,
                 const int *__restrict__ ql_ptr, const int *__restrict__ ql_col, long nqq, long nql, long nqqL,
                 const T *__restrict__ vv, const T *__restrict__ vp, const T *__restrict__ pv,
                 const T *__restrict__ pp, const T *__restrict__ x, const T *__restrict__ b, T *__restrict__ res,
                 long pres_off) {
  EXF_PDL_WAIT();
  const int lane = threadIdx.x % LPR;
  const long g = ((long)blockIdx.x * NT + threadIdx.x) / LPR;
  const bool vel = g < nrows;
  const bool prs = !vel && g < (long)nrows + npatch;
  T acc[D];
#pragma unroll
  for (int a = 0; a < D; a++) acc[a] = T(0);
  int node = 0;
  if (vel) {
    node = rows[g];
    node_row_dot<T, D, LPR, true>(node, lane, N, qq_ptr, qq_col, ql_ptr, ql_col, nqq, nql, vv, vp, x, acc);
  } else if (prs) {
    node = items[g - nrows];
    for (int k = qq_ptr[node] + lane; k < qq_ptr[node + 1]; k += LPR) {
      const int c = qq_col[k];
#pragma unroll
      for (int bb = 0; bb < D; bb++) acc[0] += pv[(long)bb * nqqL + k] * x[(long)bb * N + c];
    }
    for (int k = ql_ptr[node] + lane; k < ql_ptr[node + 1]; k += LPR) acc[0] += pp[k] * x[(long)D * N + ql_col[k]];
  }
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) acc[a] += __shfl_down_sync(0xffffffffu, acc[a], o, LPR);
  if (lane == 0) {
    if (vel) {
#pragma unroll
      for (int a = 0; a < D; a++) res[(gbase + g) * D + a] = b[(long)a * N + node] - acc[a];
    } else if (prs) {
      res[pres_off + node] = b[(long)D * N + node] - acc[0];
    }
  }
}

// per (patch, star DOF): {1/a, D/a, G/a}; per patch: {sum D G / a - c_mm, c_mm}
template <int D>
__global__ void k_vanka_prep(int NL, const int *__restrict__ pstart, const int *__restrict__ qq_ptr,
                             const int *__restrict__ qq_col, const int *__restrict__ ql_ptr,
                             const int *__restrict__ ql_col, const int *__restrict__ diag_pos,
                             const int *__restrict__ gidx, long nqq, long nql, long nqqL, const double *vv,
                             const double *vp, const double *pv, const double *pp, double *vk64, float *vk32,
                             double *pk64, float *pk32) {
  const int m = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (m >= NL) return;  // one warp per patch, uniform per warp
  const int k0 = qq_ptr[m], K = qq_ptr[m + 1] - k0;
  const long g0 = pstart[m];
  double S = 0.;
  for (int t = lane; t < K * D; t += 32) {
    const int kk = t / D, a = t % D;
    const int n = qq_col[k0 + kk];
    const double ia = 1. / vv[(long)(a * D + a) * nqq + diag_pos[n]];
    const double dd = pv[(long)a * nqqL + k0 + kk];
    const double gg = vp[(long)a * nql + gidx[k0 + kk]];
    const long e = 3 * ((g0 + kk) * D + a);
    vk64[e] = ia;
    vk64[e + 1] = dd * ia;
    vk64[e + 2] = gg * ia;
    vk32[e] = (float)ia;
    vk32[e + 1] = (float)(dd * ia);
    vk32[e + 2] = (float)(gg * ia);
    S += dd * gg * ia;
  }
  double cmm = 0.;
  for (int k = ql_ptr[m] + lane; k < ql_ptr[m + 1]; k += 32)
    if (ql_col[k] == m) cmm += pp[k];
  for (int o = 16; o > 0; o >>= 1) {
    S += __shfl_down_sync(0xffffffffu, S, o);
    cmm += __shfl_down_sync(0xffffffffu, cmm, o);
  }
  if (lane == 0) {
    pk64[2 * m] = S - cmm;
    pk64[2 * m + 1] = cmm;
    pk32[2 * m] = (float)(S - cmm);
    pk32[2 * m + 1] = (float)cmm;
  }
}

template <class T, int D, int NT>
__global__ void __launch_bounds__(NT)
    k_vanka_solve(const int *__restrict__ items, int N, const int *__restrict__ qq_ptr,
                  const int *__restrict__ vrows, const int *__restrict__ pstart, const T *__restrict__ vk,
                  const T *__restrict__ pk, const T *__restrict__ res, long pres_off, T *__restrict__ x, T omega) {
  EXF_PDL_WAIT();
  __shared__ double s_red[NT / 32];
  const int m = items[blockIdx.x];
  const int K = qq_ptr[m + 1] - qq_ptr[m];
  const long g0 = pstart[m];
  const T *rr = res + g0 * D;
  const T *w = vk + 3 * g0 * D;
  double tsum = 0.;
  for (int t = threadIdx.x; t < K * D; t += NT) tsum += (double)(w[3 * t + 1] * rr[t]);
  for (int o = 16; o > 0; o >>= 1) tsum += __shfl_down_sync(0xffffffffu, tsum, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = tsum;
  __syncthreads();
  double Tt = 0.;
  for (int k = 0; k < NT / 32; k++) Tt += s_red[k];
  const double St = (double)pk[2 * m];
  Tt -= (double)res[pres_off + m];
  const T dp = (T)(fabs(St) > 1e-300 ? Tt / St : 0.);
  for (int t = threadIdx.x; t < K * D; t += NT) {
    const int kk = t / D, a = t % D;
    const long idx = (long)a * N + vrows[g0 + kk];
    x[idx] += omega * (rr[t] * w[3 * t] - w[3 * t + 2] * dp);
  }
  if (threadIdx.x == 0) x[(long)D * N + m] += omega * dp;
}

template <class T>
struct VK;
template <>
struct VK<double> {
  static const double *vk(const SysLevel &L) { return L.vk64.p; }
  static const double *pk(const SysLevel &L) { return L.pk64.p; }
  static double *res(SysLevel &L) { return L.vres64.p; }
};
template <>
struct VK<float> {
  static const float *vk(const SysLevel &L) { return L.vk32.p; }
  static const float *pk(const SysLevel &L) { return L.pk32.p; }
  static float *res(SysLevel &L) { return L.vres32.p; }
};

template <class T, int D>
static int vanka_sweep(exf_sys *s, int lev, const exf_mg_params *p, T *x, const T *b) {
  SysLevel &L = s->L[lev];
  constexpr int NTS = D == 3 ? 128 : 64;
  constexpr int LPR = D == 3 ? 32 : 16;
  constexpr int NTR = 256;
  T *res = VK<T>::res(L);
  const long pres_off = (long)L.vrow_off[L.ncolour] * D;
  for (int cc = 0; cc < L.ncolour; cc++) {
    const int c = p->reverse_colours ? L.ncolour - 1 - cc : cc;
    const int n = L.col_off[c + 1] - L.col_off[c];
    if (n == 0) continue;
    const int nr = L.vrow_off[c + 1] - L.vrow_off[c];
    const int *items = L.col_items.p + L.col_off[c];
    EXF_CUDA(launch_pdl(k_vanka_rows<T, D, LPR, NTR>, dim3(nblk((long)(nr + n) * LPR, NTR)), dim3(NTR), 0, s->stream,
                        L.vrows.p + L.vrow_off[c], nr, L.vrow_off[c], items, n, L.N, L.qq_ptr.p, L.qq_col.p,
                        L.ql_ptr.p, L.ql_col.p, L.nqq, L.nql, L.nqqL, VT<T>::vv(L), VT<T>::vp(L), VT<T>::pv(L),
                        VT<T>::pp(L), x, b, res, pres_off));
    EXF_CUDA(launch_pdl(k_vanka_solve<T, D, NTS>, dim3(n), dim3(NTS), 0, s->stream, items, L.N, L.qq_ptr.p,
                        L.vrows.p, L.pstart.p, VK<T>::vk(L), VK<T>::pk(L), res, pres_off, x, (T)p->omega));
    EXF_COUNT(2);
  }
  return EXF_OK;
}

int vanka_prep(exf_sys *s, int lev) {
  if (s->kind != EXF_KIND_NS) return EXF_OK;
  SysLevel &L = s->L[lev];
  const unsigned grid = nblk(L.NL, 4);
  if (s->dim == 2)
    k_vanka_prep<2><<<grid, 128, 0, s->stream>>>(L.NL, L.pstart.p, L.qq_ptr.p, L.qq_col.p, L.ql_ptr.p,
                                                  L.ql_col.p, L.diag_pos.p, L.gidx.p, L.nqq, L.nql, L.nqqL,
                                                  L.A.vv.p, L.A.vp.p, L.A.pv.p, L.A.pp.p, L.vk64.p, L.vk32.p,
                                                  L.pk64.p, L.pk32.p);
  else
    k_vanka_prep<3><<<grid, 128, 0, s->stream>>>(L.NL, L.pstart.p, L.qq_ptr.p, L.qq_col.p, L.ql_ptr.p,
                                                  L.ql_col.p, L.diag_pos.p, L.gidx.p, L.nqq, L.nql, L.nqqL,
                                                  L.A.vv.p, L.A.vp.p, L.A.pv.p, L.A.pp.p, L.vk64.p, L.vk32.p,
                                                  L.pk64.p, L.pk32.p);
  EXF_LAUNCH_CHECK();
  EXF_COUNT(1);
  return EXF_OK;
}

template <class T>
static int gs_sweep(exf_sys *s, int lev, const exf_mg_params *p, T *x, const T *b) {
  SysLevel &L = s->L[lev];
  constexpr int LPR = 16;
  for (int cc = 0; cc < L.ncolour; cc++) {
    const int c = p->reverse_colours ? L.ncolour - 1 - cc : cc;
    const int n = L.col_off[c + 1] - L.col_off[c];
    if (n == 0) continue;
    EXF_CUDA(launch_pdl(k_gs_colour<T, LPR>, dim3(nblk((long)n * LPR, 256)), dim3(256), 0, s->stream,
                        L.col_items.p + L.col_off[c], n, L.qq_ptr.p, L.qq_col.p, L.diag_pos.p, VT<T>::vv(L), b, x));
    EXF_COUNT(1);
  }
  return EXF_OK;
}

template <class T>
int smooth(exf_sys *s, int lev, const exf_mg_params *p, int nsweeps, T *x, const T *b) {
  for (int it = 0; it < nsweeps; it++) {
    if (s->kind == EXF_KIND_T) {
      EXF_TRY(gs_sweep<T>(s, lev, p, x, b));
    } else if (s->dim == 2) {
      EXF_TRY((vanka_sweep<T, 2>(s, lev, p, x, b)));
    } else {
      EXF_TRY((vanka_sweep<T, 3>(s, lev, p, x, b)));
    }
  }
  return EXF_OK;
}
template int smooth<double>(exf_sys *, int, const exf_mg_params *, int, double *, const double *);
template int smooth<float>(exf_sys *, int, const exf_mg_params *, int, float *, const float *);

// -------------------------------------------------- coarsest direct solve
// In-place Gauss-Jordan inversion with partial pivoting, once per assembly, in ONE
// cooperative kernel (two grid-wide barriers per pivot).  Pivot rows are not swapped:
// step k pivots on the largest |a_ik| among unused rows p_k, which leaves
// W[p_k][j] = A0^{-1}[k][p_j]; the extraction kernel undoes the permutation.  Each coarse
// solve is then one dense GEMV in FP64.  Pressure-gauge rows become identity rows in the
// factored copy (the enclosed-flow pressure level is otherwise free).  Ties in the pivot
// search go to the smallest row index, so the factorisation is deterministic.
__global__ void k_dense_from_csr(const int *ptr, const int *col, const double *val, int n, double *W) {
  int i = blockIdx.x;
  for (int j = threadIdx.x; j < n; j += blockDim.x) W[(long)i * n + j] = 0.;
  __syncthreads();
  for (int k = ptr[i] + threadIdx.x; k < ptr[i + 1]; k += blockDim.x) W[(long)i * n + col[k]] = val[k];
}
__global__ void k_gauge_rows(double *W, int n, const double *gmask) {
  int i = blockIdx.x;
  if (gmask[i] != 0.) return;
  for (int j = threadIdx.x; j < n; j += blockDim.x) W[(long)i * n + j] = (j == i) ? 1. : 0.;
}

__device__ __forceinline__ void argmax_merge(double &v, int &i, double v2, int i2) {
  if (v2 > v || (v2 == v && i2 >= 0 && (i < 0 || i2 < i))) {
    v = v2;
    i = i2;
  }
}

template <int NT>
__device__ void block_argmax(double v, int i, double *sv, int *si, double *bm, int *bi) {
  for (int o = 16; o > 0; o >>= 1) {
    double v2 = __shfl_down_sync(0xffffffffu, v, o);
    int i2 = __shfl_down_sync(0xffffffffu, i, o);
    argmax_merge(v, i, v2, i2);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sv[w] = v;
    si[w] = i;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double bv = -1.;
    int bidx = -1;
    for (int k = 0; k < NT / 32; k++) argmax_merge(bv, bidx, sv[k], si[k]);
    bm[blockIdx.x] = bv;
    bi[blockIdx.x] = bidx;
  }
  __syncthreads();
}

template <int NT>
__global__ void __launch_bounds__(NT)
    k_gj_coop(double *W, int n, int *pivrow, double *colk, double *rowp, double *bm, int *bi, int *used, int *bad) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  __shared__ double sv[NT / 32];
  __shared__ int si[NT / 32];
  __shared__ int s_p;
  const long gt = (long)blockIdx.x * NT + threadIdx.x;
  const long nth = (long)gridDim.x * NT;
  // candidates for column 0
  {
    double v = -1.;
    int idx = -1;
    for (long i = gt; i < n; i += nth) argmax_merge(v, idx, fabs(W[i * n]), (int)i);
    block_argmax<NT>(v, idx, sv, si, bm, bi);
  }
  grid.sync();
  for (int k = 0; k < n; k++) {
    // phase A: every block selects the same pivot row and stashes row p and column k
    if (threadIdx.x == 0) {
      double bv = -1.;
      int bidx = -1;
      for (int b = 0; b < (int)gridDim.x; b++) argmax_merge(bv, bidx, bm[b], bi[b]);
      s_p = bidx;
    }
    __syncthreads();
    const int p = s_p;
    if (p < 0) {  // every remaining row is zero in this column: singular
      if (gt == 0) *bad = 1;
      return;     // uniform across the grid: every block took the same branch
    }
    if (gt == 0) {
      pivrow[k] = p;
      used[p] = 1;
      if (W[(long)p * n + k] == 0.) *bad = 1;
    }
    for (long t = gt; t < n; t += nth) {
      rowp[t] = W[(long)p * n + t];
      colk[t] = W[t * n + k];
    }
    grid.sync();
    // phase B: update every entry, collect pivot candidates of column k+1
    const double piv = rowp[k];
    const double inv = piv != 0. ? 1. / piv : 0.;
    double v = -1.;
    int idx = -1;
    const long nn = (long)n * n;
    for (long e = gt; e < nn; e += nth) {
      const int i = (int)(e / n), j = (int)(e % n);
      double a;
      if (i == p) a = (j == k) ? inv : rowp[j] * inv;
      else if (j == k) a = -colk[i] * inv;
      else a = W[e] - colk[i] * rowp[j] * inv;
      W[e] = a;
      if (j == k + 1 && i != p && !used[i]) argmax_merge(v, idx, fabs(a), i);
    }
    block_argmax<NT>(v, idx, sv, si, bm, bi);
    grid.sync();
  }
}

// inv[k][p_j] = W[p_k][j]
__global__ void k_extract_inv(const double *W, int n, const int *pivrow, double *inv) {
  const int k = blockIdx.x;
  const int pk = pivrow[k];
  for (int j = threadIdx.x; j < n; j += blockDim.x) inv[(long)k * n + pivrow[j]] = W[(long)pk * n + j];
}

int coarse_factor(exf_sys *s) {
  SysLevel &L = s->L[0];
  const int n = L.ndof;
  cudaStream_t st = s->stream;
  DBuf<double> vals, colk, rowp, bm;
  DBuf<int> bad, pivrow, used, bi;
  EXF_TRY(vals.alloc(L.nnz));
  EXF_TRY(csr_values(s, 0, vals.p));
  EXF_TRY(s->coarse_work.alloc((size_t)n * n));
  EXF_TRY(colk.alloc(n));
  EXF_TRY(rowp.alloc(n));
  EXF_TRY(pivrow.alloc(n));
  EXF_TRY(used.alloc(n));
  EXF_TRY(used.zero(st));
  EXF_TRY(bad.alloc(1));
  EXF_TRY(bad.zero(st));
  double *W = s->coarse_work.p;
  k_dense_from_csr<<<n, 128, 0, st>>>(L.csr_ptr.p, L.csr_col.p, vals.p, n, W);
  k_gauge_rows<<<n, 128, 0, st>>>(W, n, s->gmask0.p);
  EXF_LAUNCH_CHECK();
  constexpr int NT = 256;
  int dev = 0, nsm = 0, per_sm = 0;
  EXF_CUDA(cudaGetDevice(&dev));
  EXF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  EXF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gj_coop<NT>, NT, 0));
  long want = ((long)n * n + NT - 1) / NT;
  int grid = (int)std::min<long>(std::max(1, nsm * std::min(per_sm, 2)), std::max<long>(1, want));
  EXF_TRY(bm.alloc(grid));
  EXF_TRY(bi.alloc(grid));
  void *args[] = {&W, (void *)&n, &pivrow.p, &colk.p, &rowp.p, &bm.p, &bi.p, &used.p, &bad.p};
  EXF_CUDA(cudaLaunchCooperativeKernel((void *)k_gj_coop<NT>, grid, NT, args, 0, st));
  EXF_COUNT(3);
  if (s->coarse_inv.n != (size_t)n * n) {
    EXF_TRY(s->coarse_inv.alloc((size_t)n * n));
    s->buf_epoch++;
  }
  k_extract_inv<<<n, 128, 0, st>>>(W, n, pivrow.p, s->coarse_inv.p);
  EXF_LAUNCH_CHECK();
  int hbad = 0;
  EXF_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  EXF_CUDA(cudaStreamSynchronize(st));
  s->coarse_work.release();
  if (hbad) {
    set_error("coarsest matrix is singular");
    return EXF_ERR_SINGULAR;
  }
  s->coarse_ok = 1;
  return EXF_OK;
}

// x = A0^{-1} (b * gmask), one warp per row, FP64 arithmetic for either vector type
template <class T>
__global__ void k_coarse_gemv(const double *__restrict__ inv, int n, const double *__restrict__ gmask,
                              const T *__restrict__ b, T *__restrict__ x) {
  EXF_PDL_WAIT();
  const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (row >= n) return;
  double acc = 0.;
  for (int j = lane; j < n; j += 32) acc += inv[(long)row * n + j] * (gmask[j] * (double)b[j]);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) x[row] = (T)acc;
}

template <class T>
int coarse_apply(exf_sys *s, const T *b, T *x) {
  if (!s->coarse_ok) EXF_TRY(coarse_factor(s));
  const int n = s->L[0].ndof;
  EXF_CUDA(launch_pdl(k_coarse_gemv<T>, dim3(nblk(n, 8)), dim3(256), 0, s->stream, s->coarse_inv.p, n, s->gmask0.p,
                      b, x));
  EXF_COUNT(1);
  return EXF_OK;
}
template int coarse_apply<double>(exf_sys *, const double *, double *);
template int coarse_apply<float>(exf_sys *, const float *, float *);

// ---------------------------------------------------------- vector helpers
template <class T>
__global__ void k_zero(T *a, long n) {
  EXF_PDL_WAIT();
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = T(0);
}
template <class T>
int zero_vec(cudaStream_t st, T *a, long n) {
  EXF_CUDA(launch_pdl(k_zero<T>, dim3(nblk(n, 256)), dim3(256), 0, st, a, n));
  EXF_COUNT(1);
  return EXF_OK;
}
template int zero_vec<double>(cudaStream_t, double *, long);
template int zero_vec<float>(cudaStream_t, float *, long);

__global__ void k_cast_d2f(const double *a, float *b, long n) {
  EXF_PDL_WAIT();
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}
__global__ void k_add_f2d(const float *a, double *b, long n) {
  EXF_PDL_WAIT();
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] += (double)a[i];
}
int cast_d2f(cudaStream_t st, const double *a, float *b, long n) {
  EXF_CUDA(launch_pdl(k_cast_d2f, dim3(nblk(n, 256)), dim3(256), 0, st, a, b, n));
  EXF_COUNT(1);
  return EXF_OK;
}
int add_f2d(cudaStream_t st, const float *a, double *b, long n) {
  EXF_CUDA(launch_pdl(k_add_f2d, dim3(nblk(n, 256)), dim3(256), 0, st, a, b, n));
  EXF_COUNT(1);
  return EXF_OK;
}

template <int NT>
__global__ void k_norm2_part(const double *v, long n, double *part) {
  EXF_PDL_WAIT();
  __shared__ double sh[32];
  double acc = 0.;
  for (long i = (long)blockIdx.x * NT + threadIdx.x; i < n; i += (long)gridDim.x * NT) acc += v[i] * v[i];
  acc = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}
int norm2(exf_sys *s, const double *v, long n, double *d_out) {
  const int grid = 296;
  EXF_TRY(ensure_partials(s, grid));
  k_norm2_part<256><<<grid, 256, 0, s->stream>>>(v, n, s->red.part.p);
  k_reduce_partials<<<1, 1024, 0, s->stream>>>(s->red.part.p, grid, d_out);
  EXF_LAUNCH_CHECK();
  EXF_COUNT(2);
  return EXF_OK;
}

// pressure gauge: p -= p[gauge] on the top level
__global__ void k_gauge_read(const double *x, long idx, double *out) {
  EXF_PDL_WAIT(); *out = x[idx]; }
__global__ void k_gauge_sub(double *p, int n, const double *v) {
  EXF_PDL_WAIT();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] -= *v;
}
int gauge_shift(exf_sys *s, double *x) {
  if (s->kind != EXF_KIND_NS || s->gauge_node < 0) return EXF_OK;
  SysLevel &T = s->L[s->nlev - 1];
  double *p = x + (long)s->nv2 * T.N;
  EXF_CUDA(launch_pdl(k_gauge_read, dim3(1), dim3(1), 0, s->stream, (const double *)p, (long)s->gauge_node,
                      s->red.out.p + 8));
  EXF_CUDA(launch_pdl(k_gauge_sub, dim3(nblk(T.NL, 256)), dim3(256), 0, s->stream, p, T.NL,
                      (const double *)(s->red.out.p + 8)));
  EXF_COUNT(2);
  return EXF_OK;
}

}  // namespace exf
