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
    const int n = (int)g;
    const int k0 = qq_ptr[n], k1 = qq_ptr[n + 1];
    for (int k = k0 + lane; k < k1; k += LPR) {
      const int m = qq_col[k];
      T xb[D];
#pragma unroll
      for (int bb = 0; bb < D; bb++) xb[bb] = x[(long)bb * N + m];
#pragma unroll
      for (int a = 0; a < D; a++)
#pragma unroll
        for (int bb = 0; bb < D; bb++) acc[a] += vv[(long)(a * D + bb) * nqq + k] * xb[bb];
    }
    if (NS) {
      const int l0 = ql_ptr[n], l1 = ql_ptr[n + 1];
      for (int k = l0 + lane; k < l1; k += LPR) {
        const T p = x[(long)D * N + ql_col[k]];
#pragma unroll
        for (int a = 0; a < D; a++) acc[a] += vp[(long)a * nql + k] * p;
      }
    }
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
  k_spmv_resid<T, D, LPR, NS, NT><<<grid, NT, 0, s->stream>>>(
      L.N, L.NL, L.qq_ptr.p, L.qq_col.p, L.ql_ptr.p, L.ql_col.p, L.nqq, L.nql, L.nqqL, VT<T>::vv(L), VT<T>::vp(L),
      VT<T>::pv(L), VT<T>::pp(L), x, b, r, d_norm2 ? s->red.part.p : nullptr);
  EXF_LAUNCH_CHECK();
  EXF_COUNT(1);
  if (d_norm2) {
    k_reduce_partials<<<1, 1024, 0, s->stream>>>(s->red.part.p, grid, d_norm2);
    EXF_LAUNCH_CHECK();
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
  k_restrict<T><<<nblk(nrow, 256), 256, 0, s->stream>>>(
      s->nv2, s->nv1, C.N, C.NL, F.N, C.Rq.ptr.p, C.Rq.col.p, VT<T>::pq(C.Rq), s->nv1 ? C.Rl.ptr.p : nullptr,
      s->nv1 ? C.Rl.col.p : nullptr, s->nv1 ? VT<T>::pq(C.Rl) : nullptr, C.rmask.p, r_f, b_c);
  EXF_LAUNCH_CHECK();
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
  k_prolong<T><<<nblk(nrow, 256), 256, 0, s->stream>>>(
      s->nv2, s->nv1, F.N, F.NL, C.N, F.Pq.ptr.p, F.Pq.col.p, VT<T>::pq(F.Pq), s->nv1 ? F.Pl.ptr.p : nullptr,
      s->nv1 ? F.Pl.col.p : nullptr, s->nv1 ? VT<T>::pq(F.Pl) : nullptr, x_c, x_f, (T)damp, overwrite, cond);
  EXF_LAUNCH_CHECK();
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
  const int lane = threadIdx.x % LPR;
  const long g = ((long)blockIdx.x * blockDim.x + threadIdx.x) / LPR;
  const bool valid = g < nitems;  // all lanes reach the shuffles
  const int n = valid ? items[g] : 0;
  const int dp = valid ? diag_pos[n] : 0;
  T acc = T(0);
  if (valid)
    for (int k = qq_ptr[n] + lane; k < qq_ptr[n + 1]; k += LPR)
      if (k != dp) acc += vv[k] * x[qq_col[k]];
#pragma unroll
  for (int o = LPR / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, LPR);
  if (valid && lane == 0) x[n] = (b[n] - acc) / vv[dp];
}

// --------------------------------------------------------------- Vanka
// Patch of pressure node m: the velocity DOFs of pressure row m (all Q2 nodes of the
// elements around vertex m, every component) plus p_m.  With the velocity block
// approximated by its diagonal the local saddle system is solved in closed form:
//   dp = (sum_j D_mj r_j/a_jj - r_m) / (sum_j D_mj G_jm/a_jj - c_mm)
//   du_j = (r_j - G_jm dp)/a_jj ;  x += omega*(du, dp)
// Per colour: (1) the residual of every velocity row in the colour's stars is computed
// from the iterate at the start of the colour (a masked SpMV over disjoint stars, fully
// parallel); (2) one CTA per patch forms the closed-form solve (warp shuffles + a fixed
// reduction order) and writes its own star.  A patch's pressure row only reads its own
// star and pressures of other colours, so (2) needs no further synchronisation and the
// sweep is deterministic.
template <class T, int D, int LPR, int NT>
__global__ void __launch_bounds__(NT)
    k_vanka_rows(const int *__restrict__ rows, int nrows, int N, const int *__restrict__ qq_ptr,
                 const int *__restrict__ qq_col, const int *__restrict__ ql_ptr, const int *__restrict__ ql_col,
                 long nqq, long nql, const T *__restrict__ vv, const T *__restrict__ vp, const T *__restrict__ x,
                 const T *__restrict__ b, T *__restrict__ res) {
  const int lane = threadIdx.x % LPR;
  const long g = ((long)blockIdx.x * NT + threadIdx.x) / LPR;
  const bool valid = g < nrows;
  const int n = valid ? rows[g] : 0;
  T acc[D];
#pragma unroll
  for (int a = 0; a < D; a++) acc[a] = T(0);
  if (valid) {
    const int k0 = qq_ptr[n], k1 = qq_ptr[n + 1];
    for (int k = k0 + lane; k < k1; k += LPR) {
      const int c = qq_col[k];
      T xb[D];
#pragma unroll
      for (int bb = 0; bb < D; bb++) xb[bb] = x[(long)bb * N + c];
#pragma unroll
      for (int a = 0; a < D; a++)
#pragma unroll
        for (int bb = 0; bb < D; bb++) acc[a] += vv[(long)(a * D + bb) * nqq + k] * xb[bb];
    }
    const int l0 = ql_ptr[n], l1 = ql_ptr[n + 1];
    for (int k = l0 + lane; k < l1; k += LPR) {
      const T p = x[(long)D * N + ql_col[k]];
#pragma unroll
      for (int a = 0; a < D; a++) acc[a] += vp[(long)a * nql + k] * p;
    }
  }
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) acc[a] += __shfl_down_sync(0xffffffffu, acc[a], o, LPR);
  if (valid && lane == 0) {
#pragma unroll
    for (int a = 0; a < D; a++) res[(long)a * N + n] = b[(long)a * N + n] - acc[a];
  }
}

template <int NT>
__device__ __forceinline__ void block_sum4(double v[4], double (*sh)[NT / 32]) {
#pragma unroll
  for (int i = 0; i < 4; i++)
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0)
    for (int i = 0; i < 4; i++) sh[i][w] = v[i];
  __syncthreads();
  for (int i = 0; i < 4; i++) {
    double r = 0.;
    for (int k = 0; k < NT / 32; k++) r += sh[i][k];
    v[i] = r;
  }
}

template <class T, int D, int NT, int KMAX>
__global__ void __launch_bounds__(NT)
    k_vanka_solve(const int *__restrict__ items, int N, const int *__restrict__ qq_ptr,
                  const int *__restrict__ qq_col, const int *__restrict__ ql_ptr, const int *__restrict__ ql_col,
                  const int *__restrict__ diag_pos, const int *__restrict__ gidx, long nqq, long nql, long nqqL,
                  const T *__restrict__ vv, const T *__restrict__ vp, const T *__restrict__ pv,
                  const T *__restrict__ pp, T *__restrict__ x, const T *__restrict__ b, const T *__restrict__ res,
                  T omega) {
  __shared__ T s_r[KMAX * D];
  __shared__ T s_ia[KMAX * D];
  __shared__ T s_g[KMAX * D];
  __shared__ double s_red[4][NT / 32];
  const int m = items[blockIdx.x];
  const int k0 = qq_ptr[m];
  const int K = min(qq_ptr[m + 1] - k0, KMAX);  // structured hierarchies never exceed KMAX
  // v[0] = sum D G/a, v[1] = sum D r/a, v[2] = pressure-row product, v[3] = c_mm
  double v[4] = {0., 0., 0., 0.};
  for (int t = threadIdx.x; t < K * D; t += NT) {
    const int kk = t / D, a = t % D;
    const int n = qq_col[k0 + kk];
    const T r = res[(long)a * N + n];
    const T ia = T(1) / vv[(long)(a * D + a) * nqq + diag_pos[n]];
    const T g = vp[(long)a * nql + gidx[k0 + kk]];
    const T dd = pv[(long)a * nqqL + k0 + kk];
    s_r[t] = r;
    s_ia[t] = ia;
    s_g[t] = g;
    v[0] += (double)(dd * g * ia);
    v[1] += (double)(dd * r * ia);
    v[2] += (double)(dd * x[(long)a * N + n]);
  }
  for (int k = ql_ptr[m] + threadIdx.x; k < ql_ptr[m + 1]; k += NT) {
    const int c = ql_col[k];
    v[2] += (double)(pp[k] * x[(long)D * N + c]);
    if (c == m) v[3] += (double)pp[k];
  }
  block_sum4<NT>(v, s_red);  // ends with every thread holding the totals
  const double rp = (double)b[(long)D * N + m] - v[2];
  const double St = v[0] - v[3], Tt = v[1] - rp;
  const double dp = fabs(St) > 1e-300 ? Tt / St : 0.;
  const T dpt = (T)dp;
  for (int t = threadIdx.x; t < K * D; t += NT) {
    const int kk = t / D, a = t % D;
    const long idx = (long)a * N + qq_col[k0 + kk];
    x[idx] += omega * (s_r[t] - s_g[t] * dpt) * s_ia[t];
  }
  if (threadIdx.x == 0) x[(long)D * N + m] += omega * dpt;
}

template <class T, int D>
static int vanka_sweep(exf_sys *s, int lev, const exf_mg_params *p, T *x, const T *b) {
  SysLevel &L = s->L[lev];
  constexpr int NTS = D == 3 ? 128 : 64;
  constexpr int KMAX = D == 3 ? 125 : 25;
  constexpr int LPR = D == 3 ? 32 : 16;
  constexpr int NTR = 256;
  T *res = VT<T>::dx(L);
  for (int cc = 0; cc < L.ncolour; cc++) {
    const int c = p->reverse_colours ? L.ncolour - 1 - cc : cc;
    const int n = L.col_off[c + 1] - L.col_off[c];
    if (n == 0) continue;
    const int nr = L.vrow_off[c + 1] - L.vrow_off[c];
    k_vanka_rows<T, D, LPR, NTR><<<nblk((long)nr * LPR, NTR), NTR, 0, s->stream>>>(
        L.vrows.p + L.vrow_off[c], nr, L.N, L.qq_ptr.p, L.qq_col.p, L.ql_ptr.p, L.ql_col.p, L.nqq, L.nql,
        VT<T>::vv(L), VT<T>::vp(L), x, b, res);
    k_vanka_solve<T, D, NTS, KMAX><<<n, NTS, 0, s->stream>>>(
        L.col_items.p + L.col_off[c], L.N, L.qq_ptr.p, L.qq_col.p, L.ql_ptr.p, L.ql_col.p, L.diag_pos.p, L.gidx.p,
        L.nqq, L.nql, L.nqqL, VT<T>::vv(L), VT<T>::vp(L), VT<T>::pv(L), VT<T>::pp(L), x, b, res, (T)p->omega);
    EXF_LAUNCH_CHECK();
    EXF_COUNT(2);
  }
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
    k_gs_colour<T, LPR><<<nblk((long)n * LPR, 256), 256, 0, s->stream>>>(
        L.col_items.p + L.col_off[c], n, L.qq_ptr.p, L.qq_col.p, L.diag_pos.p, VT<T>::vv(L), b, x);
    EXF_LAUNCH_CHECK();
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
// Gauss-Jordan with partial pivoting on [A0 | I] gives A0^{-1} once per assembly; each
// coarse solve is then one dense GEMV in FP64.  Pressure-gauge rows become identity rows
// in the factored copy (the enclosed-flow pressure level is otherwise free).
__global__ void k_dense_from_csr(const int *ptr, const int *col, const double *val, int n, double *W) {
  int i = blockIdx.x;
  for (int k = ptr[i] + threadIdx.x; k < ptr[i + 1]; k += blockDim.x) W[(long)i * 2 * n + col[k]] = val[k];
  for (int j = threadIdx.x; j < n; j += blockDim.x) W[(long)i * 2 * n + n + j] = (i == j) ? 1. : 0.;
}
__global__ void k_gauge_rows(double *W, int n, const double *gmask) {
  int i = blockIdx.x;
  if (gmask[i] != 0.) return;
  for (int j = threadIdx.x; j < 2 * n; j += blockDim.x) W[(long)i * 2 * n + j] = (j == i) ? 1. : 0.;
}
// pivot step k: one CTA selects the pivot, swaps, scales row k, stashes column k
__global__ void k_gj_pivot(double *W, int n, int k, double *colk, int *bad) {
  __shared__ double sv[1024];
  __shared__ int si[1024];
  const int t = threadIdx.x;
  double best = -1.;
  int bi = k;
  for (int i = k + t; i < n; i += blockDim.x) {
    double v = fabs(W[(long)i * 2 * n + k]);
    if (v > best) {
      best = v;
      bi = i;
    }
  }
  sv[t] = best;
  si[t] = bi;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (t < o) {
      if (sv[t + o] > sv[t] || (sv[t + o] == sv[t] && si[t + o] < si[t])) {
        sv[t] = sv[t + o];
        si[t] = si[t + o];
      }
    }
    __syncthreads();
  }
  const int p = si[0];
  const double pv = W[(long)p * 2 * n + k];
  if (t == 0 && pv == 0.) *bad = 1;
  __syncthreads();
  if (p != k)
    for (int j = t; j < 2 * n; j += blockDim.x) {
      double a = W[(long)k * 2 * n + j];
      W[(long)k * 2 * n + j] = W[(long)p * 2 * n + j];
      W[(long)p * 2 * n + j] = a;
    }
  __syncthreads();
  const double inv = pv != 0. ? 1. / pv : 0.;
  for (int j = t; j < 2 * n; j += blockDim.x) W[(long)k * 2 * n + j] *= inv;
  for (int i = t; i < n; i += blockDim.x) colk[i] = (i == k) ? 0. : W[(long)i * 2 * n + k];
}
__global__ void k_gj_elim(double *W, int n, int k, const double *colk) {
  const int i = blockIdx.y;
  const double f = colk[i];
  if (f == 0.) return;
  for (int j = k + blockIdx.x * blockDim.x + threadIdx.x; j < 2 * n; j += gridDim.x * blockDim.x)
    W[(long)i * 2 * n + j] -= f * W[(long)k * 2 * n + j];
}
__global__ void k_extract_inv(const double *W, int n, double *inv) {
  int i = blockIdx.x;
  for (int j = threadIdx.x; j < n; j += blockDim.x) inv[(long)i * n + j] = W[(long)i * 2 * n + n + j];
}

int coarse_factor(exf_sys *s) {
  SysLevel &L = s->L[0];
  const int n = L.ndof;
  cudaStream_t st = s->stream;
  DBuf<double> vals, colk;
  DBuf<int> bad;
  EXF_TRY(vals.alloc(L.nnz));
  EXF_TRY(csr_values(s, 0, vals.p));
  EXF_TRY(s->coarse_work.alloc((size_t)n * 2 * n));
  EXF_TRY(s->coarse_work.zero(st));
  EXF_TRY(colk.alloc(n));
  EXF_TRY(bad.alloc(1));
  EXF_TRY(bad.zero(st));
  double *W = s->coarse_work.p;
  k_dense_from_csr<<<n, 128, 0, st>>>(L.csr_ptr.p, L.csr_col.p, vals.p, n, W);
  k_gauge_rows<<<n, 128, 0, st>>>(W, n, s->gmask0.p);
  EXF_LAUNCH_CHECK();
  for (int k = 0; k < n; k++) {
    k_gj_pivot<<<1, 1024, 0, st>>>(W, n, k, colk.p, bad.p);
    dim3 grid((unsigned)std::min<long>(8, nblk(2 * n - k, 256)), n);
    k_gj_elim<<<grid, 256, 0, st>>>(W, n, k, colk.p);
  }
  EXF_LAUNCH_CHECK();
  if (s->coarse_inv.n != (size_t)n * n) {
    EXF_TRY(s->coarse_inv.alloc((size_t)n * n));
    s->buf_epoch++;
  }
  k_extract_inv<<<n, 128, 0, st>>>(W, n, s->coarse_inv.p);
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
  k_coarse_gemv<T><<<nblk(n, 8), 256, 0, s->stream>>>(s->coarse_inv.p, n, s->gmask0.p, b, x);
  EXF_LAUNCH_CHECK();
  EXF_COUNT(1);
  return EXF_OK;
}
template int coarse_apply<double>(exf_sys *, const double *, double *);
template int coarse_apply<float>(exf_sys *, const float *, float *);

// ---------------------------------------------------------- vector helpers
__global__ void k_cast_d2f(const double *a, float *b, long n) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}
__global__ void k_add_f2d(const float *a, double *b, long n) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] += (double)a[i];
}
int cast_d2f(cudaStream_t st, const double *a, float *b, long n) {
  k_cast_d2f<<<nblk(n, 256), 256, 0, st>>>(a, b, n);
  EXF_LAUNCH_CHECK();
  EXF_COUNT(1);
  return EXF_OK;
}
int add_f2d(cudaStream_t st, const float *a, double *b, long n) {
  k_add_f2d<<<nblk(n, 256), 256, 0, st>>>(a, b, n);
  EXF_LAUNCH_CHECK();
  EXF_COUNT(1);
  return EXF_OK;
}

template <int NT>
__global__ void k_norm2_part(const double *v, long n, double *part) {
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
__global__ void k_gauge_read(const double *x, long idx, double *out) { *out = x[idx]; }
__global__ void k_gauge_sub(double *p, int n, const double *v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] -= *v;
}
int gauge_shift(exf_sys *s, double *x) {
  if (s->kind != EXF_KIND_NS || s->gauge_node < 0) return EXF_OK;
  SysLevel &T = s->L[s->nlev - 1];
  double *p = x + (long)s->nv2 * T.N;
  k_gauge_read<<<1, 1, 0, s->stream>>>(p, s->gauge_node, s->red.out.p + 8);
  k_gauge_sub<<<nblk(T.NL, 256), 256, 0, s->stream>>>(p, T.NL, s->red.out.p + 8);
  EXF_LAUNCH_CHECK();
  EXF_COUNT(2);
  return EXF_OK;
}

}  // namespace exf
