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
#include <atomic>
#include <cmath>
#include <cstdio>
#include <type_traits>
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

// Vector layouts.  DOF order: component a of node n at a*N + n, pressure of vertex m at
// D*N + m.  I4 (FP32 Navier-Stokes V-cycle): the node's (u, v, w, p) as one float4 at
// 4n, so a column gather is one 16-byte load; slot 3 of a non-vertex node stays zero.
template <bool I4>
struct Lay {
  static __device__ __forceinline__ long v(int a, long n, long N) { return I4 ? 4 * n + a : (long)a * N + n; }
  static __device__ __forceinline__ long p(long m, long N, int D) { return I4 ? 4 * m + 3 : (long)D * N + m; }
};

// acc[a] += sum over the node row n of the d x d blocks times x (and B^T times p);
// two blocks per lane in flight
template <class T, int D, int LPR, bool PRESSURE, bool I4 = false>
__device__ __forceinline__ void node_row_dot(int n, int lane, int N, const int *__restrict__ qq_ptr,
                                             const int *__restrict__ qq_col, const int *__restrict__ ql_ptr,
                                             const int *__restrict__ ql_col, long nqq, long nql,
                                             const T *__restrict__ vv, const T *__restrict__ vp,
                                             const T *__restrict__ x, T acc[D]) {
  const int k0 = qq_ptr[n], k1 = qq_ptr[n + 1];
  auto gather = [&](int c, T *xb) {
    if constexpr (I4) {
      const float4 v = reinterpret_cast<const float4 *>(x)[c];
      xb[0] = v.x;
      if (D > 1) xb[D > 1 ? 1 : 0] = v.y;
      if (D > 2) xb[D > 2 ? 2 : 0] = v.z;
    } else {
#pragma unroll
      for (int bb = 0; bb < D; bb++) xb[bb] = x[(long)bb * N + c];
    }
  };
  int k = k0 + lane;
  for (; k + LPR < k1; k += 2 * LPR) {
    const int c0 = qq_col[k], c1 = qq_col[k + LPR];
    T v0[D * D], v1[D * D], x0[D], x1[D];
#pragma unroll
    for (int q = 0; q < D * D; q++) {
      v0[q] = vv[(long)q * nqq + k];
      v1[q] = vv[(long)q * nqq + k + LPR];
    }
    gather(c0, x0);
    gather(c1, x1);
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int bb = 0; bb < D; bb++) acc[a] += v0[a * D + bb] * x0[bb] + v1[a * D + bb] * x1[bb];
  }
  if (k < k1) {
    T x0[D];
    gather(qq_col[k], x0);
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int bb = 0; bb < D; bb++) acc[a] += vv[(long)(a * D + bb) * nqq + k] * x0[bb];
  }
  if (PRESSURE) {
    for (int kp = ql_ptr[n] + lane; kp < ql_ptr[n + 1]; kp += LPR) {
      const T p = x[Lay<I4>::p(ql_col[kp], N, D)];
#pragma unroll
      for (int a = 0; a < D; a++) acc[a] += vp[(long)a * nql + kp] * p;
    }
  }
}

// ------------------------------------------------------------------ SpMV
// row groups: g < N -> Q2 node g (d outputs), g >= N -> Q1 node g-N (1 output).
// LPR lanes per row group; the node-block index k is shared by the d*d planes.
// CTAs per SM the register budget must allow (occupancy over per-thread depth: each
// configuration measured fastest among its neighbours); 3D FP32 also runs 16 lanes per
// node row, so each warp has two rows in flight
template <class T, int D>
constexpr int spmv_minb() {
  return D == 3 ? (sizeof(T) == 4 ? 8 : 6) : (D == 2 ? 6 : 8);
}
template <class T, int D, int LPR, bool NS, int NT, bool I4>
__global__ void __launch_bounds__(NT, spmv_minb<T, D>())
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
    node_row_dot<T, D, LPR, NS, I4>((int)g, lane, N, qq_ptr, qq_col, ql_ptr, ql_col, nqq, nql, vv, vp, x, acc);
  } else if (prs) {
    const int m = (int)(g - N);
    const int k0 = qq_ptr[m], k1 = qq_ptr[m + 1];
    for (int k = k0 + lane; k < k1; k += LPR) {
      const int nn = qq_col[k];
#pragma unroll
      for (int bb = 0; bb < D; bb++) acc[0] += pv[(long)bb * nqqL + k] * x[Lay<I4>::v(bb, nn, N)];
    }
    const int l0 = ql_ptr[m], l1 = ql_ptr[m + 1];
    for (int k = l0 + lane; k < l1; k += LPR) acc[0] += pp[k] * x[Lay<I4>::p(ql_col[k], N, D)];
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
        const long row = Lay<I4>::v(a, g, N);
        T rv = b ? b[row] - acc[a] : acc[a];
        r[row] = rv;
        nrm += (double)rv * (double)rv;
      }
    } else if (prs) {
      const long row = Lay<I4>::p(g - N, N, D);
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
  constexpr bool I4 = NS && sizeof(T) == 4;
  constexpr int LPR = spmv_lpr<T, D, NS>();
  long ngroups = (long)L.N + (NS ? L.NL : 0);
  unsigned grid = nblk(ngroups * LPR, NT);
  if (d_norm2) EXF_TRY(ensure_partials(s, grid));
  EXF_CUDA(launch_pdl(k_spmv_resid<T, D, LPR, NS, NT, I4>, dim3(grid), dim3(NT), 0, s->stream, L.N, L.NL, L.qq_ptr.p,
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
// the FP64 residual kernels that the allocation-free residual (noalloc.cu) launches with
// the same lanes per row
#define EXF_SPMV64_INST(D, NS)                                                                                  \
  template __global__ void k_spmv_resid<double, D, spmv_lpr<double, D, NS>(), NS, 256, false>(                 \
      int, int, const int *, const int *, const int *, const int *, long, long, long, const double *,            \
      const double *, const double *, const double *, const double *, const double *, double *, double *);
EXF_SPMV64_INST(1, false)
EXF_SPMV64_INST(2, true)
EXF_SPMV64_INST(3, true)
#undef EXF_SPMV64_INST

// ------------------------------------------------------------ transfers
// b_c[(a,c)] = mask[(a,c)] * sum_f R[c,f] r_f[(a,f)]   (restriction, rows = coarse DOFs)
template <class T, bool I4>
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
  long dst;
  if (row < nq) {
    int a = (int)(row / Nc), c = (int)(row % Nc);
    for (int k = rq_ptr[c]; k < rq_ptr[c + 1]; k++) acc += rq_val[k] * rf[Lay<I4>::v(a, rq_col[k], Nf)];
    dst = Lay<I4>::v(a, c, Nc);
  } else {
    int c = (int)(row - nq);
    for (int k = rl_ptr[c]; k < rl_ptr[c + 1]; k++) acc += rl_val[k] * rf[Lay<I4>::p(rl_col[k], Nf, nv2)];
    dst = Lay<I4>::p(c, Nc, nv2);
  }
  bc[dst] = (T)mask[row] * acc;
}

template <class T>
int restrict_op(exf_sys *s, int lev_c, const T *r_f, T *b_c) {
  SysLevel &C = s->L[lev_c];
  SysLevel &F = s->L[lev_c + 1];
  long nrow = C.ndof;
  auto kern = (s->nv1 && sizeof(T) == 4) ? k_restrict<T, true> : k_restrict<T, false>;
  EXF_CUDA(launch_pdl(kern, dim3(nblk(nrow, 256)), dim3(256), 0, s->stream, s->nv2, s->nv1, C.N, C.NL, F.N,
                      C.Rq.ptr.p, C.Rq.col.p, VT<T>::pq(C.Rq), s->nv1 ? C.Rl.ptr.p : nullptr,
                      s->nv1 ? C.Rl.col.p : nullptr, s->nv1 ? VT<T>::pq(C.Rl) : nullptr, C.rmask.p, r_f, b_c));
  EXF_COUNT(1);
  return EXF_OK;
}
template int restrict_op<double>(exf_sys *, int, const double *, double *);
template int restrict_op<float>(exf_sys *, int, const float *, float *);

// x_f[(a,f)] += damp * sum_c P[f,c] x_c[(a,c)]   (damp = 0 -> y = P x overwrite mode)
template <class T, bool I4>
__global__ void k_prolong(int nv2, int nv1, int Nf, int NLf, int Nc, const int *__restrict__ pq_ptr,
                          const int *__restrict__ pq_col, const T *__restrict__ pq_val,
                          const int *__restrict__ pl_ptr, const int *__restrict__ pl_col,
                          const T *__restrict__ pl_val, const T *__restrict__ xc, T *__restrict__ xf, T damp,
                          int overwrite, const double *lacc, int lf) {
  EXF_PDL_WAIT();
  // the reference's conditional correction (src/MGSolverBase.C:262-263): added only when
  // the coarse level's accuracy is below this level's pre-smoothing accuracy; lacc holds
  // per level {||b||^2, pre-smoothing r^2, post-smoothing (coarsest: solve) r^2, -}
  if (lacc) {
    const double bf = lacc[4 * lf] > 0. ? sqrt(lacc[4 * lf]) : 1.;
    const double bc = lacc[4 * (lf - 1)] > 0. ? sqrt(lacc[4 * (lf - 1)]) : 1.;
    if (!(sqrt(lacc[4 * (lf - 1) + 2]) / bc < sqrt(lacc[4 * lf + 1]) / bf)) return;
  }
  long row = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long nq = (long)nv2 * Nf;
  if (row >= nq + (long)nv1 * NLf) return;
  T acc = T(0);
  long dst;
  if (row < nq) {
    int a = (int)(row / Nf), f = (int)(row % Nf);
    for (int k = pq_ptr[f]; k < pq_ptr[f + 1]; k++) acc += pq_val[k] * xc[Lay<I4>::v(a, pq_col[k], Nc)];
    dst = Lay<I4>::v(a, f, Nf);
  } else {
    int f = (int)(row - nq);
    for (int k = pl_ptr[f]; k < pl_ptr[f + 1]; k++) acc += pl_val[k] * xc[Lay<I4>::p(pl_col[k], Nc, nv2)];
    dst = Lay<I4>::p(f, Nf, nv2);
  }
  if (overwrite) xf[dst] = acc;
  else xf[dst] += damp * acc;
}

template <class T>
static int prolong_impl(exf_sys *s, int lev_f, const T *x_c, T *x_f, double damp, int overwrite,
                        const double *acc) {
  SysLevel &F = s->L[lev_f];
  SysLevel &C = s->L[lev_f - 1];
  long nrow = F.ndof;
  auto kern = (s->nv1 && sizeof(T) == 4) ? k_prolong<T, true> : k_prolong<T, false>;
  EXF_CUDA(launch_pdl(kern, dim3(nblk(nrow, 256)), dim3(256), 0, s->stream, s->nv2, s->nv1, F.N, F.NL, C.N,
                      F.Pq.ptr.p, F.Pq.col.p, VT<T>::pq(F.Pq), s->nv1 ? F.Pl.ptr.p : nullptr,
                      s->nv1 ? F.Pl.col.p : nullptr, s->nv1 ? VT<T>::pq(F.Pl) : nullptr, x_c, x_f, (T)damp, overwrite,
                      acc, lev_f));
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
int prolong_cond(exf_sys *s, int lev_f, const T *x_c, T *x_f, double damp, const double *acc) {
  return prolong_impl<T>(s, lev_f, x_c, x_f, damp, 0, acc);
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
// Every residual of a colour is computed from the iterate at the start of the colour;
// stars of one colour are disjoint, so the sweep is deterministic and independent of
// scheduling.  Two kernel families do this per colour:
//  ROWS: k_vanka_rows computes the star-row and pressure-row residuals as a masked SpMV
//        (LPR lanes per row, residuals written in patch order), then k_vanka_solve (one
//        CTA per patch) reduces the Schur numerator in a fixed order and updates x.
//  TILE: one CTA per patch gathers the iterate on the 9^d lattice points around vertex m
//        (every column of the star rows lies within 4 lattice steps of m) into shared
//        memory, computes the residuals against that tile (columns addressed by a
//        precomputed tile step, no dependent global gather), solves, and writes compact
//        corrections; k_vanka_apply adds them once every patch has read its tile.  The
//        3D FP32 variant (k_vanka_stream) streams each warp's rows into shared memory
//        with asynchronous copies.
// The FP32 smoother reads the velocity blocks in FP16, scaled per (node, component) row
// by the row's largest magnitude (vsc); the FP64 smoother reads the FP64 blocks.

// Sources of the blocks of a row.  Planar: column in col[k], value q of block k at
// v[q*stride + k] (NQ values).  Packed16: FP16 row-scaled velocity blocks, one 16-byte
// record of values 0..7 per block plus {column, value 8} (3D), or one 8-byte record of
// values 0..3 with the column in col[k] (2D): two loads per block instead of 1 + d*d.
template <class T, int NQ>
struct PlanarBlocks {
  static constexpr bool scaled = false;
  const int *__restrict__ col;
  const T *__restrict__ v;
  long stride;
  template <int M>  // into the first NQ entries of o
  __device__ __forceinline__ void load(long k, int &c, T (&o)[M]) const {
    static_assert(M >= NQ, "block buffer too small");
    c = col[k];
#pragma unroll
    for (int q = 0; q < NQ; q++) o[q] = v[(long)q * stride + k];
  }
};

__device__ __forceinline__ float2 h2f(unsigned w) {
  __half2 h;
  memcpy(&h, &w, 4);
  return __half22float2(h);
}

template <int D>
struct Packed16 {
  static constexpr bool scaled = true;
  const int *__restrict__ col;
  const void *__restrict__ h;
  const uint2 *__restrict__ cx;
  template <int M>
  __device__ __forceinline__ void load(long k, int &c, float (&o)[M]) const {
    static_assert(M >= D * D, "block buffer too small");
    float2 f;
    if constexpr (D == 3) {
      const uint4 r = reinterpret_cast<const uint4 *>(h)[k];
      const uint2 e = cx[k];
      c = (int)e.x;
      f = h2f(r.x); o[0] = f.x; o[1] = f.y;
      f = h2f(r.y); o[2] = f.x; o[3] = f.y;
      f = h2f(r.z); o[4] = f.x; o[5] = f.y;
      f = h2f(r.w); o[6] = f.x; o[7] = f.y;
      f = h2f(e.y); o[8] = f.x;
    } else {
      const uint2 r = reinterpret_cast<const uint2 *>(h)[k];
      c = col[k];
      f = h2f(r.x); o[0] = f.x; o[1] = f.y;
      f = h2f(r.y); o[2] = f.x; o[3] = f.y;
    }
  }
};

// Row product of one star row (RA = D outputs: d x d blocks and the d planes of vp) or
// pressure row (RA = 1: the d planes of pv as 1 x d blocks, and pp) by LPR lanes, UNR
// blocks per lane in flight: all columns and values of a chunk are loaded before the
// first gather; the pressure couplings (at most LPR per row on these meshes) are loaded
// up front with them.  rsc undoes a row scaling of the blocks on each lane's sum.
// patch_row_first loads what does not change during a sweep (the couplings and the
// first chunk), so a kernel can issue it before waiting for the iterate;
// patch_row_rest gathers, multiplies and walks the remaining chunks.  LW >= RA and
// VW >= RA * D are the caller's buffer widths.
template <class T, int D, int LPR, int UNR, int RA, class BL, int LW, int VW>
__device__ __forceinline__ void patch_row_first(int lane, int k0, int nk, int l0, int nl, const BL &bl,
                                                const int *__restrict__ ql_col, long lstride,
                                                const T *__restrict__ lv, int &lc, T (&lw)[LW], int (&c)[UNR],
                                                T (&v)[UNR][VW]) {
  static_assert(LW >= RA && VW >= RA * D, "row buffers too small");
  lc = -1;
  if (lane < nl) {
    lc = ql_col[l0 + lane];
#pragma unroll
    for (int a = 0; a < RA; a++) lw[a] = lv[(long)a * lstride + l0 + lane];
  }
#pragma unroll
  for (int u = 0; u < UNR; u++) {
    const int i = u * LPR + lane;
    c[u] = -1;
    if (i < nk) bl.load(k0 + i, c[u], v[u]);
  }
}

template <class T, int D, int LPR, int UNR, bool I4, int RA, class BL, int LW, int VW>
__device__ __forceinline__ void patch_row_rest(int lane, int N, int k0, int nk, int l0, int nl, const BL &bl,
                                               const int *__restrict__ ql_col, long lstride,
                                               const T *__restrict__ lv, const T *__restrict__ x, T acc[D],
                                               const T (&rsc)[D], int lc, const T (&lw)[LW], int (&c)[UNR],
                                               T (&v)[UNR][VW]) {
  for (int base = 0; base < nk; base += UNR * LPR) {
    if (base > 0) {
#pragma unroll
      for (int u = 0; u < UNR; u++) {
        const int i = base + u * LPR + lane;
        c[u] = -1;
        if (i < nk) bl.load(k0 + i, c[u], v[u]);
      }
    }
    T xb[UNR][D];
#pragma unroll
    for (int u = 0; u < UNR; u++) {
      if constexpr (I4) {
        float4 t4 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c[u] >= 0) t4 = reinterpret_cast<const float4 *>(x)[c[u]];
        xb[u][0] = t4.x;
        if (D > 1) xb[u][D > 1 ? 1 : 0] = t4.y;
        if (D > 2) xb[u][D > 2 ? 2 : 0] = t4.z;
      } else {
#pragma unroll
        for (int bb = 0; bb < D; bb++) xb[u][bb] = c[u] >= 0 ? x[(long)bb * N + c[u]] : T(0);
      }
    }
#pragma unroll
    for (int u = 0; u < UNR; u++)
      if (c[u] >= 0)
#pragma unroll
        for (int a = 0; a < RA; a++)
#pragma unroll
          for (int bb = 0; bb < D; bb++) acc[a] += v[u][a * D + bb] * xb[u][bb];
  }
  if constexpr (BL::scaled) {
#pragma unroll
    for (int a = 0; a < RA; a++) acc[a] *= rsc[a];
  }
  if (lc >= 0) {
    const T pval = x[Lay<I4>::p(lc, N, D)];
#pragma unroll
    for (int a = 0; a < RA; a++) acc[a] += lw[a] * pval;
  }
  for (int i = LPR + lane; i < nl; i += LPR) {  // rows with more than LPR pressure couplings
    const T pval = x[Lay<I4>::p(ql_col[l0 + i], N, D)];
#pragma unroll
    for (int a = 0; a < RA; a++) acc[a] += lv[(long)a * lstride + l0 + i] * pval;
  }
}

template <class T, int D, int LPR, int UNR, bool I4, int RA, class BL>
__device__ __forceinline__ void patch_row_dot(int lane, int N, int k0, int nk, int l0, int nl, const BL &bl,
                                              const int *__restrict__ ql_col, long lstride,
                                              const T *__restrict__ lv, const T *__restrict__ x, T acc[D],
                                              const T (&rsc)[D]) {
  int lc, c[UNR];
  T lw[RA], v[UNR][RA * D];
  patch_row_first<T, D, LPR, UNR, RA>(lane, k0, nk, l0, nl, bl, ql_col, lstride, lv, lc, lw, c, v);
  patch_row_rest<T, D, LPR, UNR, I4, RA>(lane, N, k0, nk, l0, nl, bl, ql_col, lstride, lv, x, acc, rsc, lc, lw, c,
                                         v);
}

// ROWS phase 1: residuals of the star rows (g < nrows) and of the patches' pressure
// rows (g >= nrows), LPR lanes per row, written in patch order.  rinfo per star row:
// {node, qq_ptr[node], ql_ptr[node], nqq | nql << 8 | tile index << 16}; pinfo per patch
// (two int4): {m, first star entry, qq_ptr[m], ql_ptr[m]}, {nqq(m), nql(m), lattice, 0}.
template <class T, int D, int LPR, int NT, bool I4, int UNR, int MINB, class VB>
__global__ void __launch_bounds__(NT, MINB)
    k_vanka_rows(const int4 *__restrict__ rinfo, int nrows, int gbase, const int4 *__restrict__ pinfo, int npatch,
                 int N, VB vb, const T *__restrict__ vsc, const int *__restrict__ qq_col,
                 const int *__restrict__ ql_col, long nql, long nqqL, const T *__restrict__ vp,
                 const T *__restrict__ pv, const T *__restrict__ pp, const T *__restrict__ x,
                 const T *__restrict__ b, T *__restrict__ res, long pres_off) {
  const int lane = threadIdx.x % LPR;
  const long g = ((long)blockIdx.x * NT + threadIdx.x) / LPR;
  const bool vel = g < nrows;
  const bool prs = !vel && g < (long)nrows + npatch;
  // the row descriptors, scales, couplings and the first chunk of blocks do not change
  // during a sweep (only kernels that complete before their dependents start write
  // them): load them before waiting for the iterate
  int4 q0 = make_int4(0, 0, 0, 0), q1 = q0;
  if (vel) {
    q0 = rinfo[g];
  } else if (prs) {
    q0 = pinfo[2 * (g - nrows)];
    q1 = pinfo[2 * (g - nrows) + 1];
  }
  const PlanarBlocks<T, D> pb{qq_col, pv, nqqL};
  int lc = -1, c[UNR];
  T lw[D], v[UNR][D * D], sc[D];
#pragma unroll
  for (int u = 0; u < UNR; u++) c[u] = -1;
  const int node = q0.x;
  if (vel) {
#pragma unroll
    for (int a = 0; a < D; a++) sc[a] = VB::scaled ? vsc[(long)a * N + node] : T(1);
    patch_row_first<T, D, LPR, UNR, D>(lane, q0.y, q0.w & 0xff, q0.z, (q0.w >> 8) & 0xff, vb, ql_col, nql, vp, lc,
                                       lw, c, v);
  } else if (prs) {
    patch_row_first<T, D, LPR, UNR, 1>(lane, q0.z, q1.x, q0.w, q1.y, pb, ql_col, 0, pp, lc, lw, c, v);
  }
  EXF_PDL_WAIT();
  T acc[D], bv[D];
#pragma unroll
  for (int a = 0; a < D; a++) acc[a] = bv[a] = T(0);
  if (vel) {
    if (lane == 0) {
#pragma unroll
      for (int a = 0; a < D; a++) bv[a] = b[Lay<I4>::v(a, node, N)];
    }
    patch_row_rest<T, D, LPR, UNR, I4, D>(lane, N, q0.y, q0.w & 0xff, q0.z, (q0.w >> 8) & 0xff, vb, ql_col, nql, vp,
                                          x, acc, sc, lc, lw, c, v);
  } else if (prs) {
    if (lane == 0) bv[0] = b[Lay<I4>::p(node, N, D)];
    const T one[D] = {};
    patch_row_rest<T, D, LPR, UNR, I4, 1>(lane, N, q0.z, q1.x, q0.w, q1.y, pb, ql_col, 0, pp, x, acc, one, lc, lw, c,
                                          v);
  }
#pragma unroll
  for (int a = 0; a < D; a++)
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) acc[a] += __shfl_down_sync(0xffffffffu, acc[a], o, LPR);
  if (lane == 0) {
    if (vel) {
#pragma unroll
      for (int a = 0; a < D; a++) res[(gbase + g) * D + a] = bv[a] - acc[a];
    } else if (prs) {
      res[pres_off + node] = bv[0] - acc[0];
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

// ROWS phase 2: one CTA per patch; every value the update needs (residuals,
// coefficients, star nodes, current iterate) is loaded in one round before the Schur
// numerator is reduced (warp shuffles, then the warps in order).  SU entries per thread
// cover the stars of these meshes; longer stars take the loops after the first round.
template <class T, int D, int NT, bool I4, int SU>
__global__ void __launch_bounds__(NT)
    k_vanka_solve(const int4 *__restrict__ pinfo, int N, const int *__restrict__ vrows, const T *__restrict__ vk,
                  const T *__restrict__ pk, const T *__restrict__ res, long pres_off, T *__restrict__ x, T omega) {
  __shared__ double s_red[NT / 32];
  // the patch's coefficients and star rows do not change during a sweep: load them
  // before waiting for the row kernel
  const int4 pi = pinfo[2 * blockIdx.x];
  const int m = pi.x, KD = pinfo[2 * blockIdx.x + 1].x * D;
  const long g0 = pi.y;
  const T *rr = res + g0 * D;
  const T *w = vk + 3 * g0 * D;
  T r_[SU], w0[SU], w1[SU], w2[SU], xv[SU];
  long ix[SU];
#pragma unroll
  for (int u = 0; u < SU; u++) {
    const int t = threadIdx.x + u * NT;
    ix[u] = -1;
    r_[u] = w0[u] = w1[u] = w2[u] = xv[u] = T(0);
    if (t < KD) {
      w0[u] = w[3 * t];
      w1[u] = w[3 * t + 1];
      w2[u] = w[3 * t + 2];
      ix[u] = Lay<I4>::v(t % D, vrows[g0 + t / D], N);
    }
  }
  const double Sd = (double)pk[2 * m];
  EXF_PDL_WAIT();  // residuals and iterate come from the previous kernels
#pragma unroll
  for (int u = 0; u < SU; u++)
    if (ix[u] >= 0) {
      r_[u] = rr[threadIdx.x + u * NT];
      xv[u] = x[ix[u]];
    }
  const T rp = res[pres_off + m];
  T xp = T(0);
  if (threadIdx.x == 0) xp = x[Lay<I4>::p(m, N, D)];
  double tsum = 0.;
#pragma unroll
  for (int u = 0; u < SU; u++)
    if (ix[u] >= 0) tsum += (double)(w1[u] * r_[u]);
  for (int t = threadIdx.x + SU * NT; t < KD; t += NT) tsum += (double)(w[3 * t + 1] * rr[t]);
  for (int o = 16; o > 0; o >>= 1) tsum += __shfl_down_sync(0xffffffffu, tsum, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = tsum;
  __syncthreads();
  // every thread sums the warps' partials in warp order (the same value everywhere)
  double Tt = 0.;
#pragma unroll
  for (int k = 0; k < NT / 32; k++) Tt += s_red[k];
  const double num = Tt - (double)rp, den = Sd;
  const T dp = (T)(fabs(den) > 1e-300 ? num / den : 0.);
#pragma unroll
  for (int u = 0; u < SU; u++)
    if (ix[u] >= 0) x[ix[u]] = xv[u] + omega * (r_[u] * w0[u] - w2[u] * dp);
  for (int t = threadIdx.x + SU * NT; t < KD; t += NT) {
    const long idx = Lay<I4>::v(t % D, vrows[g0 + t / D], N);
    x[idx] += omega * (rr[t] * w[3 * t] - w[3 * t + 2] * dp);
  }
  if (threadIdx.x == 0) x[Lay<I4>::p(m, N, D)] = xp + omega * dp;
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

// ------------------------------------------------- TILE: one CTA per patch
// Block sources in tile mode: load() fetches a block's raw record, step() and unpack()
// give the tile step of its column and its values.
template <int D>
struct TileBlocks16 {  // FP16 row-scaled; 3D: uint4 + {value 8, step}; 2D: uint2 + step
  static constexpr bool scaled = true;
  struct Raw {
    uint4 r;
    uint32_t e;
  };
  const void *__restrict__ h;
  const uint32_t *__restrict__ qc;
  const int16_t *__restrict__ tcq;
  __device__ __forceinline__ Raw load(long k) const {
    Raw w;
    if constexpr (D == 3) {
      w.r = reinterpret_cast<const uint4 *>(h)[k];
      w.e = qc[k];
    } else {
      const uint2 r2 = reinterpret_cast<const uint2 *>(h)[k];
      w.r = make_uint4(r2.x, r2.y, 0u, 0u);
      w.e = (uint32_t)(uint16_t)tcq[k] << 16;
    }
    return w;
  }
  static __device__ __forceinline__ int step(const Raw &w) { return (int)(int16_t)(w.e >> 16); }
  static __device__ __forceinline__ void unpack(const Raw &w, float (&o)[D * D]) {
    float2 f;
    f = h2f(w.r.x); o[0] = f.x; o[1] = f.y;
    f = h2f(w.r.y); o[2] = f.x; o[3] = f.y;
    if constexpr (D == 3) {
      f = h2f(w.r.z); o[4] = f.x; o[5] = f.y;
      f = h2f(w.r.w); o[6] = f.x; o[7] = f.y;
      o[8] = h2f(w.e).x;
    }
  }
};
template <class T, int NQ>
struct TileBlocksPlanar {
  static constexpr bool scaled = false;
  struct Raw {
    T v[NQ];
    int st;
  };
  const T *__restrict__ v;
  long stride;
  const int16_t *__restrict__ tcq;
  __device__ __forceinline__ Raw load(long k) const {
    Raw w;
    w.st = tcq[k];
#pragma unroll
    for (int q = 0; q < NQ; q++) w.v[q] = v[(long)q * stride + k];
    return w;
  }
  static __device__ __forceinline__ int step(const Raw &w) { return w.st; }
  static __device__ __forceinline__ void unpack(const Raw &w, T (&o)[NQ]) {
#pragma unroll
    for (int q = 0; q < NQ; q++) o[q] = w.v[q];
  }
};

// Row product against the tile: UNR blocks per lane loaded, then used; the rest of the
// row (longer than UNR*LPR blocks), the row scale and the pressure couplings (lv planes,
// tile steps tcl, tile slot 3) in tile_row_finish.
template <class BL, int UNR>
struct RowRegs {
  bool ok[UNR];
  typename BL::Raw w[UNR];
};

template <int LPR, int UNR, class BL>
__device__ __forceinline__ void tile_row_load(int lane, int base, int k0, int nk, const BL &bl, RowRegs<BL, UNR> &R) {
#pragma unroll
  for (int u = 0; u < UNR; u++) {
    const int i = base + u * LPR + lane;
    R.ok[u] = i < nk;
    if (R.ok[u]) R.w[u] = bl.load(k0 + i);
  }
}

template <class T, int D, int UNR, int RA, class BL>
__device__ __forceinline__ void tile_row_use(const T (*tile)[4], int tb, const RowRegs<BL, UNR> &R, T acc[RA]) {
#pragma unroll
  for (int u = 0; u < UNR; u++)
    if (R.ok[u]) {
      T v[RA * D];
      BL::unpack(R.w[u], v);
      const T *xt = tile[tb + BL::step(R.w[u])];
#pragma unroll
      for (int a = 0; a < RA; a++)
#pragma unroll
        for (int bb = 0; bb < D; bb++) acc[a] += v[a * D + bb] * xt[bb];
    }
}

template <class T, int D, int LPR, int UNR, int RA, class BL>
__device__ __forceinline__ void tile_row_finish(int lane, const T (*tile)[4], int tb, int k0, int nk, int l0, int nl,
                                                const BL &bl, const int16_t *__restrict__ tcl, long lstride,
                                                const T *__restrict__ lv, T acc[RA], const T (&rsc)[RA]) {
  for (int base = UNR * LPR; base < nk; base += UNR * LPR) {
    RowRegs<BL, UNR> R;
    tile_row_load<LPR, UNR>(lane, base, k0, nk, bl, R);
    tile_row_use<T, D, UNR, RA>(tile, tb, R, acc);
  }
  if constexpr (BL::scaled) {
#pragma unroll
    for (int a = 0; a < RA; a++) acc[a] *= rsc[a];
  }
  for (int i = lane; i < nl; i += LPR) {
    const T pval = tile[tb + tcl[l0 + i]][3];
#pragma unroll
    for (int a = 0; a < RA; a++) acc[a] += lv[(long)a * lstride + l0 + i] * pval;
  }
}

// The iterate on the 9^d tile around the patch vertex whose lattice coordinates are
// packed in pz (zero outside the mesh, never referenced there).
template <class T, int D, int NT, bool I4>
__device__ __forceinline__ void load_tile(T (*tile)[4], int pz, int N, int NL, int L0, int L1, int L2,
                                          const int *__restrict__ latnode, const T *__restrict__ x) {
  constexpr int TS = D == 3 ? 729 : 81;
  const int ox = (pz & 2047) - 4, oy = ((pz >> 11) & 2047) - 4, oz = ((pz >> 22) & 1023) - 4;
  for (int t = threadIdx.x; t < TS; t += NT) {
    const int gx = ox + t % 9, gy = oy + (t / 9) % 9, gz = D == 3 ? oz + t / 81 : 0;
    T q0 = T(0), q1 = T(0), q2 = T(0), q3 = T(0);
    if (gx >= 0 && gx < L0 && gy >= 0 && gy < L1 && gz >= 0 && gz < L2) {
      const int n = latnode[((long)gz * L1 + gy) * L0 + gx];
      if constexpr (I4) {
        const float4 f = reinterpret_cast<const float4 *>(x)[n];
        q0 = f.x;
        q1 = f.y;
        q2 = f.z;
        q3 = f.w;
      } else {
        q0 = x[n];
        q1 = x[(long)N + n];
        if (D == 3) q2 = x[2L * N + n];
        if (n < NL) q3 = x[(long)D * N + n];
      }
    }
    tile[t][0] = q0;
    tile[t][1] = q1;
    tile[t][2] = q2;
    tile[t][3] = q3;
  }
}

// Schur numerator (threads in order, warps in order) and the corrections of one patch
// from its residuals res[0 .. K*D] (the last one the pressure row)
template <class T, int D, int NT>
__device__ __forceinline__ void patch_solve(const T *res, double *red, int K, int m, long g0,
                                            const T *__restrict__ vk, const T *__restrict__ pk, T *__restrict__ dlt,
                                            long pres_off, T omega) {
  constexpr int NW = NT / 32;
  const int KD = K * D;
  const T *w = vk + 3 * g0 * D;
  double tsum = 0.;
  for (int t = threadIdx.x; t < KD; t += NT) tsum += (double)(w[3 * t + 1] * res[t]);
  for (int o = 16; o > 0; o >>= 1) tsum += __shfl_down_sync(0xffffffffu, tsum, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = tsum;
  __syncthreads();
  double Tt = 0.;
  for (int k = 0; k < NW; k++) Tt += red[k];
  Tt -= (double)res[KD];
  const double Sd = (double)pk[2 * m];
  const T dp = (T)(fabs(Sd) > 1e-300 ? Tt / Sd : 0.);
  for (int t = threadIdx.x; t < KD; t += NT) dlt[g0 * D + t] = omega * (res[t] * w[3 * t] - w[3 * t + 2] * dp);
  if (threadIdx.x == 0) dlt[pres_off + m] = omega * dp;
}

template <class T, int D, int NT, int LPR, int UNR, bool I4, class BL>
__global__ void __launch_bounds__(NT)
    k_vanka_tile(const int4 *__restrict__ pinfo, const int4 *__restrict__ rinfo, int N, int NL, int L0, int L1,
                 int L2, const int *__restrict__ latnode, BL bl, const T *__restrict__ vsc,
                 const int16_t *__restrict__ tcq, const int16_t *__restrict__ tcl, long nql, long nqqL,
                 const T *__restrict__ vp, const T *__restrict__ pv, const T *__restrict__ pp,
                 const T *__restrict__ vk, const T *__restrict__ pk, const T *__restrict__ x,
                 const T *__restrict__ b, T *__restrict__ dlt, long pres_off, T omega) {
  constexpr int TS = D == 3 ? 729 : 81;
  constexpr int KMAX = D == 3 ? 125 : 25;
  constexpr int TC = D == 3 ? 364 : 40;  // tile index of the patch vertex
  constexpr int NW = NT / 32;
  constexpr int NG = NW * (32 / LPR);    // row groups of the CTA
  __shared__ T tile[TS][4];
  __shared__ T res[KMAX * D + 1];
  __shared__ int4 s_ri[KMAX];
  __shared__ double red[NW];
  EXF_PDL_WAIT();
  const int4 pi = pinfo[2 * blockIdx.x];
  const int4 pj = pinfo[2 * blockIdx.x + 1];
  const int m = pi.x, K = pj.x;
  const long g0 = pi.y;
  for (int r = threadIdx.x; r < K; r += NT) s_ri[r] = rinfo[g0 + r];
  load_tile<T, D, NT, I4>(tile, pj.z, N, NL, L0, L1, L2, latnode, x);
  __syncthreads();
  // star-row residuals, one row per row group and pass
  const int lane = threadIdx.x % LPR, grp = threadIdx.x / LPR;
  const int npass = (K + NG - 1) / NG;
  for (int ps = 0; ps < npass; ps++) {
    const int r = ps * NG + grp;
    int4 ri = make_int4(0, 0, 0, 0);
    if (r < K) ri = s_ri[r];
    RowRegs<BL, UNR> R;
    tile_row_load<LPR, UNR>(lane, 0, ri.y, r < K ? (ri.w & 0xff) : 0, bl, R);
    T sc[D], bv[D], acc[D];
#pragma unroll
    for (int a = 0; a < D; a++) {
      sc[a] = T(1);
      bv[a] = acc[a] = T(0);
      if (r < K) {
        if (BL::scaled) sc[a] = vsc[(long)a * N + ri.x];
        if (lane == 0) bv[a] = b[Lay<I4>::v(a, ri.x, N)];
      }
    }
    if (r < K) {
      tile_row_use<T, D, UNR, D>(tile, ri.w >> 16, R, acc);
      tile_row_finish<T, D, LPR, UNR, D>(lane, tile, ri.w >> 16, ri.y, ri.w & 0xff, ri.z, (ri.w >> 8) & 0xff, bl,
                                         tcl, nql, vp, acc, sc);
    }
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) acc[a] += __shfl_down_sync(0xffffffffu, acc[a], o, LPR);
    if (lane == 0 && r < K) {
#pragma unroll
      for (int a = 0; a < D; a++) res[r * D + a] = bv[a] - acc[a];
    }
  }
  // pressure row of m: one warp
  if (threadIdx.x < 32) {
    const int ln = threadIdx.x;
    T acc[1] = {T(0)};
    const T one[1] = {T(1)};
    const TileBlocksPlanar<T, D> pb{pv, nqqL, tcq};
    tile_row_finish<T, D, 32, 1, 1>(ln, tile, TC, pi.z - 32, K + 32, pi.w, pj.y, pb, tcl, 0, pp, acc, one);
    for (int o = 16; o > 0; o >>= 1) acc[0] += __shfl_down_sync(0xffffffffu, acc[0], o);
    if (ln == 0) res[K * D] = b[Lay<I4>::p(m, N, D)] - acc[0];
  }
  __syncthreads();
  patch_solve<T, D, NT>(res, red, K, m, g0, vk, pk, dlt, pres_off, omega);
}

// --------------------------------------- TILE, 3D FP32: streamed star rows
// Each warp owns star rows w, w+NW, ... of the patch and streams their FP16 records
// (16-byte values + 4-byte {value 8, tile step}) into a per-warp ring of SLOTS
// shared-memory slots with asynchronous copies (cp.async), SLOTS-1 rows ahead of the row
// it computes, so the bytes in flight do not depend on registers; the small per-row data
// (row scales, right-hand side, pressure couplings) is loaded one row ahead into
// registers.  Waits are cp.async.wait_group on the thread's own copies (no spinning).
#define EXF_ST_ROWMAX 128  // records per slot (star rows have at most 125 blocks)
#define EXF_ST_QMAX 136    // 4-byte words per slot: 125 blocks + alignment slack, 16-byte multiple

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int NT, int SLOTS>
struct StreamSmem {
  float tile[729][4];
  float res[125 * 3 + 1];
  int4 ri[125];
  double red[NT / 32];
  uint4 h[NT / 32][SLOTS][EXF_ST_ROWMAX];
  uint32_t q[NT / 32][SLOTS][EXF_ST_QMAX];
};

template <int NT, int SLOTS>
__global__ void __launch_bounds__(NT)
    k_vanka_stream(const int4 *__restrict__ pinfo, const int4 *__restrict__ rinfo, int N, int L0, int L1, int L2,
                   const int *__restrict__ latnode, const uint4 *__restrict__ h16, const uint32_t *__restrict__ h16qc,
                   const float *__restrict__ vsc, const int16_t *__restrict__ tcq, const int16_t *__restrict__ tcl,
                   long nql, long nqqL, const float *__restrict__ vp, const float *__restrict__ pv,
                   const float *__restrict__ pp, const float *__restrict__ vk, const float *__restrict__ pk,
                   const float *__restrict__ x, const float *__restrict__ b, float *__restrict__ dlt, long pres_off,
                   float omega) {
  constexpr int NW = NT / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StreamSmem<NT, SLOTS> &S = *reinterpret_cast<StreamSmem<NT, SLOTS> *>(smem_raw);
  EXF_PDL_WAIT();
  const int4 pi = pinfo[2 * blockIdx.x];
  const int4 pj = pinfo[2 * blockIdx.x + 1];
  const int m = pi.x, K = pj.x;
  const long g0 = pi.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nmine = K > warp ? (K - warp + NW - 1) / NW : 0;  // star rows of this warp
  for (int r = threadIdx.x; r < K; r += NT) S.ri[r] = rinfo[g0 + r];
  __syncthreads();
  // copies of the i-th row of this warp into slot i % SLOTS (the 4-byte records as the
  // aligned 16-byte chunks that cover them)
  auto issue = [&](int i) {
    const int4 ri = S.ri[warp + i * NW];
    const int k0 = ri.y, nk = ri.w & 0xff;
    const int sl = i % SLOTS;
    for (int j = lane; j < nk; j += 32) cp_async16(&S.h[warp][sl][j], h16 + k0 + j);
    const int qa = k0 & ~3, qn = ((k0 + nk + 3) & ~3) - qa;
    for (int j = lane * 4; j < qn; j += 128) cp_async16(&S.q[warp][sl][j], h16qc + qa + j);
  };
#pragma unroll
  for (int i = 0; i < SLOTS - 1; i++) {
    if (i < nmine) issue(i);
    cp_async_commit();
  }
  load_tile<float, 3, NT, true>(S.tile, pj.z, N, 0, L0, L1, L2, latnode, x);
  __syncthreads();
  // pressure row of m (warp 0, direct loads; B = pv plane by plane)
  if (warp == 0) {
    float acc = 0.f;
    for (int j = lane; j < K; j += 32) {
      const long k = pi.z + j;
      const float *xt = S.tile[364 + tcq[k]];
      acc += pv[k] * xt[0] + pv[nqqL + k] * xt[1] + pv[2 * nqqL + k] * xt[2];
    }
    for (int j = lane; j < pj.y; j += 32) acc += pp[pi.w + j] * S.tile[364 + tcl[pi.w + j]][3];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) S.res[K * 3] = b[4L * m + 3] - acc;
  }
  struct RowSmall {
    float sc0, sc1, sc2, l0, l1, l2;
    float4 bv;
    int lcode;
  };
  auto small = [&](int i) {
    RowSmall q;
    q.sc0 = q.sc1 = q.sc2 = q.l0 = q.l1 = q.l2 = 0.f;
    q.bv = make_float4(0.f, 0.f, 0.f, 0.f);
    q.lcode = 0;
    if (i < nmine) {
      const int4 ri = S.ri[warp + i * NW];
      const int node = ri.x, nl = (ri.w >> 8) & 0xff;
      q.sc0 = vsc[node];
      q.sc1 = vsc[(long)N + node];
      q.sc2 = vsc[2L * N + node];
      if (lane < nl) {
        q.lcode = tcl[ri.z + lane];
        q.l0 = vp[ri.z + lane];
        q.l1 = vp[nql + ri.z + lane];
        q.l2 = vp[2 * nql + ri.z + lane];
      }
      if (lane == 0) q.bv = reinterpret_cast<const float4 *>(b)[node];
    }
    return q;
  };
  RowSmall nxt = small(0);
  for (int i = 0; i < nmine; i++) {
    if (i + SLOTS - 1 < nmine) issue(i + SLOTS - 1);
    cp_async_commit();
    const RowSmall cur = nxt;
    nxt = small(i + 1);
    const int r = warp + i * NW;
    const int4 ri = S.ri[r];
    const int k0 = ri.y, nk = ri.w & 0xff, nl = (ri.w >> 8) & 0xff, tb = ri.w >> 16;
    cp_async_wait<SLOTS - 1>();
    __syncwarp();
    const int sl = i % SLOTS;
    const int qo = k0 & 3;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    for (int j = lane; j < nk; j += 32) {
      const uint4 h = S.h[warp][sl][j];
      const uint32_t e = S.q[warp][sl][qo + j];
      const float *xt = S.tile[tb + (int)(int16_t)(e >> 16)];
      float2 f;
      f = h2f(h.x);
      a0 += f.x * xt[0] + f.y * xt[1];
      f = h2f(h.y);
      a0 += f.x * xt[2];
      a1 += f.y * xt[0];
      f = h2f(h.z);
      a1 += f.x * xt[1] + f.y * xt[2];
      f = h2f(h.w);
      a2 += f.x * xt[0] + f.y * xt[1];
      a2 += h2f(e).x * xt[2];
    }
    a0 *= cur.sc0;
    a1 *= cur.sc1;
    a2 *= cur.sc2;
    if (lane < nl) {
      const float pval = S.tile[tb + cur.lcode][3];
      a0 += cur.l0 * pval;
      a1 += cur.l1 * pval;
      a2 += cur.l2 * pval;
    }
    for (int o = 16; o > 0; o >>= 1) {
      a0 += __shfl_down_sync(0xffffffffu, a0, o);
      a1 += __shfl_down_sync(0xffffffffu, a1, o);
      a2 += __shfl_down_sync(0xffffffffu, a2, o);
    }
    if (lane == 0) {
      S.res[r * 3] = cur.bv.x - a0;
      S.res[r * 3 + 1] = cur.bv.y - a1;
      S.res[r * 3 + 2] = cur.bv.z - a2;
    }
    __syncwarp();  // slot sl is refilled by the copies issued in iteration i + 1
  }
  cp_async_wait<0>();
  __syncthreads();
  patch_solve<float, 3, NT>(S.res, S.red, K, m, g0, vk, pk, dlt, pres_off, omega);
}

// ROWS phase 1 for the streaming levels of the 3D FP32 smoother: persistent warps, each
// owning star rows gw, gw + TW, ... (TW = warps of the grid), whose FP16 records
// (16-byte values, 8-byte {column, value 8}) are copied into a per-warp ring of SLOTS
// shared-memory slots with cp.async, SLOTS-1 rows ahead of the row being computed; the
// row descriptors and the small per-row data (row scales, rhs, pressure couplings) are
// loaded one row ahead into registers.  The bytes in flight per SM then do not depend
// on registers.  The patches' pressure rows follow with direct loads.  Rows have at most
// 125 blocks (the host uses this kernel only then).
#define EXF_RS_MAXB 128  // records per slot (star rows have at most 125 blocks)

template <int NW, int SLOTS>
struct RowStreamSmem {
  uint4 h[NW][SLOTS][EXF_RS_MAXB];
  uint2 c[NW][SLOTS][EXF_RS_MAXB + 2];  // + alignment slack of the 16-byte chunks
};

template <int NT, int SLOTS>
__global__ void __launch_bounds__(NT)
    k_vanka_rows_stream(const int4 *__restrict__ rinfo, int nrows, int gbase, const int4 *__restrict__ pinfo,
                        int npatch, int N, const uint4 *__restrict__ h16, const uint2 *__restrict__ cx,
                        const float *__restrict__ vsc, const int *__restrict__ qq_col,
                        const int *__restrict__ ql_col, long nql, long nqqL, const float *__restrict__ vp,
                        const float *__restrict__ pv, const float *__restrict__ pp, const float *__restrict__ x,
                        const float *__restrict__ b, float *__restrict__ res, long pres_off) {
  constexpr int NW = NT / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RowStreamSmem<NW, SLOTS> &S = *reinterpret_cast<RowStreamSmem<NW, SLOTS> *>(smem_raw);
  EXF_PDL_WAIT();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blockIdx.x * NW + warp;
  const int TW = gridDim.x * NW;
  const int nmine = gw < nrows ? (nrows - gw + TW - 1) / TW : 0;
  const float4 *x4 = reinterpret_cast<const float4 *>(x);
  auto desc = [&](int i) { return i < nmine ? rinfo[gw + (long)i * TW] : make_int4(0, 0, 0, 0); };
  auto issue = [&](int i, int4 ri) {
    const int k0 = ri.y, nk = ri.w & 0xff, sl = i % SLOTS;
    for (int j = lane; j < nk; j += 32) cp_async16(&S.h[warp][sl][j], h16 + k0 + j);
    const int ca = k0 & ~1, cn = ((k0 + nk + 1) & ~1) - ca;  // uint2 records, 16-byte chunks
    for (int j = 2 * lane; j < cn; j += 64) cp_async16(&S.c[warp][sl][j], cx + ca + j);
  };
  struct RowSmall {
    float sc0, sc1, sc2, l0, l1, l2;
    float4 bv;
    int lc;
  };
  auto small = [&](int4 ri, bool ok) {
    RowSmall q;
    q.sc0 = q.sc1 = q.sc2 = q.l0 = q.l1 = q.l2 = 0.f;
    q.bv = make_float4(0.f, 0.f, 0.f, 0.f);
    q.lc = -1;
    if (ok) {
      const int node = ri.x, nl = (ri.w >> 8) & 0xff;
      q.sc0 = vsc[node];
      q.sc1 = vsc[(long)N + node];
      q.sc2 = vsc[2L * N + node];
      if (lane < nl) {
        q.lc = ql_col[ri.z + lane];
        q.l0 = vp[ri.z + lane];
        q.l1 = vp[nql + ri.z + lane];
        q.l2 = vp[2 * nql + ri.z + lane];
      }
      if (lane == 0) q.bv = reinterpret_cast<const float4 *>(b)[node];
    }
    return q;
  };
  // descriptors: d[s] holds row i + s for the rows already issued or about to be
  int4 dcur[SLOTS];
#pragma unroll
  for (int s = 0; s < SLOTS; s++) dcur[s] = desc(s);
#pragma unroll
  for (int s = 0; s < SLOTS - 1; s++) {
    if (s < nmine) issue(s, dcur[s]);
    cp_async_commit();
  }
  // column gathers of row i (from its slot once landed): one row ahead of the products
  auto gather = [&](int i, const int4 &ri, const RowSmall &q, float4 (&xg)[4], float &pv4) {
    const int sl = i % SLOTS, co = ri.y & 1, nk = ri.w & 0xff;
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int j = lane + 32 * u;
      xg[u] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (i < nmine && j < nk) xg[u] = x4[S.c[warp][sl][co + j].x];
    }
    pv4 = (i < nmine && q.lc >= 0) ? x4[q.lc].w : 0.f;
  };
  RowSmall nxt = small(dcur[0], 0 < nmine);
  float4 xg[4], xgn[4];
  float pval = 0.f, pvaln = 0.f;
  cp_async_wait<SLOTS - 2>();
  __syncwarp();
  gather(0, dcur[0], nxt, xg, pval);
  for (int i = 0; i < nmine; i++) {
    const int4 ri = dcur[0];
    if (i + SLOTS - 1 < nmine) issue(i + SLOTS - 1, dcur[SLOTS - 1]);
    cp_async_commit();
#pragma unroll
    for (int s = 0; s < SLOTS - 1; s++) dcur[s] = dcur[s + 1];
    dcur[SLOTS - 1] = desc(i + SLOTS);
    const RowSmall cur = nxt;
    nxt = small(dcur[0], i + 1 < nmine);
    const int nk = ri.w & 0xff, nl = (ri.w >> 8) & 0xff;
    cp_async_wait<SLOTS - 2>();  // rows up to i + 1 have landed
    __syncwarp();
    gather(i + 1, dcur[0], nxt, xgn, pvaln);
    const int sl = i % SLOTS, co = ri.y & 1;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int j = lane + 32 * u;
      if (j < nk) {
        const uint4 h = S.h[warp][sl][j];
        const uint32_t e = S.c[warp][sl][co + j].y;
        const float4 xt = xg[u];
        float2 f;
        f = h2f(h.x);
        a0 += f.x * xt.x + f.y * xt.y;
        f = h2f(h.y);
        a0 += f.x * xt.z;
        a1 += f.y * xt.x;
        f = h2f(h.z);
        a1 += f.x * xt.y + f.y * xt.z;
        f = h2f(h.w);
        a2 += f.x * xt.x + f.y * xt.y;
        a2 += h2f(e).x * xt.z;
      }
    }
    a0 *= cur.sc0;
    a1 *= cur.sc1;
    a2 *= cur.sc2;
    if (cur.lc >= 0) {
      a0 += cur.l0 * pval;
      a1 += cur.l1 * pval;
      a2 += cur.l2 * pval;
    }
    for (int j = 32 + lane; j < nl; j += 32) {  // more than 32 pressure couplings
      const float pv2 = x4[ql_col[ri.z + j]].w;
      a0 += vp[ri.z + j] * pv2;
      a1 += vp[nql + ri.z + j] * pv2;
      a2 += vp[2 * nql + ri.z + j] * pv2;
    }
    for (int o = 16; o > 0; o >>= 1) {
      a0 += __shfl_down_sync(0xffffffffu, a0, o);
      a1 += __shfl_down_sync(0xffffffffu, a1, o);
      a2 += __shfl_down_sync(0xffffffffu, a2, o);
    }
    if (lane == 0) {
      const long g = gw + (long)i * TW;
      res[(gbase + g) * 3] = cur.bv.x - a0;
      res[(gbase + g) * 3 + 1] = cur.bv.y - a1;
      res[(gbase + g) * 3 + 2] = cur.bv.z - a2;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) xg[u] = xgn[u];
    pval = pvaln;
    __syncwarp();  // slot sl is refilled by the copies issued in iteration i + 1
  }
  cp_async_wait<0>();
  // the patches' pressure rows (one warp each, direct loads)
  for (int pr = gw; pr < npatch; pr += TW) {
    const int4 pi = pinfo[2 * pr];
    const int4 pj = pinfo[2 * pr + 1];
    float acc[3] = {0.f, 0.f, 0.f};
    const float one[3] = {};
    const PlanarBlocks<float, 3> pb{qq_col, pv, nqqL};
    patch_row_dot<float, 3, 32, 4, true, 1>(lane, N, pi.z, pj.x, pi.w, pj.y, pb, ql_col, 0, pp, x, acc, one);
    for (int o = 16; o > 0; o >>= 1) acc[0] += __shfl_down_sync(0xffffffffu, acc[0], o);
    if (lane == 0) res[pres_off + pi.x] = b[4L * pi.x + 3] - acc[0];
  }
}

// TILE phase 2: x += corrections of one colour (each star node and patch vertex once)
template <class T, int D, bool I4>
__global__ void k_vanka_apply(const int *__restrict__ vrows, int nr, long gbase, const int *__restrict__ items,
                              int npatch, int N, const T *__restrict__ dlt, long pres_off, T *__restrict__ x) {
  EXF_PDL_WAIT();
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nr) {
    const int n = vrows[i];
#pragma unroll
    for (int a = 0; a < D; a++) x[Lay<I4>::v(a, n, N)] += dlt[(gbase + i) * D + a];
  } else if (i < (long)nr + npatch) {
    const int m = items[i - nr];
    x[Lay<I4>::p(m, N, D)] += dlt[pres_off + m];
  }
}

// BULK phase 1 for the 3D FP32 smoother.  Each star row is stored star-major (sv: row
// after row in sweep order) as one self-contained run of 16-byte records: {row scales,
// node}, {nqq | nql << 8}, the FP16 values 0..7 of each block, the block columns (4 per
// record), the blocks' 9th values (8 per record) and the pressure couplings {vp 0..2,
// column}: 22 bytes per block, so a colour's rows are one contiguous stream.  (Reading the
// columns from qq_col through L2 instead, 18 bytes per block in the stream, was slower:
// 1.16 against 1.07 ms per channel3d fine sweep.)  Persistent CTAs own contiguous row ranges, cut on
// the host into stages of whole rows (at most 32 rows and CAPB records: the schedule,
// {first row, first record} per stage).  One producer warp fills stage buffers with two
// bulk copies (the records and the rows' record offsets) completed on the stage's "full"
// mbarrier, with no global load on its path; NWC consumer warps take the stages' row pairs
// round-robin (16 lanes per row, every column gather of a row issued at once, x gathers
// mostly L1 hits) and release a stage on its "empty" mbarrier.  Each lane visits the
// blocks and couplings of its row in the same order as the ROWS kernel, so both give the
// same sums.  Every wait is bounded: a wait that runs out sets the system's wait flag and
// the kernel leaves once its copies have landed.
#ifndef EXF_WAIT_TRIES
#define EXF_WAIT_TRIES (1 << 22)
#endif

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}
// true once the phase of parity `par` has completed; false after `tries` tries
__device__ __forceinline__ bool mbar_wait(uint64_t *b, unsigned par, int tries = EXF_WAIT_TRIES) {
  for (int t = 0; t < tries; t++) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(b)), "r"(par)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

static int star_pack(exf_sys *s, int lev);

template <int STG, int CAPB>
struct BulkSmem {
  uint4 val[STG][CAPB];   // the stage's star-row records
  long long so[STG][34];  // record offsets of the stage's rows (from an even row index)
  int nrow[STG];          // rows in the stage; 0 ends the stream
  int gfirst[STG];        // colour row index of the stage's first row
  uint64_t full[STG], empty[STG];
};

template <int NWC, int STG, int CAPB, int UNR, int LPR>
__global__ void __launch_bounds__(32 * (NWC + 1), 1)
    k_vanka_rows_bulk(const longlong2 *__restrict__ sched, const int *__restrict__ sched_off, int gbase,
                      const int4 *__restrict__ pinfo, int npatch, int N, const long long *__restrict__ soff,
                      const uint4 *__restrict__ sv, const int *__restrict__ qq_col, const int *__restrict__ ql_col, long nqqL,
                      const float *__restrict__ pv, const float *__restrict__ pp, const float *__restrict__ x,
                      const float *__restrict__ b, float *__restrict__ res, long pres_off,
                      int *__restrict__ wait_flag) {
  constexpr int RPW = 32 / LPR;  // rows per warp pass
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BulkSmem<STG, CAPB> &S = *reinterpret_cast<BulkSmem<STG, CAPB> *>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STG; s++) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], NWC);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (warp == NWC) {
    // producer: stage `it` goes to slot it % STG once its previous use is released.  It
    // reads only the star-major records, offsets and schedule, which no kernel of the
    // sweep writes, so it starts streaming without waiting for the previous kernel
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int e0 = sched_off[blockIdx.x], nst = sched_off[blockIdx.x + 1] - e0 - 1;
    longlong2 win = make_longlong2(0, 0);  // schedule entries e0 + wb + lane
    int wb = -64;
    int it = 0;
    bool ok = true;
    for (;; it++) {
      const int s = it % STG;
      if (it >= STG && !mbar_wait(&S.empty[s], ((it / STG) - 1) & 1)) {
        ok = false;
        break;
      }
      if (it >= nst) {
        if (lane == 0) {
          S.nrow[s] = 0;
          mbar_arrive(&S.full[s]);
        }
        it++;
        break;
      }
      if (it + 1 >= wb + 32) {  // entries it and it + 1 in the window
        wb = it;
        if (wb + lane <= nst) win = sched[e0 + wb + lane];
      }
      const longlong2 st = make_longlong2(__shfl_sync(0xffffffffu, win.x, it - wb),
                                          __shfl_sync(0xffffffffu, win.y, it - wb));
      const longlong2 en = make_longlong2(__shfl_sync(0xffffffffu, win.x, it + 1 - wb),
                                          __shfl_sync(0xffffffffu, win.y, it + 1 - wb));
      if (lane == 0) {
        const int r = (int)st.x, m = (int)(en.x - st.x);
        const unsigned nb = (unsigned)(en.y - st.y);  // records
        const long long ga = ((long long)gbase + r) & ~1LL;
        const unsigned ns = (unsigned)((((long long)gbase + r + m + 1 - ga) + 1) & ~1LL);  // offsets, even
        S.nrow[s] = m;
        S.gfirst[s] = r;
        mbar_arrive_tx(&S.full[s], nb * 16u + ns * 8u);
        if (nb > 0) bulk_g2s(&S.val[s][0], sv + st.y, nb * 16u, &S.full[s]);
        bulk_g2s(&S.so[s][0], soff + ga, ns * 8u, &S.full[s]);
      }
      __syncwarp();
    }
    if (!ok) {
      if (lane == 0) atomicExch(wait_flag, 1);
      // let the copies already issued land before the CTA leaves
      for (int j = max(0, it - STG); j < it; j++) mbar_wait(&S.full[j % STG], (j / STG) & 1);
    }
    return;
  }
  EXF_PDL_WAIT();  // x and b come from the previous kernels
  const float4 *x4 = reinterpret_cast<const float4 *>(x);
  const int half = lane / LPR, hl = lane % LPR;
  // the pressure rows of this CTA's share of the patches, RPW per warp, while the first
  // stages stream in
  const int p0 = (int)((long)blockIdx.x * npatch / gridDim.x);
  const int p1 = (int)((long)(blockIdx.x + 1) * npatch / gridDim.x);
  for (int q2 = p0 + RPW * warp; q2 < p1; q2 += RPW * NWC) {
    const int q = q2 + half;
    float acc[3] = {0.f, 0.f, 0.f};
    int node = 0;
    if (q < p1) {
      const int4 pi = pinfo[2 * q];
      const int4 pj = pinfo[2 * q + 1];
      node = pi.x;
      const float one[3] = {};
      const PlanarBlocks<float, 3> pb{qq_col, pv, nqqL};
      patch_row_dot<float, 3, LPR, 4, true, 1>(hl, N, pi.z, pj.x, pi.w, pj.y, pb, ql_col, 0, pp, x, acc, one);
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) acc[0] += __shfl_down_sync(0xffffffffu, acc[0], o, LPR);
    if (q < p1 && hl == 0) res[pres_off + node] = b[4L * node + 3] - acc[0];
  }
  // consumers: the row groups (RPW rows) of all stages dealt round-robin over the warps
  int cum = 0;  // row groups of the earlier stages, modulo NWC
  for (int it = 0;; it++) {
    const int s = it % STG;
    if (!mbar_wait(&S.full[s], (it / STG) & 1)) {
      if (lane == 0) atomicExch(wait_flag, 1);
      break;
    }
    const int m = S.nrow[s];
    if (m == 0) break;
    const int r = S.gfirst[s];
    const int d = (int)(((long long)gbase + r) & 1LL);
    const long long base = S.so[s][d];
    const int np = (m + RPW - 1) / RPW;
    for (int q = (warp - cum + NWC) % NWC; q < np; q += NWC) {
      const int j = RPW * q + half;
      const bool valid = j < m;
      float acc[3] = {0.f, 0.f, 0.f};
      const int of = valid ? (int)(S.so[s][d + j] - base) : 0;
      const uint4 *vr = &S.val[s][of];  // [0], [1]: header; [2, 2 + nk): blocks; columns; 9th values; couplings
      const uint4 hs = vr[0];
      const int rw = valid ? (int)vr[1].x : 0;
      const int nk = rw & 0xff, nl = (rw >> 8) & 0xff;
      const int c4 = (nk + 3) >> 2;
      const int *qc = reinterpret_cast<const int *>(vr + 2 + nk);  // the row's block columns
      const __half *v8 = reinterpret_cast<const __half *>(vr + 2 + nk + c4);
      const uint4 *cpl = vr + 2 + nk + c4 + ((nk + 7) >> 3);
      float4 bv = make_float4(0.f, 0.f, 0.f, 0.f);
      if (valid && hl == 0) bv = reinterpret_cast<const float4 *>(b)[hs.w];
      // the first two pressure couplings of the lane, gathered before the blocks (added
      // after them, in the same order)
      uint4 cq0 = make_uint4(0u, 0u, 0u, 0u), cq1 = cq0;
      float pq0 = 0.f, pq1 = 0.f;
      if (hl < nl) {
        cq0 = cpl[hl];
        pq0 = x4[(int)cq0.w].w;
      }
      if (hl + LPR < nl) {
        cq1 = cpl[hl + LPR];
        pq1 = x4[(int)cq1.w].w;
      }
      for (int i0 = 0; i0 < nk; i0 += UNR * LPR) {
        int c[UNR];
        float4 xb[UNR];
#pragma unroll
        for (int u = 0; u < UNR; u++) {
          const int i = i0 + u * LPR + hl;
          c[u] = i < nk ? qc[i] : -1;
        }
#pragma unroll
        for (int u = 0; u < UNR; u++) xb[u] = c[u] >= 0 ? x4[c[u]] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int u = 0; u < UNR; u++) {
          const int i = i0 + u * LPR + hl;
          if (c[u] >= 0) {
            const uint4 h = vr[2 + i];
            float v[9];
            float2 f;
            f = h2f(h.x); v[0] = f.x; v[1] = f.y;
            f = h2f(h.y); v[2] = f.x; v[3] = f.y;
            f = h2f(h.z); v[4] = f.x; v[5] = f.y;
            f = h2f(h.w); v[6] = f.x; v[7] = f.y;
            v[8] = __half2float(v8[i]);
            const float xx[3] = {xb[u].x, xb[u].y, xb[u].z};
#pragma unroll
            for (int a = 0; a < 3; a++)
#pragma unroll
              for (int bb = 0; bb < 3; bb++) acc[a] += v[a * 3 + bb] * xx[bb];
          }
        }
      }
      if (valid) {
        acc[0] *= __uint_as_float(hs.x);
        acc[1] *= __uint_as_float(hs.y);
        acc[2] *= __uint_as_float(hs.z);
      }
      if (hl < nl) {  // pressure couplings {vp 0..2, column}
        acc[0] += __uint_as_float(cq0.x) * pq0;
        acc[1] += __uint_as_float(cq0.y) * pq0;
        acc[2] += __uint_as_float(cq0.z) * pq0;
      }
      if (hl + LPR < nl) {
        acc[0] += __uint_as_float(cq1.x) * pq1;
        acc[1] += __uint_as_float(cq1.y) * pq1;
        acc[2] += __uint_as_float(cq1.z) * pq1;
      }
      for (int i = hl + 2 * LPR; i < nl; i += LPR) {  // further couplings
        const uint4 q4 = cpl[i];
        const float pval = x4[(int)q4.w].w;
        acc[0] += __uint_as_float(q4.x) * pval;
        acc[1] += __uint_as_float(q4.y) * pval;
        acc[2] += __uint_as_float(q4.z) * pval;
      }
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) acc[a] += __shfl_down_sync(0xffffffffu, acc[a], o, LPR);
      if (valid && hl == 0) {
        const long g = (long)gbase + r + j;
        res[g * 3] = bv.x - acc[0];
        res[g * 3 + 1] = bv.y - acc[1];
        res[g * 3 + 2] = bv.z - acc[2];
      }
    }
    cum = (cum + np) % NWC;
    __syncwarp();
    if (lane == 0) mbar_arrive(&S.empty[s]);
  }

}

// kernel tuning: levels with many waves of rows stream the matrix (occupancy first),
// small levels are latency-bound (every block of a row in flight at once)
#ifndef EXF_UNR_BIG32
#define EXF_UNR_BIG32 1
#endif
#ifndef EXF_MINB_BIG32
#define EXF_MINB_BIG32 8
#endif
#ifndef EXF_UNR_BIG64
#define EXF_UNR_BIG64 1
#endif
#ifndef EXF_MINB_BIG64
#define EXF_MINB_BIG64 6
#endif
#ifndef EXF_ST_SLOTS
#define EXF_ST_SLOTS 2
#endif
#ifndef EXF_BK_NWC
#define EXF_BK_NWC 23
#endif
#ifndef EXF_BK_STG
#define EXF_BK_STG 4
#endif
#ifndef EXF_BK_CAPB
#define EXF_BK_CAPB 3072
#endif
#ifndef EXF_BK_UNR
#define EXF_BK_UNR 4
#endif
#ifndef EXF_BK_LPR
#define EXF_BK_LPR 16
#endif
#ifndef EXF_AUTO_BULK
#define EXF_AUTO_BULK 1
#endif

// stages of the BULK row kernel: per colour and CTA (grid CTAs, rows split evenly), the
// rows cut greedily into stages of at most 32 rows and capb records, {first row, first
// record} per stage and one closing entry per CTA
static int bulk_schedule(SysLevel &L, int grid, int capb) {
  const std::vector<long long> &so = L.soff_h;
  std::vector<longlong2> e;
  std::vector<int> off;
  L.bsched_coff.assign(L.ncolour, 0);
  for (int c = 0; c < L.ncolour; c++) {
    const int gb = L.vrow_off[c], nr = L.vrow_off[c + 1] - gb;
    L.bsched_coff[c] = (int)off.size();
    for (int bk = 0; bk < grid; bk++) {
      off.push_back((int)e.size());
      const int r0 = (int)((long)bk * nr / grid), r1 = (int)((long)(bk + 1) * nr / grid);
      int r = r0;
      while (r < r1) {
        e.push_back(make_longlong2(r, so[gb + r]));
        int m = 1;
        while (m < 32 && r + m < r1 && so[gb + r + m + 1] - so[gb + r] <= capb) m++;
        r += m;
      }
      e.push_back(make_longlong2(r1, so[gb + r1]));
    }
    off.push_back((int)e.size());
  }
  EXF_TRY(L.bsched.alloc(e.size()));
  EXF_TRY(L.bsched_off.alloc(off.size()));
  EXF_CUDA(cudaMemcpy(L.bsched.p, e.data(), e.size() * sizeof(longlong2), cudaMemcpyHostToDevice));
  EXF_CUDA(cudaMemcpy(L.bsched_off.p, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
  L.bsched_G = grid;
  return EXF_OK;
}

template <class T, int D>
static int vanka_sweep_rows(exf_sys *s, int lev, const exf_mg_params *p, T *x, const T *b) {
  SysLevel &L = s->L[lev];
  constexpr bool I4 = sizeof(T) == 4;
#ifndef EXF_NTS3
#define EXF_NTS3 128
#endif
  constexpr int NTS = D == 3 ? EXF_NTS3 : 64;
  constexpr int SU = D == 3 ? (375 + NTS - 1) / NTS : 1;  // 3D stars: 125 nodes x 3; 2D: 25 x 2 <= 64
  constexpr int LPR = D == 3 ? 32 : 16;
  constexpr int NTR = 256;
  constexpr int UNR_S = sizeof(T) == 4 ? EXF_UNR_BIG32 : EXF_UNR_BIG64;
#ifndef EXF_LPR_BIG32
#define EXF_LPR_BIG32 16
#endif
  constexpr int LPR_S = (D == 3 && sizeof(T) == 4) ? EXF_LPR_BIG32 : LPR;
  constexpr int MINB_S = sizeof(T) == 4 ? EXF_MINB_BIG32 : EXF_MINB_BIG64;
  // 3D FP32 levels of one to four waves: two blocks per lane, 64 registers
#ifndef EXF_UNR_MID32
#define EXF_UNR_MID32 2
#endif
#ifndef EXF_MINB_MID32
#define EXF_MINB_MID32 4
#endif
#ifndef EXF_LPR_MID32
#define EXF_LPR_MID32 32
#endif
#ifndef EXF_UNR_SMALL32
#define EXF_UNR_SMALL32 2
#endif
#ifndef EXF_LPR_SMALL32
#define EXF_LPR_SMALL32 32
#endif
  constexpr int UNR_M = (D == 3 && sizeof(T) == 4) ? EXF_UNR_MID32 : UNR_S;
  constexpr int MINB_M = (D == 3 && sizeof(T) == 4) ? EXF_MINB_MID32 : MINB_S;
  constexpr int LPR_M = (D == 3 && sizeof(T) == 4) ? EXF_LPR_MID32 : LPR;
  constexpr int UNR_L = (D == 3 && sizeof(T) == 4) ? EXF_UNR_SMALL32 : 2;
  constexpr int LPR_L = (D == 3 && sizeof(T) == 4) ? EXF_LPR_SMALL32 : LPR;
  T *res = VK<T>::res(L);
  const long pres_off = (long)L.vrow_off[L.ncolour] * D;
  for (int cc = 0; cc < L.ncolour; cc++) {
    const int c = p->reverse_colours ? L.ncolour - 1 - cc : cc;
    const int n = L.col_off[c + 1] - L.col_off[c];
    if (n == 0) continue;
    const int nr = L.vrow_off[c + 1] - L.vrow_off[c];
    const int4 *pin = L.pinfo.p + 2L * L.col_off[c];
    const long nthr = (long)(nr + n) * LPR;
    const long wave = (long)s->nsm * 2048;  // resident threads of the GPU
    const bool big = nthr > (D == 3 ? 4 : 1) * wave;
    const bool mid = !big && nthr > wave;
    const long nthr_s = (long)(nr + n) * LPR_S;
    // STREAM (selectable, 3D FP32): measured 1.86 ms per channel3d fine sweep against
    // 1.42 ms for the register-pipelined row kernel, so AUTO does not use it
    if constexpr (sizeof(T) == 4 && D == 3) {
      // AUTO: the bulk kernel on the streaming levels (above four waves of rows)
      if (!p->fp32_blocks &&
          (p->vanka_kernel == EXF_VANKA_BULK || (p->vanka_kernel == EXF_VANKA_AUTO && EXF_AUTO_BULK && big))) {
        constexpr int NWC = EXF_BK_NWC, STG = EXF_BK_STG, CAPB = EXF_BK_CAPB, UNR = EXF_BK_UNR,
                      BLPR = EXF_BK_LPR;
        static_assert(CAPB >= 2 + 255 + 64 + 32 + 255,
                      "a stage holds the longest row (header, 255 blocks with columns and 9th values, 255 couplings)");
        using SM = BulkSmem<STG, CAPB>;
        auto kern = k_vanka_rows_bulk<NWC, STG, CAPB, UNR, BLPR>;
        // CTAs per SM, per device (threads driving systems on one device may both resolve
        // it; they store the same value)
        static std::atomic<int> per_sm[64];
        const int dev = s->mesh->device;
        if (dev < 0 || dev >= 64) {
          set_error("device ordinal %d out of range", dev);
          return EXF_ERR_ARG;
        }
        int nper = per_sm[dev].load(std::memory_order_acquire);
        if (nper == 0) {
          EXF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SM)));
          EXF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nper, kern, 32 * (NWC + 1), sizeof(SM)));
          if (nper < 1) {
            set_error("Vanka bulk row kernel does not fit on an SM");
            return EXF_ERR_UNSUPPORTED;
          }
          per_sm[dev].store(nper, std::memory_order_release);
        }
        const int grid = s->nsm * nper;
        if (!L.sv.p || L.bsched_G != grid) {  // first BULK sweep of this level (or a new grid)
          cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
          EXF_CUDA(cudaStreamIsCapturing(s->stream, &cs));
          if (cs != cudaStreamCaptureStatusNone) {
            set_error("the first BULK sweep of level %d cannot run inside a graph capture", lev);
            return EXF_ERR_STATE;
          }
          if (!L.sv.p) EXF_TRY(star_pack(s, lev));
          EXF_TRY(bulk_schedule(L, grid, CAPB));
        }
        EXF_CUDA(launch_pdl(kern, dim3(grid), dim3(32 * (NWC + 1)), sizeof(SM), s->stream,
                            (const longlong2 *)L.bsched.p, (const int *)(L.bsched_off.p + L.bsched_coff[c]),
                            L.vrow_off[c], pin, n, L.N, (const long long *)L.soff.p, (const uint4 *)L.sv.p,
                            (const int *)L.qq_col.p, (const int *)L.ql_col.p, L.nqqL,
                            (const float *)VT<T>::pv(L), (const float *)VT<T>::pp(L), (const float *)x,
                            (const float *)b, (float *)res, pres_off, s->wait_flag.p));
        EXF_CUDA(launch_pdl(k_vanka_solve<T, D, NTS, I4, SU>, dim3(n), dim3(NTS), 0, s->stream, pin, L.N, L.vrows.p,
                            VK<T>::vk(L), VK<T>::pk(L), res, pres_off, x, (T)p->omega));
        EXF_COUNT(2);
        continue;
      }
      if (p->vanka_kernel == EXF_VANKA_STREAM && !p->fp32_blocks) {
        if (!L.tile_ok) {
          set_error("Vanka row streaming: a row of level %d exceeds 125 blocks", lev);
          return EXF_ERR_UNSUPPORTED;
        }
        constexpr int RNT = 256, RSL = 4;
        using SM = RowStreamSmem<RNT / 32, RSL>;
        static bool attr_set[64] = {false};
        const int dev = s->mesh->device;
        if (dev < 0 || dev >= 64) {
          set_error("device ordinal %d out of range", dev);
          return EXF_ERR_ARG;
        }
        if (!attr_set[dev]) {
          EXF_CUDA(cudaFuncSetAttribute(k_vanka_rows_stream<RNT, RSL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sizeof(SM)));
          attr_set[dev] = true;
        }
        int per_sm = 0;
        EXF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_vanka_rows_stream<RNT, RSL>, RNT,
                                                               sizeof(SM)));
        const int grid = s->nsm * std::max(1, per_sm);
        EXF_CUDA(launch_pdl(k_vanka_rows_stream<RNT, RSL>, dim3(grid), dim3(RNT), sizeof(SM), s->stream,
                            (const int4 *)(L.vrinfo.p + L.vrow_off[c]), nr, L.vrow_off[c], pin, n, L.N,
                            (const uint4 *)L.h16.p, (const uint2 *)L.h16cx.p, (const float *)L.vsc.p,
                            (const int *)L.qq_col.p, (const int *)L.ql_col.p, L.nql, L.nqqL,
                            (const float *)VT<T>::vp(L), (const float *)VT<T>::pv(L), (const float *)VT<T>::pp(L),
                            (const float *)x, (const float *)b, (float *)res, pres_off));
        EXF_CUDA(launch_pdl(k_vanka_solve<T, D, NTS, I4, SU>, dim3(n), dim3(NTS), 0, s->stream, pin, L.N, L.vrows.p,
                            VK<T>::vk(L), VK<T>::pk(L), res, pres_off, x, (T)p->omega));
        EXF_COUNT(2);
        continue;
      }
    }
    bool launched = false;
    if constexpr (sizeof(T) == 4) {  // FP32 V-cycle: row-scaled FP16 velocity blocks
      if (!p->fp32_blocks) {
        using VB = Packed16<D>;
        const VB vb{L.qq_col.p, L.h16.p, L.h16cx.p};
        auto kern = big   ? k_vanka_rows<T, D, LPR_S, NTR, I4, UNR_S, MINB_S, VB>
                    : mid ? k_vanka_rows<T, D, LPR_M, NTR, I4, UNR_M, MINB_M, VB>
                          : k_vanka_rows<T, D, LPR_L, NTR, I4, UNR_L, 1, VB>;
        const long nthr_k = big ? nthr_s : (long)(nr + n) * (mid ? LPR_M : LPR_L);
        EXF_CUDA(launch_pdl(kern, dim3(nblk(nthr_k, NTR)), dim3(NTR), 0, s->stream,
                            L.vrinfo.p + L.vrow_off[c], nr, L.vrow_off[c], pin, n, L.N, vb, (const T *)L.vsc.p,
                            L.qq_col.p, L.ql_col.p, L.nql, L.nqqL, VT<T>::vp(L), VT<T>::pv(L), VT<T>::pp(L), x, b,
                            res, pres_off));
        launched = true;
      }
    }
    if (!launched) {  // FP64, or FP32 storage of the blocks in the FP32 V-cycle
      using VB = PlanarBlocks<T, D * D>;
      const VB vb{L.qq_col.p, VT<T>::vv(L), L.nqq};
      auto kern = big ? k_vanka_rows<T, D, LPR, NTR, I4, UNR_S, MINB_S, VB>
                      : k_vanka_rows<T, D, LPR, NTR, I4, UNR_L, 1, VB>;
      EXF_CUDA(launch_pdl(kern, dim3(nblk(nthr, NTR)), dim3(NTR), 0, s->stream, L.vrinfo.p + L.vrow_off[c], nr,
                          L.vrow_off[c], pin, n, L.N, vb, (const T *)nullptr, L.qq_col.p, L.ql_col.p, L.nql, L.nqqL,
                          VT<T>::vp(L), VT<T>::pv(L), VT<T>::pp(L), x, b, res, pres_off));
    }
    EXF_CUDA(launch_pdl(k_vanka_solve<T, D, NTS, I4, SU>, dim3(n), dim3(NTS), 0, s->stream, pin, L.N, L.vrows.p,
                        VK<T>::vk(L), VK<T>::pk(L), res, pres_off, x, (T)p->omega));
    EXF_COUNT(2);
  }
  return EXF_OK;
}

template <class T, int D>
static int vanka_sweep_tile(exf_sys *s, int lev, const exf_mg_params *p, T *x, const T *b) {
  SysLevel &L = s->L[lev];
  constexpr bool I4 = sizeof(T) == 4;
  constexpr int NT = D == 3 ? 256 : 64;
  constexpr int LPR = D == 3 ? 32 : 8;
  constexpr int UNR = sizeof(T) == 4 ? 4 : 1;
  constexpr int SNT = 256, SLOTS = EXF_ST_SLOTS;
  T *dlt = VK<T>::res(L);
  const long pres_off = (long)L.vrow_off[L.ncolour] * D;
  if constexpr (sizeof(T) == 4 && D == 3) {
    // dynamic shared memory above 48 KB: opt in once per device
    static bool attr_set[64] = {false};
    const int dev = s->mesh->device;
    if (dev < 0 || dev >= 64) {
      set_error("device ordinal %d out of range", dev);
      return EXF_ERR_ARG;
    }
    if (!attr_set[dev]) {
      EXF_CUDA(cudaFuncSetAttribute(k_vanka_stream<SNT, SLOTS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sizeof(StreamSmem<SNT, SLOTS>)));
      attr_set[dev] = true;
    }
  }
  for (int cc = 0; cc < L.ncolour; cc++) {
    const int c = p->reverse_colours ? L.ncolour - 1 - cc : cc;
    const int n = L.col_off[c + 1] - L.col_off[c];
    if (n == 0) continue;
    const int nr = L.vrow_off[c + 1] - L.vrow_off[c];
    const int4 *pin = L.pinfo.p + 2L * L.col_off[c];
    if constexpr (sizeof(T) == 4 && D == 3) {
      EXF_CUDA(launch_pdl(k_vanka_stream<SNT, SLOTS>, dim3(n), dim3(SNT), sizeof(StreamSmem<SNT, SLOTS>), s->stream,
                          pin, (const int4 *)L.vrinfo.p, L.N, L.Ll[0], L.Ll[1], L.Ll[2], (const int *)L.latnode.p,
                          (const uint4 *)L.h16.p, (const uint32_t *)L.h16qc.p, (const float *)L.vsc.p,
                          (const int16_t *)L.tcq.p, (const int16_t *)L.tcl.p, L.nql, L.nqqL,
                          (const float *)VT<T>::vp(L), (const float *)VT<T>::pv(L), (const float *)VT<T>::pp(L),
                          (const float *)VK<T>::vk(L), (const float *)VK<T>::pk(L), (const float *)x,
                          (const float *)b, (float *)dlt, pres_off, (float)p->omega));
    } else if constexpr (sizeof(T) == 4) {
      using BL = TileBlocks16<D>;
      const BL bl{L.h16.p, L.h16qc.p, L.tcq.p};
      EXF_CUDA(launch_pdl(k_vanka_tile<T, D, NT, LPR, UNR, I4, BL>, dim3(n), dim3(NT), 0, s->stream, pin,
                          (const int4 *)L.vrinfo.p, L.N, L.NL, L.Ll[0], L.Ll[1], L.Ll[2], (const int *)L.latnode.p,
                          bl, (const T *)L.vsc.p, (const int16_t *)L.tcq.p, (const int16_t *)L.tcl.p, L.nql, L.nqqL,
                          VT<T>::vp(L), VT<T>::pv(L), VT<T>::pp(L), VK<T>::vk(L), VK<T>::pk(L), x, b, dlt, pres_off,
                          (T)p->omega));
    } else {
      using BL = TileBlocksPlanar<T, D * D>;
      const BL bl{VT<T>::vv(L), L.nqq, L.tcq.p};
      EXF_CUDA(launch_pdl(k_vanka_tile<T, D, NT, LPR, UNR, I4, BL>, dim3(n), dim3(NT), 0, s->stream, pin,
                          (const int4 *)L.vrinfo.p, L.N, L.NL, L.Ll[0], L.Ll[1], L.Ll[2], (const int *)L.latnode.p,
                          bl, (const T *)nullptr, (const int16_t *)L.tcq.p, (const int16_t *)L.tcl.p, L.nql, L.nqqL,
                          VT<T>::vp(L), VT<T>::pv(L), VT<T>::pp(L), VK<T>::vk(L), VK<T>::pk(L), x, b, dlt, pres_off,
                          (T)p->omega));
    }
    EXF_CUDA(launch_pdl(k_vanka_apply<T, D, I4>, dim3(nblk((long)nr + n, 256)), dim3(256), 0, s->stream,
                        L.vrows.p + L.vrow_off[c], nr, (long)L.vrow_off[c], L.col_items.p + L.col_off[c], n, L.N,
                        (const T *)dlt, pres_off, x));
    EXF_COUNT(2);
  }
  return EXF_OK;
}

// AUTO runs the ROWS pair: on the channel, cavity and Boussinesq hierarchies it was
// measured at least as fast as the tile kernels on every level
template <class T, int D>
static int vanka_sweep(exf_sys *s, int lev, const exf_mg_params *p, T *x, const T *b) {
  SysLevel &L = s->L[lev];
  // FP32 blocks in the FP32 V-cycle are read by the row kernel only
  if (p->vanka_kernel == EXF_VANKA_TILE && !(sizeof(T) == 4 && p->fp32_blocks)) {
    if (!L.tile_ok) {
      set_error("Vanka tile kernel: a star or row of level %d exceeds the 5^d-node patch", lev);
      return EXF_ERR_UNSUPPORTED;
    }
    return vanka_sweep_tile<T, D>(s, lev, p, x, b);
  }
  return vanka_sweep_rows<T, D>(s, lev, p, x, b);
}

// FP16 copy of the velocity blocks for the FP32 smoother: row (n, a) is scaled by its
// largest magnitude over every block and column, so each stored entry lies in [-1, 1]
// (no overflow; entries below 2^-14 of the row maximum lose relative precision, which
// bounds their absolute error by 2^-25 of the row maximum).  Records as read by
// Packed16 and TileBlocks16 / k_vanka_stream.  One warp per node.
template <int D>
__global__ void k_pack16(int N, const int *__restrict__ qq_ptr, const int *__restrict__ qq_col,
                         const int16_t *__restrict__ tcq, long nqq, const double *__restrict__ vv,
                         void *__restrict__ h16, uint2 *__restrict__ cx, uint32_t *__restrict__ qc,
                         float *__restrict__ vsc) {
  const int n = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (n >= N) return;  // uniform per warp
  const int k0 = qq_ptr[n], k1 = qq_ptr[n + 1];
  double sc[D];
  for (int a = 0; a < D; a++) {
    double mx = 0.;
    for (int k = k0 + lane; k < k1; k += 32)
      for (int bb = 0; bb < D; bb++) mx = fmax(mx, fabs(vv[(long)(a * D + bb) * nqq + k]));
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    sc[a] = (mx > 0. && mx < 1e300) ? mx : 1.;
    if (lane == 0) vsc[(long)a * N + n] = (float)sc[a];
  }
  for (int k = k0 + lane; k < k1; k += 32) {
    unsigned short hv[D * D + 1];
    for (int q = 0; q < D * D; q++) {
      const __half hq = __float2half_rn((float)(vv[(long)q * nqq + k] / sc[q / D]));
      memcpy(&hv[q], &hq, 2);
    }
    hv[D * D] = 0;
    unsigned w[(D * D + 1) / 2];
    for (int i = 0; i < (D * D + 1) / 2; i++) w[i] = (unsigned)hv[2 * i] | ((unsigned)hv[2 * i + 1] << 16);
    if constexpr (D == 3) {
      reinterpret_cast<uint4 *>(h16)[k] = make_uint4(w[0], w[1], w[2], w[3]);
      cx[k] = make_uint2((unsigned)qq_col[k], w[4]);
      qc[k] = (w[4] & 0xffffu) | ((uint32_t)(uint16_t)tcq[k] << 16);
    } else {
      reinterpret_cast<uint2 *>(h16)[k] = make_uint2(w[0], w[1]);
    }
  }
}

// star-major copy of each 3D star row (one warp per row): record 0 is the header
// {vsc 0..2, node} / {nqq | nql << 8}, records 1..nqq the FP16 blocks, then one record per
// pressure coupling {vp 0..2 (FP32), column}; the pad record is zero
__global__ void k_pack_star(int nrows, const int4 *__restrict__ rinfo, const long long *__restrict__ soff, int N,
                            const uint4 *__restrict__ h16, const uint2 *__restrict__ cx,
                            const float *__restrict__ vsc, const int *__restrict__ ql_col,
                            const float *__restrict__ vp, long nql, uint4 *__restrict__ sv) {
  const long g = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= nrows) return;
  const int4 ri = rinfo[g];
  const int node = ri.x, k0 = ri.y, l0 = ri.z, nk = ri.w & 0xff, nl = (ri.w >> 8) & 0xff;
  const int c4 = (nk + 3) >> 2, n8 = (nk + 7) >> 3;
  const long long o = soff[g];
  const int w = (int)(soff[g + 1] - o);
  for (int i = lane; i < w; i += 32) {
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (i == 0) {
      v = make_uint4(__float_as_uint(vsc[node]), __float_as_uint(vsc[(long)N + node]),
                     __float_as_uint(vsc[2L * N + node]), (unsigned)node);
    } else if (i == 1) {
      v = make_uint4((unsigned)(nk | (nl << 8)), 0u, 0u, 0u);
    } else if (i < 2 + nk) {
      v = h16[k0 + i - 2];
    } else if (i < 2 + nk + c4) {  // columns of blocks 4 (i - 2 - nk) ..
      const int b0 = 4 * (i - 2 - nk);
      unsigned c[4];
#pragma unroll
      for (int t = 0; t < 4; t++) c[t] = b0 + t < nk ? cx[k0 + b0 + t].x : 0u;
      v = make_uint4(c[0], c[1], c[2], c[3]);
    } else if (i < 2 + nk + c4 + n8) {  // 9th values of blocks 8 (i - 2 - nk - c4) ..
      const int b0 = 8 * (i - 2 - nk - c4);
      unsigned h[8];
#pragma unroll
      for (int t = 0; t < 8; t++) h[t] = b0 + t < nk ? (cx[k0 + b0 + t].y & 0xffffu) : 0u;
      v = make_uint4(h[0] | (h[1] << 16), h[2] | (h[3] << 16), h[4] | (h[5] << 16), h[6] | (h[7] << 16));
    } else {
      const long q = l0 + i - 2 - nk - c4 - n8;
      v = make_uint4(__float_as_uint(vp[q]), __float_as_uint(vp[nql + q]), __float_as_uint(vp[2 * nql + q]),
                     (unsigned)ql_col[q]);
    }
    sv[o + i] = v;
  }
}

static int star_pack(exf_sys *s, int lev) {
  SysLevel &L = s->L[lev];
  if (!L.soff.p || !L.h16.p || !L.A32.vp.p) {
    set_error("star-major records need the 3D FP16 blocks of level %d", lev);
    return EXF_ERR_STATE;
  }
  EXF_TRY(L.sv.ensure((size_t)L.nstar));
  const int nrows = L.vrow_off[L.ncolour];
  if (nrows > 0)
    k_pack_star<<<nblk((long)nrows * 32, 256), 256, 0, s->stream>>>(
        nrows, L.vrinfo.p, L.soff.p, L.N, L.h16.p, L.h16cx.p, L.vsc.p, L.ql_col.p, L.A32.vp.p, L.nql, L.sv.p);
  EXF_CUDA(cudaGetLastError());
  return EXF_OK;
}

int vanka_prep(exf_sys *s, int lev) {
  if (s->kind != EXF_KIND_NS) return EXF_OK;
  SysLevel &L = s->L[lev];
  if (s->dim == 2)
    k_pack16<2><<<nblk(L.N, 8), 256, 0, s->stream>>>(L.N, L.qq_ptr.p, L.qq_col.p, L.tcq.p, L.nqq, L.A.vv.p,
                                                      L.h16.p, nullptr, nullptr, L.vsc.p);
  else
    k_pack16<3><<<nblk(L.N, 8), 256, 0, s->stream>>>(L.N, L.qq_ptr.p, L.qq_col.p, L.tcq.p, L.nqq, L.A.vv.p,
                                                      L.h16.p, L.h16cx.p, L.h16qc.p, L.vsc.p);
  EXF_LAUNCH_CHECK();
  EXF_COUNT(1);
  if (L.sv.p) EXF_TRY(star_pack(s, lev));  // the BULK smoother's copy is in use: refresh it
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

// one CTA waits, bounded, on an mbarrier phase that nothing completes: the wait runs out,
// sets the system's wait flag and the kernel returns (exercises the status path of every
// bounded wait without a fault)
__global__ void k_wait_probe(int tries, int *wait_flag) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(&bar, 0u, tries)) atomicExch(wait_flag, 1);
}

int wait_probe(exf_sys *s) {
  k_wait_probe<<<1, 32, 0, s->stream>>>(1 << 14, s->wait_flag.p);
  EXF_LAUNCH_CHECK();
  EXF_COUNT(1);
  return device_wait_status(s);
}

int device_wait_status(exf_sys *s) {
  int flag = 0;
  EXF_CUDA(cudaMemcpyAsync(&flag, s->wait_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  if (flag) {
    EXF_CUDA(cudaMemsetAsync(s->wait_flag.p, 0, sizeof(int), s->stream));
    EXF_CUDA(cudaStreamSynchronize(s->stream));
    set_error("a bounded wait of the Vanka bulk row kernel ran out");
    return EXF_ERR_CUDA;
  }
  return EXF_OK;
}

template <class T>
int smooth(exf_sys *s, int lev, const exf_mg_params *p, int nsweeps, T *x, const T *b) {
  if (p->smoother == EXF_SMOOTH_GMRES_ILU) {  // one level-solver call of nsweeps iterations
    if constexpr (sizeof(T) == 8) {
      return gmres_smooth(s, lev, p->eps, nsweeps, x, b, nullptr);
    } else {
      set_error("GMRES + ILU smoothing runs in FP64 precision only");
      return EXF_ERR_UNSUPPORTED;
    }
  }
  for (int it = 0; it < nsweeps; it++) {
    if (s->nv1 == 0) {  // scalar systems (T, kappa, omega)
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
// In-place Gauss-Jordan inversion with partial pivoting, once per assembly: blocked (a
// single-CTA panel of 16 pivots, then one rank-16 update) where the panel fits shared
// memory, otherwise ONE cooperative kernel with a grid-wide barrier per pivot.  Pivot rows are not swapped:
// step k pivots on the largest |a_ik| among unused rows p_k, which leaves
// W[p_k][j] = A0^{-1}[k][p_j]; the extraction kernel undoes the permutation.  Each coarse
// solve is then one dense GEMV in FP64.  Pressure-gauge rows become identity rows in the
// factored copy (the enclosed-flow pressure level is otherwise free).  The pivot search
// merges keys of the magnitude's top 44 bits and the row (smallest row among equal keys)
// with atomicMax, so the factorisation is deterministic.
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

// Pivot key: the top 44 bits of |a| (non-negative doubles order as unsigned integers)
// above the inverted row index, so the largest magnitude wins and, among magnitudes equal
// in those bits, the smallest row; 0 = no candidate.  Rows below 2^20.
__device__ __forceinline__ unsigned long long piv_key(double a, int i) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(a));
  return ((b >> 20) << 20) | (unsigned long long)(0xFFFFF - i);
}

// block maximum of the keys, then one atomicMax per block on *dst
template <int NT>
__device__ __forceinline__ void block_key_max(unsigned long long v, unsigned long long *sk,
                                              unsigned long long *dst) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v2 = __shfl_down_sync(0xffffffffu, v, o);
    v = v2 > v ? v2 : v;
  }
  if ((threadIdx.x & 31) == 0) sk[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long m = 0;
    for (int w = 0; w < NT / 32; w++) m = sk[w] > m ? sk[w] : m;
    if (m) atomicMax(dst, m);
  }
  __syncthreads();
}

// Step k reads the iterate from Wc and writes the next one to Wn (the two swap every
// step), so every block can read pivot row p and column k while others write: one
// grid-wide barrier per pivot.  The pivot row p of step k comes from key[k], merged by
// one atomicMax per block during step k-1 over the candidates of column k (unused rows);
// rows are distributed over blocks, columns over threads.
template <int NT>
__global__ void __launch_bounds__(NT)
    k_gj_coop(double *__restrict__ W0, double *__restrict__ W1, int n, int *__restrict__ pivrow,
              unsigned long long *__restrict__ key, int *__restrict__ used, int *__restrict__ bad) {
  namespace cg = cooperative_groups;
  cg::grid_group grid = cg::this_grid();
  __shared__ unsigned long long sk[NT / 32];
  const long gt = (long)blockIdx.x * NT + threadIdx.x;
  const long nth = (long)gridDim.x * NT;
  {
    unsigned long long v = 0;
    for (long i = gt; i < n; i += nth) {
      const unsigned long long c = piv_key(W0[i * n], (int)i);
      v = c > v ? c : v;
    }
    block_key_max<NT>(v, sk, &key[0]);
  }
  grid.sync();
  for (int k = 0; k < n; k++) {
    const double *__restrict__ Wc = (k & 1) ? W1 : W0;
    double *__restrict__ Wn = (k & 1) ? W0 : W1;
    const unsigned long long kk = __ldcg(&key[k]);
    if (kk == 0) {  // no candidate row left: singular (uniform across the grid)
      if (gt == 0) *bad = 1;
      return;
    }
    const int p = 0xFFFFF - (int)(kk & 0xFFFFFull);
    const double *rowp = Wc + (long)p * n;
    const double piv = rowp[k];
    const double inv = piv != 0. ? 1. / piv : 0.;
    if (gt == 0) {
      pivrow[k] = p;
      used[p] = 1;
      if (piv == 0.) *bad = 1;
    }
    unsigned long long best = 0;
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
      const double *Wi = Wc + (long)i * n;
      double *Oi = Wn + (long)i * n;
      const double ci = Wi[k];
      const bool cand = i != p && !used[i];
      for (int j0 = threadIdx.x; j0 < n; j0 += 4 * NT) {
        double w[4], r[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int j = j0 + u * NT;
          w[u] = r[u] = 0.;
          if (j < n) {
            w[u] = Wi[j];
            r[u] = rowp[j];
          }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int j = j0 + u * NT;
          if (j < n) {
            double a;
            if (i == p) a = (j == k) ? inv : r[u] * inv;
            else if (j == k) a = -ci * inv;
            else a = w[u] - ci * r[u] * inv;
            Oi[j] = a;
            if (j == k + 1 && cand) {
              const unsigned long long c = piv_key(a, i);
              best = c > best ? c : best;
            }
          }
        }
      }
    }
    if (k + 1 < n) block_key_max<NT>(best, sk, &key[k + 1]);
    grid.sync();
  }
}

// ---- blocked Gauss-Jordan: NB pivots per block.  The NB steps of a block change every
// column outside the block j by W[:, j] += (H - E_P) W[P, j], where P are the block's pivot
// rows, W[P, j] their values before the block, E_P the unit columns e_{p_t} and H the
// block's own columns after its NB steps (each step k is W <- (I + g_k e_{p_k}^T) W, and
// such products stay of the form I + (H - E_P) E_P^T).  One CTA factors the n x NB panel
// with the same pivot rule as k_gj_coop; a grid-wide kernel then applies the rank-NB
// change to the other columns.
//
// Every row of the panel belongs to one thread, which searches, eliminates and (as the
// pivot row) scales it.  Per pivot: the warps' candidate keys -> barrier -> every warp
// reduces the keys itself; the pivot row's owner scales its row and publishes the scaled
// copy -> barrier -> every thread eliminates its rows against the published copy.  (A
// one-barrier form that left the pivot row unscaled for the other threads and scaled it
// one step later gave wrong, run-dependent factors on B200 once a thread held two rows;
// the published copy with its own barrier is correct at every size.)

// R[t][j] = W[p_t][j]: the block's pivot rows before the block, for the columns outside
// the block (the block's own columns of W may already hold H); CH loads in flight per
// thread
template <int NT, int CH>
__device__ __forceinline__ void gj_copy_pivot_rows(const double *__restrict__ W, int n, int nb, const int *spiv,
                                                   double *__restrict__ R) {
  const long tot = (long)nb * n;
  for (long q0 = threadIdx.x; q0 < tot; q0 += (long)CH * NT) {
    double v[CH];
#pragma unroll
    for (int c = 0; c < CH; c++) {
      const long q = q0 + (long)c * NT;
      v[c] = q < tot ? W[(long)spiv[q / n] * n + q % n] : 0.;
    }
#pragma unroll
    for (int c = 0; c < CH; c++) {
      const long q = q0 + (long)c * NT;
      if (q < tot) R[q] = v[c];
    }
  }
}

// the panel in registers: thread tid holds rows tid + r * NT (r < RPT), n <= RPT * NT
template <int NB, int NT, int RPT>
__global__ void __launch_bounds__(NT, 1)
    k_gj_panel_reg(double *__restrict__ W, int n, int k0, int nb, int *__restrict__ pivrow, int *__restrict__ used,
                   double *__restrict__ Hm, double *__restrict__ R, int *__restrict__ bad) {
  __shared__ unsigned long long sk[2][NT / 32];
  __shared__ double srs[2][NB];
  __shared__ int spiv[NB];
  const int tid = threadIdx.x, lane = tid & 31;
  double a[RPT][NB];
  unsigned ub = 0;  // used (or absent) rows of this thread
#pragma unroll
  for (int r = 0; r < RPT; r++) {
    const int i = tid + r * NT;
#pragma unroll
    for (int u = 0; u < NB; u++) a[r][u] = (i < n && u < nb) ? W[(long)i * n + k0 + u] : 0.;
    if (i >= n || used[i]) ub |= 1u << r;
  }
#pragma unroll
  for (int t = 0; t < NB; t++) {
    if (t >= nb) break;
    unsigned long long v = 0;
#pragma unroll
    for (int r = 0; r < RPT; r++)
      if (!((ub >> r) & 1u)) {
        const unsigned long long c = piv_key(a[r][t], tid + r * NT);
        v = c > v ? c : v;
      }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long v2 = __shfl_xor_sync(0xffffffffu, v, o);
      v = v2 > v ? v2 : v;
    }
    if (lane == 0) sk[t & 1][tid >> 5] = v;
    __syncthreads();
    unsigned long long m = lane < NT / 32 ? sk[t & 1][lane] : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long m2 = __shfl_xor_sync(0xffffffffu, m, o);
      m = m2 > m ? m2 : m;
    }
    if (m == 0) {  // no candidate row left: singular (the same branch in every thread)
      if (tid == 0) *bad = 1;
      return;
    }
    const int p = 0xFFFFF - (int)(m & 0xFFFFFull);
    if (p % NT == tid) {
      const int r0 = p / NT;
#pragma unroll
      for (int r = 0; r < RPT; r++)
        if (r == r0) {
          const double piv = a[r][t];
          const double inv = piv != 0. ? 1. / piv : 0.;
#pragma unroll
          for (int u = 0; u < NB; u++) {
            a[r][u] = u == t ? inv : a[r][u] * inv;
            srs[t & 1][u] = a[r][u];
          }
          if (piv == 0.) *bad = 1;
        }
      ub |= 1u << r0;
      spiv[t] = p;
    }
    __syncthreads();
    const double inv = srs[t & 1][t];
#pragma unroll
    for (int r = 0; r < RPT; r++) {
      const int i = tid + r * NT;
      if (i < n && i != p) {
        const double ci = a[r][t];
#pragma unroll
        for (int u = 0; u < NB; u++) a[r][u] = u == t ? -ci * inv : a[r][u] - ci * srs[t & 1][u];
      }
    }
  }
  __syncthreads();
  if (tid < nb) pivrow[k0 + tid] = spiv[tid];
#pragma unroll
  for (int r = 0; r < RPT; r++) {
    const int i = tid + r * NT;
    if (i < n) {
      used[i] = (ub >> r) & 1u;
#pragma unroll
      for (int u = 0; u < NB; u++)
        if (u < nb) {
          W[(long)i * n + k0 + u] = a[r][u];
          Hm[(long)u * n + i] = a[r][u] - (i == spiv[u] ? 1. : 0.);
        }
    }
  }
  gj_copy_pivot_rows<NT, 16>(W, n, nb, spiv, R);
}

// the panel in shared memory ([NB][n], a warp's rows in consecutive words), for levels
// whose rows exceed RPT * NT of the register form
template <int NB, int NT>
__global__ void __launch_bounds__(NT, 1)
    k_gj_panel(double *__restrict__ W, int n, int k0, int nb, int *__restrict__ pivrow, int *__restrict__ used,
               double *__restrict__ Hm, double *__restrict__ R, int *__restrict__ bad) {
  extern __shared__ __align__(16) double sp[];  // [NB][n] panel, then n used flags (bytes)
  unsigned char *su = reinterpret_cast<unsigned char *>(sp + (size_t)NB * n);
  __shared__ unsigned long long sk[2][NT / 32];
  __shared__ double srs[2][NB];
  __shared__ int spiv[NB];
  const int tid = threadIdx.x, lane = tid & 31;
  for (long q = tid; q < (long)n * NB; q += NT) {
    const int i = (int)(q / NB), t = (int)(q % NB);
    sp[(long)t * n + i] = t < nb ? W[(long)i * n + k0 + t] : 0.;
  }
  for (int i = tid; i < n; i += NT) su[i] = (unsigned char)used[i];
  __syncthreads();
  for (int t = 0; t < nb; t++) {
    unsigned long long v = 0;
    for (int i = tid; i < n; i += NT)
      if (!su[i]) {
        const unsigned long long c = piv_key(sp[(long)t * n + i], i);
        v = c > v ? c : v;
      }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long v2 = __shfl_xor_sync(0xffffffffu, v, o);
      v = v2 > v ? v2 : v;
    }
    if (lane == 0) sk[t & 1][tid >> 5] = v;
    __syncthreads();
    unsigned long long m = lane < NT / 32 ? sk[t & 1][lane] : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long m2 = __shfl_xor_sync(0xffffffffu, m, o);
      m = m2 > m ? m2 : m;
    }
    if (m == 0) {
      if (tid == 0) *bad = 1;
      return;
    }
    const int p = 0xFFFFF - (int)(m & 0xFFFFFull);
    if (p % NT == tid) {
      const double piv = sp[(long)t * n + p];
      const double inv = piv != 0. ? 1. / piv : 0.;
      for (int u = 0; u < NB; u++) {
        const double r = u == t ? inv : sp[(long)u * n + p] * inv;
        srs[t & 1][u] = r;
        sp[(long)u * n + p] = r;
      }
      su[p] = 1;
      spiv[t] = p;
      if (piv == 0.) *bad = 1;
    }
    __syncthreads();
    const double inv = srs[t & 1][t];
    for (int i = tid; i < n; i += NT) {
      if (i == p) continue;
      const double ci = sp[(long)t * n + i];
#pragma unroll
      for (int u = 0; u < NB; u++) {
        double &w = sp[(long)u * n + i];
        w = u == t ? -ci * inv : w - ci * srs[t & 1][u];
      }
    }
  }
  __syncthreads();
  if (tid < nb) pivrow[k0 + tid] = spiv[tid];
  for (int i = tid; i < n; i += NT) used[i] = su[i];
  for (long q = tid; q < (long)n * NB; q += NT) {
    const int i = (int)(q / NB), t = (int)(q % NB);
    if (t < nb) {
      const double h = sp[(long)t * n + i];
      W[(long)i * n + k0 + t] = h;
      Hm[(long)t * n + i] = h - (i == spiv[t] ? 1. : 0.);
    }
  }
  gj_copy_pivot_rows<NT, 4>(W, n, nb, spiv, R);
}

// W[i, j] += sum_t Hm[t][i] R[t][j] (Hm = H - E_P) for every column j outside the block:
// a rank-NB update in 64 x 64 tiles, the tile's Hm and R slices staged in shared memory,
// a 4 x 4 register tile per thread; each entry sums its NB products in order t = 0, 1, ..
template <int NB>
__global__ void __launch_bounds__(256)
    k_gj_update(double *__restrict__ W, int n, int k0, int nb, const double *__restrict__ Hm,
                const double *__restrict__ R) {
  __shared__ __align__(16) double sh[NB][64];
  __shared__ __align__(16) double sr[NB][64];
  const int tid = threadIdx.x;
  const int bi = blockIdx.y * 64, bj = blockIdx.x * 64;
  for (int q = tid; q < NB * 64; q += 256) {
    const int t = q / 64, c = q % 64;
    sh[t][c] = (t < nb && bi + c < n) ? Hm[(long)t * n + bi + c] : 0.;
    sr[t][c] = (t < nb && bj + c < n) ? R[(long)t * n + bj + c] : 0.;
  }
  __syncthreads();
  const int ti = (tid >> 4) * 4, tj = (tid & 15) * 4;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int i = bi + ti + a, j = bj + tj + c;
      acc[a][c] = (i < n && j < n) ? W[(long)i * n + j] : 0.;
    }
#pragma unroll
  for (int t = 0; t < NB; t++) {
    if (t < nb) {
      const double2 h0 = *reinterpret_cast<const double2 *>(&sh[t][ti]);
      const double2 h1 = *reinterpret_cast<const double2 *>(&sh[t][ti + 2]);
      const double2 r0 = *reinterpret_cast<const double2 *>(&sr[t][tj]);
      const double2 r1 = *reinterpret_cast<const double2 *>(&sr[t][tj + 2]);
      const double h[4] = {h0.x, h0.y, h1.x, h1.y}, r[4] = {r0.x, r0.y, r1.x, r1.y};
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[a][c] += h[a] * r[c];
    }
  }
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int i = bi + ti + a, j = bj + tj + c;
      if (i < n && j < n && (j < k0 || j >= k0 + nb)) W[(long)i * n + j] = acc[a][c];
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
  #ifndef EXF_GJ_NT
#define EXF_GJ_NT 512
#endif
  constexpr int NT = EXF_GJ_NT;
  if (n >= 0xFFFFF) {
    set_error("coarsest level of %d DOFs exceeds the direct solver's %d", n, 0xFFFFF - 1);
    return EXF_ERR_UNSUPPORTED;
  }
  EXF_TRY(s->coarse_vals.ensure(L.nnz));
  EXF_TRY(s->coarse_work.ensure((size_t)n * n));
  EXF_TRY(s->coarse_work2.ensure(std::max((size_t)n * n, (size_t)n * 32)));  // also the blocked form's H, R
  EXF_TRY(s->coarse_piv.ensure(n));
  EXF_TRY(s->coarse_used.ensure(n));
  EXF_TRY(s->coarse_bad.ensure(1));
  EXF_TRY(s->coarse_key.ensure((size_t)n + 1));
  DBuf<int> &pivrow = s->coarse_piv, &used = s->coarse_used, &bad = s->coarse_bad;
  DBuf<unsigned long long> &key = s->coarse_key;
  EXF_TRY(used.zero(st));
  EXF_TRY(bad.zero(st));
  EXF_TRY(key.zero(st));
  EXF_TRY(pivrow.zero(st));  // every entry a valid row, even after a singular pivot
  EXF_TRY(csr_values(s, 0, s->coarse_vals.p));
  double *W = s->coarse_work.p;
  k_dense_from_csr<<<n, 128, 0, st>>>(L.csr_ptr.p, L.csr_col.p, s->coarse_vals.p, n, W);
  k_gauge_rows<<<n, 128, 0, st>>>(W, n, s->gmask0.p);
  EXF_LAUNCH_CHECK();
  int dev = 0, nsm = 0, per_sm = 0;
  EXF_CUDA(cudaGetDevice(&dev));
  EXF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  EXF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gj_coop<NT>, NT, 0));
  if (per_sm < 1) {
    set_error("cooperative factorisation kernel does not fit on an SM");
    return EXF_ERR_CUDA;
  }
#ifndef EXF_GJ_BLOCKS_PER_SM
#define EXF_GJ_BLOCKS_PER_SM 2
#endif
  const int grid = std::max(1, std::min(n, nsm * std::min(per_sm, EXF_GJ_BLOCKS_PER_SM)));  // rows over blocks
  double *W1p = s->coarse_work2.p;
  const double *Wfinal = W;
  // blocked form while the n x NB panel fits one CTA's shared memory
  constexpr int GNB = 16, GNT = 1024;
  const size_t psm = (size_t)n * GNB * sizeof(double) + (((size_t)n + 15) & ~(size_t)15);
  int smax = 0;
  EXF_CUDA(cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (psm + 1024 <= (size_t)smax) {
    // one value for every caller (the attribute is per function, shared by the threads
    // that factor systems of different sizes)
    EXF_CUDA(cudaFuncSetAttribute(k_gj_panel<GNB, GNT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax - 1024));
    // H - E_P (NB x n) and the block's pivot rows (NB x n) in the second work buffer
    double *Hb = W1p, *Rb = W1p + (size_t)n * GNB;
    const dim3 ugrid((unsigned)((n + 63) / 64), (unsigned)((n + 63) / 64));
    constexpr int RNT = 512, RPT = 3;
    for (int k0 = 0; k0 < n; k0 += GNB) {
      const int nb = std::min(GNB, n - k0);
      if (n <= RNT * RPT)
        k_gj_panel_reg<GNB, RNT, RPT><<<1, RNT, 0, st>>>(W, n, k0, nb, pivrow.p, used.p, Hb, Rb, bad.p);
      else
        k_gj_panel<GNB, GNT><<<1, GNT, psm, st>>>(W, n, k0, nb, pivrow.p, used.p, Hb, Rb, bad.p);
      k_gj_update<GNB><<<ugrid, 256, 0, st>>>(W, n, k0, nb, Hb, Rb);
      EXF_COUNT(2);
    }
    EXF_LAUNCH_CHECK();
  } else {
    void *args[] = {&W, &W1p, (void *)&n, &pivrow.p, &key.p, &used.p, &bad.p};
    EXF_CUDA(cudaLaunchCooperativeKernel((void *)k_gj_coop<NT>, grid, NT, args, 0, st));
    EXF_COUNT(3);
    Wfinal = (n & 1) ? W1p : W;  // step n-1 wrote buffer (n-1)&1 ? W0 : W1
  }
  int hbad = 0;
  EXF_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  EXF_CUDA(cudaStreamSynchronize(st));
  if (hbad) {
    set_error("coarsest matrix is singular");
    return EXF_ERR_SINGULAR;
  }
  if (s->coarse_inv.n != (size_t)n * n) {
    EXF_TRY(s->coarse_inv.alloc((size_t)n * n));
    s->buf_epoch++;
  }
  k_extract_inv<<<n, 128, 0, st>>>(Wfinal, n, pivrow.p, s->coarse_inv.p);
  EXF_LAUNCH_CHECK();
  s->coarse_ok = 1;
  return EXF_OK;
}

// x = A0^{-1} (b * gmask), one warp per row, FP64 arithmetic for either vector type;
// with I4 vectors DOF j is slot j / N0 of node j % N0 (pressure: slot 3 of node j - d*N0)
template <bool I4>
__device__ __forceinline__ long coarse_slot(int j, int N0, int d) {
  if (!I4) return j;
  return j < d * N0 ? 4L * (j % N0) + j / N0 : 4L * (j - d * N0) + 3;
}
template <class T, bool I4>
__global__ void k_coarse_gemv(const double *__restrict__ inv, int n, const double *__restrict__ gmask,
                              const T *__restrict__ b, T *__restrict__ x, int N0, int d) {
  EXF_PDL_WAIT();
  const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (row >= n) return;
  double acc = 0.;
  for (int j = lane; j < n; j += 32)
    acc += inv[(long)row * n + j] * (gmask[j] * (double)b[coarse_slot<I4>(j, N0, d)]);
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) x[coarse_slot<I4>(row, N0, d)] = (T)acc;
}

template <class T>
int coarse_apply(exf_sys *s, const T *b, T *x) {
  if (!s->coarse_ok) EXF_TRY(coarse_factor(s));
  const int n = s->L[0].ndof;
  auto kern = (s->nv1 && sizeof(T) == 4) ? k_coarse_gemv<T, true> : k_coarse_gemv<T, false>;
  EXF_CUDA(launch_pdl(kern, dim3(nblk(n, 8)), dim3(256), 0, s->stream, s->coarse_inv.p, n, s->gmask0.p, b, x,
                      s->L[0].N, s->nv2));
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

// FP64 DOF-order vectors <-> FP32 V-cycle vectors (I4 when i4 != 0: N nodes, d velocity
// components)
__device__ __forceinline__ long i4_slot(long i, int N, int d) {
  return i < (long)d * N ? 4 * (i % N) + i / N : 4 * (i - (long)d * N) + 3;
}
__global__ void k_cast_d2f(const double *a, float *b, long n, int i4, int N, int d) {
  EXF_PDL_WAIT();
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i4 ? i4_slot(i, N, d) : i] = (float)a[i];
}
__global__ void k_add_f2d(const float *a, double *b, long n, int i4, int N, int d) {
  EXF_PDL_WAIT();
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] += (double)a[i4 ? i4_slot(i, N, d) : i];
}
int cast_d2f(cudaStream_t st, const double *a, float *b, long n, int i4, int N, int d) {
  EXF_CUDA(launch_pdl(k_cast_d2f, dim3(nblk(n, 256)), dim3(256), 0, st, a, b, n, i4, N, d));
  EXF_COUNT(1);
  return EXF_OK;
}
int add_f2d(cudaStream_t st, const float *a, double *b, long n, int i4, int N, int d) {
  EXF_CUDA(launch_pdl(k_add_f2d, dim3(nblk(n, 256)), dim3(256), 0, st, a, b, n, i4, N, d));
  EXF_COUNT(1);
  return EXF_OK;
}

template <int NT, class T>
__global__ void k_norm2_part(const T *v, long n, double *part) {
  EXF_PDL_WAIT();
  __shared__ double sh[32];
  double acc = 0.;
  for (long i = (long)blockIdx.x * NT + threadIdx.x; i < n; i += (long)gridDim.x * NT)
    acc += (double)v[i] * (double)v[i];
  acc = block_sum<NT>(acc, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = acc;
}
// ||v||^2 into *d_out (FP64 sums in a fixed order; FP32 vectors are node-interleaved with
// zero padding slots, which add nothing)
template <class T>
int norm2(exf_sys *s, const T *v, long n, double *d_out) {
  const int grid = 296;
  EXF_TRY(ensure_partials(s, grid));
  EXF_CUDA(launch_pdl(k_norm2_part<256, T>, dim3(grid), dim3(256), 0, s->stream, v, n, s->red.part.p));
  EXF_CUDA(launch_pdl(k_reduce_partials, dim3(1), dim3(1024), 0, s->stream, (const double *)s->red.part.p, grid,
                      d_out));
  EXF_COUNT(2);
  return EXF_OK;
}
template int norm2<double>(exf_sys *, const double *, long, double *);
template int norm2<float>(exf_sys *, const float *, long, double *);

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
