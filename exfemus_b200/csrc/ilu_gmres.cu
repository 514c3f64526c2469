// ilu_gmres.cu -- the reference's default level solver for scalar equations: LASPACK's
// GMRESIter (restart 30) left-preconditioned by ILUPrecond, selected by SOLVERT GMRESM
// with the default ILU_PRECONDM (template_appl/nse/DATA/MGSclass_conf.h:101,
// contrib/matrix/linear_solverM.h:200-205, contrib/matrix/laspack_linear_solverM.C:91-96).
//
// ILU (contrib/laspack/factor.c:25-320, the non-symmetric row-wise branch): row i takes
// the set S of its columns <= i, gathers the current entries (S_a, S_b) of the rows in S
// into a dense |S| x |S| matrix, eliminates, and writes back row i's lower entries, its
// diagonal and the entries (S_a, i) of the earlier rows: the factor is stored on the
// matrix's own pattern and the preconditioner is
//   y = (D + U)^-1 D (D + L)^-1 c     (ILUPrecond, contrib/laspack/precond.c:75-110)
// with the triangular solves of MulInv_QV (contrib/laspack/operats.c:1049-1290).  Every
// elimination step, product, sum and division is done in the reference's order with
// explicitly rounded operations (no fused multiply-add), so the factor and the
// preconditioner give the reference's bits.
//
// The row recurrences run sync-free: a warp takes the next row from a ticket counter
// (rows by dependency level, see level_order), waits until the rows it depends on are
// published (bounded acquire loads: of a generation flag per row in the factorisation, of
// the value itself in the triangular solves), computes, and publishes its row (release
// store).  A warp only waits on rows with earlier tickets, which running
// warps hold, so the recurrences always progress; a wait that runs out sets the system's
// wait flag, which the host reports as EXF_ERR_CUDA.  Time is set by the dependency depth
// of the numbering (the level-nested numbering: about 770 levels for the 257 x 257 nodes
// of a 128 x 128 quad9 level), not by bandwidth.
//
// GMRES (contrib/laspack/itersolv.c:1341-1510): MaxIter = the smoothing count, modified
// Gram-Schmidt, Givens rotations, the reference's relative-residual test (rtc.c:48-70)
// before every restart cycle; the scalars live on the device and a converged call skips
// the rest of its kernels, so a smoothing call is a fixed kernel sequence that a CUDA
// graph can hold.  Vector updates use the reference's rounding (a product, then a sum);
// inner products and norms are parallel reductions, so GMRES iterates agree with the
// reference's to rounding, not bitwise.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "exf_internal.h"

namespace exf {

__device__ __forceinline__ int ld_acq(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_rel(int *p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// the triangular solves publish each row's value itself: the output vector is filled with
// this NaN pattern (which arithmetic does not produce) first, and a row's value replaces it
// with a release store
constexpr unsigned long long kNotReady = 0x7FF4C0FFEE000001ull;
__device__ __forceinline__ double ld_acq_f64(const double *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return __longlong_as_double((long long)v);
}
__device__ __forceinline__ void st_rel_f64(double *p, double v) {
  asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"((unsigned long long)__double_as_longlong(v))
               : "memory");
}
// bounded wait for the published value of row j (0 if the wait ran out; the flag is set)
__device__ __forceinline__ double wait_val(const double *v, int j, int *err) {
  for (int t = 0; t < (1 << 20); t++) {
    const double x = ld_acq_f64(v + j);
    if ((unsigned long long)__double_as_longlong(x) != kNotReady) return x;
    if ((t & 255) == 255 && *(volatile int *)err) return 0.;
    __nanosleep(32);
  }
  atomicExch(err, 1);
  return 0.;
}

// bounded wait until row j is published in generation gen; false if it ran out (or an
// earlier wait of the launch did)
__device__ __forceinline__ bool wait_row(const int *flag, int j, int gen, int *err) {
  for (int t = 0; t < (1 << 20); t++) {
    if (ld_acq(flag + j) >= gen) return true;
    if ((t & 255) == 255 && *(volatile int *)err) return false;
    __nanosleep(64);
  }
  atomicExch(err, 1);
  return false;
}

// position of c in the sorted list a[0..n), -1 if absent
__device__ __forceinline__ int bsearch_i(const int *a, int n, int c) {
  int lo = 0, hi = n - 1;
  while (lo <= hi) {
    const int m = (lo + hi) >> 1, v = a[m];
    if (v == c) return m;
    if (v < c) lo = m + 1;
    else hi = m - 1;
  }
  return -1;
}

// a[j >> 5] of a per-lane register array without a dynamic register index
template <int KU>
__device__ __forceinline__ double pick(const double (&a)[KU], int u) {
  double v = a[0];
#pragma unroll
  for (int q = 1; q < KU; q++)
    if (q == u) v = a[q];
  return v;
}

// ctl[0]: ticket, ctl[1]: generation (factorisation), ctl[2]: zero-pivot row + 1
__global__ void k_ilu_arm(int *ctl, const int *skip) {
  if (skip && *skip) return;
  ctl[0] = 0;
  ctl[1] += 1;
}
// before a triangular solve: the output marked unpublished, the ticket reset
__global__ void k_ilu_prep(double *v, long n, int *ctl, const int *skip) {
  if (skip && *skip) return;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) ctl[0] = 0;
  if (i < n) v[i] = __longlong_as_double((long long)kNotReady);
}

// one warp per row; MAXL >= the longest lower row + 1; f holds a copy of the matrix on
// entry and the factor on exit; invd[i] = 1 / the factor's diagonal
template <int MAXL, int NW>
__global__ void __launch_bounds__(32 * NW) k_ilu_factor(int N, const int *__restrict__ ord, const int *__restrict__ ptr,
                                                        const int *__restrict__ col, const int *__restrict__ dpos,
                                                        double *f, double *invd, int *flag, int *ctl, int *err) {
  constexpr int KU = (MAXL + 31) / 32;
  extern __shared__ double ilu_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double *Lm = ilu_smem + (size_t)warp * MAXL * (MAXL + 1);
  // per warp: S, each S row's first entry and entry count, the offsets of the rows'
  // entries in the flattened gather, and the position of column i in each S row
  int *Sc = reinterpret_cast<int *>(ilu_smem + (size_t)NW * MAXL * (MAXL + 1)) + warp * 5 * MAXL;
  int *Rb = Sc + MAXL, *Off = Rb + MAXL, *Pi = Off + MAXL + 1;  // Off holds MAXL + 1 entries
  const int gen = ctl[1];
  auto Lat = [&](int a, int b) -> double & { return Lm[a * (MAXL + 1) + b]; };
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(ctl, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= N) return;
    const int i = ord[t];
    const int k0 = ptr[i], kd = dpos[i], LD = kd - k0 + 1;
    if (LD > MAXL) {  // the host sizes MAXL from the pattern: not reached
      if (lane == 0) atomicExch(err, 1);
      if (lane == 0) st_rel(flag + i, gen);
      continue;
    }
    for (int a = lane; a < LD; a += 32) {
      const int r = col[k0 + a];
      Sc[a] = r;
      Rb[a] = ptr[r];
      Off[a + 1] = ptr[r + 1] - Rb[a];  // the row's entry count, summed below
      Pi[a] = -1;
    }
    for (int a = lane; a < LD - 1; a += 32) wait_row(flag, Sc[a], gen, err);
    for (int t = lane; t < LD * (MAXL + 1); t += 32) Lm[t] = 0.;
    __syncwarp();
    if (lane == 0) {
      Off[0] = 0;
      for (int a = 0; a < LD; a++) Off[a + 1] += Off[a];
    }
    __syncwarp();
    // the entries (S_a, S_b) of the rows in S, columns <= i, gathered by all lanes over the
    // rows' concatenated entries, four entries per lane in flight
    const int T = Off[LD];
    for (int e0 = 0; e0 < T; e0 += 128) {
      int kk[4], cc[4], aa[4];
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int e = e0 + 32 * q + lane;
        kk[q] = -1;
        if (e < T) {
          int lo = 0, hi = LD - 1;  // the row a with Off[a] <= e < Off[a + 1]
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (Off[mid] <= e) lo = mid;
            else hi = mid - 1;
          }
          aa[q] = lo;
          kk[q] = Rb[lo] + (e - Off[lo]);
          cc[q] = col[kk[q]];
        }
      }
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (kk[q] >= 0 && cc[q] <= i) {
          const int b = bsearch_i(Sc, LD, cc[q]);
          if (b >= 0) Lat(aa[q], b) = f[kk[q]];
          if (cc[q] == i) Pi[aa[q]] = kk[q];
        }
    }
    __syncwarp();
    const int last = LD - 1;
    double lk[KU], uk[KU];  // row i's lower entries and the column-i entries of rows S_k
#pragma unroll
    for (int u = 0; u < KU; u++) {
      const int k = lane + 32 * u;
      lk[u] = k < last ? Lat(last, k) : 0.;
      uk[u] = k < last ? Lat(k, last) : 0.;
    }
    for (int j = 0; j < last; j++) {  // L[last][k] -= L[last][j] * L[j][k] / L[j][j]
      const double lj = __shfl_sync(0xffffffffu, pick(lk, j >> 5), j & 31), djj = Lat(j, j);
#pragma unroll
      for (int u = 0; u < KU; u++) {
        const int k = lane + 32 * u;
        if (k > j && k < last) lk[u] = __dsub_rn(lk[u], __ddiv_rn(__dmul_rn(lj, Lat(j, k)), djj));
      }
    }
    for (int j = 0; j < last; j++) {  // L[k][last] -= L[j][last] * L[k][j] / L[j][j]
      const double uj = __shfl_sync(0xffffffffu, pick(uk, j >> 5), j & 31), djj = Lat(j, j);
#pragma unroll
      for (int u = 0; u < KU; u++) {
        const int k = lane + 32 * u;
        if (k > j && k < last) uk[u] = __dsub_rn(uk[u], __ddiv_rn(__dmul_rn(uj, Lat(k, j)), djj));
      }
    }
    double d = Lat(last, last);  // L[last][last] -= L[j][last] * L[last][j] / L[j][j]
    for (int j = 0; j < last; j++) {
      const double uj = __shfl_sync(0xffffffffu, pick(uk, j >> 5), j & 31);
      const double lj = __shfl_sync(0xffffffffu, pick(lk, j >> 5), j & 31);
      d = __dsub_rn(d, __ddiv_rn(__dmul_rn(uj, lj), Lat(j, j)));
    }
    if (fabs(d) < 10. * DBL_MIN && lane == 0) atomicCAS(ctl + 2, 0, i + 1);  // LASZeroPivotErr
#pragma unroll
    for (int u = 0; u < KU; u++) {
      const int k = lane + 32 * u;
      if (k < last) {
        f[k0 + k] = lk[u];
        if (Pi[k] >= 0) f[Pi[k]] = uk[u];  // entry (S_k, i) of the earlier row S_k
        else atomicExch(err, 1);           // LASILUStructErr: the pattern is symmetric here
      }
    }
    if (lane == 0) {
      f[kd] = d;
      invd[i] = __ddiv_rn(1., d);
    }
    __threadfence();
    __syncwarp();
    if (lane == 0) st_rel(flag + i, gen);
  }
}

// w = (D + L)^-1 c: Sum = 0, Sum -= l_ik w_k over the row's lower entries in column
// order, Sum += c_i, w_i = Sum / d_i (as the product with the stored inverse)
__global__ void __launch_bounds__(128) k_ilu_lower(int N, const int *__restrict__ ord, const int *__restrict__ ptr,
                                                   const int *__restrict__ col,
                                                   const int *__restrict__ dpos, const double *__restrict__ f,
                                                   const double *__restrict__ invd, const double *c, double *w,
                                                   int *ctl, int *err, const int *skip) {
  if (skip && *skip) return;
  const int lane = threadIdx.x & 31;
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(ctl, 1);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= N) return;
    const int i = ord[t];
    const int k0 = ptr[i], nl = dpos[i] - k0;
    const double ci = c[i], di = invd[i];  // loaded before the waits, off the critical path
    double s = 0.;
    for (int base = 0; base < nl; base += 32) {
      double p = 0.;
      if (base + lane < nl) {
        const int k = k0 + base + lane;
        const double fk = f[k];
        p = __dmul_rn(fk, wait_val(w, col[k], err));
      }
      const int n = min(32, nl - base);
      for (int t = 0; t < n; t++) s = __dsub_rn(s, __shfl_sync(0xffffffffu, p, t));
    }
    s = __dadd_rn(s, ci);
    if (lane == 0) st_rel_f64(w + i, __dmul_rn(s, di));
  }
}

// y = (D + U)^-1 (D w): Sum -= u_ik y_k over the upper entries from the row's end,
// Sum += d_i w_i, y_i = Sum / d_i (rows by level of the upper entries)
__global__ void __launch_bounds__(128) k_ilu_upper(int N, const int *__restrict__ ord, const int *__restrict__ ptr,
                                                   const int *__restrict__ col,
                                                   const int *__restrict__ dpos, const double *__restrict__ f,
                                                   const double *__restrict__ invd, const double *w, double *y,
                                                   int *ctl, int *err, const int *skip) {
  if (skip && *skip) return;
  const int lane = threadIdx.x & 31;
  for (;;) {
    int t0 = 0;
    if (lane == 0) t0 = atomicAdd(ctl, 1);
    t0 = __shfl_sync(0xffffffffu, t0, 0);
    if (t0 >= N) return;
    const int i = ord[t0];
    const int kd = dpos[i], k1 = ptr[i + 1], nu = k1 - 1 - kd;
    const double zi = __dadd_rn(0., __dmul_rn(f[kd], w[i])), di = invd[i];  // Mul_QV of the diagonal: 0 + d_i w_i
    double s = 0.;
    for (int base = 0; base < nu; base += 32) {
      double p = 0.;
      if (base + lane < nu) {
        const int k = k1 - 1 - base - lane;  // from the row's end
        const double fk = f[k];
        p = __dmul_rn(fk, wait_val(y, col[k], err));
      }
      const int n = min(32, nu - base);
      for (int t = 0; t < n; t++) s = __dsub_rn(s, __shfl_sync(0xffffffffu, p, t));
    }
    s = __dadd_rn(s, zi);
    if (lane == 0) st_rel_f64(y + i, __dmul_rn(s, di));
  }
}


// ------------------------------------------------------------------- GMRES scalars
// gm_sc: [0] ||b||^2, [1] ||v1||^2 (the residual), [2] the last inner product, [4] the
// norm a vector is scaled by, H(i, k) = h[i][k], S(k) = s[k], C1/C2 the rotations, Y(k)
// = y[k] (1-based as in GMRESIter); gm_ctl[0] != 0: the call has converged, skip
constexpr int kGmSteps = 30;  // SetGMRESRestart(30), laspack_linear_solverM.C:91
__host__ __device__ constexpr int gmH(int i, int k) { return 16 + i * 32 + k; }
__host__ __device__ constexpr int gmS(int k) { return 1008 + k; }
__host__ __device__ constexpr int gmC1(int k) { return 1040 + k; }
__host__ __device__ constexpr int gmC2(int k) { return 1072 + k; }
__host__ __device__ constexpr int gmY(int k) { return 1104 + k; }
constexpr int kGmScalars = 1136;

template <int NT>
__global__ void __launch_bounds__(NT) k_gm_dot_part(const double *__restrict__ a, const double *__restrict__ b,
                                                    long n, double *part) {
  __shared__ double sh[NT / 32];
  double v = 0.;
  for (long i = (long)blockIdx.x * NT + threadIdx.x; i < n; i += (long)gridDim.x * NT) v += a[i] * b[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.;
    for (int k = 0; k < NT / 32; k++) t += sh[k];
    part[blockIdx.x] = t;
  }
}
__global__ void k_gm_dot_fin(const double *__restrict__ part, int np, double *out) {
  __shared__ double sh[8];
  double v = 0.;
  for (int i = threadIdx.x; i < np; i += 256) v += part[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.;
    for (int k = 0; k < 8; k++) t += sh[k];
    *out = t;
  }
}

// RTCResult (rtc.c:48-70): converged when ||r|| < eps ||b|| (or b = 0 and 1 + ||r|| = 1)
__global__ void k_gm_rtc(const double *sc, int *ctl, double eps) {
  const double rn = sqrt(sc[1]), bn = sqrt(sc[0]);
  const bool conv = rn < eps * bn || (fabs(bn) < 10. * DBL_MIN && fabs((1. + rn) - 1.) < 10. * DBL_EPSILON);
  ctl[0] = conv ? 1 : 0;
}
__global__ void k_gm_reset(int *ctl) { ctl[0] = 0; }

// s[1] = ||v1|| after preconditioning; the vector is then scaled by 1 / s[1]
__global__ void k_gm_first(double *sc) {
  sc[gmS(1)] = __dsqrt_rn(sc[2]);
  sc[4] = sc[gmS(1)];
}

// v *= 1 / *den (MulAsgn_VS with the reciprocal formed once)
__global__ void k_gm_scale(double *v, long n, const double *den, const int *skip) {
  if (*skip) return;
  const double f = __ddiv_rn(1., *den);
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = __dmul_rn(v[i], f);
}
// v -= h vk (SubAsgn_VV(v, Mul_SV(h, vk)))
__global__ void k_gm_axpy(double *v, const double *__restrict__ vk, long n, const double *h, const int *skip) {
  if (*skip) return;
  const double hh = *h;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = __dsub_rn(v[i], __dmul_rn(hh, vk[i]));
}

// h[i][i+1] = ||v_{i+1}|| (the last inner product), then the Q-R update of column i and
// of s (itersolv.c, the "Q-R algorithm" block)
__global__ void k_gm_qr(double *sc, int i) {
  const double nrm = __dsqrt_rn(sc[2]);
  sc[gmH(i, i + 1)] = nrm;
  sc[4] = nrm;
  for (int k = 1; k < i; k++) {
    const double hk = sc[gmH(i, k)], hk1 = sc[gmH(i, k + 1)];
    const double h1 = __dadd_rn(__dmul_rn(sc[gmC1(k)], hk), __dmul_rn(sc[gmC2(k)], hk1));
    const double h2 = __dadd_rn(__dmul_rn(-sc[gmC2(k)], hk), __dmul_rn(sc[gmC1(k)], hk1));
    sc[gmH(i, k)] = h1;
    sc[gmH(i, k + 1)] = h2;
  }
  const double hii = sc[gmH(i, i)], hi1 = sc[gmH(i, i + 1)];
  const double r = __dsqrt_rn(__dadd_rn(__dmul_rn(hii, hii), __dmul_rn(hi1, hi1)));
  sc[gmC1(i)] = __ddiv_rn(hii, r);
  sc[gmC2(i)] = __ddiv_rn(hi1, r);
  sc[gmH(i, i)] = r;
  sc[gmH(i, i + 1)] = 0.;
  sc[gmS(i + 1)] = __dmul_rn(-sc[gmC2(i)], sc[gmS(i)]);
  sc[gmS(i)] = __dmul_rn(sc[gmC1(i)], sc[gmS(i)]);
}

// H y = s by back substitution (s is overwritten, as in the reference)
__global__ void k_gm_solve(double *sc, int ni) {
  for (int j = ni; j > 0; j--) {
    sc[gmY(j)] = __ddiv_rn(sc[gmS(j)], sc[gmH(j, j)]);
    for (int k = j - 1; k > 0; k--) sc[gmS(k)] = __dsub_rn(sc[gmS(k)], __dmul_rn(sc[gmH(j, k)], sc[gmY(j)]));
  }
}

// x += y_j v_j for j = ni .. 1 (AddAsgn_VV(x, Mul_SV(y[j], v[j])))
__global__ void k_gm_update(double *x, const double *__restrict__ V, long n, int ni, const double *sc,
                            const int *skip) {
  if (*skip) return;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double xi = x[i];
  for (int j = ni; j > 0; j--) xi = __dadd_rn(xi, __dmul_rn(sc[gmY(j)], V[(long)(j - 1) * n + i]));
  x[i] = xi;
}
__global__ void k_gm_copy(const double *src, double *dst) { *dst = *src; }

// ------------------------------------------------------------------- host side
static int ilu_grid(exf_sys *s) { return s->nsm * 2; }

static int dot_dev(exf_sys *s, SysLevel &L, const double *a, const double *b, long n, double *out) {
  constexpr int G = 296;
  if (L.gm_part.n < (size_t)G) EXF_TRY(L.gm_part.alloc(G));
  k_gm_dot_part<256><<<G, 256, 0, s->stream>>>(a, b, n, L.gm_part.p);
  k_gm_dot_fin<<<1, 256, 0, s->stream>>>(L.gm_part.p, G, out);
  EXF_COUNT(2);
  return EXF_OK;
}

// y = ILUPrecond(c) on level lev (y may be c); kernels skipped while *skip != 0
static int ilu_apply_dev(exf_sys *s, int lev, const double *c, double *y, const int *skip) {
  SysLevel &L = s->L[lev];
  const int N = L.N, G = ilu_grid(s);
  const unsigned g = (unsigned)((N + 255) / 256);
  k_ilu_prep<<<g, 256, 0, s->stream>>>(L.gm_w.p, N, L.ilu_ctl.p, skip);
  k_ilu_lower<<<G, 128, 0, s->stream>>>(N, L.ilu_ord_lo.p, L.qq_ptr.p, L.qq_col.p, L.diag_pos.p, L.ilu_f.p,
                                        L.ilu_inv.p, c, L.gm_w.p, L.ilu_ctl.p, s->wait_flag.p, skip);
  k_ilu_prep<<<g, 256, 0, s->stream>>>(y, N, L.ilu_ctl.p, skip);
  k_ilu_upper<<<G, 128, 0, s->stream>>>(N, L.ilu_ord_up.p, L.qq_ptr.p, L.qq_col.p, L.diag_pos.p, L.ilu_f.p,
                                        L.ilu_inv.p, L.gm_w.p, y, L.ilu_ctl.p, s->wait_flag.p, skip);
  EXF_COUNT(4);
  EXF_LAUNCH_CHECK();
  return EXF_OK;
}

template <int MAXL, int NW>
static int launch_factor(exf_sys *s, SysLevel &L) {
  const size_t smem = (size_t)NW * (MAXL * (MAXL + 1) * sizeof(double) + 5 * MAXL * sizeof(int));
  auto kern = k_ilu_factor<MAXL, NW>;
  EXF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_ilu_arm<<<1, 1, 0, s->stream>>>(L.ilu_ctl.p, nullptr);
  kern<<<s->nsm * 4, 32 * NW, smem, s->stream>>>(L.N, L.ilu_ord_lo.p, L.qq_ptr.p, L.qq_col.p, L.diag_pos.p, L.ilu_f.p, L.ilu_inv.p,
                                                   L.ilu_flag.p, L.ilu_ctl.p, s->wait_flag.p);
  EXF_COUNT(2);
  EXF_LAUNCH_CHECK();
  return EXF_OK;
}

// The rows in the order their tickets hand them out: by dependency level (the longest
// chain of lower, or upper, entries leading to the row), index order within a level.
// Every row depends only on rows of earlier levels, so a warp still waits only on earlier
// tickets, and the rows of a level run together instead of one index after the other
// (consecutive rows of the level-nested numbering mostly depend on each other).
// Returns the number of levels.
static int level_order(const std::vector<int> &ptr, const std::vector<int> &col, const std::vector<int> &dp,
                       bool upper, std::vector<int> &ord) {
  const int N = (int)dp.size();
  std::vector<int> lv(N, 0);
  int nl = 0;
  for (int q = 0; q < N; q++) {
    const int i = upper ? N - 1 - q : q;
    int l = 0;
    const int a = upper ? dp[i] + 1 : ptr[i], e = upper ? ptr[i + 1] : dp[i];
    for (int k = a; k < e; k++) l = std::max(l, lv[col[k]] + 1);
    lv[i] = l;
    nl = std::max(nl, l + 1);
  }
  std::vector<int> cnt(nl + 1, 0);
  for (int i = 0; i < N; i++) cnt[lv[i] + 1]++;
  for (int l = 0; l < nl; l++) cnt[l + 1] += cnt[l];
  ord.assign(N, 0);
  for (int i = 0; i < N; i++) ord[cnt[lv[i]]++] = i;
  return nl;
}

// ILUFactor of level lev's matrix, once per assembly (outside graph capture)
int ilu_ready(exf_sys *s, int lev) {
  SysLevel &L = s->L[lev];
  if (L.ilu_ok) return EXF_OK;
  if (s->nv1 != 0) {
    set_error("GMRES + ILU smoothing needs a scalar system: the Navier-Stokes pressure block has zero "
              "diagonal entries, on which LASPACK's ILU stops (LASZeroInDiagErr)");
    return EXF_ERR_UNSUPPORTED;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  EXF_CUDA(cudaStreamIsCapturing(s->stream, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    set_error("the ILU factor of level %d is stale inside a graph capture", lev);
    return EXF_ERR_STATE;
  }
  const int N = L.N;
  if (L.ilu_maxl == 0) {  // from the pattern, fixed per system
    std::vector<int> ptr(N + 1), dp(N), col(L.nqq);
    EXF_CUDA(cudaMemcpyAsync(ptr.data(), L.qq_ptr.p, (N + 1) * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    EXF_CUDA(cudaMemcpyAsync(dp.data(), L.diag_pos.p, N * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    EXF_CUDA(cudaMemcpyAsync(col.data(), L.qq_col.p, L.nqq * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    EXF_CUDA(cudaStreamSynchronize(s->stream));
    int m = 1;
    for (int i = 0; i < N; i++) m = std::max(m, dp[i] - ptr[i] + 1);
    std::vector<int> lo, up;
    L.ilu_depth[0] = level_order(ptr, col, dp, false, lo);
    L.ilu_depth[1] = level_order(ptr, col, dp, true, up);
    EXF_TRY(L.ilu_ord_lo.alloc(N));
    EXF_TRY(L.ilu_ord_up.alloc(N));
    EXF_CUDA(cudaMemcpyAsync(L.ilu_ord_lo.p, lo.data(), N * sizeof(int), cudaMemcpyHostToDevice, s->stream));
    EXF_CUDA(cudaMemcpyAsync(L.ilu_ord_up.p, up.data(), N * sizeof(int), cudaMemcpyHostToDevice, s->stream));
    EXF_CUDA(cudaStreamSynchronize(s->stream));
    L.ilu_maxl = m;
    s->buf_epoch++;
  }
  if (L.ilu_maxl > 128) {
    set_error("ILU: a row of level %d has %d entries left of the diagonal (at most 127 supported)", lev,
              L.ilu_maxl - 1);
    return EXF_ERR_UNSUPPORTED;
  }
  if (L.ilu_f.n != (size_t)L.nqq) {
    EXF_TRY(L.ilu_f.alloc(L.nqq));
    EXF_TRY(L.ilu_inv.alloc(N));
    EXF_TRY(L.ilu_flag.alloc(N));
    EXF_TRY(L.ilu_flag.zero(s->stream));
    EXF_TRY(L.ilu_ctl.alloc(4));
    EXF_TRY(L.ilu_ctl.zero(s->stream));
    s->buf_epoch++;
  }
  EXF_CUDA(cudaMemcpyAsync(L.ilu_f.p, L.A.vv.p, L.nqq * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
  EXF_CUDA(cudaMemsetAsync(L.ilu_ctl.p + 2, 0, sizeof(int), s->stream));
  if (L.ilu_maxl <= 16) EXF_TRY((launch_factor<16, 2>(s, L)));
  else if (L.ilu_maxl <= 32) EXF_TRY((launch_factor<32, 2>(s, L)));
  else if (L.ilu_maxl <= 64) EXF_TRY((launch_factor<64, 2>(s, L)));
  else EXF_TRY((launch_factor<128, 1>(s, L)));
  int zp = 0;
  EXF_CUDA(cudaMemcpyAsync(&zp, L.ilu_ctl.p + 2, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  EXF_TRY(device_wait_status(s));
  if (zp) {
    set_error("ILU: zero pivot in row %d of level %d (LASZeroPivotErr)", zp - 1, lev);
    return EXF_ERR_SINGULAR;
  }
  L.ilu_ok = true;
  return EXF_OK;
}

int ilu_apply(exf_sys *s, int lev, const double *c, double *y) {
  EXF_TRY(ilu_ready(s, lev));
  SysLevel &L = s->L[lev];
  if (L.gm_w.n < (size_t)L.ndof) EXF_TRY(L.gm_w.alloc(L.ndof));
  return ilu_apply_dev(s, lev, c, y, nullptr);
}

// one call of the level solver: GMRESIter(A, x, b, m, ILUPrecond) with RTC accuracy eps;
// with acc, *acc = the squared residual of its last test (LastAcc times ||b||)
int gmres_smooth(exf_sys *s, int lev, double eps, int m, double *x, const double *b, double *acc) {
  EXF_TRY(ilu_ready(s, lev));
  SysLevel &L = s->L[lev];
  const long n = L.ndof;
  const int kmax = std::min(m, kGmSteps);
  if (L.gm_V.n < (size_t)(kmax + 1) * n || L.gm_w.n < (size_t)n || L.gm_t.n < (size_t)n || !L.gm_sc.p) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    EXF_CUDA(cudaStreamIsCapturing(s->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) {
      set_error("GMRES work space of level %d sized inside a graph capture", lev);
      return EXF_ERR_STATE;
    }
    if (L.gm_V.n < (size_t)(kmax + 1) * n) EXF_TRY(L.gm_V.alloc((size_t)(kmax + 1) * n));
    if (L.gm_w.n < (size_t)n) EXF_TRY(L.gm_w.alloc(n));
    if (L.gm_t.n < (size_t)n) EXF_TRY(L.gm_t.alloc(n));
    if (!L.gm_sc.p) {
      EXF_TRY(L.gm_sc.alloc(kGmScalars));
      EXF_TRY(L.gm_sc.zero(s->stream));
      EXF_TRY(L.gm_ctl.alloc(4));
    }
    s->buf_epoch++;
  }
  double *sc = L.gm_sc.p, *V = L.gm_V.p;
  int *ctl = L.gm_ctl.p;
  auto vk = [&](int k) { return V + (long)(k - 1) * n; };  // v[k], 1-based
  const unsigned g = (unsigned)((n + 255) / 256);
  k_gm_reset<<<1, 1, 0, s->stream>>>(ctl);
  EXF_TRY(dot_dev(s, L, b, b, n, sc));                                  // bNorm
  EXF_TRY(spmv_resid<double>(s, lev, x, b, vk(1), sc + 1));             // v[1] = b - A x
  for (int iter = 0; iter < m;) {
    k_gm_rtc<<<1, 1, 0, s->stream>>>(sc, ctl, eps);
    EXF_TRY(ilu_apply_dev(s, lev, vk(1), vk(1), ctl));
    EXF_TRY(dot_dev(s, L, vk(1), vk(1), n, sc + 2));
    k_gm_first<<<1, 1, 0, s->stream>>>(sc);
    k_gm_scale<<<g, 256, 0, s->stream>>>(vk(1), n, sc + 4, ctl);
    EXF_COUNT(3);
    const int ni = std::min(kGmSteps, m - iter);
    for (int i = 1; i <= ni; i++) {
      EXF_TRY(spmv_resid<double>(s, lev, vk(i), nullptr, L.gm_t.p, nullptr));  // A v[i]
      EXF_TRY(ilu_apply_dev(s, lev, L.gm_t.p, vk(i + 1), ctl));
      for (int k = 1; k <= i; k++) {  // modified Gram-Schmidt
        EXF_TRY(dot_dev(s, L, vk(i + 1), vk(k), n, sc + gmH(i, k)));
        k_gm_axpy<<<g, 256, 0, s->stream>>>(vk(i + 1), vk(k), n, sc + gmH(i, k), ctl);
        EXF_COUNT(1);
      }
      EXF_TRY(dot_dev(s, L, vk(i + 1), vk(i + 1), n, sc + 2));
      k_gm_qr<<<1, 1, 0, s->stream>>>(sc, i);
      k_gm_scale<<<g, 256, 0, s->stream>>>(vk(i + 1), n, sc + 4, ctl);
      EXF_COUNT(2);
    }
    iter += ni;
    k_gm_solve<<<1, 1, 0, s->stream>>>(sc, ni);
    k_gm_update<<<g, 256, 0, s->stream>>>(x, V, n, ni, sc, ctl);
    EXF_COUNT(2);
    EXF_TRY(spmv_resid<double>(s, lev, x, b, vk(1), sc + 1));  // the new residual
  }
  if (acc) {
    k_gm_copy<<<1, 1, 0, s->stream>>>(sc + 1, acc);
    EXF_COUNT(1);
  }
  EXF_LAUNCH_CHECK();
  return EXF_OK;
}

}  // namespace exf
