// api.cu -- the C ABI: meshes, systems (one per equation, like an MGSolBase object),
// assembly dispatch, and the multigrid driver (MGSolve/MGStep) on device-resident state.
//
// Multigrid (src/MGSolverBase.C:163-289): recursive cycle with gamma coarse visits,
// sweeps doubled below the top level, damped coarse correction (0.95 in the reference,
// optionally conditional as in the reference), exact coarse solve.  The stop test is the
// relative residual ||b-Ax||/||b|| of the top level.  Mixed precision: the residual,
// solution update and coarse solve are FP64; the V-cycle (smoother, residuals, transfers)
// runs on FP32 copies of the level matrices (defect correction).
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstddef>
#include <cstring>
#include <vector>

#include "exf_internal.h"

namespace exf {

static thread_local char g_err[512] = "";
static unsigned long long g_launches = 0;
void count_launch(int n) { __atomic_add_fetch(&g_launches, (unsigned long long)n, __ATOMIC_RELAXED); }
void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

static inline unsigned nblk(long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// ------------------------------------------------- NB <-> DOF-level CSR values
__global__ void k_nb_to_csr(int N, int NL, int d, int ns, const int *qq_ptr, const int *ql_ptr, long nqq, long nql,
                            long nqqL, const double *vv, const double *vp, const double *pv, const double *pp,
                            const int *rowptr, double *out, int dir) {
  long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long nq = (long)d * N;
  long nrow = nq + (ns ? NL : 0);
  if (r >= nrow) return;
  long o = rowptr[r];
  double *vvw = const_cast<double *>(vv), *vpw = const_cast<double *>(vp), *pvw = const_cast<double *>(pv),
         *ppw = const_cast<double *>(pp);
  if (r < nq) {
    int a = (int)(r / N), n = (int)(r % N);
    for (int b = 0; b < d; b++)
      for (int k = qq_ptr[n]; k < qq_ptr[n + 1]; k++, o++) {
        long idx = (long)(a * d + b) * nqq + k;
        if (dir == 0) out[o] = vv[idx];
        else vvw[idx] = out[o];
      }
    if (ns)
      for (int k = ql_ptr[n]; k < ql_ptr[n + 1]; k++, o++) {
        long idx = (long)a * nql + k;
        if (dir == 0) out[o] = vp[idx];
        else vpw[idx] = out[o];
      }
  } else {
    int m = (int)(r - nq);
    for (int b = 0; b < d; b++)
      for (int k = qq_ptr[m]; k < qq_ptr[m + 1]; k++, o++) {
        long idx = (long)b * nqqL + k;
        if (dir == 0) out[o] = pv[idx];
        else pvw[idx] = out[o];
      }
    for (int k = ql_ptr[m]; k < ql_ptr[m + 1]; k++, o++) {
      if (dir == 0) out[o] = pp[k];
      else ppw[k] = out[o];
    }
  }
}

static int nb_csr(exf_sys *s, int lev, double *d_vals, int dir) {
  SysLevel &L = s->L[lev];
  k_nb_to_csr<<<nblk(L.ndof, 256), 256, 0, s->stream>>>(L.N, L.NL, s->nv2, s->nv1, L.qq_ptr.p, L.ql_ptr.p, L.nqq,
                                                         L.nql, L.nqqL, L.A.vv.p, L.A.vp.p, L.A.pv.p, L.A.pp.p,
                                                         L.csr_ptr.p, d_vals, dir);
  EXF_LAUNCH_CHECK();
  return EXF_OK;
}
int csr_values(exf_sys *s, int lev, double *d_out) { return nb_csr(s, lev, d_out, 0); }
int csr_set_values(exf_sys *s, int lev, const double *d_in) { return nb_csr(s, lev, const_cast<double *>(d_in), 1); }

__global__ void k_d2f(const double *a, float *b, long n) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}
int sync_fp32(exf_sys *s, int lev) {
  SysLevel &L = s->L[lev];
  auto cp = [&](const DBuf<double> &a, DBuf<float> &b) {
    if (a.p && b.p) {
      k_d2f<<<nblk(a.n, 256), 256, 0, s->stream>>>(a.p, b.p, a.n);
      EXF_COUNT(1);
    }
  };
  cp(L.A.vv, L.A32.vv);
  cp(L.A.vp, L.A32.vp);
  cp(L.A.pv, L.A32.pv);
  cp(L.A.pp, L.A32.pp);
  EXF_LAUNCH_CHECK();
  L.ilu_ok = false;  // the matrix changed: refactor before the next GMRES + ILU call
  return vanka_prep(s, lev);
}

// ----------------------------------------------------------------- transpose
// block (n,m) of A^T = block (m,n) of A transposed; B^T <-> B through gidx
__global__ void k_tpos(const int *qq_ptr, const int *qq_col, int N, int *tpos) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  for (int k = qq_ptr[n]; k < qq_ptr[n + 1]; k++) {
    int m = qq_col[k];
    int lo = qq_ptr[m], hi = qq_ptr[m + 1];
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (qq_col[mid] < n) lo = mid + 1;
      else hi = mid;
    }
    tpos[k] = lo;
  }
}
__global__ void k_tpos_l(const int *ql_ptr, const int *ql_col, int NL, int *tpos) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= NL) return;
  for (int k = ql_ptr[n]; k < ql_ptr[n + 1]; k++) {
    int m = ql_col[k];
    int lo = ql_ptr[m], hi = ql_ptr[m + 1];
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (ql_col[mid] < n) lo = mid + 1;
      else hi = mid;
    }
    tpos[k] = lo;
  }
}
__global__ void k_transpose_vv(const double *src, double *dst, const int *tpos, long nqq, int d) {
  long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nqq) return;
  long t = tpos[k];
  for (int a = 0; a < d; a++)
    for (int b = 0; b < d; b++) dst[(long)(a * d + b) * nqq + k] = src[(long)(b * d + a) * nqq + t];
}
__global__ void k_transpose_bp(const double *vp, const double *pv, double *vp_t, double *pv_t, const int *gidx,
                               long nql, long nqqL, int d) {
  long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nqqL) return;
  long g = gidx[k];
  for (int a = 0; a < d; a++) {
    pv_t[(long)a * nqqL + k] = vp[(long)a * nql + g];
    vp_t[(long)a * nql + g] = pv[(long)a * nqqL + k];
  }
}
__global__ void k_transpose_pp(const double *src, double *dst, const int *tpos, long n) {
  long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) dst[k] = src[tpos[k]];
}

int transpose_level(exf_sys *s, int lev) {
  SysLevel &L = s->L[lev];
  cudaStream_t st = s->stream;
  const int d = s->nv2;
  DBuf<int> tpos;
  EXF_TRY(tpos.alloc(L.nqq));
  k_tpos<<<nblk(L.N, 128), 128, 0, st>>>(L.qq_ptr.p, L.qq_col.p, L.N, tpos.p);
  DBuf<double> vv;
  EXF_TRY(vv.alloc(L.A.vv.n));
  k_transpose_vv<<<nblk(L.nqq, 256), 256, 0, st>>>(L.A.vv.p, vv.p, tpos.p, L.nqq, d);
  EXF_CUDA(cudaMemcpyAsync(L.A.vv.p, vv.p, L.A.vv.n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  if (s->nv1) {
    DBuf<double> vp, pv, pp;
    DBuf<int> tl;
    EXF_TRY(vp.alloc(L.A.vp.n));
    EXF_TRY(pv.alloc(L.A.pv.n));
    EXF_TRY(pp.alloc(L.A.pp.n));
    EXF_TRY(tl.alloc(L.nllL));
    EXF_TRY(vp.zero(st));
    k_transpose_bp<<<nblk(L.nqqL, 256), 256, 0, st>>>(L.A.vp.p, L.A.pv.p, vp.p, pv.p, L.gidx.p, L.nql, L.nqqL, d);
    k_tpos_l<<<nblk(L.NL, 128), 128, 0, st>>>(L.ql_ptr.p, L.ql_col.p, L.NL, tl.p);
    k_transpose_pp<<<nblk(L.nllL, 256), 256, 0, st>>>(L.A.pp.p, pp.p, tl.p, L.nllL);
    EXF_CUDA(cudaMemcpyAsync(L.A.vp.p, vp.p, L.A.vp.n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    EXF_CUDA(cudaMemcpyAsync(L.A.pv.p, pv.p, L.A.pv.n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    EXF_CUDA(cudaMemcpyAsync(L.A.pp.p, pp.p, L.A.pp.n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    EXF_CUDA(cudaStreamSynchronize(st));
  }
  EXF_LAUNCH_CHECK();
  EXF_CUDA(cudaStreamSynchronize(st));
  return sync_fp32(s, lev);
}

// ------------------------------------------------------------ multigrid
// MGStep (src/MGSolverBase.C:212-289) for value type T on the vectors VT of each level.
// rest/crest of the reference are kept on the device when cond_corr is requested.
template <class T>
static T *lvx(SysLevel &L);
template <>
double *lvx<double>(SysLevel &L) { return L.x.p; }
template <>
float *lvx<float>(SysLevel &L) { return L.x32.p; }
template <class T>
static T *lvb(SysLevel &L);
template <>
double *lvb<double>(SysLevel &L) { return L.b.p; }
template <>
float *lvb<float>(SysLevel &L) { return L.b32.p; }
template <class T>
static T *lvr(SysLevel &L);
template <>
double *lvr<double>(SysLevel &L) { return L.r.p; }
template <>
float *lvr<float>(SysLevel &L) { return L.r32.p; }

// the level's accuracies in the reference's sense are needed for the conditional
// correction and for the reference stop test
static bool needs_acc(const exf_mg_params *p) { return p->cond_corr || p->stop_test == EXF_STOP_REFERENCE; }

// One smoothing call of nsw sweeps.  With acc, it also leaves in *slot the squared
// residual that the reference's level solver reports as its accuracy: LASPACK's
// stationary iterations evaluate ||r||/||b|| on a residual refreshed only while
// Iter < MaxIter (SORForwIter, contrib/laspack/itersolv.c:850-894; LastAcc,
// contrib/laspack/rtc.c:48-70), i.e. the residual of the iterate before the last sweep.
// GMRESIter reports the residual of its last test, taken after its last restart cycle.
template <class T>
static int smooth_acc(exf_sys *s, int lev, const exf_mg_params *p, int nsw, T *x, const T *b, T *r, double *slot) {
  if constexpr (sizeof(T) == 8) {
    if (p->smoother == EXF_SMOOTH_GMRES_ILU) return gmres_smooth(s, lev, p->eps, nsw, x, b, slot);
  }
  if (!slot) return smooth<T>(s, lev, p, nsw, x, b);
  if (nsw > 0) EXF_TRY(smooth<T>(s, lev, p, nsw - 1, x, b));
  EXF_TRY(spmv_resid<T>(s, lev, x, b, r, slot));
  if (nsw > 0) EXF_TRY(smooth<T>(s, lev, p, 1, x, b));
  return EXF_OK;
}

template <class T>
static int mg_step(exf_sys *s, int lev, const exf_mg_params *p, bool final_resid, double *d_norm_out) {
  SysLevel &L = s->L[lev];
  T *x = lvx<T>(L), *b = lvb<T>(L), *r = lvr<T>(L);
  const int top = s->nlev - 1;
  const long len = sizeof(T) == 4 ? L.len32 : (long)L.ndof;
  double *acc = needs_acc(p) ? s->mg_acc.p + 4 * lev : nullptr;
  if (acc) EXF_TRY(norm2<T>(s, b, len, acc));
  if (lev == 0) {
    if constexpr (sizeof(T) == 8) {
      if (p->smoother == EXF_SMOOTH_GMRES_ILU && p->coarse_iters > 0) {  // _solver[0]->solve(.., 60)
        EXF_TRY(gmres_smooth(s, 0, p->eps, p->coarse_iters, x, b, acc ? acc + 2 : nullptr));
        if (final_resid) EXF_TRY(spmv_resid<T>(s, 0, x, b, r, d_norm_out));
        return EXF_OK;
      }
    }
    EXF_TRY(coarse_apply<T>(s, b, x));
    if (acc) EXF_TRY(spmv_resid<T>(s, 0, x, b, r, acc + 2));
    if (final_resid) EXF_TRY(spmv_resid<T>(s, 0, x, b, r, d_norm_out));
    return EXF_OK;
  }
  const int mul = (p->double_below_top && lev < top) ? 2 : 1;
  EXF_TRY(smooth_acc<T>(s, lev, p, p->nu_pre * mul, x, b, r, acc ? acc + 1 : nullptr));
  EXF_TRY(spmv_resid<T>(s, lev, x, b, r, nullptr));
  SysLevel &C = s->L[lev - 1];
  EXF_TRY(restrict_op<T>(s, lev - 1, r, lvb<T>(C)));
  EXF_TRY(zero_vec<T>(s->stream, lvx<T>(C), sizeof(T) == 4 ? C.len32 : (long)C.ndof));
  for (int g = 0; g < p->gamma; g++) EXF_TRY(mg_step<T>(s, lev - 1, p, false, nullptr));
  if (p->cond_corr) EXF_TRY(prolong_cond<T>(s, lev, lvx<T>(C), x, p->corr_damp, s->mg_acc.p));
  else EXF_TRY(prolong_add<T>(s, lev, lvx<T>(C), x, p->corr_damp));
  EXF_TRY(smooth_acc<T>(s, lev, p, p->nu_post * mul, x, b, r, acc ? acc + 2 : nullptr));
  if (final_resid) EXF_TRY(spmv_resid<T>(s, lev, x, b, r, d_norm_out));
  return EXF_OK;
}

// FP64 cycle on the top level: returns ||b - A x||^2 in *d_relres
int vcycle_fp64(exf_sys *s, const exf_mg_params *p, double *d_norm2) {
  EXF_TRY(mg_step<double>(s, s->nlev - 1, p, true, d_norm2));
  return gauge_shift(s, s->L[s->nlev - 1].x.p);
}

// mixed: r64 = b - A x (already in L.r), cast, FP32 cycle, x += e
int vcycle_mixed(exf_sys *s, const exf_mg_params *p) {
  SysLevel &T = s->L[s->nlev - 1];
  const int i4 = s->nv1 ? 1 : 0;
  EXF_TRY(cast_d2f(s->stream, T.r.p, T.b32.p, T.ndof, i4, T.N, s->nv2));
  EXF_TRY(zero_vec<float>(s->stream, T.x32.p, T.len32));
  EXF_TRY(mg_step<float>(s, s->nlev - 1, p, false, nullptr));
  EXF_TRY(add_f2d(s->stream, T.x32.p, T.x.p, T.ndof, i4, T.N, s->nv2));
  return gauge_shift(s, T.x.p);
}

}  // namespace exf

using namespace exf;

// ===================================================================== C ABI
extern "C" {

const char *exf_last_error(void) { return g_err; }
long long exf_launch_count(void) { return (long long)__atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

int exf_event_record(exf_sys *s, int slot) {
  CHECK_SYS(s);
  if (slot < 0 || slot >= 8) return EXF_ERR_ARG;
  if (!s->user_ev[slot]) EXF_CUDA(cudaEventCreate(&s->user_ev[slot]));
  EXF_CUDA(cudaEventRecord(s->user_ev[slot], s->stream));
  return EXF_OK;
}

int exf_event_elapsed(exf_sys *s, int a, int b, double *ms) {
  CHECK_SYS(s);
  if (!ms || a < 0 || a >= 8 || b < 0 || b >= 8 || !s->user_ev[a] || !s->user_ev[b]) return EXF_ERR_ARG;
  EXF_CUDA(cudaEventSynchronize(s->user_ev[b]));
  float f = 0.f;
  EXF_CUDA(cudaEventElapsedTime(&f, s->user_ev[a], s->user_ev[b]));
  *ms = f;
  return EXF_OK;
}
const char *exf_version(void) { return "exfemus_b200 1.0 (sm_100a)"; }

int exf_mesh_create(const exf_mesh_desc *desc, exf_mesh **out) {
  if (!desc || !out || (desc->dim != 2 && desc->dim != 3) || desc->nlev < 1 || desc->nlev > 12) {
    set_error("exf_mesh_create: bad descriptor");
    return EXF_ERR_ARG;
  }
  for (int d = 0; d < desc->dim; d++)
    if (desc->n0[d] < 1) {
      set_error("exf_mesh_create: n0 must be >= 1");
      return EXF_ERR_ARG;
    }
  EXF_CUDA(cudaSetDevice(desc->device));
  exf_mesh *m = new exf_mesh();
  m->dim = desc->dim;
  m->nlev = desc->nlev;
  m->device = desc->device;
  for (int d = 0; d < 3; d++) m->n0[d] = desc->n0[d];
  for (int d = 0; d < 6; d++) m->box[d] = desc->box[d];
  int rc = build_mesh_host(m);
  if (rc == EXF_OK) rc = upload_fe_table(m);
  if (rc != EXF_OK) {
    delete m;
    return rc;
  }
  *out = m;
  return EXF_OK;
}

int exf_mesh_destroy(exf_mesh *m) {
  if (!m) return EXF_OK;
  {
    std::lock_guard<std::mutex> g(m->sys_mu);
    if (!m->systems.empty()) {  // the last exf_sys_destroy frees it
      m->orphaned = true;
      return EXF_OK;
    }
  }
  cudaSetDevice(m->device);
  delete m;
  return EXF_OK;
}

int exf_mesh_info(const exf_mesh *m, int lev, int *nnodes, int *nel, int *nvert0) {
  if (!m || lev < 0 || lev >= m->nlev) {
    set_error("exf_mesh_info: bad level");
    return EXF_ERR_ARG;
  }
  if (nnodes) *nnodes = m->lev[lev].nnodes;
  if (nel) *nel = m->lev[lev].nel;
  if (nvert0) *nvert0 = m->nvert0;
  return EXF_OK;
}

int exf_mesh_get_xyz(const exf_mesh *m, double *xyz) {
  if (!m || !xyz) return EXF_ERR_ARG;
  EXF_TRY(mesh_pull_xyz(const_cast<exf_mesh *>(m)));
  memcpy(xyz, m->xyz.data(), m->xyz.size() * sizeof(double));
  return EXF_OK;
}

int exf_mesh_get_conn(const exf_mesh *m, int lev, int *conn, int *neigh, int *colour) {
  if (!m || lev < 0 || lev >= m->nlev) return EXF_ERR_ARG;
  const MeshLevel &ml = m->lev[lev];
  if (conn) memcpy(conn, ml.conn.data(), ml.conn.size() * sizeof(int));
  if (neigh) memcpy(neigh, ml.neigh.data(), ml.neigh.size() * sizeof(int));
  if (colour) memcpy(colour, ml.colour.data(), ml.colour.size() * sizeof(int));
  return EXF_OK;
}

static int sys_upload_bc(exf_sys *s) {
  int ntd = (int)s->bc0.size();
  EXF_CUDA(cudaMemcpyAsync(s->d_bc0.p, s->bc0.data(), ntd * sizeof(int), cudaMemcpyHostToDevice, s->stream));
  EXF_CUDA(cudaMemcpyAsync(s->d_bc1.p, s->bc1.data(), ntd * sizeof(int), cudaMemcpyHostToDevice, s->stream));
  EXF_TRY(update_rmask(s));
  // pressure gauge: first pressure node flagged Dirichlet (bc0 == 0)
  s->gauge_node = -1;
  if (s->kind == EXF_KIND_NS) {
    SysLevel &T = s->L[s->nlev - 1];
    for (int i = 0; i < T.NL; i++)
      if (s->bc0[(size_t)s->nv2 * T.N + i] == 0) {
        s->gauge_node = i;
        break;
      }
  }
  SysLevel &L0 = s->L[0];
  std::vector<double> gm(L0.ndof, 1.);
  if (s->gauge_node >= 0 && s->gauge_node < L0.NL) gm[(size_t)s->nv2 * L0.N + s->gauge_node] = 0.;
  EXF_TRY(s->gmask0.alloc(L0.ndof));
  EXF_CUDA(cudaMemcpyAsync(s->gmask0.p, gm.data(), gm.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  s->coarse_ok = 0;
  return EXF_OK;
}

int exf_sys_create(exf_mesh *m, int kind, exf_sys **out) {
  if (!m || !out || kind < EXF_KIND_T || kind > EXF_KIND_DS) {
    set_error("exf_sys_create: bad argument");
    return EXF_ERR_ARG;
  }
  EXF_CUDA(cudaSetDevice(m->device));
  exf_sys *s = new exf_sys();
  s->mesh = m;
  s->kind = kind;
  s->dim = m->dim;
  s->nlev = m->nlev;
  s->nv2 = kind == EXF_KIND_NS ? m->dim : 1;  // T, K, W, DS: one quadratic variable
  s->nv1 = kind == EXF_KIND_NS ? 1 : 0;
  s->nvars = s->nv2 + s->nv1;
  if (cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, m->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess) {
    set_error("exf_sys_create: stream/event creation failed");
    delete s;
    return EXF_ERR_CUDA;
  }
  s->L.resize(s->nlev);
  // MGSolDA::init_dof (src/MGSolverDA.C:880-951): host copy of _node_dof for the ABI
  s->node_dof.resize(s->nlev);
  for (int l = 0; l < s->nlev; l++) {
    int N = m->lev[l].nnodes, NL = l > 0 ? m->lev[l - 1].nnodes : m->nvert0;
    std::vector<int> &nd = s->node_dof[l];
    nd.assign((size_t)s->nvars * m->ntop, -1);
    int cnt = 0;
    for (int v = 0; v < s->nv2; v++)
      for (int k = 0; k < N; k++) nd[k + (size_t)v * m->ntop] = cnt++;
    for (int v = 0; v < s->nv1; v++)
      for (int k = 0; k < NL; k++) nd[k + (size_t)(s->nv2 + v) * m->ntop] = cnt++;
  }
  int rc = build_patterns(s);
  if (rc == EXF_OK) rc = build_colours(s);
  if (rc == EXF_OK) rc = build_transfers(s);
  int ntd = rc == EXF_OK ? s->L[s->nlev - 1].ndof : 0;
  if (rc == EXF_OK) {
    s->bc0.assign(ntd, 1);
    s->bc1.assign(ntd, 1);
    rc = s->d_bc0.alloc(ntd);
    if (rc == EXF_OK) rc = s->d_bc1.alloc(ntd);
    if (rc == EXF_OK) rc = s->xold.alloc(ntd);
    if (rc == EXF_OK) rc = s->xold.zero(s->stream);
    if (rc == EXF_OK) rc = s->src_qe.alloc(m->lev[s->nlev - 1].nel);
    if (rc == EXF_OK) rc = s->src_qe.zero(s->stream);
    if (rc == EXF_OK) rc = s->red.out.alloc(16);
    if (rc == EXF_OK) rc = s->wait_flag.alloc(1);
    if (rc == EXF_OK) rc = s->wait_flag.zero(s->stream);
    if (rc == EXF_OK) rc = sys_upload_bc(s);
  }
  if (rc != EXF_OK) {
    exf_sys_destroy(s);
    return rc;
  }
  {
    std::lock_guard<std::mutex> g(m->sys_mu);
    m->systems.push_back(s);
  }
  *out = s;
  return EXF_OK;
}

int exf_sys_destroy(exf_sys *s) {
  if (!s) return EXF_OK;
  exf_mesh *const m = s->mesh;
  bool drop_mesh = false;
  {  // no partner keeps a pointer to s (their next assembly reports the missing coupling)
    std::lock_guard<std::mutex> g(m->sys_mu);
    for (exf_sys *o : m->systems) {
      if (o->other == s) o->other = nullptr;
      if (o->turb == s) o->turb = nullptr;
      if (o->ns_k == s) o->ns_k = nullptr;
      if (o->ns_w == s) o->ns_w = nullptr;
      if (o->ds_x == s) o->ds_x = nullptr;
    }
    for (size_t k = 0; k < m->systems.size(); k++)
      if (m->systems[k] == s) {
        m->systems.erase(m->systems.begin() + k);
        break;
      }
    drop_mesh = m->orphaned && m->systems.empty();
  }
  cudaSetDevice(s->mesh->device);
  for (int k = 0; k < exf_sys::kGraphSlots; k++) {
    if (s->cyc_slot[k].exec) cudaGraphExecDestroy(s->cyc_slot[k].exec);
    if (s->loop_slot[k].exec) cudaGraphExecDestroy(s->loop_slot[k].exec);
  }
  if (s->stream) cudaStreamSynchronize(s->stream);
  s->L.clear();
  for (int k = 0; k < 8; k++)
    if (s->user_ev[k]) cudaEventDestroy(s->user_ev[k]);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  if (drop_mesh) {  // exf_mesh_destroy came first
    cudaSetDevice(m->device);
    delete m;
  }
  return EXF_OK;
}

int exf_sys_ndof(const exf_sys *s, int lev, int *ndof) {
  CHECK_LEV(s, lev);
  *ndof = s->L[lev].ndof;
  return EXF_OK;
}

int exf_sys_get_node_dof(const exf_sys *s, int lev, int *node_dof) {
  CHECK_LEV(s, lev);
  memcpy(node_dof, s->node_dof[lev].data(), s->node_dof[lev].size() * sizeof(int));
  return EXF_OK;
}

// bc_read presets: flags are functions of the node coordinates (GenBc_loop,
// src/MGSolverDA.C:781-865; User_NS.C bc_read)
int exf_sys_bc_preset(exf_sys *s, int preset) {
  CHECK_SYS(s);
  exf_mesh *m = s->mesh;
  const int top = s->nlev - 1, dim = m->dim;
  const SysLevel &T = s->L[top];
  std::fill(s->bc0.begin(), s->bc0.end(), 1);
  std::fill(s->bc1.begin(), s->bc1.end(), 1);
  if (preset < 1 || preset > 5) {
    set_error("unknown bc preset %d", preset);
    return EXF_ERR_ARG;
  }
  // pressure gauge node of the enclosed-flow presets: node 0 of a generated box (its
  // corner (x0, y0, z0)); on an uploaded mesh the pressure node first in (z, y, x) order
  // of the coordinates, the same physical node whatever the numbering
  int gauge = 0;
  if (!m->lattice && s->nv1) gauge = node_zyx_order(m, T.NL)[0];
  // walls: lattice planes of a generated box; for uploaded meshes the faces of the
  // coordinate bounding box (within 1e-10 of its extent)
  for (int n = 0; n < m->ntop; n++) {
    int lo[3], hi[3], onb = 0;
    for (int d = 0; d < 3; d++) {
      if (m->lattice) {
        const int *p = &m->lat[3 * n];
        lo[d] = d < dim && p[d] == 0;
        hi[d] = d < dim && p[d] == m->L[d] - 1;
      } else {
        const double x = d < dim ? m->xyz[(size_t)n + (size_t)d * m->ntop] : 0.;
        const double tol = 1e-10 * std::max(m->box[2 * d + 1] - m->box[2 * d], 1e-300);
        lo[d] = d < dim && fabs(x - m->box[2 * d]) <= tol;
        hi[d] = d < dim && fabs(x - m->box[2 * d + 1]) <= tol;
      }
      onb |= lo[d] | hi[d];
    }
    if (!onb) continue;  // interior nodes keep (1,1) (bc_intern_read)
    for (int v = 0; v < s->nvars; v++) {
      const bool quad = v < s->nv2;
      if (!quad && n >= T.NL) continue;
      const size_t dof = quad ? (size_t)v * T.N + n : (size_t)s->nv2 * T.N + n;
      int b0 = 1, b1 = 0;
      switch (preset) {
        case EXF_BC_HEAT_DIRICHLET:
          b0 = 0;
          b1 = 0;
          break;
        case EXF_BC_CAVITY:
          if (quad) {
            b0 = 0;
            b1 = (v == 0 && hi[1] && !lo[0] && !hi[0]) ? 4 : 0;
          } else if (n == gauge) {
            b0 = 0;  // pressure gauge node
          }
          break;
        case EXF_BC_CHANNEL:
          if (quad) {
            int wall = lo[1] || hi[1] || lo[2] || hi[2];
            if (wall || lo[0]) {
              b0 = 0;
              b1 = (v == 0 && lo[0] && !wall) ? 4 : 0;
            }
          }
          break;
        case EXF_BC_BOUSS_NS:
          if (quad) {
            b0 = 0;
            b1 = 0;
          } else if (n == gauge) {
            b0 = 0;
          }
          break;
        case EXF_BC_BOUSS_T:
          if (lo[0]) {
            b0 = 0;
            b1 = 1;
          } else if (hi[0]) {
            b0 = 0;
            b1 = 0;
          }
          break;
      }
      s->bc0[dof] = b0;
      s->bc1[dof] = b1;
    }
  }
  return sys_upload_bc(s);
}

int exf_sys_set_bc(exf_sys *s, const int *bc0, const int *bc1) {
  CHECK_SYS(s);
  if (!bc0 || !bc1) return EXF_ERR_ARG;
  memcpy(s->bc0.data(), bc0, s->bc0.size() * sizeof(int));
  memcpy(s->bc1.data(), bc1, s->bc1.size() * sizeof(int));
  return sys_upload_bc(s);
}

int exf_sys_get_bc(const exf_sys *s, int *bc0, int *bc1) {
  CHECK_SYS(s);
  if (bc0) memcpy(bc0, s->bc0.data(), s->bc0.size() * sizeof(int));
  if (bc1) memcpy(bc1, s->bc1.data(), s->bc1.size() * sizeof(int));
  return EXF_OK;
}

int exf_sys_nnz(const exf_sys *s, int lev, long *nnz) {
  CHECK_LEV(s, lev);
  *nnz = s->L[lev].nnz;
  return EXF_OK;
}

int exf_sys_get_pattern(exf_sys *s, int lev, int *rowptr, int *col) {
  CHECK_LEV(s, lev);
  SysLevel &L = s->L[lev];
  if (rowptr)
    EXF_CUDA(cudaMemcpyAsync(rowptr, L.csr_ptr.p, (L.ndof + 1) * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  if (col) EXF_CUDA(cudaMemcpyAsync(col, L.csr_col.p, L.nnz * sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  return EXF_OK;
}

// expand a node-level transfer to DOF level: row (a, node) -> columns (a, node')
static void expand_transfer(const exf_sys *s, const Transfer &Tq, const Transfer &Tl, int nrow_q, int ncol_q,
                            int nrow_l, int ncol_l, const double *mask, std::vector<int> &ptr,
                            std::vector<int> &col, std::vector<double> &val) {
  ptr.assign(1, 0);
  col.clear();
  val.clear();
  int row = 0;
  for (int a = 0; a < s->nv2; a++)
    for (int i = 0; i < nrow_q; i++, row++) {
      for (int q = Tq.h_ptr[i]; q < Tq.h_ptr[i + 1]; q++) {
        col.push_back(a * ncol_q + Tq.h_col[q]);
        val.push_back(Tq.h_val[q] * (mask ? mask[row] : 1.));
      }
      ptr.push_back((int)col.size());
    }
  if (s->nv1)
    for (int i = 0; i < nrow_l; i++, row++) {
      for (int q = Tl.h_ptr[i]; q < Tl.h_ptr[i + 1]; q++) {
        col.push_back(s->nv2 * ncol_q + Tl.h_col[q]);
        val.push_back(Tl.h_val[q] * (mask ? mask[row] : 1.));
      }
      ptr.push_back((int)col.size());
    }
}

int exf_sys_set_transfer(exf_sys *s, int lev, int kind, int block, const int dim[2], const int *len, const int *pos,
                         const double *val) {
  CHECK_LEV(s, lev);
  return set_transfer(s, lev, kind, block, dim, len, pos, val);
}

int exf_sys_get_transfer(exf_sys *s, int lev, int kind, int block, int dim[2], long *nnz, int *len, int *pos,
                         double *val) {
  CHECK_LEV(s, lev);
  if ((kind != 0 && kind != 1) || (block != 1 && block != 2) || !dim || !nnz || (block == 1 && !s->nv1)) {
    set_error("exf_sys_get_transfer: bad argument");
    return EXF_ERR_ARG;
  }
  const int other = kind == 0 ? lev - 1 : lev + 1;
  if (other < 0 || other >= s->nlev) {
    set_error("exf_sys_get_transfer: no level %d next to level %d", other, lev);
    return EXF_ERR_ARG;
  }
  const SysLevel &L = s->L[lev], &O = s->L[other];
  const Transfer &T = kind == 0 ? (block == 2 ? L.Pq : L.Pl) : (block == 2 ? L.Rq : L.Rl);
  const int nrow = block == 2 ? L.N : L.NL, ncol = block == 2 ? O.N : O.NL;
  if (T.nrow != nrow || (int)T.h_ptr.size() != nrow + 1) {
    set_error("exf_sys_get_transfer: the %s block %d of level %d has not been built or supplied",
              kind == 0 ? "prolongation" : "restriction", block, lev);
    return EXF_ERR_STATE;
  }
  dim[0] = nrow;
  dim[1] = ncol;
  *nnz = T.h_ptr[nrow];
  if (len) std::copy(T.h_ptr.begin(), T.h_ptr.end(), len);
  if (pos) std::copy(T.h_col.begin(), T.h_col.end(), pos);
  if (val) std::copy(T.h_val.begin(), T.h_val.end(), val);
  return EXF_OK;
}

int exf_sys_check_pattern(exf_sys *s, int lev, int block, const int dim[2], const int *len, const int *pos) {
  CHECK_LEV(s, lev);
  SysLevel &L = s->L[lev];
  if (!dim || !len || !pos || (block != 22 && block != 21 && block != 12 && block != 11) ||
      (block != 22 && !s->nv1)) {
    set_error("exf_sys_check_pattern: bad argument");
    return EXF_ERR_ARG;
  }
  const bool qrow = block / 10 == 2, qcol = block % 10 == 2;
  const int nrow = qrow ? L.N : L.NL, ncol = qcol ? L.N : L.NL;
  if (dim[0] != nrow || dim[1] != ncol) {
    set_error("exf_sys_check_pattern: block %d is %dx%d, level %d has %dx%d", block, dim[0], dim[1], lev, nrow, ncol);
    return EXF_ERR_ARG;
  }
  std::vector<int> p(L.N + 1), c(qcol ? L.nqq : L.nql);
  EXF_CUDA(cudaMemcpy(p.data(), qcol ? L.qq_ptr.p : L.ql_ptr.p, (L.N + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  EXF_CUDA(cudaMemcpy(c.data(), qcol ? L.qq_col.p : L.ql_col.p, c.size() * sizeof(int), cudaMemcpyDeviceToHost));
  std::vector<int> row;
  for (int i = 0; i < nrow; i++) {  // the pressure rows of node m use the node's lists
    if (len[i + 1] < len[i]) {
      set_error("exf_sys_check_pattern: row offsets decrease at row %d", i);
      return EXF_ERR_ARG;
    }
    row.assign(pos + len[i], pos + len[i + 1]);
    std::sort(row.begin(), row.end());
    if (row.size() != (size_t)(p[i + 1] - p[i]) || !std::equal(row.begin(), row.end(), c.begin() + p[i])) {
      set_error("exf_sys_check_pattern: block %d row %d differs from the element couplings (%zu entries, %d built)",
                block, i, row.size(), p[i + 1] - p[i]);
      return EXF_ERR_ARG;
    }
  }
  return EXF_OK;
}

static int need_transfers(const exf_sys *s) {
  if (transfers_ready(s)) return EXF_OK;
  set_error("the transfer operators are not set (exf_sys_set_transfer for every level and block)");
  return EXF_ERR_STATE;
}

int exf_sys_get_prol(exf_sys *s, int lev, long *nnz, int *rowptr, int *col, double *val) {
  CHECK_LEV(s, lev);
  if (lev == 0) {
    set_error("no prolongation into level 0");
    return EXF_ERR_ARG;
  }
  EXF_TRY(need_transfers(s));
  const SysLevel &F = s->L[lev], &C = s->L[lev - 1];
  std::vector<int> p, c;
  std::vector<double> v;
  expand_transfer(s, F.Pq, F.Pl, F.N, C.N, F.NL, C.NL, nullptr, p, c, v);
  if (nnz) *nnz = (long)c.size();
  if (rowptr) memcpy(rowptr, p.data(), p.size() * sizeof(int));
  if (col) memcpy(col, c.data(), c.size() * sizeof(int));
  if (val) memcpy(val, v.data(), v.size() * sizeof(double));
  return EXF_OK;
}

int exf_sys_get_rest(exf_sys *s, int lev, long *nnz, int *rowptr, int *col, double *val) {
  CHECK_LEV(s, lev);
  if (lev == s->nlev - 1) {
    set_error("no restriction from above the top level");
    return EXF_ERR_ARG;
  }
  EXF_TRY(need_transfers(s));
  const SysLevel &C = s->L[lev], &F = s->L[lev + 1];
  std::vector<double> mask(C.ndof);
  EXF_CUDA(cudaMemcpyAsync(mask.data(), C.rmask.p, C.ndof * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  std::vector<int> p, c;
  std::vector<double> v;
  expand_transfer(s, C.Rq, C.Rl, C.N, F.N, C.NL, F.NL, mask.data(), p, c, v);
  if (nnz) *nnz = (long)c.size();
  if (rowptr) memcpy(rowptr, p.data(), p.size() * sizeof(int));
  if (col) memcpy(col, c.data(), c.size() * sizeof(int));
  if (val) memcpy(val, v.data(), v.size() * sizeof(double));
  return EXF_OK;
}

int exf_sys_get_colours(exf_sys *s, int lev, int *ncolours, int *colour_of_item) {
  CHECK_LEV(s, lev);
  SysLevel &L = s->L[lev];
  if (ncolours) *ncolours = L.ncolour;
  if (colour_of_item)
    EXF_CUDA(cudaMemcpyAsync(colour_of_item, L.item_colour.p, L.item_colour.n * sizeof(int), cudaMemcpyDeviceToHost,
                             s->stream));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  return EXF_OK;
}

int exf_sys_couple(exf_sys *s, exf_sys *other) {
  CHECK_SYS(s);
  if (other && other->mesh != s->mesh) {
    set_error("coupled systems must share the mesh");
    return EXF_ERR_ARG;
  }
  const bool kw = s->kind == EXF_KIND_K || s->kind == EXF_KIND_W;
  if (s->kind == EXF_KIND_DS && other && other->kind == EXF_KIND_DS) {
    s->ds_x = other;  // the x displacement the boundary rows read
  } else if (s->kind == EXF_KIND_NS && other && (other->kind == EXF_KIND_K || other->kind == EXF_KIND_W)) {
    (other->kind == EXF_KIND_K ? s->ns_k : s->ns_w) = other;  // the eddy viscosity's fields
  } else if (kw && other && (other->kind == EXF_KIND_K || other->kind == EXF_KIND_W)) {
    if (other->kind == s->kind) {
      set_error("a kappa (omega) system couples to an omega (kappa) system");
      return EXF_ERR_ARG;
    }
    s->turb = other;  // the other turbulence variable
  } else {
    s->other = other;
  }
  return EXF_OK;
}

int exf_sys_set_wall(exf_sys *s, const double *dist, double nu_wall) {
  CHECK_SYS(s);
  if (!dist || (s->kind != EXF_KIND_K && s->kind != EXF_KIND_W)) return EXF_ERR_ARG;
  std::vector<long> off(1, 0);
  for (int l = 0; l < s->nlev; l++) off.push_back(off.back() + s->mesh->lev[l].nel);
  for (long e = 0; e < off.back(); e++)
    if (!(dist[e] > 0.)) {
      set_error("exf_sys_set_wall: element %ld has wall distance %g", e, dist[e]);
      return EXF_ERR_ARG;
    }
  EXF_TRY(s->wall_dist.ensure(off.back()));
  EXF_CUDA(cudaMemcpyAsync(s->wall_dist.p, dist, off.back() * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  s->wall_off = off;
  s->nu_wall = nu_wall;
  return EXF_OK;
}

int exf_sys_set_ds(exf_sys *s, int dir, double dt, const double *u_fsi, const double *d_old) {
  CHECK_SYS(s);
  if (s->kind != EXF_KIND_DS || dir < 0 || dir >= s->mesh->dim || !(dt > 0.) || (!u_fsi != !d_old)) {
    set_error("exf_sys_set_ds: needs a displacement system, 0 <= dir < dim, dt > 0 and both fields or none");
    return EXF_ERR_ARG;
  }
  s->ds_dir = dir;
  s->ds_dt = dt;
  s->ds_host = u_fsi != nullptr;
  if (!u_fsi) return EXF_OK;  // coupled: the fields are the systems' x_old on the device
  const size_t n = (size_t)s->mesh->dim * s->mesh->ntop;
  EXF_TRY(s->ds_u.ensure(n));
  EXF_TRY(s->ds_d.ensure(n));
  EXF_CUDA(cudaMemcpyAsync(s->ds_u.p, u_fsi, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  EXF_CUDA(cudaMemcpyAsync(s->ds_d.p, d_old, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  return EXF_OK;
}

int exf_sys_set_mesh_motion(exf_sys *s, int moving) {
  CHECK_SYS(s);
  if (s->kind != EXF_KIND_DS) return EXF_ERR_ARG;
  s->ds_move = moving != 0;
  return EXF_OK;
}


static int h2d(exf_sys *s, double *d, const double *h, size_t n) {
  if (!h) return EXF_ERR_ARG;
  EXF_CUDA(cudaMemcpyAsync(d, h, n * sizeof(double), cudaMemcpyHostToDevice, s->stream));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  return EXF_OK;
}
static int d2h(exf_sys *s, double *h, const double *d, size_t n) {
  if (!h) return EXF_ERR_ARG;
  EXF_CUDA(cudaMemcpyAsync(h, d, n * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  return EXF_OK;
}

int exf_sys_set_xold(exf_sys *s, const double *x) {
  CHECK_SYS(s);
  return h2d(s, s->xold.p, x, s->xold.n);
}
int exf_sys_get_xold(exf_sys *s, double *x) {
  CHECK_SYS(s);
  return d2h(s, x, s->xold.p, s->xold.n);
}
int exf_sys_set_x(exf_sys *s, const double *x) {
  CHECK_SYS(s);
  SysLevel &T = s->L[s->nlev - 1];
  return h2d(s, T.x.p, x, T.ndof);
}
int exf_sys_get_x(exf_sys *s, double *x) {
  CHECK_SYS(s);
  SysLevel &T = s->L[s->nlev - 1];
  return d2h(s, x, T.x.p, T.ndof);
}
int exf_sys_xold_update(exf_sys *s) {
  CHECK_SYS(s);
  SysLevel &T = s->L[s->nlev - 1];
  if (s->kind == EXF_KIND_DS && s->ds_move) EXF_TRY(ds_move_mesh(s));  // FINE_MOVEMENT
  EXF_CUDA(cudaMemcpyAsync(s->xold.p, T.x.p, T.ndof * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
  // coupled systems read this x_old (and the moved mesh) from their own streams
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  return EXF_OK;
}
int exf_sys_set_source(exf_sys *s, const double *qe) {
  CHECK_SYS(s);
  return h2d(s, s->src_qe.p, qe, s->src_qe.n);
}
int exf_sys_set_rhs(exf_sys *s, const double *b) {
  CHECK_SYS(s);
  SysLevel &T = s->L[s->nlev - 1];
  return h2d(s, T.b.p, b, T.ndof);
}
int exf_sys_get_rhs(exf_sys *s, double *b) {
  CHECK_SYS(s);
  SysLevel &T = s->L[s->nlev - 1];
  return d2h(s, b, T.b.p, T.ndof);
}

int exf_gen_mat_rhs(exf_sys *s, const exf_phys *ph, int lev, int mode) {
  CHECK_LEV(s, lev);
  if (!ph || (mode != 0 && mode != 1)) return EXF_ERR_ARG;
  if (s->kind == EXF_KIND_NS && s->mesh->dim == 3 && s->nv2 != 3) return EXF_ERR_STATE;
  if (s->kind == EXF_KIND_K || s->kind == EXF_KIND_W) EXF_TRY(assemble_kw_level(s, ph, lev, mode));
  else if (s->kind == EXF_KIND_DS) EXF_TRY(assemble_ds_level(s, lev, mode));
  else EXF_TRY(assemble_level(s, ph, lev, mode));
  EXF_TRY(sync_fp32(s, lev));
  if (lev == 0) s->coarse_ok = 0;
  s->assembled = 1;
  return EXF_OK;
}

// GenMatRhs of every level (the top one with its rhs); for T and NS the levels' elements
// of one colour in one launch
static int assemble_every_level(exf_sys *s, const exf_phys *ph) {
  if (s->kind == EXF_KIND_K || s->kind == EXF_KIND_W) {
    for (int l = s->nlev - 1; l >= 0; l--) EXF_TRY(assemble_kw_level(s, ph, l, l == s->nlev - 1 ? 1 : 0));
  } else if (s->kind == EXF_KIND_DS) {
    for (int l = s->nlev - 1; l >= 0; l--) EXF_TRY(assemble_ds_level(s, l, l == s->nlev - 1 ? 1 : 0));
  } else {
    EXF_TRY(assemble_all_levels(s, ph));
  }
  return EXF_OK;
}

int exf_assemble_all(exf_sys *s, const exf_phys *ph) {
  CHECK_SYS(s);
  if (!ph) return EXF_ERR_ARG;
  if (s->kind == EXF_KIND_NS && s->mesh->dim == 3 && s->nv2 != 3) return EXF_ERR_STATE;
  EXF_TRY(assemble_every_level(s, ph));
  for (int l = 0; l < s->nlev; l++) EXF_TRY(sync_fp32(s, l));
  s->coarse_ok = 0;
  s->assembled = 1;
  return EXF_OK;
}

int exf_get_matrix(exf_sys *s, int lev, double *val) {
  CHECK_LEV(s, lev);
  SysLevel &L = s->L[lev];
  DBuf<double> d;
  EXF_TRY(d.alloc(L.nnz));
  EXF_TRY(csr_values(s, lev, d.p));
  return d2h(s, val, d.p, L.nnz);
}

int exf_set_matrix(exf_sys *s, int lev, const double *val) {
  CHECK_LEV(s, lev);
  SysLevel &L = s->L[lev];
  DBuf<double> d;
  EXF_TRY(d.alloc(L.nnz));
  EXF_TRY(h2d(s, d.p, val, L.nnz));
  EXF_TRY(csr_set_values(s, lev, d.p));
  EXF_TRY(sync_fp32(s, lev));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  if (lev == 0) s->coarse_ok = 0;
  s->assembled = 1;
  return EXF_OK;
}

int exf_sys_transpose(exf_sys *s) {
  CHECK_SYS(s);
  for (int l = 0; l < s->nlev; l++) EXF_TRY(transpose_level(s, l));
  s->coarse_ok = 0;
  s->transposed ^= 1;
  return EXF_OK;
}

// ------------------------------------------------------------------ solve
// one outer cycle; leaves ||b - A x||^2 of the top level in *dnr
static int cycle_body(exf_sys *s, const exf_mg_params *p, double *dnr) {
  SysLevel &T = s->L[s->nlev - 1];
  if (p->precision == EXF_PREC_MIXED) {
    EXF_TRY(vcycle_mixed(s, p));
    return spmv_resid<double>(s, s->nlev - 1, T.x.p, T.b.p, T.r.p, dnr);
  }
  return vcycle_fp64(s, p, dnr);
}

static unsigned long long params_key(const exf_mg_params *p) {
  unsigned long long h = 1469598103934665603ull;
  auto mix = [&](unsigned long long v) {
    h ^= v;
    h *= 1099511628211ull;
  };
  mix((unsigned long long)p->gamma);
  mix((unsigned long long)p->nu_pre);
  mix((unsigned long long)p->nu_post);
  mix((unsigned long long)p->double_below_top);
  mix((unsigned long long)p->smoother);
  unsigned long long w, c;
  memcpy(&w, &p->omega, 8);
  memcpy(&c, &p->corr_damp, 8);
  mix(w);
  mix(c);
  mix((unsigned long long)p->reverse_colours);
  mix((unsigned long long)p->precision);
  mix((unsigned long long)p->vanka_kernel);
  mix((unsigned long long)p->cond_corr);
  mix((unsigned long long)p->stop_test);
  mix((unsigned long long)p->fp32_blocks);
  if (p->smoother == EXF_SMOOTH_GMRES_ILU) {  // the level solver's accuracy test is in its kernels
    unsigned long long e;
    memcpy(&e, &p->eps, 8);
    mix(e);
    mix((unsigned long long)p->coarse_iters);
  }
  return h | 1ull;
}

// the slot holding (key, current epoch), or an emptied slot to build it in (*hit false):
// a free one, else the least recently used
static exf_sys::GraphSlot *graph_slot(exf_sys *s, exf_sys::GraphSlot *slots, unsigned long long key, bool *hit) {
  exf_sys::GraphSlot *victim = &slots[0];
  for (int k = 0; k < exf_sys::kGraphSlots; k++) {
    exf_sys::GraphSlot &g = slots[k];
    if (g.exec && g.key == key && g.epoch == s->buf_epoch) {
      g.used = ++s->graph_clock;
      *hit = true;
      return &g;
    }
    if (!g.exec) {
      if (victim->exec) victim = &g;
    } else if (victim->exec && g.used < victim->used) {
      victim = &g;
    }
  }
  if (victim->exec) cudaGraphExecDestroy(victim->exec);
  *victim = exf_sys::GraphSlot();
  victim->used = ++s->graph_clock;
  *hit = false;
  return victim;
}

static int cycle_graph(exf_sys *s, const exf_mg_params *p, double *dnr) {
  const unsigned long long key = params_key(p);
  bool hit = false;
  exf_sys::GraphSlot *gs = graph_slot(s, s->cyc_slot, key, &hit);
  if (!hit) {
    cudaGraph_t g = nullptr;
    const long long c0 = exf_launch_count();
    EXF_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int rc = cycle_body(s, p, dnr);
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (rc != EXF_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) {
      set_error("graph capture failed: %s", cudaGetErrorString(e));
      return EXF_ERR_CUDA;
    }
    e = cudaGraphInstantiate(&gs->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      set_error("graph instantiation failed: %s", cudaGetErrorString(e));
      gs->exec = nullptr;
      return EXF_ERR_CUDA;
    }
    gs->key = key;
    gs->epoch = s->buf_epoch;
    gs->launches = exf_launch_count() - c0;
    count_launch(-(int)gs->launches);  // captured, not executed
  }
  EXF_CUDA(cudaGraphLaunch(gs->exec, s->stream));
  count_launch((int)gs->launches);
  return EXF_OK;
}

// The check at the end of every device-loop iteration: record the cycle's relative
// residual, apply the stop test and set the WHILE condition (continue while not converged,
// finite and below max_cycles).
__global__ void k_cycle_check(cudaGraphConditionalHandle h, LoopDev *st, const double *r2, const double *acc2) {
  const double rel = sqrt(*r2) / st->den;
  const int c = st->cycles;
  if (c < 256) st->hist[c] = rel;
  st->cycles = c + 1;
  st->rel = rel;
  const double acc = (acc2 && !st->mixed) ? sqrt(*acc2) / st->den : rel;
  st->last_acc = acc;
  const bool done = st->ref_stop ? acc < st->lim : rel <= st->lim;
  const bool go = isfinite(rel) && !done && c + 1 < st->max_cycles;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// Cycles until convergence inside one graph launch: a conditional WHILE node whose body is
// the captured V-cycle followed by k_cycle_check.  Returns EXF_ERR_UNSUPPORTED (and never
// tries again for this system) when the runtime does not build such a graph; the caller
// then loops on the host.
static int cycle_body(exf_sys *s, const exf_mg_params *p, double *dnr);
static unsigned long long params_key(const exf_mg_params *p);
static int device_loop(exf_sys *s, const exf_mg_params *p, exf_solve_stats *st, double den, double lim,
                       bool ref_stop, double *dnr) {
  const unsigned long long key = params_key(p);
  if (!s->loop_dev.p) EXF_TRY(s->loop_dev.alloc(1));
  bool hit = false;
  exf_sys::GraphSlot *gs = graph_slot(s, s->loop_slot, key, &hit);
  if (!hit) {
    cudaGraph_t g = nullptr;
    cudaGraphConditionalHandle h;
    cudaGraphNodeParams np = {};
    cudaGraphNode_t node;
    bool ok = cudaGraphCreate(&g, 0) == cudaSuccess &&
              cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
      np.type = cudaGraphNodeTypeConditional;
      np.conditional.handle = h;
      np.conditional.type = cudaGraphCondTypeWhile;
      np.conditional.size = 1;
      ok = cudaGraphAddNode(&node, g, nullptr, 0, &np) == cudaSuccess;
    }
    cudaGraph_t body = ok ? np.conditional.phGraph_out[0] : nullptr;
    const long long c0 = exf_launch_count();
    if (ok) ok = cudaStreamBeginCaptureToGraph(s->stream, body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    int rc = EXF_OK;
    if (ok) {
      rc = cycle_body(s, p, dnr);
      if (rc == EXF_OK) {
        const double *acc2 = needs_acc(p) ? s->mg_acc.p + 4 * (s->nlev - 1) + 2 : nullptr;
        k_cycle_check<<<1, 1, 0, s->stream>>>(h, s->loop_dev.p, dnr, acc2);
        count_launch(1);
      }
      cudaGraph_t cap = body;
      ok = cudaStreamEndCapture(s->stream, &cap) == cudaSuccess && rc == EXF_OK;
    }
    gs->launches = exf_launch_count() - c0;
    count_launch(-(int)gs->launches);  // captured, not executed
    if (ok) ok = cudaGraphInstantiate(&gs->exec, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    if (rc != EXF_OK) {
      if (gs->exec) cudaGraphExecDestroy(gs->exec);
      gs->exec = nullptr;
      return rc;
    }
    if (!ok) {
      gs->exec = nullptr;
      s->loop_unavailable = 1;
      return EXF_ERR_UNSUPPORTED;
    }
    gs->key = key;
    gs->epoch = s->buf_epoch;
  }
  LoopDev hd = {};
  hd.den = den;
  hd.lim = lim;
  hd.max_cycles = p->max_cycles;
  hd.cycles = st->cycles;
  hd.ref_stop = ref_stop ? 1 : 0;
  hd.mixed = p->precision == EXF_PREC_MIXED ? 1 : 0;
  EXF_CUDA(cudaMemcpyAsync(s->loop_dev.p, &hd, offsetof(LoopDev, hist), cudaMemcpyHostToDevice, s->stream));
  EXF_CUDA(cudaGraphLaunch(gs->exec, s->stream));
  EXF_CUDA(cudaMemcpyAsync(&hd, s->loop_dev.p, sizeof(LoopDev), cudaMemcpyDeviceToHost, s->stream));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  count_launch((int)(gs->launches * (hd.cycles - st->cycles)));
  for (int c = st->cycles; c < hd.cycles && c < 256; c++) st->hist[c] = hd.hist[c];
  st->cycles = hd.cycles;
  st->rel_res = hd.rel;
  st->last_acc = hd.last_acc;
  return EXF_OK;
}

static int read_scalar(exf_sys *s, const double *d, double *h) {
  EXF_CUDA(cudaMemcpyAsync(h, d, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  return EXF_OK;
}

int exf_mg_solve(exf_sys *s, const exf_mg_params *p, exf_solve_stats *st) {
  CHECK_SYS(s);
  if (!p || !st) return EXF_ERR_ARG;
  if (!s->assembled) {
    set_error("exf_mg_solve before assembly");
    return EXF_ERR_STATE;
  }
  EXF_TRY(need_transfers(s));
  if (p->gamma < 1 || p->nu_pre < 0 || p->nu_post < 0 || p->max_cycles < 0 || p->coarse_iters < 0 ||
      (p->stop_test != EXF_STOP_RELRES && p->stop_test != EXF_STOP_REFERENCE))
    return EXF_ERR_ARG;
  if (needs_acc(p) && s->mg_acc.n != (size_t)4 * s->nlev) {
    EXF_TRY(s->mg_acc.alloc(4 * (size_t)s->nlev));
    EXF_TRY(s->mg_acc.zero(s->stream));
    s->buf_epoch++;
  }
  memset(st, 0, sizeof(*st));
  SysLevel &T = s->L[s->nlev - 1];
  double *dnb = s->red.out.p, *dnr = s->red.out.p + 1;
  if (p->smoother == EXF_SMOOTH_GMRES_ILU) {
    if (p->precision != EXF_PREC_FP64) {
      set_error("GMRES + ILU smoothing runs in FP64 precision only");
      return EXF_ERR_UNSUPPORTED;
    }
    for (int l = p->coarse_iters > 0 ? 0 : 1; l < s->nlev; l++) EXF_TRY(ilu_ready(s, l));  // once per assembly
  }
  if (!s->coarse_ok) EXF_TRY(coarse_factor(s));
  EXF_CUDA(cudaEventRecord(s->ev0, s->stream));
  EXF_TRY(norm2(s, T.b.p, T.ndof, dnb));
  double bn2 = 0.;
  EXF_TRY(read_scalar(s, dnb, &bn2));
  double bn = sqrt(bn2);
  st->bnorm = bn;
  const double den = bn > 0. ? bn : 1.;
  // initial residual
  EXF_TRY(spmv_resid<double>(s, s->nlev - 1, T.x.p, T.b.p, T.r.p, dnr));
  double r2 = 0.;
  EXF_TRY(read_scalar(s, dnr, &r2));
  double rel = sqrt(r2) / den;
  st->rel_res = rel;
  int rc = EXF_OK;
  // stop tests: ||b-Ax||/||b|| <= eps, or the reference's exit test rest < eps*(1+||b||)
  // (src/MGSolverBase.C:201) with rest the top level's accuracy of the last cycle (FP64; in
  // mixed precision the top level of the FP32 cycle solves for the correction, so rest is
  // the FP64 outer relative residual there)
  const bool ref_stop = p->stop_test == EXF_STOP_REFERENCE;
  const double lim = ref_stop ? p->eps * (1. + bn) : p->eps;
  bool done = !ref_stop && rel <= p->eps;
  if (!std::isfinite(rel) || !std::isfinite(bn)) {
    set_error("multigrid diverged: non-finite initial residual or rhs");
    rc = EXF_ERR_DIVERGED;
    done = true;  // skip the cycle loop
  }
  while (!done && st->cycles < p->max_cycles) {
    // the first cycle runs eagerly (it sizes every scratch buffer); with use_graph the
    // later cycles run on the device until the stop test holds (one graph launch, no host
    // read per cycle), or, where the runtime cannot build that graph, replay a captured
    // graph of one cycle per host iteration
    if (p->use_graph && st->cycles > 0 && !s->loop_unavailable) {
      const int lrc = device_loop(s, p, st, den, lim, ref_stop, dnr);
      if (lrc == EXF_OK) {
        rel = st->rel_res;
        if (!std::isfinite(rel)) {
          rc = EXF_ERR_DIVERGED;
          set_error("multigrid diverged at cycle %d", st->cycles);
          break;
        }
        done = ref_stop ? st->last_acc < lim : rel <= p->eps;
        continue;
      }
      if (lrc != EXF_ERR_UNSUPPORTED) return lrc;
    }
    if (p->use_graph && st->cycles > 0) {
      EXF_TRY(cycle_graph(s, p, dnr));
    } else {
      EXF_TRY(cycle_body(s, p, dnr));
    }
    EXF_TRY(read_scalar(s, dnr, &r2));
    rel = sqrt(r2) / den;
    if (st->cycles < 256) st->hist[st->cycles] = rel;
    st->cycles++;
    st->rel_res = rel;
    st->last_acc = rel;
    if (needs_acc(p) && p->precision != EXF_PREC_MIXED) {
      double a2 = 0.;
      EXF_TRY(read_scalar(s, s->mg_acc.p + 4 * (s->nlev - 1) + 2, &a2));
      st->last_acc = sqrt(a2) / den;
    }
    if (!std::isfinite(rel)) {
      rc = EXF_ERR_DIVERGED;
      set_error("multigrid diverged at cycle %d", st->cycles);
      break;
    }
    done = ref_stop ? st->last_acc < lim : rel <= p->eps;
  }
  EXF_CUDA(cudaEventRecord(s->ev1, s->stream));
  EXF_CUDA(cudaEventSynchronize(s->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, s->ev0, s->ev1);
  st->seconds = ms * 1e-3;
  EXF_TRY(device_wait_status(s));
  st->converged = rc == EXF_OK && (ref_stop ? (st->cycles > 0 && st->last_acc < lim) : rel <= p->eps);
  if (rc == EXF_OK && !st->converged) {
    set_error("not converged: rel %.3e after %d cycles", rel, st->cycles);
    rc = EXF_ERR_NOT_CONVERGED;
  }
  return rc;
}

int exf_resid(exf_sys *s, int lev, const double *x, const double *b, double *r) {
  CHECK_LEV(s, lev);
  SysLevel &L = s->L[lev];
  DBuf<double> dx, db, dr;
  EXF_TRY(dx.alloc(L.ndof));
  EXF_TRY(db.alloc(L.ndof));
  EXF_TRY(dr.alloc(L.ndof));
  EXF_TRY(h2d(s, dx.p, x, L.ndof));
  if (b) EXF_TRY(h2d(s, db.p, b, L.ndof));
  EXF_TRY(spmv_resid<double>(s, lev, dx.p, b ? db.p : nullptr, dr.p, nullptr));
  return d2h(s, r, dr.p, L.ndof);
}

int exf_restrict(exf_sys *s, int lev, const double *r_fine, double *b_coarse) {
  CHECK_LEV(s, lev);
  if (lev >= s->nlev - 1) return EXF_ERR_ARG;
  EXF_TRY(need_transfers(s));
  SysLevel &C = s->L[lev], &F = s->L[lev + 1];
  DBuf<double> df, dc;
  EXF_TRY(df.alloc(F.ndof));
  EXF_TRY(dc.alloc(C.ndof));
  EXF_TRY(h2d(s, df.p, r_fine, F.ndof));
  EXF_TRY(restrict_op<double>(s, lev, df.p, dc.p));
  return d2h(s, b_coarse, dc.p, C.ndof);
}

int exf_prolong(exf_sys *s, int lev, const double *x_coarse, double *y_fine) {
  CHECK_LEV(s, lev);
  if (lev == 0) return EXF_ERR_ARG;
  EXF_TRY(need_transfers(s));
  SysLevel &F = s->L[lev], &C = s->L[lev - 1];
  DBuf<double> df, dc;
  EXF_TRY(df.alloc(F.ndof));
  EXF_TRY(dc.alloc(C.ndof));
  EXF_TRY(h2d(s, dc.p, x_coarse, C.ndof));
  EXF_TRY(prolong_add<double>(s, lev, dc.p, df.p, 0.));
  return d2h(s, y_fine, df.p, F.ndof);
}

int exf_smooth(exf_sys *s, int lev, const exf_mg_params *p, int nsweeps, double *x, const double *b) {
  CHECK_LEV(s, lev);
  if (!p || nsweeps < 0) return EXF_ERR_ARG;
  SysLevel &L = s->L[lev];
  DBuf<double> dx, db;
  EXF_TRY(dx.alloc(L.ndof));
  EXF_TRY(db.alloc(L.ndof));
  EXF_TRY(h2d(s, dx.p, x, L.ndof));
  EXF_TRY(h2d(s, db.p, b, L.ndof));
  EXF_TRY(smooth<double>(s, lev, p, nsweeps, dx.p, db.p));
  EXF_TRY(device_wait_status(s));
  return d2h(s, x, dx.p, L.ndof);
}

int exf_ilu_apply(exf_sys *s, int lev, const double *c, double *y) {
  CHECK_LEV(s, lev);
  if (!c || !y) return EXF_ERR_ARG;
  SysLevel &L = s->L[lev];
  DBuf<double> dc;
  EXF_TRY(dc.alloc(L.ndof));
  EXF_TRY(h2d(s, dc.p, c, L.ndof));
  EXF_TRY(ilu_apply(s, lev, dc.p, dc.p));
  EXF_TRY(device_wait_status(s));
  return d2h(s, y, dc.p, L.ndof);
}

int exf_coarse_solve(exf_sys *s, const double *b, double *x) {
  CHECK_SYS(s);
  SysLevel &L = s->L[0];
  DBuf<double> dx, db;
  EXF_TRY(dx.alloc(L.ndof));
  EXF_TRY(db.alloc(L.ndof));
  EXF_TRY(h2d(s, db.p, b, L.ndof));
  EXF_TRY(coarse_apply<double>(s, db.p, dx.p));
  return d2h(s, x, dx.p, L.ndof);
}

}  // extern "C"

namespace exf {
// FP64 FMA throughput probe: EXF_FMA_CHAINS independent fma chains of EXF_FMA_ITERS
// steps per thread, 4 CTAs of 256 threads per SM; the sink is written only if a chain
// ends in NaN, which keeps the chains live without a store per thread
__device__ double g_fma_sink;
__global__ void __launch_bounds__(256) k_fma_probe(double seed) {
  double a[EXF_FMA_CHAINS];
#pragma unroll
  for (int c = 0; c < EXF_FMA_CHAINS; c++) a[c] = seed * (threadIdx.x + c + 1);
  const double m = 1. - 1e-12, k = 1e-12;
  for (int it = 0; it < EXF_FMA_ITERS; it++) {
#pragma unroll
    for (int c = 0; c < EXF_FMA_CHAINS; c++) a[c] = fma(a[c], m, k);
  }
  double sum = 0.;
#pragma unroll
  for (int c = 0; c < EXF_FMA_CHAINS; c++) sum += a[c];
  if (sum != sum) g_fma_sink = sum;
}
}  // namespace exf

extern "C" {

// device time of one operation class, averaged over reps launches (CUDA events on the
// system stream, after one untimed warm-up)
int exf_time_op(exf_sys *s, int what, int lev, const exf_mg_params *p, const exf_phys *ph, int reps,
                double *avg_ms) {
  CHECK_LEV(s, lev);
  if (!p || !avg_ms || reps < 1) return EXF_ERR_ARG;
  if (what == 2 && !ph) return EXF_ERR_ARG;
  if (what != 2 && !s->assembled) return EXF_ERR_STATE;
  if (what == 3) EXF_TRY(need_transfers(s));
  if (!s->coarse_ok && what == 3) EXF_TRY(coarse_factor(s));
  SysLevel &L = s->L[lev];
  const bool f32 = p->precision == EXF_PREC_MIXED;
  auto once = [&]() -> int {
    switch (what) {
      case 0:
        return f32 ? spmv_resid<float>(s, lev, L.x32.p, L.b32.p, L.r32.p, nullptr)
                   : spmv_resid<double>(s, lev, L.x.p, L.b.p, L.r.p, nullptr);
      case 1:
        return f32 ? smooth<float>(s, lev, p, 1, L.x32.p, L.b32.p) : smooth<double>(s, lev, p, 1, L.x.p, L.b.p);
      case 2:
        EXF_TRY(assemble_every_level(s, ph));  // the exf_assemble_all path
        for (int l = 0; l < s->nlev; l++) s->L[l].ilu_ok = false;
        return EXF_OK;
      case 3: {
        SysLevel &T = s->L[s->nlev - 1];
        if (f32) {
          EXF_TRY(spmv_resid<double>(s, s->nlev - 1, T.x.p, T.b.p, T.r.p, s->red.out.p + 1));
          return vcycle_mixed(s, p);
        }
        return vcycle_fp64(s, p, s->red.out.p + 1);
      }
      case 4:
        s->coarse_ok = 0;
        return coarse_factor(s);
      case 5:
        k_fma_probe<<<4 * s->nsm, 256, 0, s->stream>>>(1e-3);
        EXF_LAUNCH_CHECK();
        return EXF_OK;
      case 7:
        L.ilu_ok = false;
        return ilu_ready(s, lev);
      case 8:
        return ilu_apply(s, lev, L.r.p, L.r.p);
      default:
        set_error("exf_time_op: unknown operation %d", what);
        return EXF_ERR_ARG;
    }
  };
  if (what == 6) {
    *avg_ms = 0.;
    return wait_probe(s);
  }
  EXF_TRY(once());
  EXF_CUDA(cudaEventRecord(s->ev0, s->stream));
  for (int i = 0; i < reps; i++) EXF_TRY(once());
  EXF_CUDA(cudaEventRecord(s->ev1, s->stream));
  EXF_CUDA(cudaEventSynchronize(s->ev1));
  float ms = 0.f;
  EXF_CUDA(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
  *avg_ms = ms / reps;
  if (what == 2)
    for (int l = 0; l < s->nlev; l++) EXF_TRY(sync_fp32(s, l));
  return EXF_OK;
}

// algorithmic bytes of one level operation in the node-block layout (value bytes vb):
// spmv   every block once (d*d values + one index), every B/B^T entry once, row pointers,
//        x read, r written, b read;
// sweep  one Vanka sweep: each pressure patch reads the rows of every velocity node of its
//        star (the colour schedule re-reads a node once per star containing it), its own
//        pressure row, b and x of its DOFs and writes x; a Gauss-Seidel sweep reads A once.
int exf_level_bytes(exf_sys *s, int lev, int precision, double *spmv_bytes, double *sweep_bytes) {
  CHECK_LEV(s, lev);
  SysLevel &L = s->L[lev];
  const double vb = precision == EXF_PREC_MIXED ? 4. : 8.;
  const int d = s->nv2;
  std::vector<int> qp(L.N + 1), lp(L.N + 1), qc(L.nqq);
  EXF_CUDA(cudaMemcpy(qp.data(), L.qq_ptr.p, (L.N + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  EXF_CUDA(cudaMemcpy(lp.data(), L.ql_ptr.p, (L.N + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  EXF_CUDA(cudaMemcpy(qc.data(), L.qq_col.p, L.nqq * sizeof(int), cudaMemcpyDeviceToHost));
  auto vrow = [&](int n) {  // bytes of the d velocity rows of node n
    return (double)(qp[n + 1] - qp[n]) * (d * d * vb + 4.) + (double)(lp[n + 1] - lp[n]) * (d * vb + 4.) + 8.;
  };
  // a star row as the Vanka row kernel reads it: FP16 values and the column in the FP32
  // smoother (3D: 18 + 4 bytes per block; 2D: 8 + 4), FP64 planes + column otherwise;
  // pressure couplings; its descriptor (16) and, for FP16, its d row scales
  const bool h16 = precision == EXF_PREC_MIXED;
  auto srow = [&](int n) {
    const double blk = h16 ? (d == 3 ? 22. : 12.) : d * d * vb + 4.;
    return (double)(qp[n + 1] - qp[n]) * blk + (double)(lp[n + 1] - lp[n]) * (d * vb + 4.) + 16. +
           (h16 ? d * 4. : 0.);
  };
  auto prow = [&](int m) {
    return (double)(qp[m + 1] - qp[m]) * (d * vb) + (double)(lp[m + 1] - lp[m]) * vb + 4.;
  };
  double A = 0.;
  for (int n = 0; n < L.N; n++) A += vrow(n);
  if (s->nv1)
    for (int m = 0; m < L.NL; m++) A += prow(m);
  const double vec = (double)L.ndof * vb;
  if (spmv_bytes) *spmv_bytes = A + 3. * vec;
  if (sweep_bytes) {
    if (s->nv1 == 0) {
      *sweep_bytes = A + 3. * vec;
    } else {
      double B = 0.;
      for (int m = 0; m < L.NL; m++) {
        for (int k = qp[m]; k < qp[m + 1]; k++) B += srow(qc[k]) + 3. * d * vb;  // rows + b, x read/write
        B += prow(m) + 3. * vb;
      }
      *sweep_bytes = B;
    }
  }
  return EXF_OK;
}

int exf_timestep_loop(exf_sys *const *sys, int nsys, const exf_phys *phys, const exf_mg_params *params,
                      int nsteps, int *cycles, double *seconds) {
  if (!sys || !phys || !params || nsys < 1 || nsteps < 0) {
    set_error("exf_timestep_loop: bad argument");
    return EXF_ERR_ARG;
  }
  for (int k = 0; k < nsys; k++)
    if (!sys[k]) {
      set_error("exf_timestep_loop: system %d is NULL", k);
      return EXF_ERR_ARG;
    }
  bool missed = false;
  for (int step = 0; step < nsteps; step++) {
    for (int k = 0; k < nsys; k++) {
      exf_solve_stats st;
      EXF_TRY(exf_assemble_all(sys[k], &phys[k]));
      const int rc = exf_mg_solve(sys[k], &params[k], &st);
      if (cycles) cycles[(long)step * nsys + k] = st.cycles;
      if (seconds) seconds[(long)step * nsys + k] = st.seconds;
      if (rc == EXF_ERR_NOT_CONVERGED) missed = true;
      else if (rc != EXF_OK) return rc;
      EXF_TRY(exf_sys_xold_update(sys[k]));
    }
  }
  if (missed) {
    set_error("exf_timestep_loop: a solve ended above its tolerance (cycles per step and system returned)");
    return EXF_ERR_NOT_CONVERGED;
  }
  return EXF_OK;
}

int exf_sync(exf_sys *s) {
  CHECK_SYS(s);
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  return EXF_OK;
}

}  // extern "C"
