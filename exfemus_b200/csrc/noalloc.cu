// noalloc.cu -- residual with its squared norm, with no device allocation.
//
// Some callers cannot allocate device memory while they run: a solver step embedded in
// a host application that owns every allocation through its own pool, code that runs
// between allocation-free checkpoints of a real-time loop, or a process whose memory is
// reserved up front.  For them exf_resid_norm_static computes r = b - A x on one level
// and ||r||^2, taking x, b, r and the norm as device buffers the caller owns, and keeps
// the per-block partial sums of the norm in a fixed file-scope device array instead of
// library-allocated scratch.  It calls no cudaMalloc/cudaFree and no allocating library
// routine.
//
// The array holds at most EXF_STATIC_PARTIALS partial sums (one per block of the
// residual kernel, 256 KB); larger levels are rejected with EXF_ERR_ARG.  The call
// returns once the system stream has finished it (it synchronizes that stream).  Every GPU that
// loads the library holds the array until the process exits.  Every call on a device
// shares the one array and leaves its last contents there; each call overwrites exactly
// the partial sums it reads, so nothing has to start at zero, but two calls whose work
// overlaps on the GPU (different streams or systems at the same time) race on it.
#include <mutex>

#include "exf_internal.h"

namespace exf {
template <class T, int D, int LPR, bool NS, int NT, bool I4>
__global__ void k_spmv_resid(int N, int NL, const int *__restrict__ qq_ptr, const int *__restrict__ qq_col,
                             const int *__restrict__ ql_ptr, const int *__restrict__ ql_col, long nqq, long nql,
                             long nqqL, const T *__restrict__ vv, const T *__restrict__ vp,
                             const T *__restrict__ pv, const T *__restrict__ pp, const T *__restrict__ x,
                             const T *__restrict__ b, T *__restrict__ r, double *__restrict__ part);
__global__ void k_reduce_partials(const double *part, int n, double *out);
}  // namespace exf

static __device__ __align__(256) double g_static_partials[EXF_STATIC_PARTIALS];

// device address of g_static_partials per device, resolved on the first call with that
// device current (the host name of the array is not a device address); the lock makes
// the first calls of threads on one device resolve it once
static double *g_partials_addr[64] = {nullptr};
static std::mutex g_partials_lock;

using namespace exf;

template <int D, bool NS>
static int resid_norm_static(exf_sys *s, int lev, const double *x, const double *b, double *r, double *norm2) {
  SysLevel &L = s->L[lev];
  constexpr int NT = 256;
  constexpr int LPR = spmv_lpr<double, D, NS>();  // the launch shape of the allocating residual
  const long ngroups = (long)L.N + (NS ? L.NL : 0);
  const long grid = (ngroups * LPR + NT - 1) / NT;
  if (grid > EXF_STATIC_PARTIALS) {
    set_error("exf_resid_norm_static: level %d needs %ld partial sums, the static array holds %d", lev, grid,
              EXF_STATIC_PARTIALS);
    return EXF_ERR_ARG;
  }
  int dev = 0;
  EXF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("exf_resid_norm_static: device ordinal %d out of range", dev);
    return EXF_ERR_ARG;
  }
  double *part = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_partials_lock);
    if (!g_partials_addr[dev]) {
      void *ptr = nullptr;
      EXF_CUDA(cudaGetSymbolAddress(&ptr, g_static_partials));
      g_partials_addr[dev] = static_cast<double *>(ptr);
    }
    part = g_partials_addr[dev];
  }
  k_spmv_resid<double, D, LPR, NS, NT, false><<<(unsigned)grid, NT, 0, s->stream>>>(
      L.N, L.NL, L.qq_ptr.p, L.qq_col.p, L.ql_ptr.p, L.ql_col.p, L.nqq, L.nql, L.nqqL, L.A.vv.p, L.A.vp.p, L.A.pv.p,
      L.A.pp.p, x, b, r, part);
  EXF_LAUNCH_CHECK();
  k_reduce_partials<<<1, 1024, 0, s->stream>>>(part, (int)grid, norm2);
  EXF_LAUNCH_CHECK();
  EXF_COUNT(2);
  return EXF_OK;
}

extern "C" int exf_resid_norm_static(exf_sys *s, int lev, const double *x, const double *b, double *r,
                                     double *norm2) {
  if (!s || lev < 0 || lev >= s->nlev || !x || !b || !r || !norm2) {
    set_error("exf_resid_norm_static: bad argument");
    return EXF_ERR_ARG;
  }
  if (!s->assembled) {
    set_error("exf_resid_norm_static before assembly");
    return EXF_ERR_STATE;
  }
  EXF_CUDA(cudaSetDevice(s->mesh->device));
  // the call waits for its result on the system stream; a stream that is being captured
  // cannot be waited on, so the call is refused there and leaves the capture intact
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  EXF_CUDA(cudaStreamIsCapturing(s->stream, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    set_error("exf_resid_norm_static synchronizes the system stream, which is being captured");
    return EXF_ERR_STATE;
  }
  const bool ns = s->kind == EXF_KIND_NS;
  int rc;
  if (s->dim == 2) rc = ns ? resid_norm_static<2, true>(s, lev, x, b, r, norm2)
                           : resid_norm_static<1, false>(s, lev, x, b, r, norm2);
  else rc = ns ? resid_norm_static<3, true>(s, lev, x, b, r, norm2)
               : resid_norm_static<1, false>(s, lev, x, b, r, norm2);
  if (rc != EXF_OK) return rc;
  EXF_CUDA(cudaStreamSynchronize(s->stream));
  return EXF_OK;
}
