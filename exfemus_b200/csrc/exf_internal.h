// exf_internal.h -- internal data structures of the B200 assembly + multigrid library.
//
// HBM layout per level (one equation system):
//   node pattern   qq_ptr/qq_col (Q2 node -> sorted Q2 neighbour nodes),
//                  ql_ptr/ql_col (Q2 node -> sorted Q1 neighbour nodes)
//   values         node-block planar arrays ("NB" layout): for d velocity components
//                  vv[(a*d+b)*nqq + k]  velocity row comp a, column comp b, block k
//                  vp[a*nql + k]        velocity row comp a, pressure column (B^T)
//                  pv[b*nqqL + k]       pressure row, velocity column comp b (B)
//                  pp[k]                pressure-pressure (k < ql_ptr[NL])
//                  one index per block instead of one per entry; planes make every
//                  warp load contiguous.  The reference's DOF-level CSR (all four
//                  blocks qq/ql/lq/ll, sorted columns) is produced from it on demand.
//   vectors        DOF order of MGSolDA::init_dof: component-major Q2 variables, then
//                  the Q1 variable on the first NL nodes.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/exfemus_b200.h"

namespace exf {

void set_error(const char *fmt, ...);
void count_launch(int n);  // kernels launched by the library (all streams)
#define EXF_COUNT(n) exf::count_launch(n)

#define EXF_CUDA(call)                                                                 \
  do {                                                                                 \
    cudaError_t e__ = (call);                                                          \
    if (e__ != cudaSuccess) {                                                          \
      exf::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e__)); \
      return EXF_ERR_CUDA;                                                             \
    }                                                                                  \
  } while (0)

#define EXF_LAUNCH_CHECK()                                                             \
  do {                                                                                 \
    cudaError_t e__ = cudaGetLastError();                                              \
    if (e__ != cudaSuccess) {                                                          \
      exf::set_error("%s:%d launch: %s", __FILE__, __LINE__, cudaGetErrorString(e__)); \
      return EXF_ERR_CUDA;                                                             \
    }                                                                                  \
  } while (0)

#define EXF_TRY(expr)          \
  do {                         \
    int rc__ = (expr);         \
    if (rc__ != EXF_OK) return rc__; \
  } while (0)

// Programmatic dependent launch: kernels of the multigrid chain are launched with
// programmatic stream serialisation so the next launch is set up while the previous grid
// drains; every such kernel starts with EXF_PDL_WAIT (griddepcontrol.wait), before its
// first global read, so it still observes all writes of the preceding grid.  Right after
// the wait it releases its own dependents (griddepcontrol.launch_dependents): their
// blocks may then be scheduled onto free SM slots, where they block in their own wait
// until this grid has completed and its writes are visible.  Launched without the
// attribute both instructions are no-ops.
#define EXF_PDL_WAIT()                                                \
  do {                                                                \
    asm volatile("griddepcontrol.wait;" ::: "memory");                \
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");   \
  } while (0)

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// device buffer with RAII
template <class T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  DBuf(DBuf &&o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DBuf &operator=(DBuf &&o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  int ensure(size_t count) { return (p && n == (count ? count : 1)) ? EXF_OK : alloc(count); }
  int alloc(size_t count) {
    release();
    if (count == 0) count = 1;
    if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      set_error("cudaMalloc of %zu bytes failed", count * sizeof(T));
      return EXF_ERR_NOMEM;
    }
    n = count;
    return EXF_OK;
  }
  int zero(cudaStream_t s) { return cudaMemsetAsync(p, 0, n * sizeof(T), s) == cudaSuccess ? EXF_OK : EXF_ERR_CUDA; }
};

struct MeshLevel {
  int nnodes = 0, nel = 0, ne[3] = {1, 1, 1};  // ne: elements per axis (structured boxes)
  std::vector<int> conn, neigh, colour;   // host copies
  std::vector<int> parent;                // uploaded meshes: parent element on level - 1
  DBuf<int> d_conn, d_neigh;
  DBuf<int> d_elist;                      // elements sorted by colour
  std::vector<int> ecol_off;              // [element colours + 1] offsets into d_elist
};

}  // namespace exf

struct exf_mesh {
  int dim = 2, nlev = 1, nen = 9, nvx = 4, nsides = 4, nsn = 3;
  // generated box (exf_mesh_create): nodes on an integer lattice, colourings and
  // transfers from lattice indices; uploaded (exf_mesh_upload): from the arrays
  bool lattice = true;
  bool has_parent = false;                // uploaded with parent elements
  int n0[3] = {1, 1, 1}, L[3] = {1, 1, 1};
  int ntop = 0, nvert0 = 0;
  int device = 0;
  double box[6] = {0, 1, 0, 1, 0, 1};
  std::vector<int> lat;       // [ntop*3]
  std::vector<double> xyz;    // [dim*ntop]
  std::vector<exf::MeshLevel> lev;
  exf::DBuf<double> d_xyz;
  bool xyz_moved = false;  // d_xyz moved on the device (displacement mesh motion): xyz is stale
  // the live systems on this mesh: a destroyed system is cleared from its partners' couplings
  std::mutex sys_mu;
  std::vector<exf_sys *> systems;
  bool orphaned = false;  // exf_mesh_destroy called while systems lived: freed with the last
  exf::DBuf<int> d_lat;
  // FE tables of the assembly (Gauss points, shape values and derivatives, surface
  // rules) on the mesh's device: written once in exf_mesh_create, read-only after
  exf::DBuf<unsigned char> d_fetab;
};

namespace exf {

template <class T>
struct LevelVals {
  DBuf<T> vv, vp, pv, pp;
};

// node-level transfer operator (CSR) applied per variable component
struct Transfer {
  int nrow = 0;
  DBuf<int> ptr, col;
  DBuf<double> val;
  DBuf<float> val32;
  std::vector<int> h_ptr, h_col;
  std::vector<double> h_val;
};

struct SysLevel {
  int N = 0, NL = 0, ndof = 0, nel = 0;
  long nqq = 0, nql = 0, nqqL = 0, nllL = 0, nnz = 0;
  DBuf<int> qq_ptr, qq_col, ql_ptr, ql_col;
  DBuf<int> diag_pos;    // [N] absolute block index of n in qq(n)
  DBuf<int> gidx;        // [nqqL] for pressure-row block k: index into vp of G(., n_k; m)
  DBuf<uint8_t> pos_qq;  // [nel*nen*nen]
  DBuf<uint8_t> pos_ql;  // [nel*nen*nvx]
  DBuf<int> csr_ptr, csr_col;  // DOF-level CSR (built on device)
  // smoother colouring: items = DOFs (T) or pressure nodes (NS), grouped by colour
  int ncolour = 0;
  std::vector<int> col_off;    // [ncolour+1]
  DBuf<int> col_items;
  DBuf<int> item_colour;
  // Vanka: velocity nodes of the stars of each colour's patches, patch by patch; entry
  // g of vrows is the (patch, star node) pair g, so per-entry data is stored compactly
  std::vector<int> vrow_off;   // [ncolour+1]
  DBuf<int> vrows;
  DBuf<int4> vrinfo;           // per vrows entry: {node, qq_ptr[node], ql_ptr[node],
                               //   nqq | nql << 8 | index of the node in its patch's tile << 16}
  DBuf<int4> pinfo;            // per patch in colour order, two int4: {m, pstart[m], qq_ptr[m],
                               //   ql_ptr[m]}, {nqq(m), nql(m), lattice coordinates of m packed, 0}
  int Ll[3] = {1, 1, 1};       // Q2 node lattice of this level
  DBuf<int> latnode;           // [N] node at each lattice point (x fastest)
  DBuf<int16_t> tcq, tcl;      // per qq / ql block: column minus row as a 9^d-tile index step
  bool tile_ok = false;        // every star and row fits the tile kernels (5^d nodes)
  DBuf<int> pstart;            // [NL] first vrows entry of each patch (by pressure node)
  DBuf<double> vk64, pk64;     // per entry*D: {1/a, D/a, G/a}; per patch: {S, c_mm}
  DBuf<float> vk32, pk32;
  DBuf<double> vres64;         // compact star-row residuals [nvrows*D] + pressure rows [NL]
  DBuf<float> vres32;
  LevelVals<double> A;
  LevelVals<float> A32;
  // NS, FP32 smoother only: velocity blocks in FP16 scaled per (node, component) row by
  // the row's largest magnitude vsc[a*N+n] (entries in [-1,1]; value = stored * vsc).
  // 3D: per block a 16-byte record of values 0..7 (h16), {column, value 8} (h16cx) and
  // {value 8, tile step} (h16qc, padded for 16-byte chunk reads); 2D: per block an
  // 8-byte record of values 0..3 (h16), columns from qq_col
  DBuf<uint4> h16;
  DBuf<uint2> h16cx;
  DBuf<uint32_t> h16qc;
  DBuf<float> vsc;
  // BULK smoother (3D FP32): every star row as 16-byte records, row after row in sweep
  // order (row scales and node; counts; the FP16 values 0..7 of each block; the block
  // columns, 4 per record; the 9th values, 8 per record; the pressure couplings), so that
  // the rows of a colour are one contiguous stream; allocated on the first BULK sweep,
  // refreshed after assembly.
  DBuf<long long> soff;        // [nvrows + 2] first record of each star row (last repeated)
  std::vector<long long> soff_h;
  long long nstar = 0;         // soff[nvrows]
  DBuf<longlong2> bsched;      // BULK stage schedule for a grid of bsched_G CTAs
  DBuf<int> bsched_off;
  std::vector<int> bsched_coff;
  int bsched_G = 0;
  DBuf<uint4> sv;
  // transfers: Pq/Pl from level-1 to this level (fine rows), Rq/Rl from this level+1
  Transfer Pq, Pl, Rq, Rl;
  DBuf<double> rmask;    // [ndof] restriction row mask (bc0 % 2 of the top DOF)
  // GMRES + ILU level solver (scalar systems): the factor on the qq pattern and the
  // inverse of its diagonal, per-row publication flags and {ticket, generation, zero
  // pivot}; the Krylov vectors, two scratch vectors, the scalars and a control word
  DBuf<double> ilu_f, ilu_inv;
  DBuf<int> ilu_flag, ilu_ctl;
  DBuf<int> ilu_ord_lo, ilu_ord_up;  // rows by dependency level of the lower / upper solve
  bool ilu_ok = false;
  int ilu_maxl = 0, ilu_depth[2] = {0, 0};
  DBuf<double> gm_V, gm_w, gm_t, gm_sc, gm_part;
  DBuf<int> gm_ctl;
  // vectors
  DBuf<double> x, b, r, dx;     // dx: smoother scratch (Vanka star-row residuals)
  DBuf<float> x32, b32, r32, dx32;  // NS: node-interleaved float4 per node (4N floats)
  long len32 = 0;                   // length of the FP32 V-cycle vectors
};

// device state of the device-resident solve loop (cycles 2.. of exf_mg_solve run inside
// one graph launch whose conditional WHILE node repeats the V-cycle body while the check
// kernel says so)
struct LoopDev {
  double den;       // ||b|| (1 when b = 0)
  double lim;       // eps, or eps (1 + ||b||) for the reference stop test
  int max_cycles;
  int cycles;       // cycles done so far (set before the launch, advanced on the device)
  int ref_stop;     // 1: stop on the top level's accuracy (FP64 cycles)
  int mixed;        // 1: mixed precision (the accuracy is the FP64 relative residual)
  double rel, last_acc;
  double hist[256];
};

struct Partials {
  DBuf<double> part;   // per-block partial sums
  DBuf<double> out;    // reduced scalars
  int nblk = 0;
};

}  // namespace exf

struct exf_sys {
  exf_mesh *mesh = nullptr;
  int kind = 0, nv2 = 1, nv1 = 0, nvars = 1, nlev = 1, dim = 2;
  cudaStream_t stream = nullptr;
  std::vector<std::vector<int>> node_dof;   // host, [nvars*ntop] per level
  std::vector<int> bc0, bc1;                // top-level DOFs (host)
  exf::DBuf<int> d_bc0, d_bc1;
  std::vector<exf::SysLevel> L;
  exf::DBuf<double> xold, src_qe, rhs_top;  // top-level fields
  exf::DBuf<double> coarse_inv;             // dense inverse of the (gauged) coarsest matrix
  exf::DBuf<double> coarse_work, coarse_work2;  // Gauss-Jordan ping-pong pair [n x n] each
  exf::DBuf<double> coarse_vals;            // CSR values of the coarsest matrix
  exf::DBuf<int> coarse_piv, coarse_used, coarse_bad;
  exf::DBuf<unsigned long long> coarse_key; // pivot keys, one per step
  // (the factorisation workspace is kept between assemblies: no allocation per solve)
  exf::DBuf<double> gmask0;                 // coarse gauge mask (0 at gauge DOFs)
  int coarse_ok = 0;
  int nsm = 148;                             // SMs of the system's device
  int gauge_node = -1;                      // top-level pressure gauge node (-1 none)
  int assembled = 0;
  int transposed = 0;
  exf_sys *other = nullptr;                 // coupled system (T <- NS velocity, NS <- T)
  exf_sys *turb = nullptr;                  // kappa <-> omega partner of a K / W system
  exf_sys *ns_k = nullptr, *ns_w = nullptr; // NS: the kappa and omega systems of the eddy viscosity
  exf::DBuf<double> wall_dist;              // K / W: element wall distances, all levels
  std::vector<long> wall_off;               // first element of each level in wall_dist
  double nu_wall = 0.;
  exf::DBuf<double> ds_u, ds_d;             // DS: u_fsi and d_old, [dim][ntop] node fields
  int ds_dir = -1;                          // DS: the direction (-1: exf_sys_set_ds not called)
  double ds_dt = 0.;
  bool ds_host = false;                     // DS: fields from ds_u / ds_d, else from couplings
  bool ds_move = false;                     // DS: move the mesh at each x_old update
  exf_sys *ds_x = nullptr;                  // DS: the dx system (old x displacement)
  exf::Partials red;
  exf::DBuf<int> wait_flag;                 // set by a bounded in-kernel wait that ran out
  // per level {||b_L||^2, r^2 before the last pre-smoothing sweep, r^2 before the last
  // post-smoothing sweep (coarsest: after the solve), -}: the accuracies the reference's
  // level solver reports, for the conditional correction and the reference stop test
  exf::DBuf<double> mg_acc;
  // scratch of exf_adjoint_backward, kept between calls: the forward x and b, x_old, the
  // element sources, dB/dx_old, the adjoint state, the source gradient
  exf::DBuf<double> adj_x, adj_b, adj_xold, adj_qe, adj_w, adj_lam, adj_gq;
  // exf_assemble_all: per colour the {level, element} work list of every level (top level
  // first) and the levels' argument blocks
  exf::DBuf<unsigned char> asm_work, asm_args;
  std::vector<int> asm_work_off;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t user_ev[8] = {nullptr};
  // captured graphs, a few per system so that alternating parameter sets (a forward and
  // an adjoint solve, the two precisions) each keep theirs: one V-cycle per launch, and
  // the device-resident solve loop (a WHILE node whose body is the V-cycle and the stop
  // test); each keyed by the multigrid parameters and the buffer epoch, least recently
  // used replaced
  static constexpr int kGraphSlots = 4;
  struct GraphSlot {
    cudaGraphExec_t exec = nullptr;
    unsigned long long key = 0;
    unsigned epoch = 0;
    long long launches = 0;                 // kernels per launch (loop: per iteration)
    unsigned long long used = 0;
  };
  GraphSlot cyc_slot[kGraphSlots], loop_slot[kGraphSlots];
  unsigned long long graph_clock = 0;
  unsigned buf_epoch = 1;                   // bumped when a buffer baked into a graph moves
  int loop_unavailable = 0;                 // the runtime refused the conditional graph
  exf::DBuf<exf::LoopDev> loop_dev;
};

// Entry-point guards: a null handle is an argument error; otherwise the system's device
// becomes current for the calling thread, so one thread may drive systems on several
// devices and threads with different current devices may each drive their own systems.
#define CHECK_SYS(s)                                                            \
  do {                                                                          \
    if (!(s)) {                                                                 \
      exf::set_error("null system handle");                                     \
      return EXF_ERR_ARG;                                                       \
    }                                                                           \
    EXF_CUDA(cudaSetDevice((s)->mesh->device));                                 \
  } while (0)
#define CHECK_LEV(s, lev)                                                       \
  do {                                                                          \
    CHECK_SYS(s);                                                               \
    if ((lev) < 0 || (lev) >= (s)->nlev) {                                      \
      exf::set_error("level %d out of range", (int)(lev));                      \
      return EXF_ERR_ARG;                                                       \
    }                                                                           \
  } while (0)

namespace exf {
// lanes per node row of the residual kernel k_spmv_resid<T, D, LPR, NS, ...>: one choice
// shared by every launcher of the kernel (3D FP32 runs two rows per warp)
template <class T, int D, bool NS>
constexpr int spmv_lpr() {
  return D == 3 ? (sizeof(T) == 4 ? 16 : 32) : (NS ? 16 : 8);
}

// kernels / launchers implemented in the .cu files
int build_mesh_host(exf_mesh *m);
int mesh_finish_levels(exf_mesh *m);  // element colours, colour lists, device copies
// uploaded meshes: node indices 0..n-1 in (z, y, x) order of their coordinates, and a
// first-fit colouring of items in that order under the conflict lists cptr/cidx
std::vector<int> node_zyx_order(const exf_mesh *m, int n);
int colour_items_greedy(const exf_mesh *m, int nitem, const std::vector<int> &order,
                        const std::vector<int> &cptr, const std::vector<int> &cidx, std::vector<int> &colour);
int upload_fe_table(exf_mesh *m);  // FE tables of the mesh's element type, on its device
int build_patterns(exf_sys *s);
int build_transfers(exf_sys *s);
int set_transfer(exf_sys *s, int lev, int kind, int block, const int dim[2], const int *len, const int *pos,
                 const double *val);
bool transfers_ready(const exf_sys *s);
int update_rmask(exf_sys *s);
int build_colours(exf_sys *s);
int assemble_level(exf_sys *s, const exf_phys *ph, int lev, int mode);
int assemble_all_levels(exf_sys *s, const exf_phys *ph);  // every level, one launch per colour
int assemble_kw_level(exf_sys *s, const exf_phys *ph, int lev, int mode);  // K / W systems
int assemble_ds_level(exf_sys *s, int lev, int mode);  // DS systems
int ds_move_mesh(exf_sys *s);       // DS: xyz[dir] += x - x_old on the device
int mesh_pull_xyz(exf_mesh *m);     // refresh the host xyz after device mesh motion
int sync_fp32(exf_sys *s, int lev);  // FP32 copy + smoother coefficients after a matrix change
int vanka_prep(exf_sys *s, int lev);
int csr_values(exf_sys *s, int lev, double *d_out);         // NB -> CSR order (device)
int csr_set_values(exf_sys *s, int lev, const double *d_in);
int coarse_factor(exf_sys *s);
int transpose_level(exf_sys *s, int lev);

// solver primitives (templated on value type; launched on s->stream)
template <class T>
int spmv_resid(exf_sys *s, int lev, const T *x, const T *b, T *r, double *d_norm2);
template <class T>
int restrict_op(exf_sys *s, int lev_c, const T *r_f, T *b_c);
template <class T>
int prolong_add(exf_sys *s, int lev_f, const T *x_c, T *x_f, double damp);
template <class T>
int smooth(exf_sys *s, int lev, const exf_mg_params *p, int nsweeps, T *x, const T *b);
// EXF_ERR_CUDA (and clears the flag) when a bounded in-kernel wait ran out since the last call
int device_wait_status(exf_sys *s);
// GMRES + ILU level solver (ilu_gmres.cu)
int ilu_ready(exf_sys *s, int lev);
int ilu_apply(exf_sys *s, int lev, const double *c, double *y);
int gmres_smooth(exf_sys *s, int lev, double eps, int m, double *x, const double *b, double *acc);
// runs a bounded wait that nothing completes; returns the resulting device_wait_status
int wait_probe(exf_sys *s);
template <class T>
int coarse_apply(exf_sys *s, const T *b, T *x);
int gauge_shift(exf_sys *s, double *x);
int cast_d2f(cudaStream_t st, const double *a, float *b, long n, int i4, int N, int d);
template <class T>
int zero_vec(cudaStream_t st, T *a, long n);
int add_f2d(cudaStream_t st, const float *a, double *b, long n, int i4, int N, int d);
template <class T>
int norm2(exf_sys *s, const T *v, long n, double *d_out);
// x_f += damp * P x_c only where the reference's conditional correction applies (acc:
// per level {||b||^2, pre-smoothing r^2, post-smoothing r^2, -}, see mg_step)
template <class T>
int prolong_cond(exf_sys *s, int lev_f, const T *x_c, T *x_f, double damp, const double *acc);
int vcycle_fp64(exf_sys *s, const exf_mg_params *p, double *d_relres);
int vcycle_mixed(exf_sys *s, const exf_mg_params *p);
}  // namespace exf
