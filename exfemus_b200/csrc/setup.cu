// setup.cu -- one-time integer work on the device: node patterns, the DOF-level CSR
// pattern, element->slot maps, smoother colouring, and the transfer operators.
//
// Reference: the sparsity pattern is gencase's compute_mat_qq (union of the nodes of
// every element containing a node, USER_APPL/gencase/src/MGGenCase.C:1781-1862) read by
// MGSolDA::ReadMatrix (src/MGSolverDA.C:1785-2009) into LASPACK rows, which LASPACK
// sorts before the first product (contrib/laspack/operats.c:813).  Here the rows are
// built sorted; every result is independent of thread scheduling.
#include <algorithm>
#include <cmath>
#include <cstdio>

#include "exf_internal.h"
#include "fe_topology.h"

namespace exf {

// ------------------------------------------------------------------ exclusive scan
// in-place exclusive scan of n ints, returns total in *total (host)
__global__ void k_scan_tiles(int *a, long n, int *tile_sum) {
  __shared__ int s[1024];
  long i = (long)blockIdx.x * 1024 + threadIdx.x;
  int v = i < n ? a[i] : 0;
  s[threadIdx.x] = v;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    int t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
    __syncthreads();
    s[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) a[i] = s[threadIdx.x] - v;
  if (threadIdx.x == 1023) tile_sum[blockIdx.x] = s[1023];
}
__global__ void k_scan_sums(int *tile_sum, int ntiles, int *total) {
  if (threadIdx.x == 0) {
    int run = 0;
    for (int t = 0; t < ntiles; t++) {
      int v = tile_sum[t];
      tile_sum[t] = run;
      run += v;
    }
    *total = run;
  }
}
__global__ void k_scan_add(int *a, long n, const int *tile_sum) {
  long i = (long)blockIdx.x * 1024 + threadIdx.x;
  if (i < n) a[i] += tile_sum[blockIdx.x];
}

static int exclusive_scan(int *d, long n, int *total, cudaStream_t st) {
  long ntiles = (n + 1023) / 1024;
  DBuf<int> ts, tot;
  EXF_TRY(ts.alloc(ntiles));
  EXF_TRY(tot.alloc(1));
  k_scan_tiles<<<ntiles, 1024, 0, st>>>(d, n, ts.p);
  k_scan_sums<<<1, 32, 0, st>>>(ts.p, (int)ntiles, tot.p);
  k_scan_add<<<ntiles, 1024, 0, st>>>(d, n, ts.p);
  EXF_LAUNCH_CHECK();
  EXF_CUDA(cudaMemcpyAsync(total, tot.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  EXF_CUDA(cudaStreamSynchronize(st));
  return EXF_OK;
}

// ------------------------------------------------------------- node incidence
__global__ void k_count_incidence(const int *conn, long nentries, int *cnt) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nentries) atomicAdd(&cnt[conn[i]], 1);
}
__global__ void k_fill_incidence(const int *conn, long nentries, int nen, const int *ptr, int *fill, int *elist) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nentries) {
    int n = conn[i];
    int slot = atomicAdd(&fill[n], 1);
    elist[ptr[n] + slot] = (int)(i / nen);
  }
}
// sort each node's element list (<= 8 entries): makes the lists schedule-independent
__global__ void k_sort_incidence(const int *ptr, int *elist, int N) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  int b = ptr[n], e = ptr[n + 1];
  for (int i = b + 1; i < e; i++) {
    int v = elist[i], j = i - 1;
    while (j >= b && elist[j] > v) {
      elist[j + 1] = elist[j];
      j--;
    }
    elist[j + 1] = v;
  }
}

// sorted-unique insertion into a small local list
__device__ __forceinline__ int insert_unique(int *lst, int cnt, int v, int cap) {
  int lo = 0, hi = cnt;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (lst[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  if (lo < cnt && lst[lo] == v) return cnt;
  if (cnt >= cap) return cnt + 1;  // overflow: reported by the caller, never written
  for (int k = cnt; k > lo; k--) lst[k] = lst[k - 1];
  lst[lo] = v;
  return cnt + 1;
}

// node pattern: union of the nodes (qq) and of the vertices (ql) of the elements
// containing each node.  pass 0 writes counts, pass 1 writes the sorted lists.
template <int NEN, int NVX, int MAXQ, int MAXL>
__global__ void k_node_pattern(const int *conn, const int *eptr, const int *elist, int N, int pass, int *qq_cnt,
                               int *ql_cnt, const int *qq_ptr, const int *ql_ptr, int *qq_col, int *ql_col,
                               int *bad) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  int lq[MAXQ], ll[MAXL];
  int cq = 0, cl = 0;
  for (int k = eptr[n]; k < eptr[n + 1]; k++) {
    const int *c = conn + (long)elist[k] * NEN;
    for (int j = 0; j < NEN; j++) cq = min(insert_unique(lq, cq, c[j], MAXQ), MAXQ + 1);
    for (int j = 0; j < NVX; j++) cl = min(insert_unique(ll, cl, c[j], MAXL), MAXL + 1);
  }
  if (cq > MAXQ || cl > MAXL) {  // not a structured quad9/hex27 hierarchy
    atomicExch(bad, 1);
    cq = min(cq, MAXQ);
    cl = min(cl, MAXL);
  }
  if (pass == 0) {
    qq_cnt[n] = cq;
    ql_cnt[n] = cl;
  } else {
    for (int j = 0; j < cq; j++) qq_col[qq_ptr[n] + j] = lq[j];
    for (int j = 0; j < cl; j++) ql_col[ql_ptr[n] + j] = ll[j];
  }
}

__device__ __forceinline__ int bsearch_dev(const int *a, int lo, int hi, int v) {
  // returns index in [lo,hi) with a[idx]==v, or -1
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    int x = a[mid];
    if (x == v) return mid;
    if (x < v) lo = mid + 1;
    else hi = mid;
  }
  return -1;
}

__global__ void k_diag_pos(const int *qq_ptr, const int *qq_col, int N, int *diag) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < N) diag[n] = bsearch_dev(qq_col, qq_ptr[n], qq_ptr[n + 1], n);
}

// element slot maps: pos_qq[e][i][j] = position of node j in qq(node i) (relative),
// pos_ql[e][i][jv] = position of vertex jv in ql(node i)
__global__ void k_elem_pos(const int *conn, int nel, int nen, int nvx, const int *qq_ptr, const int *qq_col,
                           const int *ql_ptr, const int *ql_col, uint8_t *pos_qq, uint8_t *pos_ql, int *bad) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)nel * nen) return;
  long e = t / nen;
  int i = (int)(t % nen);
  const int *c = conn + e * nen;
  int ni = c[i];
  for (int j = 0; j < nen; j++) {
    int p = bsearch_dev(qq_col, qq_ptr[ni], qq_ptr[ni + 1], c[j]);
    if (p < 0) atomicExch(bad, 1);
    pos_qq[(e * nen + i) * nen + j] = (uint8_t)(p - qq_ptr[ni]);
  }
  for (int j = 0; j < nvx; j++) {
    int p = bsearch_dev(ql_col, ql_ptr[ni], ql_ptr[ni + 1], c[j]);
    if (p < 0) atomicExch(bad, 1);
    pos_ql[(e * nen + i) * nvx + j] = (uint8_t)(p - ql_ptr[ni]);
  }
}

// for the pressure row of Q1 node m and its block k (velocity node n_k): index of the
// B^T entry (row n_k, pressure column m) inside vp
__global__ void k_gidx(const int *qq_ptr, const int *qq_col, const int *ql_ptr, const int *ql_col, int NL, int *gidx,
                       int *bad) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= NL) return;
  for (int k = qq_ptr[m]; k < qq_ptr[m + 1]; k++) {
    int n = qq_col[k];
    int p = bsearch_dev(ql_col, ql_ptr[n], ql_ptr[n + 1], m);
    if (p < 0) atomicExch(bad, 1);
    gidx[k] = p;
  }
}

// DOF-level CSR: row (a,n) = [b*N + qq(n)] for b < nv2, then [nv2*N + ql(n)]
__global__ void k_csr_rowlen(const int *qq_ptr, const int *ql_ptr, int N, int NL, int nv2, int nv1, int *rowlen) {
  long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long nrow = (long)nv2 * N + (long)nv1 * NL;
  if (r >= nrow) return;
  int n = r < (long)nv2 * N ? (int)(r % N) : (int)(r - (long)nv2 * N);
  rowlen[r] = nv2 * (qq_ptr[n + 1] - qq_ptr[n]) + nv1 * (ql_ptr[n + 1] - ql_ptr[n]);
}
__global__ void k_csr_fill(const int *qq_ptr, const int *qq_col, const int *ql_ptr, const int *ql_col, int N, int NL,
                           int nv2, int nv1, const int *rowptr, int *col) {
  long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long nrow = (long)nv2 * N + (long)nv1 * NL;
  if (r >= nrow) return;
  int n = r < (long)nv2 * N ? (int)(r % N) : (int)(r - (long)nv2 * N);
  int o = rowptr[r];
  for (int b = 0; b < nv2; b++)
    for (int k = qq_ptr[n]; k < qq_ptr[n + 1]; k++) col[o++] = b * N + qq_col[k];
  if (nv1)
    for (int k = ql_ptr[n]; k < ql_ptr[n + 1]; k++) col[o++] = nv2 * N + ql_col[k];
}

static inline unsigned nblk(long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

int build_patterns(exf_sys *s) {
  exf_mesh *m = s->mesh;
  cudaStream_t st = s->stream;
  const int nen = m->nen, nvx = m->nvx;
  for (int l = 0; l < s->nlev; l++) {
    SysLevel &L = s->L[l];
    const MeshLevel &ml = m->lev[l];
    L.N = ml.nnodes;
    L.NL = l > 0 ? m->lev[l - 1].nnodes : m->nvert0;
    L.nel = ml.nel;
    L.ndof = s->nv2 * L.N + s->nv1 * L.NL;
    long nent = (long)ml.nel * nen;
    DBuf<int> eptr, fill, elist;
    EXF_TRY(eptr.alloc(L.N + 1));
    EXF_TRY(fill.alloc(L.N));
    EXF_TRY(elist.alloc(nent));
    EXF_TRY(eptr.zero(st));
    EXF_TRY(fill.zero(st));
    k_count_incidence<<<nblk(nent, 256), 256, 0, st>>>(ml.d_conn.p, nent, eptr.p);
    EXF_LAUNCH_CHECK();
    int tot = 0;
    EXF_TRY(exclusive_scan(eptr.p, L.N + 1, &tot, st));
    k_fill_incidence<<<nblk(nent, 256), 256, 0, st>>>(ml.d_conn.p, nent, nen, eptr.p, fill.p, elist.p);
    k_sort_incidence<<<nblk(L.N, 256), 256, 0, st>>>(eptr.p, elist.p, L.N);
    EXF_LAUNCH_CHECK();
    DBuf<int> bad;
    EXF_TRY(bad.alloc(1));
    EXF_TRY(bad.zero(st));
    EXF_TRY(L.qq_ptr.alloc(L.N + 1));
    EXF_TRY(L.ql_ptr.alloc(L.N + 1));
    EXF_TRY(L.qq_ptr.zero(st));
    EXF_TRY(L.ql_ptr.zero(st));
    auto launch_pattern = [&](int pass) {
      if (m->dim == 2)
        k_node_pattern<9, 4, 25, 9><<<nblk(L.N, 128), 128, 0, st>>>(
            ml.d_conn.p, eptr.p, elist.p, L.N, pass, L.qq_ptr.p, L.ql_ptr.p, L.qq_ptr.p, L.ql_ptr.p, L.qq_col.p,
            L.ql_col.p, bad.p);
      else
        k_node_pattern<27, 8, 125, 27><<<nblk(L.N, 128), 128, 0, st>>>(
            ml.d_conn.p, eptr.p, elist.p, L.N, pass, L.qq_ptr.p, L.ql_ptr.p, L.qq_ptr.p, L.ql_ptr.p, L.qq_col.p,
            L.ql_col.p, bad.p);
    };
    launch_pattern(0);
    EXF_LAUNCH_CHECK();
    int nqq = 0, nql = 0;
    EXF_TRY(exclusive_scan(L.qq_ptr.p, L.N + 1, &nqq, st));
    EXF_TRY(exclusive_scan(L.ql_ptr.p, L.N + 1, &nql, st));
    L.nqq = nqq;
    L.nql = nql;
    EXF_TRY(L.qq_col.alloc(nqq));
    EXF_TRY(L.ql_col.alloc(nql));
    launch_pattern(1);
    EXF_LAUNCH_CHECK();
    int hq = 0, hl = 0;
    EXF_CUDA(cudaMemcpyAsync(&hq, L.qq_ptr.p + L.NL, sizeof(int), cudaMemcpyDeviceToHost, st));
    EXF_CUDA(cudaMemcpyAsync(&hl, L.ql_ptr.p + L.NL, sizeof(int), cudaMemcpyDeviceToHost, st));
    EXF_CUDA(cudaStreamSynchronize(st));
    L.nqqL = hq;
    L.nllL = hl;
    // derived maps
    EXF_TRY(L.diag_pos.alloc(L.N));
    k_diag_pos<<<nblk(L.N, 256), 256, 0, st>>>(L.qq_ptr.p, L.qq_col.p, L.N, L.diag_pos.p);
    EXF_TRY(L.pos_qq.alloc((size_t)ml.nel * nen * nen));
    EXF_TRY(L.pos_ql.alloc((size_t)ml.nel * nen * nvx));
    k_elem_pos<<<nblk(nent, 128), 128, 0, st>>>(ml.d_conn.p, ml.nel, nen, nvx, L.qq_ptr.p, L.qq_col.p, L.ql_ptr.p,
                                                L.ql_col.p, L.pos_qq.p, L.pos_ql.p, bad.p);
    if (s->nv1) {
      EXF_TRY(L.gidx.alloc(L.nqqL));
      k_gidx<<<nblk(L.NL, 128), 128, 0, st>>>(L.qq_ptr.p, L.qq_col.p, L.ql_ptr.p, L.ql_col.p, L.NL, L.gidx.p,
                                              bad.p);
    }
    EXF_LAUNCH_CHECK();
    // DOF CSR
    long nrow = L.ndof;
    EXF_TRY(L.csr_ptr.alloc(nrow + 1));
    EXF_TRY(L.csr_ptr.zero(st));
    k_csr_rowlen<<<nblk(nrow, 256), 256, 0, st>>>(L.qq_ptr.p, L.ql_ptr.p, L.N, L.NL, s->nv2, s->nv1,
                                                  L.csr_ptr.p);
    EXF_LAUNCH_CHECK();
    int nnz = 0;
    EXF_TRY(exclusive_scan(L.csr_ptr.p, nrow + 1, &nnz, st));
    L.nnz = nnz;
    EXF_TRY(L.csr_col.alloc(nnz));
    k_csr_fill<<<nblk(nrow, 256), 256, 0, st>>>(L.qq_ptr.p, L.qq_col.p, L.ql_ptr.p, L.ql_col.p, L.N, L.NL, s->nv2,
                                                s->nv1, L.csr_ptr.p, L.csr_col.p);
    EXF_LAUNCH_CHECK();
    int hbad = 0;
    EXF_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    EXF_CUDA(cudaStreamSynchronize(st));
    if (hbad) {
      set_error("pattern build: inconsistent node pattern on level %d", l);
      return EXF_ERR_STATE;
    }
    // values
    const int d = s->nv2;
    EXF_TRY(L.A.vv.alloc((size_t)d * d * L.nqq));
    EXF_TRY(L.A32.vv.alloc((size_t)d * d * L.nqq));
    if (s->nv1) {
      EXF_TRY(L.A.vp.alloc((size_t)d * L.nql));
      EXF_TRY(L.A.pv.alloc((size_t)d * L.nqqL));
      EXF_TRY(L.A.pp.alloc(L.nllL));
      EXF_TRY(L.A32.vp.alloc((size_t)d * L.nql));
      EXF_TRY(L.A32.pv.alloc((size_t)d * L.nqqL));
      EXF_TRY(L.A32.pp.alloc(L.nllL));
      EXF_TRY(L.h16.alloc(d == 3 ? (size_t)L.nqq : ((size_t)L.nqq + 1) / 2));
      if (d == 3) EXF_TRY(L.h16cx.alloc((size_t)L.nqq + 2));  // 16-byte chunk reads past the end
      if (d == 3) EXF_TRY(L.h16qc.alloc(((size_t)L.nqq + 7) & ~(size_t)3));  // 16-byte chunk reads past the end
      EXF_TRY(L.vsc.alloc((size_t)d * L.N));
    }
    // vectors
    EXF_TRY(L.x.alloc(L.ndof));
    EXF_TRY(L.b.alloc(L.ndof));
    EXF_TRY(L.r.alloc(L.ndof));
    EXF_TRY(L.dx.alloc(L.ndof));
    L.len32 = s->nv1 ? 4L * L.N : (long)L.ndof;
    EXF_TRY(L.x32.alloc(L.len32));
    EXF_TRY(L.b32.alloc(L.len32));
    EXF_TRY(L.r32.alloc(L.len32));
    EXF_TRY(L.dx32.alloc(L.len32));
    EXF_TRY(L.x32.zero(st));
    EXF_TRY(L.b32.zero(st));
    EXF_TRY(L.r32.zero(st));
    EXF_TRY(L.rmask.alloc(L.ndof));
    EXF_TRY(L.x.zero(st));
    EXF_TRY(L.x32.zero(st));
    EXF_TRY(L.dx.zero(st));
    EXF_TRY(L.dx32.zero(st));
  }
  return EXF_OK;
}

// --------------------------------------------------------------- colouring
// T (Gauss-Seidel): item = node, colour = lattice index of level l mod 3 per axis;
// two nodes of one colour never share an element.  NS (Vanka): item = pressure node,
// colour = vertex index mod 3 per axis; the velocity stars of one colour are disjoint.
__global__ void k_item_colour(const int *lat, int nitem, int step, int dim, int *colour) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nitem) return;
  int c = 0, mul = 1;
  for (int d = 0; d < dim; d++) {
    c += ((lat[3 * i + d] / step) % 3) * mul;
    mul *= 3;
  }
  colour[i] = c;
}

// Uploaded meshes (no lattice): greedy first-fit colouring with items in (z, y, x) order of
// their node coordinates.  T: nodes sharing an element conflict (qq); NS: pressure
// vertices whose stars share a node conflict -- the stars holding node n are the vertices
// of ql(n), so the conflicts of vertex m are the union of ql(n) over n in qq(m).  On a
// structured box this reproduces the lattice colouring (the conflicts are the items within
// two lattice steps in every direction, and first fit in lattice order takes
// i%3 + 3 (j%3) + 9 (k%3)).
static int colour_general(exf_sys *s, int l, int nitem, std::vector<int> &col) {
  exf_mesh *m = s->mesh;
  SysLevel &L = s->L[l];
  std::vector<int> qp(L.N + 1), qc(L.nqq), lp(L.N + 1), lc(L.nql);
  EXF_CUDA(cudaMemcpy(qp.data(), L.qq_ptr.p, (L.N + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  EXF_CUDA(cudaMemcpy(qc.data(), L.qq_col.p, L.nqq * sizeof(int), cudaMemcpyDeviceToHost));
  EXF_CUDA(cudaMemcpy(lp.data(), L.ql_ptr.p, (L.N + 1) * sizeof(int), cudaMemcpyDeviceToHost));
  EXF_CUDA(cudaMemcpy(lc.data(), L.ql_col.p, L.nql * sizeof(int), cudaMemcpyDeviceToHost));
  std::vector<int> cptr(nitem + 1, 0), cidx;
  if (s->nv1 == 0) {
    cptr.assign(qp.begin(), qp.begin() + nitem + 1);
    cidx.assign(qc.begin(), qc.begin() + qp[nitem]);
  } else {
    std::vector<int> stamp(nitem, -1);
    for (int v = 0; v < nitem; v++) {
      for (int k = qp[v]; k < qp[v + 1]; k++) {
        const int n = qc[k];
        for (int j = lp[n]; j < lp[n + 1]; j++)
          if (stamp[lc[j]] != v) {
            stamp[lc[j]] = v;
            cidx.push_back(lc[j]);
          }
      }
      cptr[v + 1] = (int)cidx.size();
    }
  }
  const std::vector<int> order = node_zyx_order(m, nitem);
  return colour_items_greedy(m, nitem, order, cptr, cidx, col);
}

int build_colours(exf_sys *s) {
  exf_mesh *m = s->mesh;
  cudaStream_t st = s->stream;
  for (int l = 0; l < s->nlev; l++) {
    SysLevel &L = s->L[l];
    int sl = 1 << (m->nlev - 1 - l);
    int nitem = s->nv1 == 0 ? L.N : L.NL;  // scalar systems colour DOFs, NS pressure nodes
    int step = s->nv1 == 0 ? sl : 2 * sl;
    EXF_TRY(L.item_colour.alloc(nitem));
    std::vector<int> col(nitem);
    if (m->lattice) {
      k_item_colour<<<nblk(nitem, 256), 256, 0, st>>>(m->d_lat.p, nitem, step, m->dim, L.item_colour.p);
      EXF_LAUNCH_CHECK();
      EXF_CUDA(cudaMemcpyAsync(col.data(), L.item_colour.p, nitem * sizeof(int), cudaMemcpyDeviceToHost, st));
      EXF_CUDA(cudaStreamSynchronize(st));
      L.ncolour = m->dim == 2 ? 9 : 27;
    } else {
      L.ncolour = colour_general(s, l, nitem, col);
      EXF_CUDA(cudaMemcpy(L.item_colour.p, col.data(), nitem * sizeof(int), cudaMemcpyHostToDevice));
    }
    L.col_off.assign(L.ncolour + 1, 0);
    for (int i = 0; i < nitem; i++) L.col_off[col[i] + 1]++;
    for (int c = 0; c < L.ncolour; c++) L.col_off[c + 1] += L.col_off[c];
    std::vector<int> items(nitem), pos(L.col_off.begin(), L.col_off.end() - 1);
    for (int i = 0; i < nitem; i++) items[pos[col[i]]++] = i;
    EXF_TRY(L.col_items.alloc(nitem));
    EXF_CUDA(cudaMemcpyAsync(L.col_items.p, items.data(), nitem * sizeof(int), cudaMemcpyHostToDevice, st));
    EXF_CUDA(cudaStreamSynchronize(st));
    if (s->kind == EXF_KIND_NS) {
      // star rows of every colour: the velocity nodes of pressure row m (qq(m)), patch by
      // patch; stars of one colour are disjoint, so each node appears once per colour
      std::vector<int> qp(L.N + 1), qc(L.nqq), lp(L.N + 1), lc(L.nql);
      EXF_CUDA(cudaMemcpy(qp.data(), L.qq_ptr.p, (L.N + 1) * sizeof(int), cudaMemcpyDeviceToHost));
      EXF_CUDA(cudaMemcpy(qc.data(), L.qq_col.p, L.nqq * sizeof(int), cudaMemcpyDeviceToHost));
      EXF_CUDA(cudaMemcpy(lp.data(), L.ql_ptr.p, (L.N + 1) * sizeof(int), cudaMemcpyDeviceToHost));
      EXF_CUDA(cudaMemcpy(lc.data(), L.ql_col.p, L.nql * sizeof(int), cudaMemcpyDeviceToHost));
      // lattice of this level (Q2 nodes): the node at each lattice point, and the offset of
      // every block's column from its row node as an index step in a 9^d tile (TILE
      // kernels; uploaded meshes have no lattice: codes zero, the TILE kernels refused)
      const int dim = m->dim;
      const bool lat = m->lattice;
      for (int d = 0; d < 3; d++) L.Ll[d] = (lat && d < dim) ? 2 * m->lev[l].ne[d] + 1 : 1;
      if (L.Ll[0] > 2048 || L.Ll[1] > 2048 || L.Ll[2] > 1024) {
        set_error("build_colours: level lattice %dx%dx%d exceeds the packed patch origin", L.Ll[0], L.Ll[1], L.Ll[2]);
        return EXF_ERR_UNSUPPORTED;
      }
      auto latl = [&](int n, int d) { return (lat && d < dim) ? m->lat[3 * (size_t)n + d] / sl : 0; };
      std::vector<int> lnode(L.N, 0);
      if (lat)
        for (int n = 0; n < L.N; n++) lnode[((size_t)latl(n, 2) * L.Ll[1] + latl(n, 1)) * L.Ll[0] + latl(n, 0)] = n;
      const int tstep[3] = {1, 9, 81};
      bool far = false;
      auto tcode = [&](int n, int c) {
        int v = 0;
        for (int d = 0; d < dim; d++) {
          const int dd = latl(c, d) - latl(n, d);
          if (dd < -2 || dd > 2) far = true;
          v += dd * tstep[d];
        }
        return (int16_t)v;
      };
      std::vector<int16_t> tq(L.nqq, 0), tl(L.nql, 0);
      if (lat)
        for (int n = 0; n < L.N; n++) {
          for (int k = qp[n]; k < qp[n + 1]; k++) tq[k] = tcode(n, qc[k]);
          for (int k = lp[n]; k < lp[n + 1]; k++) tl[k] = tcode(n, lc[k]);
        }
      if (far) {
        set_error("build_colours: a block couples nodes more than 2 lattice steps apart");
        return EXF_ERR_UNSUPPORTED;
      }
      EXF_TRY(L.latnode.alloc(L.N));
      EXF_CUDA(cudaMemcpy(L.latnode.p, lnode.data(), L.N * sizeof(int), cudaMemcpyHostToDevice));
      EXF_TRY(L.tcq.alloc(L.nqq));
      EXF_CUDA(cudaMemcpy(L.tcq.p, tq.data(), L.nqq * sizeof(int16_t), cudaMemcpyHostToDevice));
      EXF_TRY(L.tcl.alloc(L.nql));
      EXF_CUDA(cudaMemcpy(L.tcl.p, tl.data(), L.nql * sizeof(int16_t), cudaMemcpyHostToDevice));
      // order in which each colour's patches are swept: lattice order (z, y, x) of the
      // vertex, reversed in every other colour, so that a colour starts where the previous
      // one ended and finds the star rows both read still in L2 (the order inside a
      // colour does not change its result: its patches are independent)
      std::vector<int> sweep(items);
      std::vector<long long> rank;
      if (!lat) {  // (z, y, x) order of the vertex coordinates
        const std::vector<int> ord = node_zyx_order(m, nitem);
        rank.assign(nitem, 0);
        for (int i = 0; i < nitem; i++) rank[ord[i]] = i;
      }
      auto lkey = [&](int v) {
        if (!lat) return rank[v];
        return ((long long)latl(v, 2) * L.Ll[1] + latl(v, 1)) * L.Ll[0] + latl(v, 0);
      };
      for (int c = 0; c < L.ncolour; c++) {
        auto b0 = sweep.begin() + L.col_off[c], b1 = sweep.begin() + L.col_off[c + 1];
        std::sort(b0, b1, [&](int a, int b) { return lkey(a) < lkey(b); });
        if (c & 1) std::reverse(b0, b1);
      }
      std::vector<int> rows;
      std::vector<int> pst(L.NL, 0);
      L.vrow_off.assign(L.ncolour + 1, 0);
      for (int c = 0; c < L.ncolour; c++) {
        L.vrow_off[c] = (int)rows.size();
        for (int t = L.col_off[c]; t < L.col_off[c + 1]; t++) {
          int mm = sweep[t];
          pst[mm] = (int)rows.size();
          for (int k = qp[mm]; k < qp[mm + 1]; k++) rows.push_back(qc[k]);
        }
      }
      L.vrow_off[L.ncolour] = (int)rows.size();
      EXF_TRY(L.vrows.alloc(rows.size()));
      EXF_CUDA(cudaMemcpy(L.vrows.p, rows.data(), rows.size() * sizeof(int), cudaMemcpyHostToDevice));
      EXF_TRY(L.pstart.alloc(L.NL));
      EXF_CUDA(cudaMemcpy(L.pstart.p, pst.data(), pst.size() * sizeof(int), cudaMemcpyHostToDevice));
      // row descriptors of the star rows and of the patches (so the sweep kernels start
      // their row products one dependent load earlier), in colour order
      std::vector<int4> vri(rows.size()), pin(2 * (size_t)nitem);
      int kmax = 0, rmax = 0;
      for (int t = 0; t < nitem; t++) {
        const int mm = sweep[t];
        const int K = qp[mm + 1] - qp[mm];
        kmax = std::max(kmax, K);
        for (int g = pst[mm]; g < pst[mm] + K; g++) {
          const int n = rows[g], nq = qp[n + 1] - qp[n], nl = lp[n + 1] - lp[n];
          if (nq > 0xff || nl > 0xff) {
            set_error("build_colours: node row of %d/%d blocks exceeds the packed range", nq, nl);
            return EXF_ERR_UNSUPPORTED;
          }
          rmax = std::max(rmax, nq);
          int tb = 0;
          for (int d = 0; d < dim; d++) tb += (latl(n, d) - latl(mm, d) + 4) * tstep[d];
          vri[g] = make_int4(n, qp[n], lp[n], nq | (nl << 8) | (tb << 16));
        }
        pin[2 * t] = make_int4(mm, pst[mm], qp[mm], lp[mm]);
        pin[2 * t + 1] = make_int4(K, lp[mm + 1] - lp[mm], latl(mm, 0) | (latl(mm, 1) << 11) | (latl(mm, 2) << 22), 0);
      }
      const int smax = dim == 3 ? 125 : 25;
      L.tile_ok = lat && kmax <= smax && rmax <= smax;
      EXF_TRY(L.vrinfo.alloc(vri.size()));
      EXF_CUDA(cudaMemcpy(L.vrinfo.p, vri.data(), vri.size() * sizeof(int4), cudaMemcpyHostToDevice));
      if (dim == 3) {  // star-major record offsets of the BULK smoother
        std::vector<long long> so(vri.size() + 1, 0);
        for (size_t g = 0; g < vri.size(); g++) {  // 2 header records, blocks, columns, 9th values, couplings
          const int nk = vri[g].w & 0xff, nl = (vri[g].w >> 8) & 0xff;
          so[g + 1] = so[g] + 2 + nk + ((nk + 3) >> 2) + ((nk + 7) >> 3) + nl;
        }
        L.nstar = so.back();
        so.push_back(so.back());  // 16-byte copies of offset pairs may read one entry past the end
        EXF_TRY(L.soff.alloc(so.size()));
        EXF_CUDA(cudaMemcpy(L.soff.p, so.data(), so.size() * sizeof(long long), cudaMemcpyHostToDevice));
        L.soff_h = std::move(so);
        L.bsched_G = 0;
      }
      EXF_TRY(L.pinfo.alloc(pin.size()));
      EXF_CUDA(cudaMemcpy(L.pinfo.p, pin.data(), pin.size() * sizeof(int4), cudaMemcpyHostToDevice));
      const size_t ne = rows.size() * (size_t)s->nv2;
      EXF_TRY(L.vk64.alloc(3 * ne));
      EXF_TRY(L.vk32.alloc(3 * ne));
      EXF_TRY(L.pk64.alloc(2 * (size_t)L.NL));
      EXF_TRY(L.pk32.alloc(2 * (size_t)L.NL));
      EXF_TRY(L.vres64.alloc(ne + L.NL));
      EXF_TRY(L.vres32.alloc(ne + L.NL));
    }
  }
  return EXF_OK;
}

// ---------------------------------------------------------------- transfers
// 1D Lagrange bases on {-1,0,+1} and the linear basis on {-1,+1} (src/MGFE.C:252-263)
static double lag1(int a, double x) {
  if (a == 0) return .5 * x * (x - 1.);
  if (a == 2) return .5 * x * (x + 1.);
  return 1. - x * x;
}
static double lin1(int a, double x) { return a == 0 ? .5 * (1. - x) : .5 * (1. + x); }

// Prolongation rows: the fine node's row holds the parent element's shape functions at
// the node, |v| > 1e-8 kept, columns sorted (gencase compute_prol_qq,
// MGGenCase.C:2308-2393; the values equal the embedding matrices of
// src/MGGeomEl.C:182-600).  Restriction = transposed prolongation, |v| > 1e-6
// (compute_res_qq, MGGenCase.C:2452-2569).  Both are node-level; every variable
// component uses the same node operator (no inter-variable coupling).
static void build_prol_host(const exf_mesh *m, int l, bool quad, Transfer &P) {
  const int dim = m->dim, nen = m->nen, nvx = m->nvx;
  const MeshLevel &fl = m->lev[l], &cl = m->lev[l - 1];
  int nrow = quad ? fl.nnodes : cl.nnodes;  // Q1 nodes of level l = Q2 nodes of level l-1
  int s_f = 1 << (m->nlev - 1 - l), s_c = 2 * s_f;
  std::vector<int> own(fl.nnodes, -1);
  for (int e = 0; e < fl.nel; e++)
    for (int k = 0; k < nen; k++) {
      int nd = fl.conn[(size_t)e * nen + k];
      if (own[nd] < 0) own[nd] = e;
    }
  P.nrow = nrow;
  P.h_ptr.assign(nrow + 1, 0);
  P.h_col.clear();
  P.h_val.clear();
  for (int i = 0; i < nrow; i++) {
    int e = own[i];
    int ex[3] = {e % fl.ne[0], (e / fl.ne[0]) % fl.ne[1], e / (fl.ne[0] * fl.ne[1])};
    int pe[3] = {ex[0] >> 1, ex[1] >> 1, ex[2] >> 1};
    int pel = (pe[2] * cl.ne[1] + pe[1]) * cl.ne[0] + pe[0];
    const int *pc = &cl.conn[(size_t)pel * nen];
    double xi[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) xi[d] = -1. + (double)(m->lat[3 * i + d] - 2 * pe[d] * s_c) / (double)s_c;
    std::vector<std::pair<int, double>> ent;
    int nsh = quad ? nen : nvx;
    for (int kj = 0; kj < nsh; kj++) {
      const int *abc = dim == 2 ? Q9_ABC[kj] : H27_ABC[kj];
      double v = 1.;
      for (int d = 0; d < dim; d++) v *= quad ? lag1(abc[d], xi[d]) : lin1(abc[d], xi[d]);
      if (fabs(v) > 1e-8) ent.push_back({pc[kj], v});
    }
    std::sort(ent.begin(), ent.end());
    for (auto &pv : ent) {
      P.h_col.push_back(pv.first);
      P.h_val.push_back(pv.second);
    }
    P.h_ptr[i + 1] = (int)P.h_col.size();
  }
}

// Uploaded meshes: the same rows from the parent elements.  A fine element lies in the
// sub-cell of its parent at the corner it shares with the parent: its local vertex k is
// the parent's vertex k (uniform refinement keeps the parent's orientation), so its local
// node with offsets (a,b,c) sits at xi = -1 + (2 pos + (a,b,c)) / 2 in the parent, pos =
// (parent vertex k's offsets) / 2.  Returns false when an element breaks that rule or the
// quadratic rows do not reproduce the fine node coordinates (the parent's Q2 map places a
// uniform refinement's nodes, curved elements included; the linear rows share the
// placement, and a bilinear interpolation of curved coordinates is not expected to match).
static bool build_prol_parent(const exf_mesh *m, int l, bool quad, Transfer &P) {
  const int dim = m->dim, nen = m->nen, nvx = m->nvx;
  const MeshLevel &fl = m->lev[l], &cl = m->lev[l - 1];
  const int nrow = quad ? fl.nnodes : cl.nnodes;
  std::vector<int> own(fl.nnodes, -1), ownk(fl.nnodes, -1);
  for (int e = 0; e < fl.nel; e++)
    for (int k = 0; k < nen; k++) {
      const int nd = fl.conn[(size_t)e * nen + k];
      if (own[nd] < 0) {
        own[nd] = e;
        ownk[nd] = k;
      }
    }
  P.nrow = nrow;
  P.h_ptr.assign(nrow + 1, 0);
  P.h_col.clear();
  P.h_val.clear();
  for (int i = 0; i < nrow; i++) {
    const int e = own[i];
    if (e < 0) return false;
    const int pel = fl.parent[e];
    const int *fc = &fl.conn[(size_t)e * nen];
    const int *pc = &cl.conn[(size_t)pel * nen];
    int corner = -1;
    for (int k = 0; k < nvx; k++)
      if (fc[k] == pc[k]) corner = corner < 0 ? k : -2;
    if (corner < 0) return false;
    const int *cabc = dim == 2 ? Q9_ABC[corner] : H27_ABC[corner];
    const int *fabc = dim == 2 ? Q9_ABC[ownk[i]] : H27_ABC[ownk[i]];
    double xi[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) xi[d] = -1. + (double)(cabc[d] + fabc[d]) / 2.;
    std::vector<std::pair<int, double>> ent;
    const int nsh = quad ? nen : nvx;
    double xr[3] = {0, 0, 0};
    for (int kj = 0; kj < nsh; kj++) {
      const int *abc = dim == 2 ? Q9_ABC[kj] : H27_ABC[kj];
      double v = 1.;
      for (int d = 0; d < dim; d++) v *= quad ? lag1(abc[d], xi[d]) : lin1(abc[d], xi[d]);
      for (int d = 0; d < dim; d++) xr[d] += v * m->xyz[(size_t)pc[kj] + (size_t)d * m->ntop];
      if (fabs(v) > 1e-8) ent.push_back({pc[kj], v});
    }
    for (int d = 0; quad && d < dim; d++) {
      const double ext = m->box[2 * d + 1] - m->box[2 * d];
      if (fabs(xr[d] - m->xyz[(size_t)i + (size_t)d * m->ntop]) > 1e-9 * (ext > 0 ? ext : 1.)) return false;
    }
    std::sort(ent.begin(), ent.end());
    for (auto &pv : ent) {
      P.h_col.push_back(pv.first);
      P.h_val.push_back(pv.second);
    }
    P.h_ptr[i + 1] = (int)P.h_col.size();
  }
  return true;
}

static void transpose_host(const Transfer &P, int ncol, Transfer &R) {
  R.nrow = ncol;
  R.h_ptr.assign(ncol + 1, 0);
  for (int i = 0; i < P.nrow; i++)
    for (int q = P.h_ptr[i]; q < P.h_ptr[i + 1]; q++)
      if (fabs(P.h_val[q]) > 1e-6) R.h_ptr[P.h_col[q] + 1]++;
  for (int i = 0; i < ncol; i++) R.h_ptr[i + 1] += R.h_ptr[i];
  R.h_col.assign(R.h_ptr[ncol], 0);
  R.h_val.assign(R.h_ptr[ncol], 0.);
  std::vector<int> fill(R.h_ptr.begin(), R.h_ptr.end() - 1);
  for (int i = 0; i < P.nrow; i++)
    for (int q = P.h_ptr[i]; q < P.h_ptr[i + 1]; q++)
      if (fabs(P.h_val[q]) > 1e-6) {
        int c = P.h_col[q];
        R.h_col[fill[c]] = i;
        R.h_val[fill[c]] = P.h_val[q];
        fill[c]++;
      }
}

static int upload_transfer(Transfer &T) {
  EXF_TRY(T.ptr.alloc(T.h_ptr.size()));
  EXF_TRY(T.col.alloc(T.h_col.size()));
  EXF_TRY(T.val.alloc(T.h_val.size()));
  EXF_TRY(T.val32.alloc(T.h_val.size()));
  std::vector<float> v32(T.h_val.begin(), T.h_val.end());
  EXF_CUDA(cudaMemcpy(T.ptr.p, T.h_ptr.data(), T.h_ptr.size() * sizeof(int), cudaMemcpyHostToDevice));
  if (!T.h_col.empty()) {
    EXF_CUDA(cudaMemcpy(T.col.p, T.h_col.data(), T.h_col.size() * sizeof(int), cudaMemcpyHostToDevice));
    EXF_CUDA(cudaMemcpy(T.val.p, T.h_val.data(), T.h_val.size() * sizeof(double), cudaMemcpyHostToDevice));
    EXF_CUDA(cudaMemcpy(T.val32.p, v32.data(), v32.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  return EXF_OK;
}

// Transfers of every level pair: from the lattice (generated boxes), from the parent
// elements (uploaded with parents), or left empty until exf_sys_set_transfer supplies
// them (uploaded without parents; solves refuse to start until then).
int build_transfers(exf_sys *s) {
  exf_mesh *m = s->mesh;
  if (!m->lattice && !m->has_parent) return EXF_OK;
  for (int l = 1; l < s->nlev; l++) {
    SysLevel &F = s->L[l];
    SysLevel &C = s->L[l - 1];
    for (int q = 0; q < (s->nv1 ? 2 : 1); q++) {
      const bool quad = q == 0;
      Transfer &P = quad ? F.Pq : F.Pl;
      Transfer &R = quad ? C.Rq : C.Rl;
      if (m->lattice) {
        build_prol_host(m, l, quad, P);
      } else if (!build_prol_parent(m, l, quad, P)) {
        set_error("build_transfers: level %d: a child element is not a sub-cell of its parent with the parent's "
                  "orientation, or the prolongation does not reproduce the node coordinates", l);
        return EXF_ERR_ARG;
      }
      EXF_TRY(upload_transfer(P));
      transpose_host(P, quad ? C.N : C.NL, R);
      EXF_TRY(upload_transfer(R));
    }
  }
  return EXF_OK;
}

// one block of a transfer operator in gencase's dataset layout (rows, columns, cumulative
// row offsets, level-local column nodes, values): columns sorted per row, uploaded
int set_transfer(exf_sys *s, int lev, int kind, int block, const int dim[2], const int *len, const int *pos,
                 const double *val) {
  if (lev < 0 || lev >= s->nlev || (kind != 0 && kind != 1) || (block != 1 && block != 2) || !dim || !len ||
      (!pos && dim[0] > 0) || (block == 1 && !s->nv1)) {
    set_error("exf_sys_set_transfer: bad argument");
    return EXF_ERR_ARG;
  }
  const int other = kind == 0 ? lev - 1 : lev + 1;
  if (other < 0 || other >= s->nlev) {
    set_error("exf_sys_set_transfer: no level %d next to level %d", other, lev);
    return EXF_ERR_ARG;
  }
  SysLevel &L = s->L[lev], &O = s->L[other];
  const int nrow = block == 2 ? L.N : L.NL, ncol = block == 2 ? O.N : O.NL;
  if (dim[0] != nrow || dim[1] != ncol) {
    set_error("exf_sys_set_transfer: block is %dx%d, level %d needs %dx%d", dim[0], dim[1], lev, nrow, ncol);
    return EXF_ERR_ARG;
  }
  if (len[0] != 0) {
    set_error("exf_sys_set_transfer: row offsets must start at 0");
    return EXF_ERR_ARG;
  }
  Transfer T;
  T.nrow = nrow;
  T.h_ptr.assign(len, len + nrow + 1);
  for (int i = 0; i < nrow; i++) {
    if (len[i + 1] < len[i]) {
      set_error("exf_sys_set_transfer: row offsets decrease at row %d", i);
      return EXF_ERR_ARG;
    }
    std::vector<std::pair<int, double>> ent;
    for (int q = len[i]; q < len[i + 1]; q++) {
      if (pos[q] < 0 || pos[q] >= ncol) {
        set_error("exf_sys_set_transfer: column %d of row %d outside 0..%d", pos[q], i, ncol - 1);
        return EXF_ERR_ARG;
      }
      ent.push_back({pos[q], val ? val[q] : 0.});
    }
    std::stable_sort(ent.begin(), ent.end(), [](const std::pair<int, double> &a, const std::pair<int, double> &b) {
      return a.first < b.first;
    });
    for (auto &e : ent) {
      T.h_col.push_back(e.first);
      T.h_val.push_back(e.second);
    }
  }
  EXF_TRY(upload_transfer(T));
  Transfer &dst = kind == 0 ? (block == 2 ? L.Pq : L.Pl) : (block == 2 ? L.Rq : L.Rl);
  dst = std::move(T);
  s->buf_epoch++;
  return EXF_OK;
}

// every transfer a V-cycle needs is present
bool transfers_ready(const exf_sys *s) {
  for (int l = 1; l < s->nlev; l++) {
    const SysLevel &F = s->L[l], &C = s->L[l - 1];
    if (F.Pq.nrow != F.N || C.Rq.nrow != C.N) return false;
    if (s->nv1 && (F.Pl.nrow != F.NL || C.Rl.nrow != C.NL)) return false;
  }
  return true;
}

// restriction row mask: bc[0][top dof] % 2 (src/MGSolverDA.C:2423-2425)
__global__ void k_rmask(const int *bc0, int N, int NL, int Ntop, int nv2, int nv1, double *mask) {
  long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long nrow = (long)nv2 * N + (long)nv1 * NL;
  if (r >= nrow) return;
  long td;
  if (r < (long)nv2 * N) td = (r / N) * (long)Ntop + (r % N);
  else td = (long)nv2 * Ntop + (r - (long)nv2 * N);
  mask[r] = (double)(bc0[td] % 2);
}

int update_rmask(exf_sys *s) {
  int Ntop = s->L[s->nlev - 1].N;
  for (int l = 0; l < s->nlev; l++) {
    SysLevel &L = s->L[l];
    k_rmask<<<nblk(L.ndof, 256), 256, 0, s->stream>>>(s->d_bc0.p, L.N, L.NL, Ntop, s->nv2, s->nv1, L.rmask.p);
    EXF_LAUNCH_CHECK();
  }
  return EXF_OK;
}

// ---------------------------------------------------------------- wall distances
// MGMesh::B_dist (src/MGMesh.C:1285-1350): per element of a level, the distance from its
// centre (the mean of its Q2 nodes) to the nearest centre (the mean of the side's nodes) of
// a wall side of the same level; one thread per element, the sides' centres in order
__global__ void k_wall_dist(int nel, int nen, const int *__restrict__ conn, const double *__restrict__ xyz, int ntop,
                            int dim, const double *__restrict__ wc, int nw, double *__restrict__ dist) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  double xm[3] = {0., 0., 0.};
  for (int d = 0; d < dim; d++) {
    for (int k = 0; k < nen; k++) xm[d] += xyz[conn[(long)e * nen + k] + (long)d * ntop];
    xm[d] /= nen;
  }
  double dmin = 1.e+20;
  for (int w = 0; w < nw; w++) {
    double dq = 0.;
    for (int d = 0; d < dim; d++) {
      const double t = xm[d] - wc[(long)w * 3 + d];
      dq += t * t;
    }
    if (dq < dmin) dmin = dq;
  }
  dist[e] = sqrt(dmin);
}

}  // namespace exf

using namespace exf;

int exf_mesh_wall_dist(const exf_mesh *m, const int *wall_node, double *dist) {
  if (!m || !wall_node || !dist) {
    set_error("exf_mesh_wall_dist: bad argument");
    return EXF_ERR_ARG;
  }
  EXF_CUDA(cudaSetDevice(m->device));
  EXF_TRY(mesh_pull_xyz(const_cast<exf_mesh *>(m)));
  const int dim = m->dim, nen = m->nen, nsn = m->nsn, nside = m->nsides;
  long off = 0;
  for (int l = 0; l < m->nlev; l++) {
    const MeshLevel &ml = m->lev[l];
    // the level's wall sides: boundary sides whose nodes are all wall nodes, centres as
    // the mean of the side's nodes (the boundary element's NDOF_FEMB nodes)
    std::vector<double> wc;
    for (int e = 0; e < ml.nel; e++)
      for (int sd = 0; sd < nside; sd++) {
        if (ml.neigh[(size_t)e * nside + sd] != -1) continue;
        bool wall = true;
        double c[3] = {0., 0., 0.};
        for (int k = 0; k < nsn; k++) {
          const int n = ml.conn[(size_t)e * nen + (dim == 2 ? Q9_SIDE[sd][k] : H27_FACE[sd][k])];
          wall = wall && wall_node[n] != 0;
          for (int d = 0; d < dim; d++) c[d] += m->xyz[(size_t)n + (size_t)d * m->ntop];
        }
        if (!wall) continue;
        for (int d = 0; d < 3; d++) wc.push_back(d < dim ? c[d] / nsn : 0.);
      }
    DBuf<double> d_wc, d_dist;
    EXF_TRY(d_wc.alloc(std::max<size_t>(1, wc.size())));
    EXF_TRY(d_dist.alloc(ml.nel));
    if (!wc.empty()) EXF_CUDA(cudaMemcpy(d_wc.p, wc.data(), wc.size() * sizeof(double), cudaMemcpyHostToDevice));
    k_wall_dist<<<(ml.nel + 127) / 128, 128>>>(ml.nel, nen, ml.d_conn.p, m->d_xyz.p, m->ntop, dim, d_wc.p,
                                               (int)(wc.size() / 3), d_dist.p);
    EXF_LAUNCH_CHECK();
    EXF_COUNT(1);
    EXF_CUDA(cudaMemcpy(dist + off, d_dist.p, ml.nel * sizeof(double), cudaMemcpyDeviceToHost));
    off += ml.nel;
  }
  return EXF_OK;
}
