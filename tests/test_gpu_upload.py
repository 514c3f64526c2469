"""Meshes and operators from host arrays (needs a B200).

exf_mesh_upload takes the hierarchy MGMesh::read_c holds (coordinates, per-level element
connectivity in top node numbers, neighbours, and the parent elements gencase records);
exf_sys_set_transfer takes the transfer operators in gencase's dataset layout; and
exf_sys_check_pattern checks a level's sparsity against gencase's matrix datasets.

  * the structured box pushed through the upload path gives the same bits as
    exf_mesh_create (colourings, patterns, transfers, matrices, solutions) for the
    Navier-Stokes systems; for the temperature system the Gauss-Seidel colouring of the
    upload path is first fit on the element-sharing graph, which is not the lattice's
    mod-3 colouring (two midpoints two lattice steps apart share no element), so there the
    solutions agree within 1e-11 at a tight tolerance;
  * a copy with nodes permuted inside each nesting class and elements permuted inside
    each level gives the permuted solution (within 1e-12);
  * transfers supplied as gencase blocks give the same bits as those built from parents,
    and solves refuse to start before they are set;
  * gencase-ordered (unsorted) pattern rows are accepted, a row missing a coupling is not.
"""
import numpy as np
import pytest

import exfemus_b200 as ex
from exfemus_b200 import _lib, workloads

from conftest import rel

pytestmark = pytest.mark.gpu

CASES = {
    "heat2d": (2, 3, (4, 4), (0, 1, 0, 1), _lib.KIND_T, _lib.BC_HEAT_DIRICHLET, dict()),
    "cavity2d": (2, 3, (4, 4), (0, 1, 0, 1), _lib.KIND_NS, _lib.BC_CAVITY, dict(inv_re=1 / 400.)),
    "channel3d": (3, 2, (4, 2, 2), (0, 4, 0, 1, 0, 1), _lib.KIND_NS, _lib.BC_CHANNEL, dict(inv_re=0.01)),
}


def structured_arrays(gm, n0):
    """The upload arrays of a generated box, with the parent of element (ex, ey, ez) the
    coarse element (ex/2, ey/2, ez/2)."""
    dim, nlev = gm.dim, gm.nlev
    conn, neigh, parent = [], [], [None]
    for lev in range(nlev):
        c, nb, _ = gm.conn(lev)
        conn.append(c)
        neigh.append(nb)
        if lev > 0:
            ne = [(n0[d] << lev) if d < dim else 1 for d in range(3)]
            nc = [(n0[d] << (lev - 1)) if d < dim else 1 for d in range(3)]
            e = np.arange(c.shape[0])
            ex_, ey_, ez_ = e % ne[0], (e // ne[0]) % ne[1], e // (ne[0] * ne[1])
            parent.append(((ez_ // 2) * nc[1] + ey_ // 2) * nc[0] + ex_ // 2)
    return dict(dim=dim, nnodes=[gm.nnodes(l) for l in range(nlev)], nvert0=gm.nvert0, xyz=gm.xyz(), conn=conn,
                neigh=neigh, parent=parent)


def make_sys(mesh, name, xold_of=None):
    dim, nlev, n0, box, kind, preset, pk = CASES[name]
    s = (ex.MGSolNS if kind == _lib.KIND_NS else ex.MGSolT)(mesh)
    s.GenBc(preset)
    s.phys = ex.phys(**pk)
    xyz = mesh.xyz()
    if kind == _lib.KIND_NS:
        x0 = workloads.ns_initial(dict(box=box, bc=preset), xyz, mesh.ntop, s.ntop_dof)
        N = mesh.ntop
        for a in range(dim):  # a smooth interior field, so the advection terms are exercised
            x0[a * N:(a + 1) * N] += 0.3 * np.sin(3 * xyz[0] + a) * np.cos(2 * xyz[1])
        b0, _ = s.bc()
        x0[:dim * N][b0[:dim * N] == 0] = workloads.ns_initial(dict(box=box, bc=preset), xyz, N,
                                                               s.ntop_dof)[:dim * N][b0[:dim * N] == 0]
    else:
        x0 = np.zeros(s.ntop_dof)
        c, _, _ = mesh.conn(nlev - 1)  # a source that follows the element's position
        cx, cy = xyz[0][c[:, :4]].mean(axis=1), xyz[1][c[:, :4]].mean(axis=1)
        s.set_source(1.0 + 0.1 * np.sin(7 * cx) * np.cos(5 * cy))
    s.set_xold(x0)
    return s, x0


def params(name, **kw):
    ns = CASES[name][4] == _lib.KIND_NS
    return ex.mg_params(eps=kw.pop("eps", 1e-11), max_cycles=200, nu_pre=3 if ns else 2, nu_post=3 if ns else 2,
                        smoother=_lib.SMOOTH_VANKA if ns else _lib.SMOOTH_GS, omega=0.4, **kw)


@pytest.mark.parametrize("name", list(CASES))
def test_structured_box_through_upload_is_bit_identical(name, gpu_lib):
    dim, nlev, n0, box, kind, preset, pk = CASES[name]
    gm = ex.Mesh(dim, nlev, n0, box)
    um = ex.Mesh.upload(**structured_arrays(gm, n0))
    for lev in range(nlev):
        for a, b in zip(gm.conn(lev), um.conn(lev)):
            assert np.array_equal(a, b)
    gs, x0 = make_sys(gm, name)
    us, ux0 = make_sys(um, name)
    assert np.array_equal(x0, ux0)
    for a, b in zip(gs.bc(), us.bc()):
        assert np.array_equal(a, b)
    same_colours = kind == _lib.KIND_NS
    for lev in range(nlev):
        if same_colours:
            assert gs.colours(lev)[0] == us.colours(lev)[0]
            assert np.array_equal(gs.colours(lev)[1], us.colours(lev)[1])
        for a, b in zip(gs.pattern(lev), us.pattern(lev)):
            assert np.array_equal(a, b)
        if lev > 0:
            for a, b in zip(gs.prol(lev), us.prol(lev)):
                assert np.array_equal(a, b)
        if lev < nlev - 1:
            for a, b in zip(gs.rest(lev), us.rest(lev)):
                assert np.array_equal(a, b)
    gs.assemble_all()
    us.assemble_all()
    for lev in range(nlev):
        assert np.array_equal(gs.matrix(lev), us.matrix(lev))
    assert np.array_equal(gs.rhs(), us.rhs())
    for prec in (_lib.PREC_FP64, _lib.PREC_MIXED):
        out = []
        for s in (gs, us):
            s.set_x(x0)
            st = s.solve(params(name, precision=prec, eps=1e-11 if same_colours else 1e-13))
            assert st.converged
            out.append((s.x(), list(st.hist[:st.cycles])))
        if same_colours:
            assert np.array_equal(out[0][0], out[1][0])
            assert out[0][1] == out[1][1]
        else:
            assert rel(out[1][0], out[0][0]) < 1e-11


def permuted_arrays(arr, seed):
    """Nodes permuted inside each nesting class ([0, nvert0), [nvert0, nnodes[0]),
    [nnodes[L-1], nnodes[L])) and elements inside each level; returns the arrays and the
    node permutation (new index of old node i)."""
    rng = np.random.default_rng(seed)
    bounds = [0, arr["nvert0"]] + list(arr["nnodes"])
    pi = np.arange(bounds[-1])
    for a, b in zip(bounds[:-1], bounds[1:]):
        pi[a:b] = a + rng.permutation(b - a)
    xyz = np.zeros_like(arr["xyz"])
    xyz[:, pi] = arr["xyz"]
    conn, neigh, parent, sig = [], [], [None], []
    for lev, (c, nb) in enumerate(zip(arr["conn"], arr["neigh"])):
        s = rng.permutation(c.shape[0])  # new index of old element e
        sig.append(s)
        cn = np.empty_like(c)
        cn[s] = pi[c]
        nn = np.empty_like(nb)
        nn[s] = np.where(nb >= 0, s[np.maximum(nb, 0)], -1)
        conn.append(cn)
        neigh.append(nn)
        if lev > 0:
            pn = np.empty(c.shape[0], np.int64)
            pn[s] = sig[lev - 1][arr["parent"][lev]]
            parent.append(pn)
    return dict(arr, xyz=xyz, conn=conn, neigh=neigh, parent=parent), pi


@pytest.mark.parametrize("name", list(CASES))
def test_permuted_copy_gives_the_permuted_solution(name, gpu_lib):
    dim, nlev, n0, box, kind, preset, pk = CASES[name]
    gm = ex.Mesh(dim, nlev, n0, box)
    arr = structured_arrays(gm, n0)
    parr, pi = permuted_arrays(arr, seed=5)
    pm = ex.Mesh.upload(**parr)
    gs, x0 = make_sys(gm, name)
    ps, px0 = make_sys(pm, name)
    N, top = gm.ntop, nlev - 1
    # DOF permutation of the top level: component blocks of N nodes, then the pressure
    nv2 = dim if kind == _lib.KIND_NS else 1
    dperm = np.concatenate([a * N + pi for a in range(nv2)] +
                           ([nv2 * N + pi[:gm.nnodes(top - 1)]] if kind == _lib.KIND_NS else []))
    assert np.array_equal(px0[dperm], x0)
    for a, b in zip(gs.bc(), ps.bc()):
        assert np.array_equal(b[dperm], a)
    gs.assemble_all()
    ps.assemble_all()
    assert rel(ps.rhs()[dperm], gs.rhs()) < 1e-14
    for s, x in ((gs, x0), (ps, px0)):
        s.set_x(x)
        assert s.solve(params(name, eps=1e-12)).converged
    assert rel(ps.x()[dperm], gs.x()) < 1e-12


@pytest.mark.parametrize("name", list(CASES))
def test_transfers_from_gencase_blocks(name, gpu_lib):
    dim, nlev, n0, box, kind, preset, pk = CASES[name]
    gm = ex.Mesh(dim, nlev, n0, box)
    arr = structured_arrays(gm, n0)
    ref_mesh = ex.Mesh.upload(**arr)
    bare = ex.Mesh.upload(**dict(arr, parent=None))
    rs, x0 = make_sys(ref_mesh, name)
    bs, _ = make_sys(bare, name)
    bs.assemble_all()
    with pytest.raises(ex.ExfError) as e:
        bs.solve(params(name))
    assert e.value.code == _lib.EXF_ERR_STATE
    nv2 = dim if kind == _lib.KIND_NS else 1
    for lev in range(1, nlev):
        rp, col, val = rs.prol(lev)
        Nf, Nc = gm.nnodes(lev), gm.nnodes(lev - 1)
        NLf = gm.nnodes(lev - 1)
        NLc = gm.nnodes(lev - 2) if lev >= 2 else gm.nvert0
        import scipy.sparse as sp
        P = sp.csr_matrix((val, col, rp), shape=(rs.ndof(lev), rs.ndof(lev - 1)))
        blocks = [(2, P[:Nf, :Nc], Nf, Nc)]
        if kind == _lib.KIND_NS:
            blocks.append((1, P[nv2 * Nf:nv2 * Nf + NLf, nv2 * Nc:nv2 * Nc + NLc], NLf, NLc))
        for block, B, nr, nc in blocks:
            B = sp.csr_matrix(B)
            # gencase writes rows in its own column order: reverse each row
            pos = np.concatenate([B.indices[B.indptr[i]:B.indptr[i + 1]][::-1] for i in range(nr)])
            vals = np.concatenate([B.data[B.indptr[i]:B.indptr[i + 1]][::-1] for i in range(nr)])
            bs.set_transfer(lev, 0, block, (nr, nc), B.indptr, pos, vals)
            R = sp.csr_matrix(B.T)  # compute_res_qq: the transposed embedding, |v| > 1e-6
            R.data[np.abs(R.data) <= 1e-6] = 0.0
            R.eliminate_zeros()
            R.sort_indices()
            bs.set_transfer(lev - 1, 1, block, (nc, nr), R.indptr, R.indices, R.data)
    for lev in range(nlev):
        if lev > 0:
            for a, b in zip(rs.prol(lev), bs.prol(lev)):
                assert np.array_equal(a, b)
        if lev < nlev - 1:
            for a, b in zip(rs.rest(lev), bs.rest(lev)):
                assert np.array_equal(a, b)
    rs.assemble_all()
    out = []
    for s in (rs, bs):
        s.set_x(x0)
        st = s.solve(params(name))
        assert st.converged
        out.append(s.x())
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("name", list(CASES))
def test_transfer_blocks_written_and_read_back(name, gpu_lib):
    """exf_sys_get_transfer writes each Prol/Rest block in gencase's layout: the blocks
    equal the node blocks of the DOF-level operators, and supplied to an uploaded mesh
    without parents they give that system the same operators and solution."""
    import scipy.sparse as sp
    dim, nlev, n0, box, kind, preset, pk = CASES[name]
    gm = ex.Mesh(dim, nlev, n0, box)
    gs, x0 = make_sys(gm, name)
    bare = ex.Mesh.upload(**dict(structured_arrays(gm, n0), parent=None))
    bs, _ = make_sys(bare, name)
    blocks = (2, 1) if kind == _lib.KIND_NS else (2,)
    for lev in range(nlev):
        for kk in (0, 1):
            if (kk == 0 and lev == 0) or (kk == 1 and lev == nlev - 1):
                continue
            rp, col, val = gs.prol(lev) if kk == 0 else gs.rest(lev)
            other = lev - 1 if kk == 0 else lev + 1
            D = sp.csr_matrix((val, col, rp), shape=(gs.ndof(lev), gs.ndof(other)))
            for block in blocks:
                dm, ln, pos, v = gs.get_transfer(lev, kk, block)
                B = sp.csr_matrix((v, pos, ln), shape=tuple(dm))
                if block == 2:
                    R = D[:dm[0], :dm[1]]
                else:
                    r0, c0 = dim * gm.nnodes(lev), dim * gm.nnodes(other)
                    R = D[r0:r0 + dm[0], c0:c0 + dm[1]]
                if kk == 1:  # the DOF-level restriction carries the bc0 % 2 row mask
                    keep = np.asarray(abs(R).sum(axis=1)).ravel() > 0
                    B = sp.diags(keep.astype(float)) @ B
                assert abs(B - R).max() == 0.0, (lev, kk, block)
                bs.set_transfer(lev, kk, block, dm, ln, pos, v)
    for lev in range(nlev):
        if lev > 0:
            for a, b in zip(gs.prol(lev), bs.prol(lev)):
                assert np.array_equal(a, b)
        if lev < nlev - 1:
            for a, b in zip(gs.rest(lev), bs.rest(lev)):
                assert np.array_equal(a, b)
    gs.assemble_all()
    bs.assemble_all()
    out = []
    for s_ in (gs, bs):
        s_.set_x(x0)
        st = s_.solve(params(name))
        assert st.converged
        out.append(s_.x())
    if kind == _lib.KIND_NS:
        assert np.array_equal(out[0], out[1])
    else:  # the uploaded T system colours its Gauss-Seidel sweep differently
        assert rel(out[1], out[0]) < 1e-9
    with pytest.raises(ex.ExfError) as e:
        bs.get_transfer(0, 0, 2)  # level 0 has no prolongation
    assert e.value.code == _lib.EXF_ERR_ARG


@pytest.mark.parametrize("name", ["heat2d", "cavity2d"])
def test_pattern_check_against_gencase_blocks(name, gpu_lib):
    dim, nlev, n0, box, kind, preset, pk = CASES[name]
    gm = ex.Mesh(dim, nlev, n0, box)
    s, _ = make_sys(gm, name)
    rng = np.random.default_rng(2)
    for lev in range(nlev):
        rp, col = s.pattern(lev)
        N = gm.nnodes(lev)
        NL = gm.nnodes(lev - 1) if lev else gm.nvert0
        nv2 = dim if kind == _lib.KIND_NS else 1
        blocks = {22: (0, N, 0, N)}
        if kind == _lib.KIND_NS:
            blocks.update({21: (0, N, nv2 * N, NL), 12: (nv2 * N, NL, 0, N), 11: (nv2 * N, NL, nv2 * N, NL)})
        for block, (r0, nr, c0, nc) in blocks.items():
            rows = []
            for i in range(nr):
                c = col[rp[r0 + i]:rp[r0 + i + 1]]
                c = c[(c >= c0) & (c < c0 + nc)] - c0
                rows.append(rng.permutation(c))
            length = np.concatenate([[0], np.cumsum([len(r) for r in rows])])
            pos = np.concatenate(rows)
            assert s.check_pattern(lev, block, (nr, nc), length, pos) == _lib.EXF_OK
            bad = np.concatenate([rows[0][1:]] + rows[1:])
            blen = np.concatenate([[0], np.cumsum([len(rows[0]) - 1] + [len(r) for r in rows[1:]])])
            assert s.check_pattern(lev, block, (nr, nc), blen, bad) == _lib.EXF_ERR_ARG


def coord_match(xa, xb):
    """sigma with xb[:, sigma[i]] == xa[:, i] (both point sets equal up to 1e-12)."""
    def order(x):
        r = np.round(np.asarray(x, float).T, 12)
        return np.lexsort(r.T[::-1])
    oa, ob = order(xa), order(xb)
    assert np.abs(xa[:, oa] - xb[:, ob]).max() < 1e-12
    sigma = np.empty(xa.shape[1], dtype=np.int64)
    sigma[oa] = ob
    return sigma


@pytest.mark.parametrize("name", list(CASES))
def test_refined_box_solves_like_the_generated_box(name, gpu_lib):
    """exf_mesh_refine on a generated box's level-0 mesh: the refined hierarchy (its own
    node numbering) gives the generated box's solution, matched node by node by
    coordinates, within 1e-10."""
    dim, nlev, n0, box, kind, preset, pk = CASES[name]
    gm = ex.Mesh(dim, nlev, n0, box)
    c0 = gm.conn(0)[0]
    rm = ex.Mesh.refine(dim, nlev, gm.nvert0, gm.xyz()[:, :gm.nnodes(0)], c0)
    assert [rm.nnodes(l) for l in range(nlev)] == [gm.nnodes(l) for l in range(nlev)]
    gs, x0 = make_sys(gm, name)
    rs, rx0 = make_sys(rm, name)
    sigma = coord_match(gm.xyz(), rm.xyz())
    N = gm.ntop
    nv2 = dim if kind == _lib.KIND_NS else 1
    dmap = np.concatenate([a * N + sigma for a in range(nv2)] +
                          ([nv2 * N + sigma[:gm.nnodes(nlev - 2)]] if kind == _lib.KIND_NS else []))
    assert np.all(sigma[:gm.nnodes(nlev - 2)] < gm.nnodes(nlev - 2))  # nesting kept
    for a, b in zip(gs.bc(), rs.bc()):
        assert np.array_equal(b[dmap], a)
    assert np.array_equal(rx0[dmap], x0)
    gs.assemble_all()
    rs.assemble_all()
    assert rel(rs.rhs()[dmap], gs.rhs()) < 1e-13
    for s_, x in ((gs, x0), (rs, rx0)):
        s_.set_x(x)
        assert s_.solve(params(name, eps=1e-12)).converged
    assert rel(rs.x()[dmap], gs.x()) < 1e-10


Q9_ABC = [(0, 0, 0), (2, 0, 0), (2, 2, 0), (0, 2, 0), (1, 0, 0), (2, 1, 0), (1, 2, 0), (0, 1, 0), (1, 1, 0)]
H27_ABC = [(0, 0, 0), (2, 0, 0), (2, 2, 0), (0, 2, 0), (0, 0, 2), (2, 0, 2), (2, 2, 2), (0, 2, 2),
           (1, 0, 0), (2, 1, 0), (1, 2, 0), (0, 1, 0), (0, 0, 1), (2, 0, 1), (2, 2, 1), (0, 2, 1),
           (1, 0, 2), (2, 1, 2), (1, 2, 2), (0, 1, 2), (1, 1, 0), (1, 0, 1), (2, 1, 1), (1, 2, 1),
           (0, 1, 1), (1, 1, 2), (1, 1, 1)]
Q9_SIDE = [[0, 1, 4], [1, 2, 5], [2, 3, 6], [3, 0, 7]]
H27_FACE = [[0, 1, 2, 3, 8, 9, 10, 11, 20], [0, 1, 5, 4, 8, 13, 16, 12, 21], [1, 2, 6, 5, 9, 14, 17, 13, 22],
            [2, 3, 7, 6, 10, 15, 18, 14, 23], [3, 0, 4, 7, 11, 12, 19, 15, 24], [4, 5, 6, 7, 16, 17, 18, 19, 25]]


def skewed_coarse(dim, ne, corners):
    """A coarse grid of ne elements per axis mapped by the (tri)linear map of `corners`
    (2^dim points, lexicographic): straight-sided elements that are not parallelograms.
    Returns nvert0, xyz0 [dim][n], conn0 [nel][9 | 27] with the vertices numbered first."""
    abc = Q9_ABC if dim == 2 else H27_ABC
    ne3 = list(ne) + [1] * (3 - dim)
    lat = [(i, j, k) for k in range(2 * ne3[2] + 1 if dim == 3 else 1)
           for j in range(2 * ne3[1] + 1) for i in range(2 * ne3[0] + 1)]
    lat.sort(key=lambda p: (any(v % 2 for v in p[:dim]), p[2], p[1], p[0]))  # vertices first
    idx = {p: n for n, p in enumerate(lat)}
    nvert0 = sum(1 for p in lat if not any(v % 2 for v in p[:dim]))
    C = np.asarray(corners, float)
    xyz0 = np.zeros((dim, len(lat)))
    for n, p in enumerate(lat):
        t = [p[d] / (2.0 * ne3[d]) for d in range(dim)]
        w = []
        for m in range(2 ** dim):
            b = [(m >> d) & 1 for d in range(dim)]
            w.append(np.prod([t[d] if b[d] else 1 - t[d] for d in range(dim)]))
        xyz0[:, n] = np.asarray(w) @ C
    conn = []
    for ez in range(ne3[2]):
        for ey in range(ne3[1]):
            for ex_ in range(ne3[0]):
                o = (2 * ex_, 2 * ey, 2 * ez)
                conn.append([idx[(o[0] + a, o[1] + b, o[2] + (c if dim == 3 else 0))] for a, b, c in abc])
    return nvert0, xyz0, np.array(conn)


@pytest.mark.parametrize("dim,nlev,ne,corners", [
    (2, 4, (2, 2), [(0.0, 0.0), (2.0, 0.1), (0.3, 1.2), (1.7, 1.5)]),
    (3, 3, (2, 1, 1), [(0, 0, 0), (2, 0, 0.2), (0, 1, 0), (1.8, 1.1, 0), (0.1, 0, 1), (2.1, 0, 1.2),
                       (0, 1.3, 1), (2, 1, 0.9)]),
])
def test_refined_skewed_mesh_reproduces_a_linear_field(dim, nlev, ne, corners, gpu_lib):
    """Heat with Dirichlet data from a linear field and no source on a refined non-affine
    mesh: isoparametric Q2 elements reproduce the field at every node."""
    nvert0, xyz0, conn0 = skewed_coarse(dim, ne, corners)
    m = ex.Mesh.refine(dim, nlev, nvert0, xyz0, conn0)
    t = ex.MGSolT(m)
    top = nlev - 1
    c, nb, _ = m.conn(top)
    sides = Q9_SIDE if dim == 2 else H27_FACE
    bnd = np.zeros(m.ntop, bool)
    for e, s in zip(*np.nonzero(nb < 0)):
        bnd[c[e, sides[s]]] = True
    b0 = np.where(bnd, 0, 1).astype(np.int32)
    b1 = np.ones(m.ntop, np.int32)
    t.set_bc(b0, b1)
    xyz = m.xyz()
    g = 0.3 + 0.7 * xyz[0] - 0.4 * xyz[1] + (0.2 * xyz[2] if dim == 3 else 0.0)
    t.set_xold(g)
    t.set_source(np.zeros(m.nel(top)))
    t.phys = ex.phys()
    t.assemble_all()
    t.set_x(np.zeros(t.ntop_dof))
    st = t.solve(ex.mg_params(eps=1e-13, max_cycles=200, smoother=_lib.SMOOTH_GS, nu_pre=2, nu_post=2))
    assert st.converged
    assert np.abs(t.x() - g).max() < 1e-9 * np.abs(g).max()
