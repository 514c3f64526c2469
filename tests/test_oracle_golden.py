"""Pin the CPU oracle against the reference's own tables and known answers (no GPU)."""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import or_mg, or_phys, rel

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mggeomel.json")))

QUAD_ABC = [(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1)]


def lag(a, x):
    return {0: .5 * x * (x - 1.), 1: 1. - x * x, 2: .5 * x * (x + 1.)}[a]


def table(key):
    g = GOLD[key]
    return np.array(g["data"]).reshape(g["shape"])


def test_side_topology_matches_surf_top(oracle_mod):
    """The restated side tables equal _surf_top (src/MGGeomEl.C:172-177, :310-317)."""
    L = oracle_mod.oracle_lib()
    for dim, key in ((2, "quad9_surf_top"), (3, "hex27_surf_top")):
        ref = table(key)
        out = np.zeros(ref.size, np.int32)
        L.or_side_table(dim, out)
        assert np.array_equal(out.reshape(ref.shape), ref)


def _child_embedding(dim, quad, pos):
    """Coarse shape functions at the fine nodes of the child at sub-cell pos."""
    from oracle.pyoracle import OrMesh  # noqa: F401
    nen = (9 if dim == 2 else 27) if quad else (4 if dim == 2 else 8)
    abc_all = _abc(dim)
    E = np.zeros((nen, nen))
    for f in range(nen):
        xi = [-1. + (2 * pos[d] + abc_all[f][d]) / 2. for d in range(dim)]
        for k in range(nen):
            v = 1.
            for d in range(dim):
                a = abc_all[k][d]
                v *= lag(a, xi[d]) if quad else (.5 * (1 - xi[d]) if a == 0 else .5 * (1 + xi[d]))
            E[f, k] = v
    return E


def _abc(dim):
    if dim == 2:
        return QUAD_ABC
    return [(0, 0, 0), (2, 0, 0), (2, 2, 0), (0, 2, 0), (0, 0, 2), (2, 0, 2), (2, 2, 2), (0, 2, 2),
            (1, 0, 0), (2, 1, 0), (1, 2, 0), (0, 1, 0), (0, 0, 1), (2, 0, 1), (2, 2, 1), (0, 2, 1),
            (1, 0, 2), (2, 1, 2), (1, 2, 2), (0, 1, 2), (1, 1, 0), (1, 0, 1), (2, 1, 1), (1, 2, 1),
            (0, 1, 1), (1, 1, 2), (1, 1, 1)]


@pytest.mark.parametrize("dim,quad,key", [(2, True, "quad9_embedding_q"), (2, False, "quad4_embedding_l"),
                                          (3, True, "hex27_embedding_q"), (3, False, "hex8_embedding_l")])
def test_lagrange_embedding_equals_reference_tables(dim, quad, key):
    """Each reference child matches exactly one sub-cell's Lagrange embedding, bit for bit
    after rounding to float (the tables are float constants, src/MGGeomEl.C:182-600)."""
    ref = table(key).astype(np.float32)
    subcells = [(i, j) for j in range(2) for i in range(2)] if dim == 2 else \
        [(i, j, k) for k in range(2) for j in range(2) for i in range(2)]
    used = set()
    for c in range(ref.shape[0]):
        hits = [p for p in subcells if np.array_equal(_child_embedding(dim, quad, p).astype(np.float32), ref[c])]
        assert len(hits) == 1, "child %d matched %s" % (c, hits)
        used.add(hits[0])
    assert len(used) == len(subcells)


@pytest.mark.parametrize("dim,n0,nlev", [(2, (2, 2), 3), (3, (2, 1, 1), 3)])
def test_oracle_prolongation_rows_are_embedding_entries(oracle_mod, dim, n0, nlev):
    """Oracle P entries equal the reference embedding values (float -> double exact)."""
    box = (0, 1, 0, 1, 0, 1)[:2 * dim]
    m = oracle_mod.OrMesh(dim, nlev, n0, box)
    s = oracle_mod.OrSys(m, 1)
    vals = set()
    for key in (("quad9_embedding_q", "quad4_embedding_l") if dim == 2 else ("hex27_embedding_q", "hex8_embedding_l")):
        t = table(key)
        vals |= set(float(np.float32(v)) for v in t.ravel() if abs(v) > 1e-8)
    for lev in range(1, nlev):
        rp, col, val = s.prol(lev)
        assert set(np.unique(val)) <= vals
        P = sp.csr_matrix((val, col, rp))
        # partition of unity per component block
        assert np.allclose(np.asarray(P.sum(axis=1)).ravel(), 1.0, atol=0, rtol=0)


def test_oracle_restriction_is_masked_transpose(oracle_mod):
    m = oracle_mod.OrMesh(2, 3, (2, 2), (0, 1, 0, 1))
    s = oracle_mod.OrSys(m, 1)
    s.bc_preset(2)
    b0, _ = s.bc()
    nd_top = s.node_dof(2)
    for lev in range(2):
        rp, col, val = s.prol(lev + 1)
        P = sp.csr_matrix((val, col, rp), shape=(s.ndof(lev + 1), s.ndof(lev)))
        rp, col, val = s.rest(lev)
        R = sp.csr_matrix((val, col, rp), shape=(s.ndof(lev), s.ndof(lev + 1)))
        nd = s.node_dof(lev)
        mask = np.ones(s.ndof(lev))
        ntop = m.ntop
        for v in range(3):
            for node in range(ntop):
                d = nd[node + v * ntop]
                if d >= 0:
                    mask[d] = b0[nd_top[node + v * ntop]] % 2
        assert abs(R - sp.diags(mask) @ P.T).max() == 0.0


def test_gencase_sizes(oracle_mod):
    """DOF and nonzero counts of the workloads (gencase rules, MGGenCase.C:1781-1862)."""
    m = oracle_mod.OrMesh(2, 4, (4, 4), (0, 1, 0, 1))
    s = oracle_mod.OrSys(m, 0)
    assert s.ndof(3) == 4225 and len(s.pattern(3)[1]) == 66049
    m = oracle_mod.OrMesh(2, 6, (4, 4), (0, 1, 0, 1))
    s = oracle_mod.OrSys(m, 1)
    assert s.ndof(5) == 2 * 66049 + 16641 and len(s.pattern(5)[1]) == 5994249


def test_dof_map_nesting(oracle_mod):
    """init_dof: Q1 nodes of level L are the Q2 nodes of level L-1 (src/MGSolverDA.C:895-897)."""
    m = oracle_mod.OrMesh(2, 3, (2, 2), (0, 1, 0, 1))
    s = oracle_mod.OrSys(m, 1)
    for lev in range(3):
        nd = s.node_dof(lev)
        N = m.nnodes(lev)
        NL = m.nnodes(lev - 1) if lev else m.nvert0
        ntop = m.ntop
        assert np.array_equal(nd[:N], np.arange(N))
        assert np.array_equal(nd[ntop:ntop + N], N + np.arange(N))
        assert np.array_equal(nd[2 * ntop:2 * ntop + NL], 2 * N + np.arange(NL))
        assert (nd[2 * ntop + NL:3 * ntop] == -1).all()
        assert s.ndof(lev) == 2 * N + NL


def _heat_sys(oracle_mod, n0=4, nlev=3, natural=False):
    m = oracle_mod.OrMesh(2, nlev, (n0, n0), (0, 1, 0, 1))
    s = oracle_mod.OrSys(m, 0)
    if natural:
        n = s.ndof(nlev - 1)
        s.set_bc(np.ones(n, np.int32), np.zeros(n, np.int32))
    else:
        s.bc_preset(1)
    return m, s


def test_mass_matrix_sums_to_area(oracle_mod):
    m, s = _heat_sys(oracle_mod, natural=True)
    s.assemble(2, 1, or_phys(oracle_mod, inv_re=0.0, inv_dt=1.0), xold=np.zeros(s.ndof(2)))
    assert abs(s.matrix(2).sum() - 1.0) < 1e-13


def test_quadratic_reproduction(oracle_mod):
    """Interior rows: (K p)_i = -lap(p) * int(phi_i) for quadratic p (exact Gauss)."""
    m, s = _heat_sys(oracle_mod, natural=True)
    n = s.ndof(2)
    s.assemble(2, 1, or_phys(oracle_mod), xold=np.zeros(n))
    rp, col = s.pattern(2)
    K = sp.csr_matrix((s.matrix(2), col, rp))
    s.assemble(2, 1, or_phys(oracle_mod, inv_re=0.0, inv_dt=1.0), xold=np.zeros(n))
    M = sp.csr_matrix((s.matrix(2), col, rp))
    x, y = m.xyz()
    p = x * x + x * y + 2 * y * y
    lap = 2 + 4
    lat = m.lattice()
    interior = (lat[:, 0] > 0) & (lat[:, 0] < lat[:, 0].max()) & (lat[:, 1] > 0) & (lat[:, 1] < lat[:, 1].max())
    lhs = (K @ p)[interior]
    rhs = (-lap * (M @ np.ones(n)))[interior]
    assert rel(lhs, rhs) < 1e-12


def test_divergence_kills_constant_pressure(oracle_mod):
    """Interior velocity rows: B^T 1 = 0 (enclosed flow has a constant-pressure kernel)."""
    m = oracle_mod.OrMesh(2, 2, (2, 2), (0, 1, 0, 1))
    s = oracle_mod.OrSys(m, 1)
    s.bc_preset(2)
    n = s.ndof(1)
    s.assemble(1, 1, or_phys(oracle_mod), xold=np.zeros(n))
    A = sp.csr_matrix((s.matrix(1), s.pattern(1)[1], s.pattern(1)[0]))
    N = m.nnodes(1)
    e = np.zeros(n)
    e[2 * N:] = 1.0
    assert np.abs((A @ e)[:2 * N]).max() < 1e-14


def test_oracle_mg_heat_converges(oracle_mod):
    m, s = _heat_sys(oracle_mod, n0=4, nlev=4)
    n = s.ndof(3)
    qe = 1 + 0.1 * np.random.default_rng(0).random(m.nel(3))
    s.assemble_all(or_phys(oracle_mod), xold=np.zeros(n), qe=qe)
    x, st = s.mg_solve(or_mg(oracle_mod))
    assert st.converged and st.rel_res <= 1e-10 and st.cycles <= 15
    A = sp.csr_matrix((s.matrix(3), s.pattern(3)[1], s.pattern(3)[0]))
    assert np.linalg.norm(A @ x - s.rhs()) / np.linalg.norm(s.rhs()) <= 1e-10


@pytest.mark.skipif(not __import__("oracle").laspack_available(), reason="reference LASPACK not built")
def test_laspack_agrees_with_oracle(oracle_mod):
    """The reference's Mul_QV and GMRESIter (compiled from contrib/laspack) on the oracle matrices."""
    m, s = _heat_sys(oracle_mod, n0=4, nlev=3)
    n = s.ndof(2)
    qe = 1 + 0.1 * np.random.default_rng(0).random(m.nel(2))
    s.assemble_all(or_phys(oracle_mod), xold=np.zeros(n), qe=qe)
    rp, col, val = s.csr(2)
    lp = oracle_mod.Laspack()
    xr = np.random.default_rng(1).random(n)
    assert rel(lp.spmv(rp, col, val, xr), s.spmv(2, xr)) < 1e-14
    x_mg, st = s.mg_solve(or_mg(oracle_mod, eps=1e-13))
    x_lp, it, acc = lp.gmres(rp, col, val, s.rhs(), tol=1e-13, maxit=5000)
    assert acc < 1e-12
    assert rel(x_mg, x_lp) < 1e-9


def test_oracle_vanka_mg_cavity_small(oracle_mod):
    """Q2-Q1 cavity, 3 levels: the restated multigrid converges with the Vanka smoother."""
    m = oracle_mod.OrMesh(2, 3, (4, 4), (0, 1, 0, 1))
    s = oracle_mod.OrSys(m, 1)
    s.bc_preset(2)
    n = s.ndof(2)
    N = m.nnodes(2)
    x, y = m.xyz()
    xold = np.zeros(n)
    xold[:N][(y == 1) & (x > 0) & (x < 1)] = 1.0
    s.assemble_all(or_phys(oracle_mod, inv_re=1 / 400.), xold=xold)
    xs, st = s.mg_solve(or_mg(oracle_mod, smoother=1, nu_pre=3, nu_post=3, max_cycles=60), x0=xold)
    assert st.converged


def _upwind_f(up, rho, mod, h, diff):
    """f_upwind of the NS volume terms (template_appl/nse/SRC/MGSolverNS.C:336-339)."""
    pe = 0.5 * mod * h / diff
    return up * rho * 0.5 * (1.0 / np.tanh(pe) - 1.0 / pe) * h / mod


@pytest.mark.parametrize("dim", [2, 3])
def test_ns_operator_reproduces_quadratic_flow(oracle_mod, dim):
    """Manufactured solution for the Navier-Stokes volume terms (MGSolverNS.C:401-489).

    Velocity u = (y^2, x^2) in 2D, (y^2, z^2, x^2) in 3D (divergence-free, exactly in the
    Q2 space), pressure p = x + 2y (+ 3z) (exactly in the Q1 space), advecting field
    v = x_old = (1, 0, 0), natural flags everywhere (no boundary terms).  For a row whose
    test function vanishes on the boundary, the weak form integrates by parts to
    int phi_i [ v.grad u_a - sum_k (nu + f_k v_k^2) d_kk u_a - (nu + f_a v_a^2) d_aa u_a
               - sum_{b != a} (nu + f_a v_a v_b) d_ab u_b + d_a p ]
    and every bracket is affine in x, so on a uniform mesh the row equals the bracket at
    the node times int phi_i (1D weights h/3 at vertices, 2h/3 at midpoints).  Every
    pressure row is int psi_m div u = 0."""
    nu = 0.01
    if dim == 2:
        n0, box, nlev = (4, 4), (0, 1, 0, 1), 2
    else:
        n0, box, nlev = (3, 2, 2), (0, 1.5, 0, 1, 0, 1), 2
    m = oracle_mod.OrMesh(dim, nlev, n0, box)
    s = oracle_mod.OrSys(m, 1)
    top = nlev - 1
    n, N, NL = s.ndof(top), m.nnodes(top), m.nnodes(top - 1)
    X = m.xyz()
    h = [(box[2 * d + 1] - box[2 * d]) / (n0[d] << top) for d in range(dim)]
    xold = np.zeros(n)
    xold[:N] = 1.0  # v = (1, 0, 0)
    s.assemble(top, 1, or_phys(oracle_mod, inv_re=nu), xold=xold)
    A = sp.csr_matrix((s.matrix(top), s.pattern(top)[1], s.pattern(top)[0]), shape=(n, n))
    x = np.zeros(n)
    if dim == 2:
        x[:N], x[N:2 * N] = X[1] ** 2, X[0] ** 2
        x[2 * N:] = X[0][:NL] + 2 * X[1][:NL]
    else:
        x[:N], x[N:2 * N], x[2 * N:3 * N] = X[1] ** 2, X[2] ** 2, X[0] ** 2
        x[3 * N:] = X[0][:NL] + 2 * X[1][:NL] + 3 * X[2][:NL]
    y = A @ x
    fx = _upwind_f(0.1, 1.0, 1.0, h[0], nu)
    lat = m.lattice()[:N]
    interior = np.ones(N, bool)
    W = np.ones(N)
    for d in range(dim):
        k = np.rint((X[d] - box[2 * d]) / (h[d] / 2)).astype(int)
        interior &= (k > 0) & (k < 2 * (n0[d] << top))
        W *= np.where(k % 2 == 0, h[d] / 3, 2 * h[d] / 3)
    assert lat.shape[0] == N
    xi = X[0]
    if dim == 2:
        expect = [W * (-2 * nu + 1.0), W * (2 * xi - 2 * (nu + fx) + 2.0)]
    else:
        expect = [W * (-2 * nu + 1.0), W * (-2 * nu + 2.0), W * (2 * xi - 2 * (nu + fx) + 3.0)]
    for a in range(dim):
        got = y[a * N:(a + 1) * N][interior]
        ref = expect[a][interior]
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), (a, np.abs(got - ref).max())
    assert np.abs(y[dim * N:]).max() <= 1e-13 * np.abs(y[:dim * N]).max()


@pytest.mark.parametrize("dim", [2, 3])
def test_ns_neumann_sides(oracle_mod, dim):
    """The natural-side branch of MGSolNS::GenMatRhs (template_appl/nse/SRC/MGSolverNS.C:
    604-681) on the outlet x = L of a box, every other wall Dirichlet:
      bc1 = 1 (normal):     velocity row a gains n_a^2 int_side phi_i   (lumped Robin)
      bc1 = 2 (tangential): row a gains (1 - n_a^2) int_side phi_i
      bc1 = 4 (rhs) with traction on: rhs row a gains -n_a int_side phi_i p_old
    with n the outward normal (1, 0, 0); rows of nodes on a Dirichlet wall take nothing."""
    n0 = (2, 2) if dim == 2 else (2, 1, 1)
    box = (0, 2, 0, 1) if dim == 2 else (0, 2, 0, 1, 0, 1)
    m = oracle_mod.OrMesh(dim, 2, n0, box)
    X = m.xyz()
    N = m.nnodes(1)
    NL = m.nnodes(0)
    ntop = m.ntop
    h = [(box[2 * d + 1] - box[2 * d]) / (n0[d] << 1) for d in range(dim)]
    outlet = np.abs(X[0] - box[1]) < 1e-12
    wall = np.zeros(ntop, bool)
    for d in range(dim):
        wall |= np.abs(X[d] - box[2 * d]) < 1e-12
        if d > 0:
            wall |= np.abs(X[d] - box[2 * d + 1]) < 1e-12
    # int over the outlet face of phi_i: product of the 1D Simpson weights of the face axes
    W = np.ones(ntop)
    for d in range(1, dim):
        k = np.rint((X[d] - box[2 * d]) / (h[d] / 2)).astype(int)
        kmax = 2 * (n0[d] << 1)
        w1 = np.where(k % 2 == 1, 4 * h[d] / 6, np.where((k == 0) | (k == kmax), h[d] / 6, 2 * h[d] / 6))
        W *= w1
    W[~outlet] = 0.0

    def run(flags, traction, p_old=0.0):
        s = oracle_mod.OrSys(m, 1)
        n = s.ndof(1)
        b0 = np.ones(n, np.int32)
        b1 = np.zeros(n, np.int32)
        for a in range(dim):
            b0[a * N:(a + 1) * N][wall] = 0  # the outlet's corners and edges belong to the walls
            b1[a * N:(a + 1) * N][outlet & ~wall] = flags[a]
        s.set_bc(b0, b1)
        xold = np.zeros(n)
        xold[dim * N:] = p_old
        s.assemble(1, 1, or_phys(oracle_mod, inv_re=0.1, traction=traction), xold=xold)
        rp, col = s.pattern(1)
        return sp.csr_matrix((s.matrix(1), col, rp), shape=(n, n)), s.rhs(), b0

    A0, r0, b0 = run([0] * dim, 0.0)
    free = np.concatenate([b0[a * N:(a + 1) * N] for a in range(dim)]).astype(bool)
    A1, _, _ = run([1] * dim, 0.0)
    D = (A1 - A0).tocsr()
    expect = np.concatenate([W * (1.0 if a == 0 else 0.0) for a in range(dim)]) * free
    assert abs(D - sp.diags(np.concatenate([expect, np.zeros(NL)]))).max() < 1e-14
    A2, _, _ = run([2] * dim, 0.0)
    D = (A2 - A0).tocsr()
    expect = np.concatenate([W * (0.0 if a == 0 else 1.0) for a in range(dim)]) * free
    assert abs(D - sp.diags(np.concatenate([expect, np.zeros(NL)]))).max() < 1e-14
    P = 0.75
    _, r4, _ = run([4] * dim, 1.0, p_old=P)
    _, r4off, _ = run([4] * dim, 0.0, p_old=P)
    expect = np.concatenate([-P * W * (1.0 if a == 0 else 0.0) for a in range(dim)]) * free
    assert np.abs((r4 - r4off)[:dim * N] - expect).max() < 1e-14
    assert np.abs(r4off - r0).max() == 0.0


def test_face0_normal_follows_the_reference_side_order(oracle_mod):
    """MGFE::normal_g (src/MGFE.C:1601-1646) takes (x1 - x0) x (x3 - x0) on the side's nodes;
    on the hex27 face {0, 1, 2, 3, ...} of _surf_top (z = z0) that is +z, so the traction
    term there has the sign of an inward normal (outward on every other face)."""
    m = oracle_mod.OrMesh(3, 1, (1, 1, 1), (0, 1, 0, 1, 0, 1))
    X = m.xyz()
    bottom = np.abs(X[2]) < 1e-12
    s = oracle_mod.OrSys(m, 1)
    n = s.ndof(0)
    N = m.nnodes(0)
    b0 = np.ones(n, np.int32)
    b1 = np.zeros(n, np.int32)
    b1[2 * N:3 * N][bottom] = 4
    s.set_bc(b0, b1)
    xold = np.zeros(n)
    xold[3 * N:] = 1.0
    s.assemble(0, 1, or_phys(oracle_mod, inv_re=0.1, traction=1.0), xold=xold)
    r = s.rhs()[2 * N:3 * N]
    assert r[bottom].sum() < 0 and abs(r[bottom].sum() + 1.0) < 1e-13  # -n_z int p = -(+1)(1)


def _ds_oracle(oracle_mod, dim, direction):
    """The oracle's displacement system (MGSolverDS.C:321-700) on the box of the GPU
    displacement tests, assembled on every level."""
    import test_gpu_ds as T
    box, nlev, n0 = T.CASES[dim]
    om = oracle_mod.OrMesh(dim, nlev, n0, box)
    xyz = om.xyz()
    b0, b1 = T.flags(xyz)
    u, d = T.fields(xyz)
    o = oracle_mod.OrSys(om, 0)
    o.set_bc(b0, b1)
    for lev in range(nlev):
        o.ds_assemble(lev, 1 if lev == nlev - 1 else 0, direction, T.DT, u, d)
    return o, xyz, b0, b1, u, d, T.DT


@pytest.mark.parametrize("dim,direction", [(2, 0), (2, 1), (3, 2)])
def test_displacement_restatement_known_answers(oracle_mod, dim, direction):
    """Fixed answers of MGSolDS's element rules: solid and interface rows solve to
    u_fsi dt + d_old of the direction (:664-671); the Dirichlet moving wall takes the x
    components (:640, fsi_idx and disp_idx without _dir); the fixed inlet (bc1 0) is 0
    away from the corners; fluid interior rows are 100 dt times a Laplacian, whose rows
    sum to zero."""
    o, xyz, b0, b1, u, d, dt = _ds_oracle(oracle_mod, dim, direction)
    x, st = o.mg_solve(or_mg(oracle_mod, eps=1e-12, max_cycles=100))
    assert st.converged
    solid = b0 >= 2
    assert np.abs(x[solid] - (u[direction][solid] * dt + d[direction][solid])).max() <= 1e-15
    top = (np.abs(xyz[1] - 1.0) < 1e-12) & (b0 == 0) & (b1 == 1)
    assert top.any() and np.abs(x[top] - (u[0][top] * dt + d[0][top])).max() <= 1e-14
    inlet = (np.abs(xyz[0]) < 1e-12) & (np.abs(xyz[1]) > 1e-12) & (np.abs(xyz[1] - 1.0) > 1e-12)
    assert np.abs(x[inlet]).max() <= 1e-14
    rp, col, val = o.csr(o.mesh.nlev - 1)
    interior = np.flatnonzero(b0 == 1)
    for i in interior[:: max(1, interior.size // 40)]:
        row = val[rp[i]:rp[i + 1]]
        assert abs(row.sum()) <= 1e-12 * np.abs(row).max(), i
