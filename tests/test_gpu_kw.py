"""The turbulence template's kappa-omega equations on the assembly engine (needs a B200):
both variables assembled on every level against the oracle's restatement of
MGSolTBK::GenMatRhs (template_appl/turb-ckw/SRC/MGSolverTBKW.C) on a channel with
no-slip walls (Dirichlet, omega's wall value), a prescribed inlet and a Neumann outlet,
advected by a parabolic Navier-Stokes velocity, then solved by multigrid against the
oracle's solution."""
import numpy as np
import pytest

import exfemus_b200 as ex
from exfemus_b200 import _lib

from conftest import or_mg, or_phys, rel

pytestmark = pytest.mark.gpu

BOX = (0.0, 2.0, 0.0, 1.0)
NU_WALL = 0.01


def flags(xyz):
    """(bc0, bc1) per node: walls y = 0, 1 Dirichlet (bc1 2: omega's wall value, kappa
    0), inlet x = 0 Dirichlet on the old value (bc1 1), outlet x = 2 Neumann (bc0 1,
    bc1 1), interior (1, 0)."""
    x, y = xyz
    n = x.size
    b0, b1 = np.ones(n, np.int32), np.zeros(n, np.int32)
    out = np.abs(x - BOX[1]) < 1e-12
    b1[out] = 1
    inl = np.abs(x - BOX[0]) < 1e-12
    b0[inl], b1[inl] = 0, 1
    wall = (np.abs(y - BOX[2]) < 1e-12) | (np.abs(y - BOX[3]) < 1e-12)
    b0[wall], b1[wall] = 0, 2
    return b0, b1


def fields(xyz):
    x, y = xyz
    u = 4.0 * y * (1.0 - y) * (1.0 + 0.1 * np.sin(2.0 * x))
    v = 0.05 * np.sin(np.pi * y) * x
    k = 0.01 + 0.02 * y * (1.0 - y) * (1.0 + 0.2 * x)
    w = 40.0 + 30.0 * (y - 0.5) ** 2 + 2.0 * x
    return u, v, k, w


def wall_dist(conns, xyz):
    """Centroid distance of every element to the nearest wall, level after level."""
    d = []
    for c in conns:
        yc = xyz[1][c].mean(axis=1)
        d.append(np.minimum(yc - BOX[2], BOX[3] - yc))
    return np.concatenate(d)


@pytest.fixture(scope="module")
def kw_case(oracle_mod):
    nlev, n0 = 3, (4, 2)
    m = ex.Mesh(2, nlev, n0, BOX)
    xyz = m.xyz()
    N = m.ntop
    u, v, k, w = fields(xyz)
    ns = ex.MGSolNS(m)
    xns = np.zeros(ns.ntop_dof)
    xns[:N], xns[N:2 * N] = u, v
    ns.set_xold(xns)
    ph = ex.phys(inv_re=0.01, inv_dt=10.0)
    conns = [m.conn(l)[0] for l in range(nlev)]
    dist = wall_dist(conns, xyz)
    b0, b1 = flags(xyz)
    sys = []
    for var, old in ((0, k), (1, w)):
        s = ex.MGSolTBK(m, var)
        s.set_bc(b0, b1)
        s.set_xold(old)
        s.set_wall(dist, NU_WALL)
        s.phys = ph
        sys.append(s)
    for s, other in ((sys[0], sys[1]), (sys[1], sys[0])):
        s.couple(ns)
        s.couple(other)
    om = oracle_mod.OrMesh(2, nlev, n0, BOX)
    osys = []
    oph = or_phys(oracle_mod, inv_re=0.01, inv_dt=10.0)
    off = np.cumsum([0] + [c.shape[0] for c in conns])
    for var in (0, 1):
        o = oracle_mod.OrSys(om, 0)
        o.set_bc(b0, b1)
        for lev in range(nlev):
            o.kw_assemble(lev, 1 if lev == nlev - 1 else 0, var, oph, xns[:2 * N], k, w,
                          dist[off[lev]:off[lev + 1]], NU_WALL)
        osys.append(o)
    return dict(mesh=m, ns=ns, sys=sys, osys=osys, nlev=nlev)


def test_kappa_omega_assembly_matches_the_oracle(gpu_lib, kw_case):
    for s, o in zip(kw_case["sys"], kw_case["osys"]):
        s.assemble_all()
        for lev in range(kw_case["nlev"]):
            rp, col, val = s.csr(lev)
            orp, ocol, oval = o.csr(lev)
            assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
            assert rel(val, oval) <= 1e-12, (s.var, lev)
        assert rel(s.rhs(), o.rhs()) <= 1e-12, s.var
        assert np.all(np.isfinite(s.rhs()))


def test_kappa_omega_solves_match_the_oracle(gpu_lib, oracle_mod, kw_case):
    for s, o in zip(kw_case["sys"], kw_case["osys"]):
        s.assemble_all()
        s.set_x(np.zeros(s.ntop_dof))
        st = s.solve(ex.mg_params(eps=1e-11, max_cycles=100, smoother=_lib.SMOOTH_GS))
        xo, sto = o.mg_solve(or_mg(oracle_mod, eps=1e-11, max_cycles=100))
        assert st.converged and sto.converged
        assert rel(s.x(), xo) <= 1e-9, s.var
    xk, xw = kw_case["sys"][0].x(), kw_case["sys"][1].x()
    xyz = kw_case["mesh"].xyz()
    wall = (np.abs(xyz[1]) < 1e-12) | (np.abs(xyz[1] - 1.0) < 1e-12)
    assert np.abs(xk[wall]).max() < 1e-10  # kappa = 0 on the no-slip walls


def test_kappa_omega_needs_partner_and_wall(gpu_lib):
    m = ex.Mesh(2, 2, (2, 2), (0, 1, 0, 1))
    s = ex.MGSolTBK(m, 1)
    s.phys = ex.phys(inv_dt=1.0)
    with pytest.raises(_lib.ExfError) as e:
        s.assemble_all()
    assert e.value.code == _lib.EXF_ERR_STATE
    other = ex.MGSolTBK(m, 1)
    with pytest.raises(_lib.ExfError) as e:
        s.couple(other)  # omega with omega
    assert e.value.code == _lib.EXF_ERR_ARG
    with pytest.raises(_lib.ExfError) as e:
        s.set_wall(np.zeros(m.nel(0) + m.nel(1)), 1e-3)  # distances must be positive
    assert e.value.code == _lib.EXF_ERR_ARG


def test_eddy_viscosity_in_the_momentum_equation_matches_the_oracle(gpu_lib, oracle_mod, kw_case):
    """The NS system coupled to the kappa and omega systems assembles the turbulence
    template's momentum equation (IRe_eff = IRe (1 + mu_t)) on every level, as the
    oracle does with the same fields; without them it stays laminar."""
    m, nlev = kw_case["mesh"], kw_case["nlev"]
    xyz = m.xyz()
    u, v, k, w = fields(xyz)
    N = m.ntop
    ph = ex.phys(inv_re=0.01, inv_dt=10.0)

    def gpu_ns(turb):
        ns = ex.MGSolNS(m)
        ns.GenBc(_lib.BC_CHANNEL)
        x = np.zeros(ns.ntop_dof)
        x[:N], x[N:2 * N] = u, v
        ns.set_xold(x)
        ns.phys = ph
        if turb:
            for s in kw_case["sys"]:
                ns.couple(s)
        ns.assemble_all()
        return ns, x

    ns, x = gpu_ns(True)
    lam, _ = gpu_ns(False)
    om = oracle_mod.OrMesh(2, nlev, (4, 2), BOX)
    o = oracle_mod.OrSys(om, 1)
    o.bc_preset(_lib.BC_CHANNEL)
    o.set_turb(k, w)
    o.assemble_all(or_phys(oracle_mod, inv_re=0.01, inv_dt=10.0), xold=x)
    for lev in range(nlev):
        _, _, val = ns.csr(lev)
        _, _, oval = o.csr(lev)
        assert rel(val, oval) <= 1e-12, lev
        assert rel(lam.csr(lev)[2], val) > 1e-6  # the eddy viscosity changed the operator
    assert rel(ns.rhs(), o.rhs()) <= 1e-12


def b_dist_here(m, wall_node):
    """MGMesh::B_dist restated: element centre to the nearest wall-side centre."""
    xyz = m.xyz()
    side = [(0, 1, 4), (1, 2, 5), (2, 3, 6), (3, 0, 7)]
    out = []
    for lev in range(m.nlev):
        conn, neigh = m.conn(lev)[:2]
        wc = []
        for e in range(conn.shape[0]):
            for sd in range(4):
                if neigh[e, sd] == -1 and all(wall_node[conn[e, k]] for k in side[sd]):
                    wc.append(xyz[:, conn[e, list(side[sd])]].sum(axis=1) / 3)
        wc = np.array(wc)
        xm = xyz[:, conn].sum(axis=2) / conn.shape[1]
        d2 = ((xm.T[:, None, :] - wc[None, :, :]) ** 2).sum(axis=2)
        out.append(np.sqrt(d2.min(axis=1)))
    return np.concatenate(out)


def test_wall_distances_are_b_dist(gpu_lib, kw_case):
    m = kw_case["mesh"]
    x, y = m.xyz()
    wall = ((np.abs(y) < 1e-12) | (np.abs(y - 1.0) < 1e-12)).astype(np.int32)
    d = m.wall_dist(wall)
    assert d.size == sum(m.nel(l) for l in range(m.nlev))
    assert np.allclose(d, b_dist_here(m, wall), rtol=1e-14, atol=0)
    assert np.all(d > 0)
