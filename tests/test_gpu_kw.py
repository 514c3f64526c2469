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

NU_WALL = 0.01
# dim: box, levels, level-0 elements (walls: the y and z faces)
CASES = {2: ((0.0, 2.0, 0.0, 1.0), 3, (4, 2)), 3: ((0.0, 2.0, 0.0, 1.0, 0.0, 1.0), 2, (2, 1, 1))}


def on_wall(xyz):
    w = (np.abs(xyz[1]) < 1e-12) | (np.abs(xyz[1] - 1.0) < 1e-12)
    if len(xyz) == 3:
        w |= (np.abs(xyz[2]) < 1e-12) | (np.abs(xyz[2] - 1.0) < 1e-12)
    return w


def flags(xyz):
    """(bc0, bc1) per node: walls Dirichlet (bc1 2: omega's wall value, kappa 0), inlet
    x = 0 Dirichlet on the old value (bc1 1), outlet x = 2 Neumann (bc0 1, bc1 1),
    interior (1, 0)."""
    x = xyz[0]
    n = x.size
    b0, b1 = np.ones(n, np.int32), np.zeros(n, np.int32)
    b1[np.abs(x - 2.0) < 1e-12] = 1
    inl = np.abs(x) < 1e-12
    b0[inl], b1[inl] = 0, 1
    wall = on_wall(xyz)
    b0[wall], b1[wall] = 0, 2
    return b0, b1


def fields(xyz):
    """Velocity components, kappa, omega at the nodes."""
    x, y = xyz[0], xyz[1]
    zf = 4.0 * xyz[2] * (1.0 - xyz[2]) if len(xyz) == 3 else 1.0
    u = 4.0 * y * (1.0 - y) * zf * (1.0 + 0.1 * np.sin(2.0 * x))
    vel = [u, 0.05 * np.sin(np.pi * y) * x]
    if len(xyz) == 3:
        vel.append(0.03 * np.sin(np.pi * xyz[2]) * y)
    k = 0.01 + 0.02 * y * (1.0 - y) * (1.0 + 0.2 * x)
    w = 40.0 + 30.0 * (y - 0.5) ** 2 + 2.0 * x
    return vel, k, w


def wall_dist(conns, xyz):
    """Centroid distance of every element to the nearest wall plane, level after level."""
    d = []
    for c in conns:
        cen = [xyz[a][c].mean(axis=1) for a in range(1, len(xyz))]
        d.append(np.min([np.minimum(q, 1.0 - q) for q in cen], axis=0))
    return np.concatenate(d)


@pytest.fixture(scope="module", params=[2, 3])
def kw_case(oracle_mod, request):
    dim = request.param
    box, nlev, n0 = CASES[dim]
    m = ex.Mesh(dim, nlev, n0, box)
    xyz = m.xyz()
    N = m.ntop
    vel, k, w = fields(xyz)
    ns = ex.MGSolNS(m)
    xns = np.zeros(ns.ntop_dof)
    for a in range(dim):
        xns[a * N:(a + 1) * N] = vel[a]
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
    om = oracle_mod.OrMesh(dim, nlev, n0, box)
    osys = []
    oph = or_phys(oracle_mod, inv_re=0.01, inv_dt=10.0)
    off = np.cumsum([0] + [c.shape[0] for c in conns])
    for var in (0, 1):
        o = oracle_mod.OrSys(om, 0)
        o.set_bc(b0, b1)
        for lev in range(nlev):
            o.kw_assemble(lev, 1 if lev == nlev - 1 else 0, var, oph, xns[:dim * N], k, w,
                          dist[off[lev]:off[lev + 1]], NU_WALL)
        osys.append(o)
    return dict(mesh=m, ns=ns, sys=sys, osys=osys, nlev=nlev, dim=dim, box=box, n0=n0)


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
    xk = kw_case["sys"][0].x()
    assert np.abs(xk[on_wall(kw_case["mesh"].xyz())]).max() < 1e-10  # kappa = 0 on the walls


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
    m, nlev, dim = kw_case["mesh"], kw_case["nlev"], kw_case["dim"]
    xyz = m.xyz()
    vel, k, w = fields(xyz)
    N = m.ntop
    ph = ex.phys(inv_re=0.01, inv_dt=10.0)

    def gpu_ns(turb):
        ns = ex.MGSolNS(m)
        ns.GenBc(_lib.BC_CHANNEL)
        x = np.zeros(ns.ntop_dof)
        for a in range(dim):
            x[a * N:(a + 1) * N] = vel[a]
        ns.set_xold(x)
        ns.phys = ph
        if turb:
            for s in kw_case["sys"]:
                ns.couple(s)
        ns.assemble_all()
        return ns, x

    ns, x = gpu_ns(True)
    lam, _ = gpu_ns(False)
    om = oracle_mod.OrMesh(dim, nlev, kw_case["n0"], kw_case["box"])
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
    """MGMesh::B_dist restated: element centre to the nearest wall-side centre; the sides
    are the reference's _surf_top (tests/golden/mggeomel.json)."""
    import json
    import os
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mggeomel.json")))
    t = gold["quad9_surf_top" if m.dim == 2 else "hex27_surf_top"]
    side = np.array(t["data"], dtype=int).reshape(t["shape"])
    xyz = m.xyz()
    out = []
    for lev in range(m.nlev):
        conn, neigh = m.conn(lev)[:2]
        wc = []
        for e in range(conn.shape[0]):
            for sd in range(side.shape[0]):
                if neigh[e, sd] == -1 and all(wall_node[conn[e, k]] for k in side[sd]):
                    wc.append(xyz[:, conn[e, side[sd]]].sum(axis=1) / side.shape[1])
        wc = np.array(wc)
        xm = xyz[:, conn].sum(axis=2) / conn.shape[1]
        d2 = ((xm.T[:, None, :] - wc[None, :, :]) ** 2).sum(axis=2)
        out.append(np.sqrt(d2.min(axis=1)))
    return np.concatenate(out)


def test_wall_distances_are_b_dist(gpu_lib, kw_case):
    m = kw_case["mesh"]
    wall = on_wall(m.xyz()).astype(np.int32)
    d = m.wall_dist(wall)
    assert d.size == sum(m.nel(l) for l in range(m.nlev))
    assert np.allclose(d, b_dist_here(m, wall), rtol=1e-14, atol=0)
    assert np.all(d > 0)


def channel_kw_systems(nlev=3):
    """NS (parabolic start), kappa and omega on the 2D channel, all coupled, eddy
    viscosity on."""
    box, _, n0 = CASES[2]
    m = ex.Mesh(2, nlev, n0, box)
    xyz = m.xyz()
    N = m.ntop
    vel, k, w = fields(xyz)
    ph = ex.phys(inv_re=0.01, inv_dt=10.0)
    ns = ex.MGSolNS(m)
    ns.GenBc(_lib.BC_CHANNEL)
    x = np.zeros(ns.ntop_dof)
    x[:N], x[N:2 * N] = vel[0], vel[1]
    ns.set_xold(x)
    ns.set_x(x)
    ns.phys = ph
    b0, b1 = flags(xyz)
    dist = m.wall_dist(on_wall(xyz).astype(np.int32))
    tk = []
    for var, old in ((0, k), (1, w)):
        s = ex.MGSolTBK(m, var)
        s.set_bc(b0, b1)
        s.set_xold(old)
        s.set_wall(dist, NU_WALL)
        s.phys = ph
        tk.append(s)
    for s, o in ((tk[0], tk[1]), (tk[1], tk[0])):
        s.couple(ns)
        s.couple(o)
        ns.couple(s)
    params = [ex.mg_params(eps=1e-10, max_cycles=200, smoother=_lib.SMOOTH_VANKA, nu_pre=3, nu_post=3, omega=0.4)]
    params += [ex.mg_params(eps=1e-10, max_cycles=200, smoother=_lib.SMOOTH_GS) for _ in tk]
    return m, [ns] + tk, params


def test_turbulent_channel_time_loop_matches_the_host_loop(gpu_lib):
    """exf_timestep_loop over NS (with the eddy viscosity), kappa and omega gives the bits
    of the same MGTimeStep sequence driven from here, with the same cycle counts."""
    _, a, pa = channel_kw_systems()
    _, b, pb = channel_kw_systems()
    nsteps = 3
    host = []
    for _ in range(nsteps):
        row = []
        for s, p in zip(a, pa):
            s.assemble_all()
            st = s.solve(p)
            assert st.converged
            s.xold_update()
            row.append(st.cycles)
        host.append(row)
    cyc, sec = ex.timestep_loop(b, pb, nsteps)
    assert cyc.tolist() == host
    for sa, sb in zip(a, b):
        assert np.array_equal(sa.x(), sb.x())
    assert np.all(np.isfinite(b[1].x())) and b[2].x().min() > 0  # omega stays positive
