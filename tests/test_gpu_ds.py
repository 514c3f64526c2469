"""The fluid-structure template's mesh displacement (MGSolDS::GenMatRhs with ALE_MOVING,
template_appl/fsi/SRC/MGSolverDS.C:321-700) on the assembly engine (needs a B200): every
direction assembled on every level against the oracle's restatement, on a box whose
right half is solid, with Dirichlet, natural and interface nodes, then solved by
multigrid against the oracle's solution."""
import numpy as np
import pytest

import exfemus_b200 as ex
from exfemus_b200 import _lib

from conftest import or_mg, rel

pytestmark = pytest.mark.gpu

DT = 0.05
# dim: box, levels, level-0 elements; the solid is x >= 1 (a level-0 element boundary)
CASES = {2: ((0.0, 2.0, 0.0, 1.0), 3, (4, 2)), 3: ((0.0, 2.0, 0.0, 1.0, 0.0, 1.0), 2, (2, 1, 1))}


def flags(xyz):
    """(bc0, bc1) per node, the reference's volume and boundary flags: fluid interior 1;
    solid (x > 1) 2; interface (x = 1) 4; fluid inlet x = 0 Dirichlet (0, bc1 0); fluid
    top y = 1 Dirichlet moving with the structure (0, bc1 1); fluid bottom y = 0 (and the
    z faces) natural (odd bc0, no penalty)."""
    x, y = xyz[0], xyz[1]
    n = x.size
    b0, b1 = np.ones(n, np.int32), np.zeros(n, np.int32)
    top = np.abs(y - 1.0) < 1e-12
    b0[top], b1[top] = 0, 1
    inl = np.abs(x) < 1e-12
    b0[inl], b1[inl] = 0, 0
    b0[x > 1.0 + 1e-12] = 2
    b0[np.abs(x - 1.0) < 1e-12] = 4
    return b0, b1


def fields(xyz):
    """u_fsi and d_old [dim][n], smooth and different per component."""
    dim = len(xyz)
    x, y = xyz[0], xyz[1]
    u = np.stack([0.3 * np.sin(1.5 * x + a) * (0.5 + y) + 0.1 * a for a in range(dim)])
    d = np.stack([0.02 * np.cos(x + 2.0 * y + a) for a in range(dim)])
    return u, d


@pytest.fixture(scope="module", params=[2, 3])
def ds_case(oracle_mod, request):
    dim = request.param
    box, nlev, n0 = CASES[dim]
    m = ex.Mesh(dim, nlev, n0, box)
    xyz = m.xyz()
    b0, b1 = flags(xyz)
    u, d = fields(xyz)
    om = oracle_mod.OrMesh(dim, nlev, n0, box)
    sys, osys = [], []
    for direction in range(dim):
        s = ex.MGSolDS(m, direction)
        s.set_bc(b0, b1)
        s.set_fields(DT, u, d)
        sys.append(s)
        o = oracle_mod.OrSys(om, 0)
        o.set_bc(b0, b1)
        for lev in range(nlev):
            o.ds_assemble(lev, 1 if lev == nlev - 1 else 0, direction, DT, u, d)
        osys.append(o)
    return dict(mesh=m, sys=sys, osys=osys, nlev=nlev, dim=dim, xyz=xyz, u=u, d=d, b0=b0, b1=b1)


def test_displacement_assembly_matches_the_oracle(gpu_lib, ds_case):
    for s, o in zip(ds_case["sys"], ds_case["osys"]):
        s.assemble_all()
        for lev in range(ds_case["nlev"]):
            rp, col, val = s.csr(lev)
            orp, ocol, oval = o.csr(lev)
            assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
            assert rel(val, oval) <= 1e-12, (s.direction, lev)
        assert rel(s.rhs(), o.rhs()) <= 1e-12, s.direction
        assert np.all(np.isfinite(s.rhs()))


def test_displacement_solves_match_the_oracle(gpu_lib, oracle_mod, ds_case):
    xyz, u, d, b0, b1 = (ds_case[k] for k in ("xyz", "u", "d", "b0", "b1"))
    solid = b0 >= 2  # solid and interface nodes: d = u_fsi dt + d_old of the direction
    top = (np.abs(xyz[1] - 1.0) < 1e-12) & (b0 == 0) & (b1 == 1)
    for s, o in zip(ds_case["sys"], ds_case["osys"]):
        s.assemble_all()
        s.set_x(np.zeros(s.ntop_dof))
        st = s.solve(ex.mg_params(eps=1e-12, max_cycles=100, smoother=_lib.SMOOTH_GS))
        xo, sto = o.mg_solve(or_mg(oracle_mod, eps=1e-12, max_cycles=100))
        assert st.converged and sto.converged
        assert rel(s.x(), xo) <= 1e-9, s.direction
        x = s.x()
        a = s.direction
        assert np.abs(x[solid] - (u[a][solid] * DT + d[a][solid])).max() <= 1e-12
        # the moving fluid wall takes the x components in every direction, as the
        # reference's penalty rhs reads fsi_idx and disp_idx without _dir
        assert np.abs(x[top] - (u[0][top] * DT + d[0][top])).max() <= 1e-10


def test_displacement_needs_its_fields(gpu_lib):
    m = ex.Mesh(2, 2, (2, 2), (0, 1, 0, 1))
    s = ex.MGSolDS(m, 0)
    with pytest.raises(_lib.ExfError) as e:
        s.assemble_all()
    assert e.value.code == _lib.EXF_ERR_STATE
    u = np.zeros((2, m.ntop))
    with pytest.raises(_lib.ExfError) as e:
        ex.MGSolDS(m, 2).set_fields(DT, u, u)  # no z direction in 2D
    assert e.value.code == _lib.EXF_ERR_ARG
    with pytest.raises(_lib.ExfError) as e:
        s.set_fields(0.0, u, u)
    assert e.value.code == _lib.EXF_ERR_ARG
    t = ex.MGSolT(m)
    with pytest.raises(_lib.ExfError) as e:
        _lib.check(t.L.exf_sys_set_ds(t.h, 0, DT, _lib.dptr(np.ascontiguousarray(u)), _lib.dptr(np.ascontiguousarray(u))))
    assert e.value.code == _lib.EXF_ERR_ARG


def coupled_systems(dim, moving):
    """A fresh mesh with the velocity system (x_old = u_fsi, not stepped) and the
    displacement systems in coupled mode (their fields are the systems' x_old)."""
    box, nlev, n0 = CASES[dim]
    m = ex.Mesh(dim, nlev, n0, box)
    xyz = m.xyz()
    N = m.ntop
    b0, b1 = flags(xyz)
    u, d = fields(xyz)
    ns = ex.MGSolNS(m)
    xns = np.zeros(ns.ntop_dof)
    xns[:dim * N] = u.reshape(-1)
    ns.set_xold(xns)
    ds = []
    for a in range(dim):
        s = ex.MGSolDS(m, a)
        s.set_bc(b0, b1)
        s.set_xold(d[a])
        s.set_fields(DT)
        s.couple(ns)
        if moving:
            s.set_mesh_motion(True)
        ds.append(s)
    for s in ds[1:]:
        s.couple(ds[0])
    params = [ex.mg_params(eps=1e-11, max_cycles=100, smoother=_lib.SMOOTH_GS) for _ in ds]
    return m, ds, params, ns


def test_coupled_fields_give_the_host_field_operators_bitwise(gpu_lib, ds_case):
    """The coupled mode reads the velocity system's and the displacement systems' x_old
    in place of the node fields: the same matrices and rhs, bit for bit."""
    _, ds, _, _ns = coupled_systems(ds_case["dim"], False)
    for s, h in zip(ds, ds_case["sys"]):
        s.assemble_all()
        h.assemble_all()
        for lev in range(ds_case["nlev"]):
            assert np.array_equal(s.csr(lev)[2], h.csr(lev)[2]), (s.direction, lev)
        assert np.array_equal(s.rhs(), h.rhs())


@pytest.mark.parametrize("dim", [2, 3])
def test_time_loop_moves_the_mesh_as_the_host_loop(gpu_lib, dim):
    """exf_timestep_loop over the displacement systems with mesh motion gives the bits,
    cycle counts and node coordinates of the same MGTimeStep sequence driven from here;
    each update moves the direction's coordinates by x - x_old."""
    ma, a, pa, _nsa = coupled_systems(dim, True)
    mb, b, pb, _nsb = coupled_systems(dim, True)
    nsteps = 2
    host = []
    for _ in range(nsteps):
        row = []
        for s, p in zip(a, pa):
            s.assemble_all()
            st = s.solve(p)
            assert st.converged
            before, xo, x = ma.xyz(), s.xold(), s.x()
            s.xold_update()
            after = ma.xyz()
            k = s.direction
            assert np.array_equal(after[k], before[k] + (x - xo))
            assert np.array_equal(np.delete(after, k, 0), np.delete(before, k, 0))
            row.append(st.cycles)
        host.append(row)
    cyc, _ = ex.timestep_loop(b, pb, nsteps)
    assert cyc.tolist() == host
    for sa, sb in zip(a, b):
        assert np.array_equal(sa.x(), sb.x())
    assert np.array_equal(ma.xyz(), mb.xyz())
    assert not np.array_equal(mb.xyz(), ex.Mesh(dim, *CASES[dim][1:], CASES[dim][0]).xyz())


def test_coupled_mode_needs_its_partners(gpu_lib):
    m = ex.Mesh(2, 2, (2, 2), (0, 1, 0, 1))
    s = ex.MGSolDS(m, 1)
    s.set_fields(DT)
    with pytest.raises(_lib.ExfError) as e:
        s.assemble_all()  # no velocity system, no dx system
    assert e.value.code == _lib.EXF_ERR_STATE
    s.couple(ex.MGSolNS(m))
    with pytest.raises(_lib.ExfError) as e:
        s.assemble_all()  # still no dx system
    assert e.value.code == _lib.EXF_ERR_STATE
    with pytest.raises(_lib.ExfError) as e:
        _lib.check(s.L.exf_sys_set_ds(s.h, 1, DT, _lib.dptr(np.zeros(2 * m.ntop)), None))  # one field only
    assert e.value.code == _lib.EXF_ERR_ARG


def test_a_closed_partner_leaves_no_coupling(gpu_lib):
    """Closing a coupled system clears it from its partners: their next assembly reports
    the missing coupling instead of reading a destroyed system."""
    m, ds, _, ns = coupled_systems(2, False)
    ds[1].assemble_all()
    ns.close()
    for s in ds:
        with pytest.raises(_lib.ExfError) as e:
            s.assemble_all()
        assert e.value.code == _lib.EXF_ERR_STATE
    m2, ds2, _, ns2 = coupled_systems(2, False)
    ds2[0].close()
    with pytest.raises(_lib.ExfError) as e:
        ds2[1].assemble_all()  # its dx system is gone
    assert e.value.code == _lib.EXF_ERR_STATE
