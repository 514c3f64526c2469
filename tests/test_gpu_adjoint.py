"""Discrete adjoint of the heat solve (needs a B200): gradients with respect to the
per-element sources q_e and the Dirichlet data, checked against central finite
differences (h = 1e-6) along seeded random directions and against the reference's
LASPACK GMRESIter on Transp_Q(A) (the transposed system)."""
import numpy as np
import pytest

import exfemus_b200 as ex
from exfemus_b200 import _lib, workloads

from conftest import or_phys, rel

pytestmark = pytest.mark.gpu

N0, NLEV = (4, 4), 3


def _velocity(xyz, n_nodes):
    x, y = xyz
    u = np.sin(np.pi * x) ** 2 * np.sin(2 * np.pi * y)
    v = -np.sin(2 * np.pi * x) * np.sin(np.pi * y) ** 2
    out = np.zeros(2 * n_nodes + 0)
    out[:n_nodes], out[n_nodes:] = u, v
    return out


def _top_wall_weights(xyz, L):
    """w_i = int_{y=1} phi_i ds (Simpson weights of each quad9 side)."""
    x, y = xyz
    w = np.zeros(x.size)
    top = np.where(y == 1.0)[0]
    order = top[np.argsort(x[top])]
    xs = x[order]
    for k in range(0, len(order) - 2, 2):
        h = xs[k + 2] - xs[k]
        w[order[k]] += h / 6
        w[order[k + 1]] += 4 * h / 6
        w[order[k + 2]] += h / 6
    return w


@pytest.fixture(scope="module")
def setup(gpu_lib):
    mesh = ex.Mesh(2, NLEV, N0, (0, 1, 0, 1))
    ns = ex.MGSolNS(mesh)
    ns.GenBc(_lib.BC_BOUSS_NS)
    t = ex.MGSolT(mesh)
    t.GenBc(_lib.BC_BOUSS_T)
    xyz = mesh.xyz()
    N = mesh.ntop
    xns = np.zeros(ns.ntop_dof)
    xns[:2 * N] = 0.5 * _velocity(xyz, N)
    ns.set_xold(xns)
    t.couple(ns)
    ph_ns, ph_t = workloads.bouss_phys(dict(ra=1e4, pr=0.71))
    t.phys = ex.phys(**ph_t)
    g = np.random.default_rng(1).standard_normal(4)
    w = dict(box=(0, 1, 0, 1))
    x0 = workloads.t_initial(w, xyz, t.ntop_dof, g_modes=g)
    qe = workloads.lognormal_source(mesh.nel(NLEV - 1), seed=3)
    t.set_xold(x0)
    t.set_source(qe)
    wj = _top_wall_weights(xyz, None)
    return dict(mesh=mesh, ns=ns, t=t, x0=x0, qe=qe, wj=wj, xns=xns, ph_t=ph_t)


def _params():
    return ex.mg_params(eps=1e-13, max_cycles=200, smoother=_lib.SMOOTH_GS, nu_pre=2, nu_post=2)


def _J(s, xold, qe):
    """J = w^T T from a fixed number of cycles started at zero: the solve is then one
    linear map of the data, so the central difference carries no solver noise."""
    t = s["t"]
    t.set_xold(xold)
    t.set_source(qe)
    t.set_x(np.zeros(t.ntop_dof))
    st = _lib.ExfSolveStats()
    L = _lib.load()
    import ctypes as C
    p = _params()
    p.eps, p.max_cycles = 1e-30, 40
    rc = L.exf_adjoint_forward(t.h, C.byref(t.phys), C.byref(p), C.byref(st))
    assert rc in (_lib.EXF_OK, _lib.EXF_ERR_NOT_CONVERGED) and st.cycles == 40 and st.rel_res < 1e-13
    return float(s["wj"] @ t.x())


def _grad(s):
    import ctypes as C
    t = s["t"]
    L = _lib.load()
    t.set_xold(s["x0"])
    t.set_source(s["qe"])
    st = _lib.ExfSolveStats()
    _lib.check(L.exf_adjoint_forward(t.h, C.byref(t.phys), C.byref(_params()), C.byref(st)))
    nel = s["mesh"].nel(NLEV - 1)
    djdq = np.zeros(nel)
    djdg = np.zeros(t.ntop_dof)
    wj = np.ascontiguousarray(s["wj"])
    rc = L.exf_adjoint_backward(t.h, C.byref(t.phys), C.byref(_params()), _lib.dptr(wj), _lib.dptr(djdq),
                                _lib.dptr(djdg), C.byref(st))
    _lib.check(rc)
    assert st.converged
    return djdq, djdg


def test_source_gradient_matches_central_fd(setup):
    djdq, _ = _grad(setup)
    rng = np.random.default_rng(11)
    for _ in range(4):
        dq = rng.standard_normal(djdq.size)
        h = 1e-6
        fd = (_J(setup, setup["x0"], setup["qe"] + h * dq) - _J(setup, setup["x0"], setup["qe"] - h * dq)) / (2 * h)
        assert abs(fd - djdq @ dq) <= 1e-6 * abs(fd), (fd, djdq @ dq)


def test_dirichlet_gradient_matches_central_fd(setup):
    _, djdg = _grad(setup)
    b0, b1 = setup["t"].bc()
    dirichlet_nonhom = (b0 == 0) & (b1 % 2 == 1)
    rng = np.random.default_rng(12)
    for _ in range(4):
        dg = np.where(dirichlet_nonhom, rng.standard_normal(djdg.size), 0.0)
        h = 1e-6
        fd = (_J(setup, setup["x0"] + h * dg, setup["qe"]) - _J(setup, setup["x0"] - h * dg, setup["qe"])) / (2 * h)
        assert abs(fd - djdg @ dg) <= 1e-6 * abs(fd), (fd, djdg @ dg)
    # gradient vanishes off the non-homogeneous Dirichlet DOFs
    assert np.all(djdg[~(b0 == 0)] == 0)


def test_forward_state_restored_after_backward(setup):
    t = setup["t"]
    J0 = _J(setup, setup["x0"], setup["qe"])
    _grad(setup)
    assert abs(float(setup["wj"] @ t.x()) - J0) <= 1e-12 * abs(J0)


@pytest.mark.skipif(not __import__("oracle").laspack_available(), reason="reference LASPACK not built")
def test_gradient_matches_laspack_transposed_solve(setup, oracle_mod):
    """lambda from the reference's GMRESIter on Transp_Q(A) of the oracle matrix."""
    djdq, djdg = _grad(setup)
    om = oracle_mod.OrMesh(2, NLEV, N0, (0, 1, 0, 1))
    os_ = oracle_mod.OrSys(om, 0)
    os_.bc_preset(_lib.BC_BOUSS_T)
    N = om.ntop
    ph = or_phys(oracle_mod, **setup["ph_t"])
    vel = setup["xns"][:2 * N]
    os_.assemble_all(ph, xold=setup["x0"], vel=vel, qe=setup["qe"])
    rp, col, val = os_.csr(NLEV - 1)
    lam, it, acc = oracle_mod.Laspack().gmres(rp, col, val, setup["wj"], tol=1e-13, maxit=20000, restart=60,
                                             transpose=True)
    assert acc < 1e-11
    rng = np.random.default_rng(13)
    dq = rng.standard_normal(djdq.size)
    os_.assemble(NLEV - 1, 1, ph, xold=np.zeros(N), vel=vel, qe=dq)
    assert rel(lam @ os_.rhs(), djdq @ dq) < 1e-8
    b0, b1 = setup["t"].bc()
    dg = np.where((b0 == 0) & (b1 % 2 == 1), rng.standard_normal(N), 0.0)
    os_.assemble(NLEV - 1, 1, ph, xold=dg, vel=vel, qe=np.zeros(djdq.size))
    assert rel(lam @ os_.rhs(), djdg @ dg) < 1e-8
