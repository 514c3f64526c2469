"""GPU parity against the CPU oracle on the five workloads at their stated sizes (B200).

  c1 heat2d     Q2 heat, 32x32, 4 levels, GS 2/2: integer work, assembly, full solve
  c2 cavity2d   Q2-Q1 lid cavity, 128x128, 6 levels, Re 400, Vanka 3/3: integer work,
                every level's assembly, the first Picard system solved to 1e-10 (FP64 per
                cycle; mixed precision against the oracle's FP64 solution)
  c3 channel3d  hex27/hex8 channel, 64x16x16, 4 levels, Re 100: the same at 440,228 DOFs
                (89.9 M nonzeros on the fine level)
  c4 bouss2d    Q2-Q1 + Q2 Boussinesq cavity, 256x256, 7 levels: the first segregated
                Picard step (NS solve, then T solve on the NS solution)
  c5 adjoint2d  the steady T problem of c4 on its converged velocity, 65,536 lognormal
                element sources and 64 Legendre modes of left-wall data: the adjoint
                gradient against the oracle's transposed solve, the transposed operator
                against the reference's own Transp_Q (LASPACK, compiled from its sources),
                and central differences along 16 seeded directions

Tolerances: integer work bit-exact; FP64 matrix and rhs entries within 1e-12 relative;
per-cycle relative residuals within 1e-6 relative with the same cycle count; solutions
within 1e-9 relative L2 (FP64 and mixed precision against the FP64 oracle); adjoint
gradients within 1e-8 of the oracle's and within 1e-6 of central differences.
The oracle runs its colour-parallel loops on every host core (results do not depend
on the thread count).
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

import exfemus_b200 as ex
from exfemus_b200 import _lib, workloads

from conftest import or_mg, or_phys, rel

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


# ------------------------------------------------------------------ helpers
def _oracle_pair(oracle, w, kind, preset):
    om = oracle.OrMesh(w["dim"], w["nlev"], w["n0"], w["box"])
    osys = oracle.OrSys(om, kind)
    osys.bc_preset(preset)
    return om, osys


def _integer_parity(gmesh, gs, om, os_, nlev):
    """Mesh tables, DOF maps, flags, level patterns, colouring and transfers, bit for bit."""
    assert np.array_equal(gmesh.xyz(), om.xyz())
    for lev in range(nlev):
        gc, gn, gcol = gmesh.conn(lev)
        oc, on, ocol = om.conn(lev)
        assert np.array_equal(gc, oc) and np.array_equal(gn, on) and np.array_equal(gcol, ocol)
        assert gs.ndof(lev) == os_.ndof(lev)
        assert np.array_equal(gs.node_dof(lev), os_.node_dof(lev))
        grp, gcl = gs.pattern(lev)
        orp, ocl = os_.pattern(lev)
        assert np.array_equal(grp, orp) and np.array_equal(gcl, ocl), lev
        gnc, gco = gs.colours(lev)
        onc, oco = os_.colours(lev)
        assert gnc == onc and np.array_equal(gco, oco)
    for lev in range(1, nlev):
        for a, b in zip(gs.prol(lev), os_.prol(lev)):
            assert np.array_equal(a, b)
    for lev in range(nlev - 1):
        for a, b in zip(gs.rest(lev), os_.rest(lev)):
            assert np.array_equal(a, b)
    g0, g1 = gs.bc()
    o0, o1 = os_.bc()
    assert np.array_equal(g0, o0) and np.array_equal(g1, o1)


def _assembly_parity(gs, os_, nlev, rhs=True):
    for lev in range(nlev):
        g, o = gs.matrix(lev), os_.matrix(lev)
        assert np.abs(g - o).max() <= 1e-12 * np.abs(o).max(), (lev, np.abs(g - o).max() / np.abs(o).max())
    if rhs:
        g, o = gs.rhs(), os_.rhs()
        assert np.abs(g - o).max() <= 1e-12 * max(np.abs(o).max(), 1e-300)


def _solve_parity(gs, os_, gp, op, x0):
    """FP64 multigrid on both sides from x0: same cycles, per-cycle residuals, solution."""
    gs.set_x(x0)
    st = gs.solve(gp)
    xo, sto = os_.mg_solve(op, x0=x0)
    assert st.converged and sto.converged
    assert st.cycles == sto.cycles, (st.cycles, sto.cycles)
    hg = np.array(st.hist[:st.cycles])
    ho = np.array(sto.hist[:sto.cycles])
    assert np.all(np.abs(hg - ho) <= 1e-6 * ho + 1e-14), (hg, ho)
    assert rel(gs.x(), xo) < 1e-9
    return xo, st


def _mixed_vs_oracle(gs, gp, x0, xo):
    p = ex.mg_params(**{f[0]: getattr(gp, f[0]) for f in gp._fields_})
    p.precision = _lib.PREC_MIXED
    gs.set_x(x0)
    st = gs.solve(p)
    assert st.converged and st.rel_res <= p.eps
    err = rel(gs.x(), xo)
    assert err < 1e-9, err
    return err


def _ns_params(w, eps=1e-10):
    return (ex.mg_params(eps=eps, max_cycles=200, nu_pre=w["nu"][0], nu_post=w["nu"][1],
                         smoother=_lib.SMOOTH_VANKA, omega=workloads.vanka_omega(w)),
            dict(eps=eps, max_cycles=200, nu_pre=w["nu"][0], nu_post=w["nu"][1], smoother=1,
                 omega=workloads.vanka_omega(w)))


# ------------------------------------------------------------------------ c1
def test_c1_heat2d_full_size(oracle_mod, gpu_lib):
    case = workloads.make_case("heat2d")
    w, gm, t = case["w"], case["mesh"], case["T"]
    nlev, top = w["nlev"], w["nlev"] - 1
    om, ot = _oracle_pair(oracle_mod, w, 0, w["bc"])
    _integer_parity(gm, t, om, ot, nlev)
    qe = workloads.heat_source(om.nel(top))
    t.assemble_all()
    ot.assemble_all(or_phys(oracle_mod, **w["phys"]), xold=np.zeros(ot.ndof(top)), qe=qe)
    _assembly_parity(t, ot, nlev)
    gp = ex.mg_params(eps=1e-10, max_cycles=100, nu_pre=2, nu_post=2, smoother=_lib.SMOOTH_GS)
    op = or_mg(oracle_mod, eps=1e-10, max_cycles=100, nu_pre=2, nu_post=2, smoother=0)
    x0 = np.zeros(t.ntop_dof)
    xo, _ = _solve_parity(t, ot, gp, op, x0)
    _mixed_vs_oracle(t, gp, x0, xo)


# ------------------------------------------------------------------------ c2
def test_c2_cavity2d_full_size(oracle_mod, gpu_lib):
    case = workloads.make_case("cavity2d")
    w, gm, ns = case["w"], case["mesh"], case["NS"]
    nlev, top = w["nlev"], w["nlev"] - 1
    om, ons = _oracle_pair(oracle_mod, w, 1, w["bc"])
    _integer_parity(gm, ns, om, ons, nlev)
    x0 = workloads.ns_initial(w, om.xyz(), om.ntop, ons.ndof(top))
    assert np.array_equal(x0, ns.xold())
    ns.assemble_all()
    ons.assemble_all(or_phys(oracle_mod, **w["phys"]), xold=x0)
    _assembly_parity(ns, ons, nlev)
    gp, opk = _ns_params(w)
    xo, _ = _solve_parity(ns, ons, gp, or_mg(oracle_mod, **opk), x0)
    _mixed_vs_oracle(ns, gp, x0, xo)


# ------------------------------------------------------------------------ c3
def test_c3_channel3d_full_size(oracle_mod, gpu_lib):
    """440,228 DOFs: the oracle's full FP64 solve to 1e-10 (about 23 cycles) is the
    reference for both the GPU FP64 cycles and the mixed-precision solution."""
    case = workloads.make_case("channel3d")
    w, gm, ns = case["w"], case["mesh"], case["NS"]
    nlev, top = w["nlev"], w["nlev"] - 1
    om, ons = _oracle_pair(oracle_mod, w, 1, w["bc"])
    _integer_parity(gm, ns, om, ons, nlev)
    x0 = workloads.ns_initial(w, om.xyz(), om.ntop, ons.ndof(top))
    ns.assemble_all()
    ons.assemble_all(or_phys(oracle_mod, **w["phys"]), xold=x0)
    _assembly_parity(ns, ons, nlev)
    gp, opk = _ns_params(w)
    xo, st = _solve_parity(ns, ons, gp, or_mg(oracle_mod, **opk), x0)
    assert 15 <= st.cycles <= 40
    _mixed_vs_oracle(ns, gp, x0, xo)


# ------------------------------------------------------------------------ c4
def _bouss_oracle(oracle_mod, w):
    om = oracle_mod.OrMesh(w["dim"], w["nlev"], w["n0"], w["box"])
    ons = oracle_mod.OrSys(om, 1)
    ons.bc_preset(w["bc"])
    ot = oracle_mod.OrSys(om, 0)
    ot.bc_preset(w["bc_t"])
    return om, ons, ot


def test_c4_bouss2d_first_picard_step_full_size(oracle_mod, gpu_lib):
    case = workloads.make_case("bouss2d")
    w, gm, ns, t = case["w"], case["mesh"], case["NS"], case["T"]
    nlev, top = w["nlev"], w["nlev"] - 1
    om, ons, ot = _bouss_oracle(oracle_mod, w)
    _integer_parity(gm, ns, om, ons, nlev)
    _integer_parity(gm, t, om, ot, nlev)
    p_ns, p_t = workloads.bouss_phys(w)
    xyz = om.xyz()
    x0_ns = workloads.ns_initial(w, xyz, om.ntop, ons.ndof(top))
    x0_t = workloads.t_initial(w, xyz, ot.ndof(top))
    assert np.array_equal(x0_t, t.xold()) and np.array_equal(x0_ns, ns.xold())
    # NS of the first step: buoyancy from the initial temperature
    ns.assemble_all()
    ons.assemble_all(or_phys(oracle_mod, **p_ns), xold=x0_ns, temp=x0_t)
    _assembly_parity(ns, ons, nlev)
    gp, opk = _ns_params(w)
    xo_ns, _ = _solve_parity(ns, ons, gp, or_mg(oracle_mod, **opk), x0_ns)
    _mixed_vs_oracle(ns, gp, x0_ns, xo_ns)
    # T of the first step on the same velocity (the oracle's NS solution on both sides)
    ns.set_xold(xo_ns)
    t.assemble_all()
    ot.assemble_all(or_phys(oracle_mod, **p_t), xold=x0_t, vel=xo_ns)
    _assembly_parity(t, ot, nlev)
    gpt = ex.mg_params(eps=1e-10, max_cycles=200, nu_pre=w["nu"][0], nu_post=w["nu"][1], smoother=_lib.SMOOTH_GS)
    opt = or_mg(oracle_mod, eps=1e-10, max_cycles=200, nu_pre=w["nu"][0], nu_post=w["nu"][1], smoother=0)
    xo_t, _ = _solve_parity(t, ot, gpt, opt, x0_t)
    _mixed_vs_oracle(t, gpt, x0_t, xo_t)


# ------------------------------------------------------------------------ c5
def _elem_shape_integrals(om, lev):
    """int_e phi_k for each element and local node of a uniform quad9 level (tensor
    product of Simpson weights h/6, 4h/6, h/6)."""
    conn, _, _ = om.conn(lev)
    X, Y = om.xyz()
    c = conn
    hx = X[c[:, 1]] - X[c[:, 0]]
    hy = Y[c[:, 3]] - Y[c[:, 0]]
    wt = {0: 1 / 6, 1: 4 / 6, 2: 1 / 6}
    abc = [(0, 0), (2, 0), (2, 2), (0, 2), (1, 0), (2, 1), (1, 2), (0, 1), (1, 1)]
    W = np.array([wt[a] * wt[b] for a, b in abc])
    return conn, (hx * hy)[:, None] * W[None, :]


def test_c5_adjoint_gradient_full_size(oracle_mod, gpu_lib):
    """dJ/dq_e and dJ/dg of J = w^T T on the c4 mesh at its converged velocity."""
    L = _lib.load()
    case = workloads.make_case("bouss2d")
    w = dict(workloads.WORKLOADS["adjoint2d"])
    workloads.picard(case, w["picard"], precision=_lib.PREC_MIXED)
    gm, ns, t = case["mesh"], case["NS"], case["T"]
    top = w["nlev"] - 1
    vel = ns.xold()
    t.phys.inv_dt = 0.0
    om, _, ot = _bouss_oracle(oracle_mod, w)
    xyz = om.xyz()
    qe = workloads.lognormal_source(om.nel(top), seed=0)
    g = np.zeros(w["modes"])
    g[0] = 1.0
    g[1:] = 0.1 * np.random.default_rng(1).standard_normal(w["modes"] - 1) / np.arange(2, w["modes"] + 1)
    x0 = workloads.t_initial(w, xyz, t.ntop_dof, g_modes=g)
    wj = np.random.default_rng(7).random(t.ntop_dof)
    # GPU forward + backward
    p = ex.mg_params(eps=1e-11, max_cycles=400, smoother=_lib.SMOOTH_GS, nu_pre=3, nu_post=3)
    t.set_xold(x0)
    t.set_source(qe)
    stf, stb = _lib.ExfSolveStats(), _lib.ExfSolveStats()
    _lib.check(L.exf_adjoint_forward(t.h, C.byref(t.phys), C.byref(p), C.byref(stf)))
    djdq = np.zeros(qe.size)
    djdg = np.zeros(t.ntop_dof)
    _lib.check(L.exf_adjoint_backward(t.h, C.byref(t.phys), C.byref(p), _lib.dptr(wj), _lib.dptr(djdq),
                                      _lib.dptr(djdg), C.byref(stb)))
    assert stf.converged and stb.converged
    # oracle: the same system, its transpose pinned to LASPACK's Transp_Q, the adjoint solve
    _, p_t = workloads.bouss_phys(w)
    p_t = dict(p_t, inv_dt=0.0)
    oph = or_phys(oracle_mod, **p_t)
    ot.assemble_all(oph, xold=x0, vel=vel, qe=qe)
    G = t.matrix(top)
    O = ot.matrix(top)
    assert np.abs(G - O).max() <= 1e-12 * np.abs(O).max()
    rp, col, val = ot.csr(top)
    n = ot.ndof(top)
    v = np.random.default_rng(3).standard_normal(n)
    if oracle_mod.laspack_available():
        at_ref = oracle_mod.Laspack().spmv_t(rp, col, val, v)
    else:
        at_ref = sp.csr_matrix((val, col, rp), shape=(n, n)).T @ v
    ot.transpose_all()
    assert rel(ot.spmv(top, v), at_ref) < 1e-14
    ot.set_rhs(wj)
    lam, sto = ot.mg_solve(or_mg(oracle_mod, eps=1e-11, max_cycles=400, nu_pre=3, nu_post=3, smoother=0,
                                 reverse_colours=1), x0=np.zeros(n))
    assert sto.converged
    b0, _ = ot.bc()
    conn, ws = _elem_shape_integrals(om, top)
    djdq_o = ((lam * b0)[conn] * ws).sum(axis=1)
    # W = d b / d x_old: the rhs of x_old = 1 with no sources and no mass term
    ot.transpose_all()
    ow = oracle_mod.OrSys(om, 0)
    ow.bc_preset(w["bc_t"])
    ow.assemble(top, 1, oph, xold=np.ones(n), vel=vel, qe=np.zeros(qe.size))
    djdg_o = lam * ow.rhs()
    assert rel(djdq, djdq_o) < 1e-8, rel(djdq, djdq_o)
    assert rel(djdg, djdg_o) < 1e-8, rel(djdg, djdg_o)
    # central differences along 16 seeded directions of (q, g) (fixed 100-cycle solves,
    # which are linear in the data)
    left = xyz[0] == w["box"][0]
    s_left = 2.0 * xyz[1][left] - 1.0
    djdmode = np.array([djdg[left] @ workloads.legendre(k, s_left) for k in range(w["modes"])])

    def J(q, gm_):
        t.set_xold(workloads.t_initial(w, xyz, t.ntop_dof, g_modes=gm_))
        t.set_source(q)
        t.set_x(np.zeros(t.ntop_dof))
        pf = ex.mg_params(eps=1e-30, max_cycles=100, smoother=_lib.SMOOTH_GS, nu_pre=3, nu_post=3)
        stj = _lib.ExfSolveStats()
        rc = L.exf_adjoint_forward(t.h, C.byref(t.phys), C.byref(pf), C.byref(stj))
        assert rc in (_lib.EXF_OK, _lib.EXF_ERR_NOT_CONVERGED)
        return float(wj @ t.x())

    rng = np.random.default_rng(16)
    h = 1e-6
    for _ in range(16):
        dq = rng.standard_normal(qe.size)
        dg = rng.standard_normal(w["modes"])
        fd = (J(qe + h * dq, g + h * dg) - J(qe - h * dq, g - h * dg)) / (2 * h)
        ad = float(djdq @ dq + djdmode @ dg)
        assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)
