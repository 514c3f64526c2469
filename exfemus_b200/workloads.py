"""The five synthetic workloads of the path and their initial/boundary data.

Each workload is a structured box hierarchy, a physics parameter set, boundary flags
(a bc_read preset) and the x_old initial field that carries the Dirichlet data (the
reference reads Dirichlet values from x_old at boundary nodes, MGSolverNS.C:546-568,
MGSolverT.C Dirichlet block).  Steady problems use no mass term (inv_dt = 0) and a
Dirichlet penalty scale of 1 (Ipenalty = det_side); the rows at Dirichlet DOFs are
pure diagonal, so the scale does not change the solution.

  heat2d     Q2 heat, unit square 32x32, 4 levels, f = 1 + 0.1 u_e, T = 0 on walls, GS 2/2
  cavity2d   Q2-Q1 lid cavity 128x128, 6 levels, Re = 400, 10 Picard steps, Vanka 3/3
  channel3d  hex27/hex8 channel 4x1x1, 64x16x16, 4 levels, Re = 100, 8 Picard steps
  bouss2d    Q2-Q1 + Q2 differentially heated cavity 256x256, 7 levels, Ra 1e5, Pr 0.71;
             every segregated Picard step is an implicit pseudo-time step dt = 1 (the
             reference's transient mass terms, inv_dt = 1): started from rest, the plain
             steady Picard iterate is a Stokes flow with |u| ~ 1/nu, and the next
             linearisation is so convection-dominated that the multigrid diverges
  adjoint2d  the steady heat problem on the converged bouss2d velocity, with per-element
             sources and 64 Legendre modes of left-wall data
"""
import math

import numpy as np

from . import _lib

WORKLOADS = {
    "heat2d": dict(dim=2, nlev=4, n0=(4, 4), box=(0, 1, 0, 1), kind="T", bc=_lib.BC_HEAT_DIRICHLET,
                   phys=dict(inv_re=1.0, inv_prdl=1.0), nu=(2, 2), picard=1),
    "cavity2d": dict(dim=2, nlev=6, n0=(4, 4), box=(0, 1, 0, 1), kind="NS", bc=_lib.BC_CAVITY,
                     phys=dict(inv_re=1.0 / 400.0), nu=(3, 3), picard=10),
    "channel3d": dict(dim=3, nlev=4, n0=(8, 2, 2), box=(0, 4, 0, 1, 0, 1), kind="NS", bc=_lib.BC_CHANNEL,
                      phys=dict(inv_re=0.01), nu=(3, 3), picard=8, omega=0.5),
    "bouss2d": dict(dim=2, nlev=7, n0=(4, 4), box=(0, 1, 0, 1), kind="NS+T", bc=_lib.BC_BOUSS_NS,
                    bc_t=_lib.BC_BOUSS_T, ra=1e5, pr=0.71, nu=(3, 3), picard=15, inv_dt=1.0),
    "adjoint2d": dict(dim=2, nlev=7, n0=(4, 4), box=(0, 1, 0, 1), kind="NS+T", bc=_lib.BC_BOUSS_NS,
                      bc_t=_lib.BC_BOUSS_T, ra=1e5, pr=0.71, nu=(3, 3), picard=15, inv_dt=1.0, modes=64),
}

VANKA_OMEGA = 0.4


def vanka_omega(w):
    """Vanka damping of a workload: its own "omega" where one was measured (channel3d: 0.5
    takes the first Picard system from 23 V-cycles at 0.4 to 17, and every one of the 8
    steps takes fewer; 0.7 and above diverge), otherwise VANKA_OMEGA."""
    return w.get("omega", VANKA_OMEGA)


def scaled(name, nlev=None, n0=None):
    """A copy of a workload on a smaller hierarchy (test sizes)."""
    w = dict(WORKLOADS[name])
    if nlev is not None:
        w["nlev"] = nlev
    if n0 is not None:
        w["n0"] = n0
    return w


def bouss_phys(w):
    """Nondimensional Boussinesq scaling: nu = sqrt(Pr/Ra), alpha = 1/sqrt(Ra Pr), f = T e_y."""
    nu = math.sqrt(w["pr"] / w["ra"])
    alpha = 1.0 / math.sqrt(w["ra"] * w["pr"])
    inv_dt = w.get("inv_dt", 0.0)
    ns = dict(inv_re=nu, buoy=1.0, dirg=(0.0, 1.0, 0.0), inv_dt=inv_dt)
    t = dict(inv_re=nu, inv_prdl=alpha / nu, inv_dt=inv_dt)
    return ns, t


def heat_source(nel, seed=0):
    """f_e = 1 + 0.1 u_e, u_e ~ U[0,1) per top-level element (PCG64 seed)."""
    return 1.0 + 0.1 * np.random.default_rng(seed).random(nel)


def lognormal_source(nel, seed=0):
    """q_e ~ lognormal(0, 0.5) per top-level element (PCG64 seed)."""
    return np.random.default_rng(seed).lognormal(0.0, 0.5, nel)


def legendre(k, s):
    """Legendre polynomial P_k on [-1,1] by the three-term recurrence."""
    p0, p1 = np.ones_like(s), s
    if k == 0:
        return p0
    for n in range(1, k):
        p0, p1 = p1, ((2 * n + 1) * s * p1 - n * p0) / (n + 1)
    return p1


def ns_initial(w, xyz, ntop_nodes, ndof):
    """x_old of the NS system: Dirichlet data on the boundary, zero inside."""
    x = np.zeros(ndof)
    N = ntop_nodes
    if w["bc"] == _lib.BC_CAVITY:
        X, Y = xyz[0], xyz[1]
        lid = (Y == w["box"][3]) & (X > w["box"][0]) & (X < w["box"][1])
        x[:N][lid] = 1.0
    elif w["bc"] == _lib.BC_CHANNEL:
        X, Y, Z = xyz[0], xyz[1], xyz[2]
        inlet = X == w["box"][0]
        x[:N][inlet] = 16.0 * Y[inlet] * (1 - Y[inlet]) * Z[inlet] * (1 - Z[inlet])
    return x


def t_initial(w, xyz, ndof, g_modes=None):
    """x_old of the T system: left wall g(y) = sum_k g_k P_k(2y-1) (default T=1), right wall 0."""
    x = np.zeros(ndof)
    X, Y = xyz[0], xyz[1]
    left = X == w["box"][0]
    if g_modes is None:
        x[left] = 1.0
    else:
        s = 2.0 * Y[left] - 1.0
        x[left] = sum(g_modes[k] * legendre(k, s) for k in range(len(g_modes)))
    return x


def make_case(name, device=0, **over):
    """Build mesh + systems of a workload on the GPU; returns a dict of handles."""
    from .mgsolver import MGSolNS, MGSolT, Mesh, mg_params, phys
    w = dict(WORKLOADS[name])
    w.update(over)
    mesh = Mesh(w["dim"], w["nlev"], w["n0"], w["box"], device=device)
    xyz = mesh.xyz()
    out = dict(w=w, mesh=mesh)
    nu_pre, nu_post = w["nu"]
    if w["kind"] == "T":
        t = MGSolT(mesh)
        t.GenBc(w["bc"])
        t.phys = phys(**w["phys"])
        t.set_xold(np.zeros(t.ntop_dof))
        t.set_source(heat_source(mesh.nel(w["nlev"] - 1)))
        out["T"] = t
        out["mg_T"] = mg_params(nu_pre=nu_pre, nu_post=nu_post, smoother=_lib.SMOOTH_GS)
    else:
        ns = MGSolNS(mesh)
        ns.GenBc(w["bc"])
        out["NS"] = ns
        out["mg_NS"] = mg_params(nu_pre=nu_pre, nu_post=nu_post, smoother=_lib.SMOOTH_VANKA, omega=vanka_omega(w),
                                 max_cycles=200)
        if w["kind"] == "NS":
            ns.phys = phys(**w["phys"])
        else:
            p_ns, p_t = bouss_phys(w)
            ns.phys = phys(**p_ns)
            t = MGSolT(mesh)
            t.GenBc(w["bc_t"])
            t.phys = phys(**p_t)
            t.set_xold(t_initial(w, xyz, t.ntop_dof))
            ns.couple(t)
            t.couple(ns)
            out["T"] = t
            out["mg_T"] = mg_params(nu_pre=nu_pre, nu_post=nu_post, smoother=_lib.SMOOTH_GS, max_cycles=200)
        ns.set_xold(ns_initial(w, xyz, mesh.ntop, ns.ntop_dof))
        ns.set_x(ns.xold())
    return out


def picard(case, steps, precision=None, on_step=None):
    """Segregated Picard iteration: every step runs MGTimeStep of each equation in map
    order (NS, then T), as MGEquationsSystem::eqnmap_timestep_loop does
    (src/MGEquationsSystem.C:422-432); each MGTimeStep assembles every level, solves and
    updates x_old."""
    stats = []
    for it in range(steps):
        row = {}
        for key in ("NS", "T"):
            if key not in case:
                continue
            s, p = case[key], case["mg_" + key]
            if precision is not None:
                p.precision = precision
            st = s.MGTimeStep(0.0, p)
            if not st.converged:
                raise RuntimeError("%s solve at Picard step %d: rel %.3e after %d cycles"
                                   % (key, it, st.rel_res, st.cycles))
            row[key] = (st.cycles, st.seconds, st.rel_res)
        stats.append(row)
        if on_step:
            on_step(it, row)
    return stats
