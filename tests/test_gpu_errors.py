"""Failure detection on the device path, injected on the host (needs a B200): every
failure comes back as a status code with a message and the context stays usable.
No test faults, traps or hangs the GPU."""
import ctypes as C

import numpy as np
import pytest

import exfemus_b200 as ex
from exfemus_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.fixture()
def heat(gpu_lib):
    m = ex.Mesh(2, 3, (4, 4), (0, 1, 0, 1))
    t = ex.MGSolT(m)
    t.GenBc(_lib.BC_HEAT_DIRICHLET)
    t.set_source(np.ones(m.nel(2)))
    return t


def _solve_rc(t, **kw):
    st = _lib.ExfSolveStats()
    p = ex.mg_params(**kw)
    return _lib.load().exf_mg_solve(t.h, C.byref(p), C.byref(st)), st


def test_solve_before_assembly_is_a_state_error(heat):
    rc, _ = _solve_rc(heat)
    assert rc == _lib.EXF_ERR_STATE


def test_nan_in_rhs_reports_divergence_and_context_survives(heat):
    heat.assemble_all()
    b = heat.rhs()
    b[7] = np.nan
    heat.set_rhs(b)
    rc, st = _solve_rc(heat, max_cycles=5)
    assert rc == _lib.EXF_ERR_DIVERGED
    assert b"diverged" in _lib.load().exf_last_error()
    heat.assemble_all()  # the same context keeps working
    rc, st = _solve_rc(heat)
    assert rc == _lib.EXF_OK and st.converged


def test_cycle_limit_reports_not_converged(heat):
    heat.assemble_all()
    heat.set_x(np.zeros(heat.ntop_dof))
    rc, st = _solve_rc(heat, max_cycles=1, eps=1e-14)
    assert rc == _lib.EXF_ERR_NOT_CONVERGED and st.cycles == 1


def test_bad_arguments(heat):
    L = _lib.load()
    n = C.c_int()
    assert L.exf_sys_ndof(heat.h, 99, C.byref(n)) == _lib.EXF_ERR_ARG
    rc, _ = _solve_rc(heat)
    assert rc == _lib.EXF_ERR_STATE  # not assembled yet
    heat.assemble_all()
    rc, _ = _solve_rc(heat, stop_test=7)
    assert rc == _lib.EXF_ERR_ARG
    rc, _ = _solve_rc(heat, nu_pre=-1)
    assert rc == _lib.EXF_ERR_ARG


def test_tile_kernels_refused_on_uploaded_meshes(gpu_lib):
    """The tile kernels need the lattice of a generated box: on an uploaded mesh they are
    refused with EXF_ERR_UNSUPPORTED and the context keeps working."""
    gm = ex.Mesh(2, 2, (2, 2), (0, 1, 0, 1))
    conn = [gm.conn(l)[0] for l in range(2)]
    neigh = [gm.conn(l)[1] for l in range(2)]
    e = np.arange(conn[1].shape[0])
    parent = [None, ((e // 4) // 2) * 2 + (e % 4) // 2]
    um = ex.Mesh.upload(2, [gm.nnodes(0), gm.nnodes(1)], gm.nvert0, gm.xyz(), conn, neigh, parent)
    ns = ex.MGSolNS(um)
    ns.GenBc(_lib.BC_CAVITY)
    ns.phys = ex.phys(inv_re=1 / 400.)
    ns.assemble_all()
    rp, col, val = ns.csr(1)  # a consistent right-hand side b = A x (enclosed flow)
    xr = np.random.default_rng(0).random(ns.ntop_dof)
    ns.set_rhs(np.array([val[rp[i]:rp[i + 1]] @ xr[col[rp[i]:rp[i + 1]]] for i in range(ns.ntop_dof)]))
    st = _lib.ExfSolveStats()
    p = ex.mg_params(smoother=_lib.SMOOTH_VANKA, vanka_kernel=_lib.VANKA_TILE)
    assert _lib.load().exf_mg_solve(ns.h, C.byref(p), C.byref(st)) == _lib.EXF_ERR_UNSUPPORTED
    st = ns.solve(ex.mg_params(smoother=_lib.SMOOTH_VANKA, nu_pre=3, nu_post=3))
    assert st.converged


def test_graph_and_eager_cycles_agree_bitwise(heat):
    heat.assemble_all()
    xs = []
    for g in (0, 1):
        heat.set_x(np.zeros(heat.ntop_dof))
        st = heat.solve(ex.mg_params(use_graph=g, precision=_lib.PREC_MIXED))
        assert st.converged
        xs.append(heat.x())
    assert np.array_equal(xs[0], xs[1])


def test_graph_cache_eviction_keeps_results(gpu_lib):
    """Six parameter sets on one system (more than its four cached solve graphs, so graphs
    are evicted and rebuilt) solved twice in turn: every solve gives the bits of the same
    parameters solved on a fresh system."""
    def make():
        m = ex.Mesh(2, 3, (4, 4), (0, 1, 0, 1))
        t = ex.MGSolT(m)
        t.GenBc(_lib.BC_HEAT_DIRICHLET)
        t.set_source(np.ones(m.nel(2)))
        t.assemble_all()
        return m, t

    sets = [dict(nu_pre=a, nu_post=a, precision=pr, reverse_colours=rv, eps=1e-11)
            for a in (1, 2, 3) for pr, rv in ((_lib.PREC_FP64, 0), (_lib.PREC_MIXED, 1))]
    fresh = []
    for kw in sets:
        m, t = make()
        t.set_x(np.zeros(t.ntop_dof))
        st = t.solve(ex.mg_params(**kw))
        fresh.append((st.cycles, t.x()))
    m, t = make()
    for _ in range(2):
        for kw, (cyc, x) in zip(sets, fresh):
            t.set_x(np.zeros(t.ntop_dof))
            st = t.solve(ex.mg_params(**kw))
            assert st.cycles == cyc and np.array_equal(t.x(), x), kw


def test_timing_probes_and_refactorisation(heat):
    """exf_time_op 4 (coarse refactorisation), 5 (FP64 FMA probe), 7 and 8 (ILU factor and
    application) run on an assembled system; a solve after them gives the same bits as
    before."""
    L = _lib.load()
    heat.assemble_all()
    p = ex.mg_params(precision=_lib.PREC_MIXED)
    heat.set_x(np.zeros(heat.ntop_dof))
    heat.solve(p)
    x0 = heat.x()
    tv = C.c_double()
    for what, lev in ((4, 0), (5, 0), (7, 2), (8, 2)):  # 7, 8: ILU factorisation and application
        _lib.check(L.exf_time_op(heat.h, what, lev, C.byref(p), C.byref(heat.phys), 2, C.byref(tv)))
        assert tv.value > 0.0
    heat.set_x(np.zeros(heat.ntop_dof))
    heat.solve(p)
    assert np.array_equal(heat.x(), x0)


def test_bounded_wait_reports_run_out(heat):
    """exf_time_op 6 runs a bounded in-kernel wait on a barrier phase that nothing
    completes: the call returns EXF_ERR_CUDA with the run-out message, the flag is cleared,
    and the context stays usable (a solve afterwards gives the bits of one before)."""
    L = _lib.load()
    heat.assemble_all()
    p = ex.mg_params(precision=_lib.PREC_MIXED)
    heat.set_x(np.zeros(heat.ntop_dof))
    heat.solve(p)
    x0 = heat.x()
    tv = C.c_double()
    rc = L.exf_time_op(heat.h, 6, 0, C.byref(p), C.byref(heat.phys), 1, C.byref(tv))
    assert rc == _lib.EXF_ERR_CUDA
    assert b"ran out" in L.exf_last_error()
    heat.set_x(np.zeros(heat.ntop_dof))
    heat.solve(p)
    assert np.array_equal(heat.x(), x0)


def test_timestep_loop_matches_host_loop(gpu_lib):
    """exf_timestep_loop (NS then T, every step) gives the bits of the same MGTimeStep
    sequence driven from here, with the same cycle counts."""
    from exfemus_b200 import workloads

    def case():
        return ex.make_case("bouss2d", nlev=3, n0=(4, 4))

    a, b = case(), case()
    rows = workloads.picard(a, 3)
    cyc, sec = ex.timestep_loop([b["NS"], b["T"]], [b["mg_NS"], b["mg_T"]], 3)
    assert [[r["NS"][0], r["T"][0]] for r in rows] == cyc.tolist()
    assert np.all(sec > 0)
    assert np.array_equal(a["NS"].x(), b["NS"].x()) and np.array_equal(a["T"].x(), b["T"].x())
    with pytest.raises(_lib.ExfError) as e:
        ex.timestep_loop([], [], 1)
    assert e.value.code == _lib.EXF_ERR_ARG
