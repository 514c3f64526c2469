"""The GMRES + ILU level solver (needs a B200) against the reference's own LASPACK code
(GMRESIter, ILUFactor, ILUPrecond compiled from contrib/laspack into oracle/_ref):
ILUPrecond bitwise on every level of 2D and 3D heat systems, single smoother calls to
rounding, one V-cycle against the same cycle composed here from the unit operations and
LASPACK's solver, and a full solve against the oracle's solution."""
import numpy as np
import pytest

import exfemus_b200 as ex
from exfemus_b200 import _lib

import gpu_cases
from conftest import or_mg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def laspack(oracle_mod):
    if not oracle_mod.laspack_available():
        pytest.skip("oracle/_ref/liblaspack_ref.so not built")
    return oracle_mod.Laspack()


def assembled(name, oracle_mod):
    c = gpu_cases.make(name, oracle_mod)
    c["gs"].assemble_all()
    return c


def gmres_params(**kw):
    kw.setdefault("smoother", _lib.SMOOTH_GMRES_ILU)
    return ex.mg_params(**kw)


@pytest.mark.parametrize("name", ["heat2d", "heat3d"])
def test_ilu_apply_is_the_reference_bitwise(gpu_lib, oracle_mod, laspack, name):
    c = assembled(name, oracle_mod)
    s = c["gs"]
    for lev in range(c["nlev"]):
        rp, col, val = s.csr(lev)
        rp, col = rp.astype(np.int32), col.astype(np.int32)
        v = np.random.default_rng(lev).standard_normal(s.ndof(lev))
        assert np.array_equal(s.ilu_apply(lev, v), laspack.ilu_apply(rp, col, val, v)), lev


@pytest.mark.parametrize("name", ["heat2d", "heat3d"])
@pytest.mark.parametrize("m", [1, 2, 4, 33])
def test_gmres_smoother_call_matches_laspack(gpu_lib, oracle_mod, laspack, name, m):
    """exf_smooth with GMRES + ILU and m iterations = LASPACK GMRESIter(A, x, b, m,
    ILUPrecond) with restart 30 (m = 33: one restart) from the same x and b."""
    c = assembled(name, oracle_mod)
    s = c["gs"]
    rng = np.random.default_rng(m)
    p = gmres_params(eps=1e-14)
    for lev in range(c["nlev"]):
        rp, col, val = s.csr(lev)
        rp, col = rp.astype(np.int32), col.astype(np.int32)
        n = s.ndof(lev)
        x0, b = rng.standard_normal(n), rng.standard_normal(n)
        xg = s.smooth(lev, p, m, x0, b)
        xl, it, _ = laspack.gmres(rp, col, val, b, x0=x0, tol=1e-14, maxit=m, restart=30, ilu=True)
        assert it == m or (m > 30 and it == 30)  # a restart test may end it after 30
        assert np.linalg.norm(xg - xl) <= 1e-11 * np.linalg.norm(xl), (lev, m)


def test_converged_call_leaves_x(gpu_lib, oracle_mod, laspack):
    """A residual already below eps ||b|| ends GMRESIter before its first iteration."""
    c = assembled("heat2d", oracle_mod)
    s = c["gs"]
    lev = c["nlev"] - 1
    x = np.random.default_rng(3).standard_normal(s.ndof(lev))
    b = s.spmv(lev, x)
    xg = s.smooth(lev, gmres_params(eps=1e-6), 4, x, b)
    assert np.array_equal(xg, x)


def mg_step_here(s, lev, x, b, p, laspack):
    """MGStep (src/MGSolverBase.C:212-289) from the library's unit operations with
    LASPACK's GMRES + ILU as the level solver (corrections added with corr_damp)."""
    top = s.nlev - 1
    rp, col, val = s.csr(lev)
    rp, col = rp.astype(np.int32), col.astype(np.int32)
    if lev == 0:
        if p.coarse_iters > 0:  # _solver[0]->solve(A, x, b, Eps1, 60) from x = 0
            return laspack.gmres(rp, col, val, b, x0=x, tol=p.eps, maxit=p.coarse_iters, restart=30, ilu=True)[0]
        return s.coarse_solve(b)
    mul = 2 if (p.double_below_top and lev < top) else 1
    x, _, _ = laspack.gmres(rp, col, val, b, x0=x, tol=p.eps, maxit=p.nu_pre * mul, restart=30, ilu=True)
    r = s.resid(lev, x, b)
    bc = s.restrict(lev - 1, r)
    xc = mg_step_here(s, lev - 1, np.zeros(s.ndof(lev - 1)), bc, p, laspack)
    x = x + p.corr_damp * s.prolong(lev, xc)
    x, _, _ = laspack.gmres(rp, col, val, b, x0=x, tol=p.eps, maxit=p.nu_post * mul, restart=30, ilu=True)
    return x


@pytest.mark.parametrize("name", ["heat2d", "heat3d"])
def test_one_vcycle_matches_the_composed_reference_cycle(gpu_lib, oracle_mod, laspack, name):
    c = assembled(name, oracle_mod)
    s = c["gs"]
    top = c["nlev"] - 1
    b = s.rhs()
    p = gmres_params(max_cycles=1, eps=1e-30, use_graph=0)
    s.set_x(np.zeros(s.ntop_dof))
    st = s.solve(p)  # one cycle, which cannot reach 1e-30
    assert st.cycles == 1 and not st.converged
    xg = s.x()
    xh = mg_step_here(s, top, np.zeros(s.ntop_dof), b, p, laspack)
    assert np.linalg.norm(xg - xh) <= 1e-11 * np.linalg.norm(xh)


@pytest.mark.parametrize("name", ["heat2d", "heat3d"])
def test_one_vcycle_with_the_coarse_level_solver(gpu_lib, oracle_mod, laspack, name):
    """coarse_iters = 60: level 0 runs the same GMRES + ILU for 60 iterations (or to the
    accuracy test), as MGStep does, instead of the direct solve."""
    c = assembled(name, oracle_mod)
    s = c["gs"]
    b = s.rhs()
    p = gmres_params(max_cycles=1, eps=1e-10, use_graph=0, coarse_iters=60)
    s.set_x(np.zeros(s.ntop_dof))
    st = s.solve(p)
    assert st.cycles == 1
    xh = mg_step_here(s, c["nlev"] - 1, np.zeros(s.ntop_dof), b, p, laspack)
    assert np.linalg.norm(s.x() - xh) <= 1e-9 * np.linalg.norm(xh)
    s.set_x(np.zeros(s.ntop_dof))
    st = s.solve(gmres_params(eps=1e-10, coarse_iters=60))
    assert st.converged


@pytest.mark.parametrize("name", ["heat2d", "heat3d"])
def test_solve_reaches_the_oracle_solution(gpu_lib, oracle_mod, name):
    c = assembled(name, oracle_mod)
    s, o = c["gs"], c["os"]
    o.assemble_all(c["oph"], xold=c["xold"], qe=c["qe"])
    xo, sto = o.mg_solve(or_mg(oracle_mod, eps=1e-13, max_cycles=200))
    assert sto.converged
    s.set_x(np.zeros(s.ntop_dof))
    st = s.solve(gmres_params(eps=1e-11, max_cycles=100))
    assert st.converged
    assert np.linalg.norm(s.x() - xo) <= 1e-9 * np.linalg.norm(xo)


def test_graph_and_eager_cycles_agree_bitwise(gpu_lib, oracle_mod):
    xs = []
    for g in (0, 1):
        c = assembled("heat2d", oracle_mod)
        s = c["gs"]
        s.set_x(np.zeros(s.ntop_dof))
        st = s.solve(gmres_params(use_graph=g, eps=1e-11))
        assert st.converged
        xs.append(s.x())
    assert np.array_equal(xs[0], xs[1])


def test_refused_for_navier_stokes_and_mixed_precision(gpu_lib, oracle_mod):
    c = gpu_cases.make("cavity2d", oracle_mod)
    ns = c["gs"]
    ns.assemble_all()
    with pytest.raises(_lib.ExfError) as e:
        ns.solve(gmres_params())
    assert e.value.code == _lib.EXF_ERR_UNSUPPORTED
    t = assembled("heat2d", oracle_mod)["gs"]
    with pytest.raises(_lib.ExfError) as e:
        t.solve(gmres_params(precision=_lib.PREC_MIXED))
    assert e.value.code == _lib.EXF_ERR_UNSUPPORTED
    st = t.solve(gmres_params())  # the context keeps working
    assert st.converged
