"""The time / Picard loop inside the library against the oracle (needs a B200).

exf_timestep_loop runs MGEquationsSystem::eqnmap_timestep_loop (src/MGEquationsSystem.C:
422-432): per step, every equation's MGTimeStep in map order (assemble every level,
solve, x_old = x), the coupled systems reading each other's x_old.  On a 16x16 Boussinesq
cavity (3 levels) the oracle runs the same segregated steps (NS with the temperature of
the previous step, then T on the new velocity); per step the cycle counts agree and the
final fields are within 1e-9."""
import numpy as np
import pytest

import exfemus_b200 as ex
from exfemus_b200 import _lib, workloads

from conftest import or_mg, or_phys, rel

pytestmark = pytest.mark.gpu


def test_timestep_loop_matches_oracle_segregated_picard(oracle_mod, gpu_lib):
    over = dict(nlev=3, n0=(4, 4))
    case = workloads.make_case("bouss2d", **over)
    w, mesh, ns, t = case["w"], case["mesh"], case["NS"], case["T"]
    top = w["nlev"] - 1
    nsteps = 3
    pn = ex.mg_params(eps=1e-10, max_cycles=200, nu_pre=3, nu_post=3, smoother=_lib.SMOOTH_VANKA,
                      omega=workloads.VANKA_OMEGA)
    pt = ex.mg_params(eps=1e-10, max_cycles=200, nu_pre=3, nu_post=3, smoother=_lib.SMOOTH_GS)
    cyc, _ = ex.timestep_loop([ns, t], [pn, pt], nsteps)
    xg_ns, xg_t = ns.x(), t.x()

    om = oracle_mod.OrMesh(w["dim"], w["nlev"], w["n0"], w["box"])
    ons = oracle_mod.OrSys(om, 1)
    ons.bc_preset(w["bc"])
    ot = oracle_mod.OrSys(om, 0)
    ot.bc_preset(w["bc_t"])
    p_ns, p_t = workloads.bouss_phys(w)
    xyz = om.xyz()
    x_ns = workloads.ns_initial(w, xyz, om.ntop, ons.ndof(top))
    x_t_old = workloads.t_initial(w, xyz, ot.ndof(top))
    x_t = np.zeros(ot.ndof(top))  # the T system starts from x = 0, x_old = the initial field
    on = or_mg(oracle_mod, eps=1e-10, max_cycles=200, nu_pre=3, nu_post=3, smoother=1, omega=workloads.VANKA_OMEGA)
    ogt = or_mg(oracle_mod, eps=1e-10, max_cycles=200, nu_pre=3, nu_post=3, smoother=0)
    for step in range(nsteps):
        ons.assemble_all(or_phys(oracle_mod, **p_ns), xold=x_ns, temp=x_t_old)
        x_ns, st = ons.mg_solve(on, x0=x_ns)
        assert st.converged and st.cycles == cyc[step, 0], (step, st.cycles, cyc[step, 0])
        ot.assemble_all(or_phys(oracle_mod, **p_t), xold=x_t_old, vel=x_ns)
        x_t, st = ot.mg_solve(ogt, x0=x_t)
        assert st.converged and st.cycles == cyc[step, 1], (step, st.cycles, cyc[step, 1])
        x_t_old = x_t
    assert rel(xg_ns, x_ns) < 1e-9
    assert rel(xg_t, x_t) < 1e-9


def test_unconverged_solves_do_not_stop_the_loop(gpu_lib):
    """MGSolve ending at its cycle limit does not stop MGTimeStep: every step runs (one
    cycle each here), x_old follows x, and the loop reports EXF_ERR_NOT_CONVERGED at the
    end (strict) or returns the cycle counts (strict=False)."""
    over = dict(nlev=3, n0=(4, 4))
    nsteps = 3
    for strict in (True, False):
        case = workloads.make_case("bouss2d", **over)
        ns, t = case["NS"], case["T"]
        p = [ex.mg_params(eps=1e-30, max_cycles=1, smoother=s, omega=workloads.VANKA_OMEGA)
             for s in (_lib.SMOOTH_VANKA, _lib.SMOOTH_GS)]
        if strict:
            with pytest.raises(_lib.ExfError) as e:
                ex.timestep_loop([ns, t], p, nsteps)
            assert e.value.code == _lib.EXF_ERR_NOT_CONVERGED
        else:
            cyc, _ = ex.timestep_loop([ns, t], p, nsteps, strict=False)
            assert cyc.tolist() == [[1, 1]] * nsteps
        assert np.array_equal(t.xold(), t.x()) and np.array_equal(ns.xold(), ns.x())
