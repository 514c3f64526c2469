"""Independent systems driven from two host threads (needs a B200).

The C ABI promises that independent systems are thread-safe (one CUDA stream per system;
the mesh owns its FE tables; per-device caches are resolved under a lock).  Each thread
builds its own mesh and system, assembles every level and solves; ctypes releases the
interpreter lock during the library calls, so the two threads' calls interleave.  Every
result must equal, bit for bit, the same work done by one thread alone.
"""
import threading

import numpy as np
import pytest

import exfemus_b200 as ex
from exfemus_b200 import _lib, workloads

pytestmark = pytest.mark.gpu


def _heat_run():
    m = ex.Mesh(2, 3, (4, 4), (0, 1, 0, 1))
    t = ex.MGSolT(m)
    t.GenBc(_lib.BC_HEAT_DIRICHLET)
    t.set_source(workloads.heat_source(m.nel(2), seed=3))
    t.set_xold(np.zeros(t.ntop_dof))
    out = []
    for _ in range(3):
        t.assemble_all()
        t.set_x(np.zeros(t.ntop_dof))
        st = t.solve(ex.mg_params(eps=1e-11))
        out.append((st.cycles, t.matrix(2), t.x()))
    return out


def _channel_run():
    m = ex.Mesh(3, 2, (4, 2, 2), (0, 4, 0, 1, 0, 1))
    ns = ex.MGSolNS(m)
    ns.GenBc(_lib.BC_CHANNEL)
    ns.phys = ex.phys(inv_re=0.01)
    w = dict(box=(0, 4, 0, 1, 0, 1), bc=_lib.BC_CHANNEL)
    x0 = workloads.ns_initial(w, m.xyz(), m.ntop, ns.ntop_dof)
    ns.set_xold(x0)
    out = []
    for prec in (_lib.PREC_FP64, _lib.PREC_MIXED):
        ns.assemble_all()
        ns.set_x(x0)
        st = ns.solve(ex.mg_params(eps=1e-10, nu_pre=3, nu_post=3, smoother=_lib.SMOOTH_VANKA, precision=prec))
        out.append((st.cycles, ns.matrix(1), ns.x()))
    return out


def _same(a, b):
    assert len(a) == len(b)
    for (ca, ma, xa), (cb, mb, xb) in zip(a, b):
        assert ca == cb
        assert np.array_equal(ma, mb)
        assert np.array_equal(xa, xb)


def test_two_threads_match_single_thread_runs(gpu_lib):
    ref_heat, ref_ch = _heat_run(), _channel_run()
    res, errs = {}, []

    def work(name, fn):
        try:
            res[name] = fn()
        except Exception as e:  # reported below, in the main thread
            errs.append((name, e))

    for _ in range(2):
        th = [threading.Thread(target=work, args=("heat", _heat_run)),
              threading.Thread(target=work, args=("channel", _channel_run))]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert not errs, errs
        _same(res["heat"], ref_heat)
        _same(res["channel"], ref_ch)
