"""The allocation-free residual entry point (needs a B200).

exf_resid_norm_static serves callers that cannot allocate device memory while they run:
it takes caller-owned device buffers and keeps its norm partial sums in a fixed device
array.  This file is collected last so a failure here cannot hide another test.  It
compares two calls in a row with the allocating entry point exf_resid and a norm taken
on the host."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _static_resid(L, sys, lev, x, b):
    import torch
    dev = torch.device("cuda", 0)
    tx = torch.tensor(x, dtype=torch.float64, device=dev)
    tb = torch.tensor(b, dtype=torch.float64, device=dev)
    tr = torch.full_like(tx, float("nan"))
    tn = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    rc = L.exf_resid_norm_static(sys.h, lev, C.c_void_p(tx.data_ptr()), C.c_void_p(tb.data_ptr()),
                                 C.c_void_p(tr.data_ptr()), C.c_void_p(tn.data_ptr()))
    return rc, tr.cpu().numpy(), float(tn.cpu().item())


@pytest.mark.parametrize("kind", ["heat", "heat3d", "ns2d", "ns3d"])
def test_static_resid_matches_allocating_entry_point(kind):
    import exfemus_b200 as ex
    from exfemus_b200 import _lib
    L = _lib.load()
    if kind == "heat":
        m = ex.Mesh(2, 3, (4, 4), (0, 1, 0, 1))
        s = ex.MGSolT(m)
        s.GenBc(_lib.BC_HEAT_DIRICHLET)
        s.set_source(np.ones(m.nel(2)))
    elif kind == "heat3d":
        m = ex.Mesh(3, 2, (2, 2, 2), (0, 1, 0, 1, 0, 1))
        s = ex.MGSolT(m)
        s.GenBc(_lib.BC_HEAT_DIRICHLET)
        s.set_source(np.ones(m.nel(1)))
    elif kind == "ns2d":
        m = ex.Mesh(2, 3, (4, 4), (0, 1, 0, 1))
        s = ex.MGSolNS(m)
        s.GenBc(_lib.BC_CAVITY)
        s.phys = ex.phys(inv_re=1 / 400.)
    else:
        m = ex.Mesh(3, 2, (4, 2, 2), (0, 4, 0, 1, 0, 1))
        s = ex.MGSolNS(m)
        s.GenBc(_lib.BC_CHANNEL)
        s.phys = ex.phys(inv_re=0.01)
    rng = np.random.default_rng(21)
    s.set_xold(0.1 * rng.standard_normal(s.ntop_dof))
    s.assemble_all()
    for lev in range(m.nlev):
        for call in range(2):  # two calls in a row share the static array
            x = rng.standard_normal(s.ndof(lev))
            b = rng.standard_normal(s.ndof(lev))
            rc, r, n2 = _static_resid(L, s, lev, x, b)
            assert rc == _lib.EXF_OK, L.exf_last_error()
            r_ref = s.resid(lev, x, b)
            assert np.array_equal(r, r_ref)
            assert abs(n2 - float(r_ref @ r_ref)) <= 1e-12 * float(r_ref @ r_ref)


def test_static_resid_rejects_bad_calls():
    import exfemus_b200 as ex
    from exfemus_b200 import _lib
    L = _lib.load()
    m = ex.Mesh(2, 2, (2, 2), (0, 1, 0, 1))
    s = ex.MGSolT(m)
    s.GenBc(_lib.BC_HEAT_DIRICHLET)
    null = C.c_void_p(0)
    assert L.exf_resid_norm_static(s.h, 0, null, null, null, null) == _lib.EXF_ERR_ARG
    x = np.zeros(s.ndof(0))
    rc, _, _ = _static_resid(L, s, 0, x, x)
    assert rc == _lib.EXF_ERR_STATE  # not assembled yet


def test_static_resid_rejects_levels_above_the_array():
    """A level needing more partial sums than the fixed array holds is refused with
    EXF_ERR_ARG before any launch: 1025 x 1025 Q2 nodes at 8 lanes per row need 32,833
    blocks of 256 threads, one more than 32,768 would allow."""
    import exfemus_b200 as ex
    from exfemus_b200 import _lib
    L = _lib.load()
    m = ex.Mesh(2, 1, (512, 512), (0, 1, 0, 1))
    s = ex.MGSolT(m)
    s.GenBc(_lib.BC_HEAT_DIRICHLET)
    s.assemble_all()
    n = s.ndof(0)
    assert n == 1025 * 1025 and (n * 8 + 255) // 256 > 32768
    x = np.zeros(n)
    rc, _, _ = _static_resid(L, s, 0, x, x)
    assert rc == _lib.EXF_ERR_ARG
    assert b"static array holds 32768" in L.exf_last_error()
