import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")
    config.addinivalue_line("markers", "slow: a workload at its full size (minutes; still part of -m gpu)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library; a GPU test fails (never falls back) if it is missing."""
    import exfemus_b200
    from exfemus_b200 import _lib
    assert os.path.exists(_lib.LIB_PATH), "libexfemus_b200.so is not built"
    return exfemus_b200


def or_phys(oracle, **kw):
    p = oracle.OrPhys()
    p.inv_re, p.inv_prdl, p.rho, p.rhocp = 1.0, 1.0, 1.0, 1.0
    p.inv_dt, p.penalty, p.upwind_ns, p.upwind_t = 0.0, 1.0, 0.1, 1.0
    p.ifr, p.buoy = 0.0, 0.0
    for k, v in kw.items():
        if k == "dirg":
            for i, x in enumerate(v):
                p.dirg[i] = x
        else:
            setattr(p, k, v)
    return p


def or_mg(oracle, **kw):
    p = oracle.OrMgParams()
    p.eps, p.max_cycles, p.gamma, p.nu_pre, p.nu_post = 1e-10, 100, 1, 2, 2
    p.double_below_top, p.smoother, p.omega, p.corr_damp = 1, 0, 0.4, 0.95
    p.cond_corr, p.reverse_colours = 0, 0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (d if d > 0 else 1.0)
