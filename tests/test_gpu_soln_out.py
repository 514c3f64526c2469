"""exf_print_soln on solved systems (needs a B200): the written datasets are the systems'
top-level x through their node_dof maps, scaled per variable, with the linear pressure
interpolated to every node; read back through the XDMF file."""
import os

import numpy as np
import pytest

import exfemus_b200 as ex
from exfemus_b200 import workloads

pytestmark = pytest.mark.gpu


def node_values(s, v):
    """Variable v of system s at every top-level node (NaN where it has no DOF)."""
    nd = s.node_dof(s.nlev - 1).reshape(s.nvars, -1)[v]
    x = s.x()
    out = np.full(nd.size, np.nan)
    out[nd >= 0] = x[nd[nd >= 0]]
    return out


@pytest.mark.parametrize("name,n0,nlev", [("bouss2d", (4, 4), 3), ("channel3d", (4, 2, 2), 2)])
def test_print_soln_writes_the_solution(gpu_lib, tmp_path, name, n0, nlev):
    case = ex.make_case(name, nlev=nlev, n0=n0)
    workloads.picard(case, 2)
    systems = [case[k] for k in ("NS", "T") if k in case]
    m = case["mesh"]
    dim = m.dim
    nvar = sum(s.nvars for s in systems)
    ref = 1.0 + 0.5 * np.arange(nvar)
    path = ex.print_soln(systems, 3, 0.3, out_dir=str(tmp_path), refvalue=ref)
    d = ex.read_xdmf(path)
    names = ["u", "v", "w"][:dim] + ["p"] + (["T"] if "T" in case else [])
    assert list(d["fields"]) == names
    assert d["time"] == 0.3
    conn = m.conn(m.nlev - 1)[0]
    assert d["cells"].shape == (conn.shape[0] * 2 ** dim, 2 ** dim)
    assert np.array_equal(d["xyz"][:dim], m.xyz())
    var = 0
    for s in systems:
        for v in range(s.nvars):
            got = d["fields"][names[var]]
            want = node_values(s, v) * ref[var]
            if s.kind == 1 and v == dim:  # pressure: vertices as solved, the rest interpolated
                vx = ~np.isnan(want)
                assert np.array_equal(got[vx], want[vx])
                assert np.all(np.isfinite(got))
                # on the box every edge node is the average of its edge's vertices
                e = conn[0]
                mid01 = e[4] if dim == 2 else e[8]  # the node on the edge of vertices 0 and 1
                assert got[mid01] == 0.5 * got[e[0]] + 0.5 * got[e[1]]
            else:
                assert np.array_equal(got, want)
            var += 1


@pytest.mark.parametrize("name,n0,nlev", [("bouss2d", (4, 4), 3), ("channel3d", (4, 2, 2), 2)])
def test_print_case_writes_the_initial_state_and_flags(gpu_lib, tmp_path, name, n0, nlev):
    """print_case: x_old and the flags bc[1] (<name>bd) and bc[0] (<name>vl) of every
    variable; a linear variable's flags reach the other nodes by the element's linear map,
    truncated to integers."""
    case = ex.make_case(name, nlev=nlev, n0=n0)
    systems = [case[k] for k in ("NS", "T") if k in case]
    m = case["mesh"]
    dim = m.dim
    rng = np.random.default_rng(5)
    for s in systems:
        s.set_xold(rng.standard_normal(s.ntop_dof))
    path = ex.print_case(systems, 0, out_dir=str(tmp_path))
    assert os.path.basename(path) == "case.0000.xmf"
    d = ex.read_xdmf(path)
    assert d["time"] is None
    names = ["u", "v", "w"][:dim] + ["p"] + (["T"] if "T" in case else [])
    assert list(d["fields"]) == [n + t for n in names for t in ("", "bd", "vl")]
    conn = m.conn(m.nlev - 1)[0]
    var = 0
    for s in systems:
        bc0, bc1 = s.bc()
        nd = s.node_dof(s.nlev - 1).reshape(s.nvars, -1)
        xo = s.xold()
        for v in range(s.nvars):
            n = names[var]
            has = nd[v] >= 0
            assert np.array_equal(d["fields"][n][has], xo[nd[v][has]])
            for tag, flag in (("bd", bc1), ("vl", bc0)):
                got = d["fields"][n + tag]
                assert np.array_equal(got[has], flag[nd[v][has]].astype(float))
                if not has.all():  # the linear pressure: flags from the vertices, truncated
                    e = conn[0]
                    mid = e[4] if dim == 2 else e[8]
                    assert got[mid] == float(int(0.5 * got[e[0]] + 0.5 * got[e[1]]))
                    assert np.all(got == np.trunc(got))
            var += 1
