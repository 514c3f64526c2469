"""Matched GPU / oracle cases at test sizes (same mesh, flags, fields)."""
import numpy as np

import exfemus_b200 as ex
from exfemus_b200 import _lib, workloads

from conftest import or_phys

CASES = {
    # name: dim, nlev, n0, box, kind, preset, phys kwargs
    "heat2d": (2, 3, (4, 4), (0, 1, 0, 1), 0, _lib.BC_HEAT_DIRICHLET, dict()),
    "cavity2d": (2, 3, (4, 4), (0, 1, 0, 1), 1, _lib.BC_CAVITY, dict(inv_re=1 / 400.)),
    "channel3d": (3, 2, (4, 2, 2), (0, 4, 0, 1, 0, 1), 1, _lib.BC_CHANNEL, dict(inv_re=0.01)),
    "heat3d": (3, 2, (2, 2, 2), (0, 1, 0, 1, 0, 1), 0, _lib.BC_HEAT_DIRICHLET, dict()),
}


def initial(name, mesh_xyz, ntop, ndof, preset):
    w = dict(box=CASES[name][3], bc=preset)
    if CASES[name][4] == 1:
        return workloads.ns_initial(w, mesh_xyz, ntop, ndof)
    return np.zeros(ndof)


def make(name, oracle):
    dim, nlev, n0, box, kind, preset, pk = CASES[name]
    gm = ex.Mesh(dim, nlev, n0, box)
    gs = (ex.MGSolNS if kind == 1 else ex.MGSolT)(gm)
    gs.GenBc(preset)
    gs.phys = ex.phys(**pk)
    om = oracle.OrMesh(dim, nlev, n0, box)
    osys = oracle.OrSys(om, kind)
    osys.bc_preset(preset)
    xyz = om.xyz()
    top = nlev - 1
    xold = initial(name, xyz, om.ntop, osys.ndof(top), preset)
    if kind == 1:
        # a non-trivial advecting field: the Dirichlet data plus a smooth interior field
        N = om.ntop
        b0, _ = osys.bc()
        for a in range(dim):
            free = b0[a * N:(a + 1) * N] != 0
            xold[a * N:(a + 1) * N][free] += 0.3 * np.sin(3 * xyz[0][free] + a) * np.cos(2 * xyz[1][free])
    qe = None
    if kind == 0:
        qe = workloads.heat_source(om.nel(top), seed=0)
        gs.set_source(qe)
    gs.set_xold(xold)
    return dict(gm=gm, gs=gs, om=om, os=osys, xold=xold, qe=qe, oph=or_phys(oracle, **pk), nlev=nlev, kind=kind,
                dim=dim)
