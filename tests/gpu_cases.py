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
    # the channel with Neumann / Robin outlet sides (MGSolverNS.C:604-681): velocity flags
    # normal + rhs, tangential, tangential + rhs, and the pressure traction on
    "outlet3d": (3, 2, (4, 2, 2), (0, 4, 0, 1, 0, 1), 1, _lib.BC_CHANNEL, dict(inv_re=0.01, traction=1.0)),
}
# natural-side flags per velocity component on the outlet (nodes off the walls)
OUTLET_FLAGS = {"outlet3d": (5, 2, 6)}


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
    if name in OUTLET_FLAGS:
        b0, b1 = osys.bc()
        N = om.ntop
        outlet = np.abs(xyz[0] - box[1]) < 1e-12
        for a, f in enumerate(OUTLET_FLAGS[name]):
            sel = outlet & (b0[a * N:(a + 1) * N] != 0)
            b1[a * N:(a + 1) * N][sel] = f
        osys.set_bc(b0, b1)
        gs.set_bc(b0, b1)
    xold = initial(name, xyz, om.ntop, osys.ndof(top), preset)
    if kind == 1:
        # a non-trivial advecting field: the Dirichlet data plus a smooth interior field
        N = om.ntop
        b0, _ = osys.bc()
        for a in range(dim):
            free = b0[a * N:(a + 1) * N] != 0
            xold[a * N:(a + 1) * N][free] += 0.3 * np.sin(3 * xyz[0][free] + a) * np.cos(2 * xyz[1][free])
        if name in OUTLET_FLAGS:  # a pressure for the traction term
            NL = om.nnodes(top - 1)
            xold[dim * N:] = 0.5 - 0.1 * xyz[0][:NL] + 0.05 * xyz[1][:NL]
    qe = None
    if kind == 0:
        qe = workloads.heat_source(om.nel(top), seed=0)
        gs.set_source(qe)
    gs.set_xold(xold)
    return dict(gm=gm, gs=gs, om=om, os=osys, xold=xold, qe=qe, oph=or_phys(oracle, **pk), nlev=nlev, kind=kind,
                dim=dim)
