"""Host-side mirror of exFEMuS's MGSolBase / MGSolDA interface over the C ABI.

Method names follow the reference (include/MGSolverBase.h:118-361): MGDofBcOp,
GenBc, GenMatRhs(time, Level, mode), MGSolve(Eps, MaxIter, Gamma, Nc_pre, Nc_coarse,
Nc_post), MGStep, MGTimeStep(time).  Errors raise ExfError with the library message
(the reference aborts; the C ABI returns a status).  Everything runs on the GPU; there
is no CPU path.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import (ExfMeshDesc, ExfMgParams, ExfPhys, ExfSolveStats, check, dptr, iptr, load)


def phys(**kw):
    """Physics parameters with the reference defaults (UP_WIND_NS=0.1, UP_WIND_T=1)."""
    p = ExfPhys()
    p.inv_re, p.inv_prdl, p.rho, p.rhocp = 1.0, 1.0, 1.0, 1.0
    p.inv_dt, p.penalty = 0.0, 1.0
    p.upwind_ns, p.upwind_t = 0.1, 1.0
    p.ifr, p.buoy = 0.0, 0.0
    for k, v in kw.items():
        if k == "dirg":
            for i, x in enumerate(v):
                p.dirg[i] = x
        else:
            setattr(p, k, v)
    return p


def mg_params(**kw):
    """Multigrid parameters (MGSolve defaults of the reference where they apply)."""
    p = ExfMgParams()
    p.eps, p.max_cycles, p.gamma = 1e-10, 100, 1
    p.nu_pre, p.nu_post, p.double_below_top = 2, 2, 1
    p.smoother, p.omega, p.corr_damp = _lib.SMOOTH_GS, 0.4, 0.95
    p.cond_corr, p.reverse_colours, p.precision, p.use_graph = 0, 0, _lib.PREC_FP64, 1
    p.vanka_kernel = _lib.VANKA_AUTO
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class Mesh:
    """Structured multilevel quad9/hex27 hierarchy (MGMesh analogue)."""

    def __init__(self, dim, nlev, n0, box, device=0):
        L = load()
        d = ExfMeshDesc()
        d.dim, d.nlev, d.device = dim, nlev, device
        n0 = list(n0) + [1] * (3 - len(n0))
        box = list(box) + [0.0] * (6 - len(box))
        for i in range(3):
            d.n0[i] = n0[i]
        for i in range(6):
            d.box[i] = box[i]
        h = C.c_void_p()
        check(L.exf_mesh_create(C.byref(d), C.byref(h)))
        self.h, self.L, self.dim, self.nlev = h, L, dim, nlev

    @classmethod
    def upload(cls, dim, nnodes, nvert0, xyz, conn, neigh, parent=None, device=0):
        """A hierarchy from host arrays, as MGMesh::read_c holds it (src/MGMesh.C:493-908):
        nnodes[L] Q2 nodes per level (level-nested numbering), nvert0 vertices of level 0,
        xyz [dim][ntop], conn[L] [nel][9|27] top node numbers, neigh[L] [nel][4|6]
        level-local neighbours (-1 boundary), parent[L] (L >= 1) parent elements or None."""
        L = load()
        nlev = len(nnodes)
        d = _lib.ExfMeshData()
        keep = [np.ascontiguousarray(nnodes, np.int32), np.ascontiguousarray(xyz, np.float64).ravel(),
                np.ascontiguousarray([len(c) for c in conn], np.int32),
                np.ascontiguousarray(np.concatenate([np.asarray(c, np.int32).ravel() for c in conn])),
                np.ascontiguousarray(np.concatenate([np.asarray(c, np.int32).ravel() for c in neigh]))]
        if parent is not None:
            keep.append(np.ascontiguousarray(np.concatenate([np.asarray(p, np.int32).ravel() for p in parent[1:]])))
        d.dim, d.nlev, d.device, d.nvert0 = dim, nlev, device, nvert0
        d.nnodes, d.xyz, d.nel = keep[0].ctypes.data, keep[1].ctypes.data, keep[2].ctypes.data
        d.conn, d.neigh = keep[3].ctypes.data, keep[4].ctypes.data
        d.parent = keep[5].ctypes.data if parent is not None else None
        h = C.c_void_p()
        check(L.exf_mesh_upload(C.byref(d), C.byref(h)))
        self = cls.__new__(cls)
        self.h, self.L, self.dim, self.nlev = h, L, dim, nlev
        return self

    @staticmethod
    def _coarse(dim, nlev, nvert0, xyz0, conn0, device):
        xyz0 = np.ascontiguousarray(xyz0, np.float64)
        conn0 = np.ascontiguousarray(conn0, np.int32)
        c = _lib.ExfMeshCoarse()
        c.dim, c.nlev, c.device, c.nvert0 = dim, nlev, device, nvert0
        c.nnode0, c.nel0 = xyz0.shape[1], conn0.shape[0]
        c.xyz0, c.conn0 = xyz0.ctypes.data, conn0.ctypes.data
        return c, (xyz0, conn0)

    @classmethod
    def refine(cls, dim, nlev, nvert0, xyz0, conn0, device=0):
        """A hierarchy by uniform refinement of a coarse quad9 / hex27 mesh (gencase's role):
        xyz0 [dim][nnode0] with the nvert0 vertices first, conn0 [nel0][9|27] libMesh order."""
        L = load()
        c, keep = cls._coarse(dim, nlev, nvert0, xyz0, conn0, device)
        h = C.c_void_p()
        check(L.exf_mesh_refine(C.byref(c), C.byref(h)))
        self = cls.__new__(cls)
        self.h, self.L, self.dim, self.nlev = h, L, dim, nlev
        return self

    @staticmethod
    def refine_arrays(dim, nlev, nvert0, xyz0, conn0):
        """The refined hierarchy as host arrays (no device work): dict of nnodes, nel, xyz
        [dim][ntop], conn, neigh and parent per level."""
        L = load()
        c, keep = Mesh._coarse(dim, nlev, nvert0, xyz0, conn0, 0)
        d = _lib.ExfMeshData()
        check(L.exf_mesh_refine_arrays(C.byref(c), C.byref(d)))
        try:
            nnodes = np.ctypeslib.as_array(C.cast(d.nnodes, C.POINTER(C.c_int)), (nlev,)).copy()
            nel = np.ctypeslib.as_array(C.cast(d.nel, C.POINTER(C.c_int)), (nlev,)).copy()
            ntop = int(nnodes[-1])
            xyz = np.ctypeslib.as_array(C.cast(d.xyz, C.POINTER(C.c_double)), (dim, ntop)).copy()
            nen, ns = (9, 4) if dim == 2 else (27, 6)
            tot = int(nel.sum())
            conn = np.ctypeslib.as_array(C.cast(d.conn, C.POINTER(C.c_int)), (tot, nen)).copy()
            neigh = np.ctypeslib.as_array(C.cast(d.neigh, C.POINTER(C.c_int)), (tot, ns)).copy()
            parent = (np.ctypeslib.as_array(C.cast(d.parent, C.POINTER(C.c_int)), (tot - int(nel[0]),)).copy()
                      if nlev > 1 else np.zeros(0, np.int32))
        finally:
            L.exf_mesh_data_free(C.byref(d))
        off = np.concatenate([[0], np.cumsum(nel)])
        return dict(nnodes=nnodes, nel=nel, nvert0=nvert0, xyz=xyz,
                    conn=[conn[off[l]:off[l + 1]] for l in range(nlev)],
                    neigh=[neigh[off[l]:off[l + 1]] for l in range(nlev)],
                    parent=[None] + [parent[off[l] - off[1]:off[l + 1] - off[1]] for l in range(1, nlev)])

    def wall_dist(self, wall_node):
        """MGMesh::B_dist: per element of every level (level 0's first) the distance from
        its centre to the nearest wall-side centre of its level; wall_node [ntop] marks
        the wall nodes."""
        w = np.ascontiguousarray(wall_node, np.int32)
        out = np.zeros(sum(self.nel(l) for l in range(self.nlev)))
        check(self.L.exf_mesh_wall_dist(self.h, iptr(w), dptr(out)))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.L.exf_mesh_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def info(self, lev):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(self.L.exf_mesh_info(self.h, lev, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def nnodes(self, lev):
        return self.info(lev)[0]

    def nel(self, lev):
        return self.info(lev)[1]

    @property
    def nvert0(self):
        return self.info(0)[2]

    @property
    def ntop(self):
        return self.nnodes(self.nlev - 1)

    @property
    def nen(self):
        return 9 if self.dim == 2 else 27

    def xyz(self):
        a = np.zeros(self.dim * self.ntop)
        check(self.L.exf_mesh_get_xyz(self.h, dptr(a)))
        return a.reshape(self.dim, self.ntop)

    def conn(self, lev):
        ne = self.nel(lev)
        ns = 4 if self.dim == 2 else 6
        c = np.zeros(ne * self.nen, np.int32)
        nb = np.zeros(ne * ns, np.int32)
        col = np.zeros(ne, np.int32)
        check(self.L.exf_mesh_get_conn(self.h, lev, iptr(c), iptr(nb), iptr(col)))
        return c.reshape(ne, self.nen), nb.reshape(ne, ns), col


class MGSolBase:
    """One equation system on the GPU (MGSolBase/MGSolDA analogue)."""

    kind = None

    def __init__(self, mesh, kind=None):
        self.L = load()
        self.mesh = mesh
        if kind is not None:
            self.kind = kind
        h = C.c_void_p()
        check(self.L.exf_sys_create(mesh.h, self.kind, C.byref(h)))  # init_dof + pattern (MGDofBcOp)
        self.h = h
        self.nlev = mesh.nlev
        self.nvars = mesh.dim + 1 if self.kind == _lib.KIND_NS else 1
        self.phys = phys()
        self._keep = None

    def close(self):
        if getattr(self, "h", None):
            self.L.exf_sys_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # ---- DOF / operators
    def MGDofBcOp(self, preset=None):
        if preset is not None:
            self.GenBc(preset)

    def ndof(self, lev):
        n = C.c_int()
        check(self.L.exf_sys_ndof(self.h, lev, C.byref(n)))
        return n.value

    @property
    def ntop_dof(self):
        return self.ndof(self.nlev - 1)

    def node_dof(self, lev):
        a = np.zeros(self.nvars * self.mesh.ntop, np.int32)
        check(self.L.exf_sys_get_node_dof(self.h, lev, iptr(a)))
        return a

    def GenBc(self, preset):
        check(self.L.exf_sys_bc_preset(self.h, preset))

    def set_bc(self, bc0, bc1):
        bc0 = np.ascontiguousarray(bc0, np.int32)
        bc1 = np.ascontiguousarray(bc1, np.int32)
        check(self.L.exf_sys_set_bc(self.h, iptr(bc0), iptr(bc1)))

    def bc(self):
        n = self.ntop_dof
        b0 = np.zeros(n, np.int32)
        b1 = np.zeros(n, np.int32)
        check(self.L.exf_sys_get_bc(self.h, iptr(b0), iptr(b1)))
        return b0, b1

    def nnz(self, lev):
        v = C.c_long()
        check(self.L.exf_sys_nnz(self.h, lev, C.byref(v)))
        return v.value

    def pattern(self, lev):
        rp = np.zeros(self.ndof(lev) + 1, np.int32)
        col = np.zeros(self.nnz(lev), np.int32)
        check(self.L.exf_sys_get_pattern(self.h, lev, iptr(rp), iptr(col)))
        return rp, col

    def _transfer(self, fn, lev, nrow):
        nnz = C.c_long()
        check(fn(self.h, lev, C.byref(nnz), None, None, None))
        rp = np.zeros(nrow + 1, np.int32)
        col = np.zeros(nnz.value, np.int32)
        val = np.zeros(nnz.value)
        check(fn(self.h, lev, C.byref(nnz), iptr(rp), iptr(col), dptr(val)))
        return rp, col, val

    def prol(self, lev):  # Prl[lev]: level lev-1 -> lev (ReadProl)
        return self._transfer(self.L.exf_sys_get_prol, lev, self.ndof(lev))

    def rest(self, lev):  # Rst[lev]: level lev+1 -> lev (ReadRest)
        return self._transfer(self.L.exf_sys_get_rest, lev, self.ndof(lev))

    def colours(self, lev):
        nitem = self.mesh.nnodes(lev) if self.kind != _lib.KIND_NS else (
            self.mesh.nnodes(lev - 1) if lev > 0 else self.mesh.nvert0)
        out = np.zeros(nitem, np.int32)
        nc = C.c_int()
        check(self.L.exf_sys_get_colours(self.h, lev, C.byref(nc), iptr(out)))
        return nc.value, out

    def set_transfer(self, lev, kind, block, dim, length, pos, val):
        """One block of a Prol/Rest operator in gencase's dataset layout (DIM0/LEN0/POS0/VAL0)."""
        a = np.ascontiguousarray(dim, np.int32)
        b = np.ascontiguousarray(length, np.int32)
        c = np.ascontiguousarray(pos, np.int32)
        v = np.ascontiguousarray(val, np.float64)
        check(self.L.exf_sys_set_transfer(self.h, lev, kind, block, iptr(a), iptr(b), iptr(c), dptr(v)))

    def get_transfer(self, lev, kind, block):
        """One block of a Prol/Rest operator in gencase's dataset layout: (dim, len, pos, val)."""
        dim = np.zeros(2, np.int32)
        nnz = C.c_long()
        check(self.L.exf_sys_get_transfer(self.h, lev, kind, block, iptr(dim), C.byref(nnz), None, None, None))
        ln = np.zeros(dim[0] + 1, np.int32)
        pos = np.zeros(nnz.value, np.int32)
        val = np.zeros(nnz.value)
        check(self.L.exf_sys_get_transfer(self.h, lev, kind, block, iptr(dim), C.byref(nnz), iptr(ln), iptr(pos),
                                          dptr(val)))
        return dim, ln, pos, val

    def check_pattern(self, lev, block, dim, length, pos):
        """Status of exf_sys_check_pattern for one block of gencase's matrix datasets."""
        a = np.ascontiguousarray(dim, np.int32)
        b = np.ascontiguousarray(length, np.int32)
        c = np.ascontiguousarray(pos, np.int32)
        return self.L.exf_sys_check_pattern(self.h, lev, block, iptr(a), iptr(b), iptr(c))

    def couple(self, other):
        """exf_sys_couple; keep the partner open while this system assembles (closing it
        clears the coupling, and the next assembly that needs it fails)."""
        check(self.L.exf_sys_couple(self.h, other.h if other is not None else None))

    # ---- fields
    def set_xold(self, x):
        x = np.ascontiguousarray(x, np.float64)
        check(self.L.exf_sys_set_xold(self.h, dptr(x)))

    def xold(self):
        x = np.zeros(self.ntop_dof)
        check(self.L.exf_sys_get_xold(self.h, dptr(x)))
        return x

    def set_x(self, x):
        x = np.ascontiguousarray(x, np.float64)
        check(self.L.exf_sys_set_x(self.h, dptr(x)))

    def x(self):
        x = np.zeros(self.ntop_dof)
        check(self.L.exf_sys_get_x(self.h, dptr(x)))
        return x

    def xold_update(self):
        check(self.L.exf_sys_xold_update(self.h))

    def set_source(self, qe):
        qe = np.ascontiguousarray(qe, np.float64)
        check(self.L.exf_sys_set_source(self.h, dptr(qe)))

    def set_rhs(self, b):
        b = np.ascontiguousarray(b, np.float64)
        check(self.L.exf_sys_set_rhs(self.h, dptr(b)))

    def rhs(self):
        b = np.zeros(self.ntop_dof)
        check(self.L.exf_sys_get_rhs(self.h, dptr(b)))
        return b

    # ---- assembly (GenMatRhs)
    def GenMatRhs(self, time, Level, mode):
        del time  # steady / pseudo-time: the time level enters through phys.inv_dt
        check(self.L.exf_gen_mat_rhs(self.h, C.byref(self.phys), Level, mode))

    def assemble_all(self):
        check(self.L.exf_assemble_all(self.h, C.byref(self.phys)))

    def matrix(self, lev):
        v = np.zeros(self.nnz(lev))
        check(self.L.exf_get_matrix(self.h, lev, dptr(v)))
        return v

    def set_matrix(self, lev, v):
        v = np.ascontiguousarray(v, np.float64)
        check(self.L.exf_set_matrix(self.h, lev, dptr(v)))

    def csr(self, lev):
        rp, col = self.pattern(lev)
        return rp, col, self.matrix(lev)

    def transpose(self):
        check(self.L.exf_sys_transpose(self.h))

    # ---- solve (MGSolve / MGStep)
    def solve(self, params):
        st = ExfSolveStats()
        rc = self.L.exf_mg_solve(self.h, C.byref(params), C.byref(st))
        if rc not in (_lib.EXF_OK, _lib.EXF_ERR_NOT_CONVERGED):
            check(rc)
        return st

    def MGSolve(self, Eps, MaxIter, Gamma=1, Nc_pre=8, Nc_coarse=40, Nc_post=8, **kw):
        del Nc_coarse  # the coarsest level is solved directly
        p = mg_params(eps=Eps, max_cycles=MaxIter, gamma=Gamma, nu_pre=Nc_pre, nu_post=Nc_post,
                      smoother=_lib.SMOOTH_VANKA if self.kind == _lib.KIND_NS else _lib.SMOOTH_GS, **kw)
        return self.solve(p)

    def MGTimeStep(self, time, params):
        """GenMatRhs(top,1) + GenMatRhs(L<top,0) + MGSolve + x_old update (MGSolverNS.C:722-750)."""
        del time
        self.assemble_all()
        st = self.solve(params)
        self.xold_update()
        return st

    # ---- unit operations on host arrays
    def resid(self, lev, x, b=None):
        """r = b - A x on level lev (NumericVectorM::resid); with b=None returns A x."""
        r = np.zeros(self.ndof(lev))
        x = np.ascontiguousarray(x, np.float64)
        bb = None if b is None else np.ascontiguousarray(b, np.float64)
        check(self.L.exf_resid(self.h, lev, dptr(x), None if bb is None else dptr(bb), dptr(r)))
        return r

    def spmv(self, lev, x):
        return self.resid(lev, x, None)

    def restrict(self, lev, r_fine):
        out = np.zeros(self.ndof(lev))
        r_fine = np.ascontiguousarray(r_fine, np.float64)
        check(self.L.exf_restrict(self.h, lev, dptr(r_fine), dptr(out)))
        return out

    def prolong(self, lev, x_coarse):
        out = np.zeros(self.ndof(lev))
        x_coarse = np.ascontiguousarray(x_coarse, np.float64)
        check(self.L.exf_prolong(self.h, lev, dptr(x_coarse), dptr(out)))
        return out

    def smooth(self, lev, params, nsweeps, x, b):
        x = np.array(x, dtype=np.float64)
        b = np.ascontiguousarray(b, np.float64)
        check(self.L.exf_smooth(self.h, lev, C.byref(params), nsweeps, dptr(x), dptr(b)))
        return x

    def ilu_apply(self, lev, c):
        """ILUPrecond of level lev: (D + U)^-1 D (D + L)^-1 c with LASPACK's ILU(0) factor."""
        c = np.ascontiguousarray(c, np.float64)
        y = np.zeros(self.ndof(lev))
        check(self.L.exf_ilu_apply(self.h, lev, dptr(c), dptr(y)))
        return y

    def coarse_solve(self, b):
        x = np.zeros(self.ndof(0))
        b = np.ascontiguousarray(b, np.float64)
        check(self.L.exf_coarse_solve(self.h, dptr(b), dptr(x)))
        return x

    def sync(self):
        check(self.L.exf_sync(self.h))


class MGSolT(MGSolBase):
    """Temperature equation (MGSolT, template_appl/nse/SRC/MGSolverT.h)."""
    kind = _lib.KIND_T


class MGSolNS(MGSolBase):
    """Coupled Navier-Stokes, Taylor-Hood Q2-Q1 (MGSolNS, NS_EQUATIONS==1)."""
    kind = _lib.KIND_NS


class MGSolTBK(MGSolBase):
    """One variable of the turbulence template's coupled kappa-omega system (MGSolTBK,
    template_appl/turb-ckw/SRC/MGSolverTBKW.C, TBK_EQUATIONS 5): var 0 kappa, 1 omega.
    Couple it to the Navier-Stokes system (velocity) and to the other variable; the
    element wall distances come from set_wall."""

    def __init__(self, mesh, var):
        super().__init__(mesh, _lib.KIND_K if var == 0 else _lib.KIND_W)
        self.var = var

    def set_wall(self, dist, nu_wall):
        """dist: the wall distance of every element, level 0's first (_mgmesh._dist);
        nu_wall = mu / rho of the omega wall value 6 nu_wall / (BETASTAR y^2)."""
        d = np.ascontiguousarray(dist, np.float64)
        self._wall = d
        check(self.L.exf_sys_set_wall(self.h, dptr(d), float(nu_wall)))


class MGSolDS(MGSolBase):
    """One direction of the fluid-structure template's mesh displacement (MGSolDS,
    template_appl/fsi/SRC/MGSolverDS.C, ALE_MOVING): direction 0 dx, 1 dy, 2 dz.  Its
    element matrices read the FSI velocity and the old displacements given to set_fields;
    bc0 carries the reference's volume flags (element phase from the centre node: < 2
    fluid, else solid; > 3 on interface nodes) and bc1 the boundary flags."""

    def __init__(self, mesh, direction):
        super().__init__(mesh, _lib.KIND_DS)
        self.direction = direction

    def set_fields(self, dt, u_fsi=None, d_old=None):
        """u_fsi, d_old: [dim][ntop] node fields (the FSI velocity, the old displacement
        of every direction); dt the time step.  Without fields the element matrices read
        the coupled systems' x_old on the device: the velocity of the coupled NS system,
        this system's own x_old and the coupled dx system's."""
        if u_fsi is None and d_old is None:
            check(self.L.exf_sys_set_ds(self.h, int(self.direction), float(dt), None, None))
            return
        u = np.ascontiguousarray(u_fsi, np.float64)
        d = np.ascontiguousarray(d_old, np.float64)
        check(self.L.exf_sys_set_ds(self.h, int(self.direction), float(dt), dptr(u), dptr(d)))

    def set_mesh_motion(self, moving=True):
        """moving_mesh with FINE_MOVEMENT: each x_old update moves the mesh's coordinates
        of this direction by x - x_old."""
        check(self.L.exf_sys_set_mesh_motion(self.h, int(bool(moving))))


def timestep_loop(systems, params, nsteps, strict=True):
    """MGEquationsSystem::eqnmap_timestep_loop (src/MGEquationsSystem.C:422-432) in the
    library: nsteps times the MGTimeStep of every system in order (assembly, solve,
    x_old update) without returning here between them.  params: one exf_mg_params per
    system.  Returns (cycles, seconds), arrays [nsteps, len(systems)].  Every step runs
    even when a solve ends above its tolerance; that raises EXF_ERR_NOT_CONVERGED at the
    end unless strict is False."""
    L = _lib.load()
    n = len(systems)
    hs = (C.c_void_p * n)(*[s.h for s in systems])
    phs = (_lib.ExfPhys * n)(*[s.phys for s in systems])
    ps = (_lib.ExfMgParams * n)(*params)
    cyc = np.zeros((nsteps, n), dtype=np.int32)
    sec = np.zeros((nsteps, n))
    rc = L.exf_timestep_loop(hs, n, phs, ps, nsteps, iptr(cyc), dptr(sec))
    if strict or rc != _lib.EXF_ERR_NOT_CONVERGED:
        check(rc)
    return cyc, sec

