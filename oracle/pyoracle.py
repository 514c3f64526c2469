"""ctypes bindings of the CPU oracle (test infrastructure only)."""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_LP = None


def build(quiet=True):
    """Compile liboracle.so (and _ref/liblaspack_ref.so when the reference tree exists)."""
    out = subprocess.run(["make", "-C", _HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


class OrPhys(C.Structure):
    _fields_ = [("inv_re", C.c_double), ("inv_prdl", C.c_double), ("rho", C.c_double),
                ("rhocp", C.c_double), ("inv_dt", C.c_double), ("penalty", C.c_double),
                ("upwind_ns", C.c_double), ("upwind_t", C.c_double), ("ifr", C.c_double),
                ("dirg", C.c_double * 3), ("buoy", C.c_double), ("traction", C.c_double)]


class OrMgParams(C.Structure):
    _fields_ = [("eps", C.c_double), ("max_cycles", C.c_int), ("gamma", C.c_int),
                ("nu_pre", C.c_int), ("nu_post", C.c_int), ("double_below_top", C.c_int),
                ("smoother", C.c_int), ("omega", C.c_double), ("corr_damp", C.c_double),
                ("cond_corr", C.c_int), ("reverse_colours", C.c_int), ("stop_test", C.c_int)]


class OrMgStats(C.Structure):
    _fields_ = [("cycles", C.c_int), ("converged", C.c_int), ("rel_res", C.c_double),
                ("bnorm", C.c_double), ("hist", C.c_double * 256), ("last_acc", C.c_double)]


def oracle_lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P = C.c_void_p
        I = C.c_int
        ip = np.ctypeslib.ndpointer(np.int32, flags="C")
        dp = np.ctypeslib.ndpointer(np.float64, flags="C")
        L.or_mesh_new.restype = P
        L.or_mesh_new.argtypes = [I, I, ip, dp]
        L.or_mesh_free.argtypes = [P]
        for f in ("or_mesh_nnodes", "or_mesh_nel"):
            getattr(L, f).argtypes = [P, I]
            getattr(L, f).restype = I
        L.or_mesh_nvert0.argtypes = [P]
        L.or_mesh_nen.argtypes = [P]
        L.or_mesh_get_xyz.argtypes = [P, dp]
        L.or_mesh_get_lattice.argtypes = [P, ip]
        L.or_mesh_get_conn.argtypes = [P, I, ip, ip, ip]
        L.or_sys_new.restype = P
        L.or_sys_new.argtypes = [P, I]
        L.or_sys_free.argtypes = [P]
        L.or_sys_ndof.argtypes = [P, I]
        L.or_sys_node_dof.argtypes = [P, I, ip]
        L.or_sys_bc_preset.argtypes = [P, I]
        L.or_sys_set_bc.argtypes = [P, ip, ip]
        L.or_sys_get_bc.argtypes = [P, ip, ip]
        for f in ("or_sys_nnz", "or_sys_prol_nnz", "or_sys_rest_nnz"):
            getattr(L, f).argtypes = [P, I]
            getattr(L, f).restype = C.c_long
        L.or_sys_pattern.argtypes = [P, I, ip, ip]
        L.or_sys_prol.argtypes = [P, I, ip, ip, dp]
        L.or_sys_rest.argtypes = [P, I, ip, ip, dp]
        L.or_sys_colours.argtypes = [P, I, C.POINTER(C.c_int), ip]
        L.or_sys_assemble.argtypes = [P, I, I, C.POINTER(OrPhys), P, P, P, P]
        L.or_kw_assemble.argtypes = [P, I, I, I, C.POINTER(OrPhys), P, P, P, P, C.c_double]
        L.or_sys_set_turb.argtypes = [P, P, P]
        L.or_ds_assemble.argtypes = [P, I, I, I, C.c_double, P, P]
        L.or_sys_get_matrix.argtypes = [P, I, dp]
        L.or_sys_set_matrix.argtypes = [P, I, dp]
        L.or_sys_get_rhs.argtypes = [P, dp]
        L.or_sys_set_rhs.argtypes = [P, dp]
        L.or_sys_transpose_all.argtypes = [P]
        L.or_spmv.argtypes = [P, I, dp, dp]
        L.or_mg_solve.argtypes = [P, C.POINTER(OrMgParams), dp, C.POINTER(OrMgStats)]
        L.or_mg_solve.restype = I
        L.or_coarse_solve.argtypes = [P, dp, dp]
        L.or_smooth.argtypes = [P, I, C.POINTER(OrMgParams), I, dp, dp]
        L.or_set_threads.argtypes = [I]
        L.or_get_threads.restype = I
        L.or_fe_tables.argtypes = [I, dp, dp, dp, dp]
        L.or_side_table.argtypes = [I, ip]
        _LIB = L
    return _LIB


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class OrMesh:
    """Structured multilevel quad9/hex27 hierarchy (restated gencase ordering)."""

    def __init__(self, dim, nlev, n0, box):
        self.L = oracle_lib()
        n0 = np.array(list(n0) + [1] * (3 - len(n0)), dtype=np.int32)
        box = np.array(list(box) + [0.0] * (6 - len(box)), dtype=np.float64)
        self.dim, self.nlev = dim, nlev
        self.h = self.L.or_mesh_new(dim, nlev, n0, box)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_mesh_free(self.h)
            self.h = None

    def nnodes(self, lev):
        return self.L.or_mesh_nnodes(self.h, lev)

    @property
    def ntop(self):
        return self.nnodes(self.nlev - 1)

    @property
    def nvert0(self):
        return self.L.or_mesh_nvert0(self.h)

    def nel(self, lev):
        return self.L.or_mesh_nel(self.h, lev)

    @property
    def nen(self):
        return 9 if self.dim == 2 else 27

    def xyz(self):
        a = np.zeros(self.dim * self.ntop)
        self.L.or_mesh_get_xyz(self.h, a)
        return a.reshape(self.dim, self.ntop)

    def lattice(self):
        a = np.zeros(3 * self.ntop, dtype=np.int32)
        self.L.or_mesh_get_lattice(self.h, a)
        return a.reshape(self.ntop, 3)

    def conn(self, lev):
        ns = 4 if self.dim == 2 else 6
        ne = self.nel(lev)
        c = np.zeros(ne * self.nen, dtype=np.int32)
        nb = np.zeros(ne * ns, dtype=np.int32)
        col = np.zeros(ne, dtype=np.int32)
        self.L.or_mesh_get_conn(self.h, lev, c, nb, col)
        return c.reshape(ne, self.nen), nb.reshape(ne, ns), col


class OrSys:
    """One equation system (kind 0 = temperature, 1 = coupled Navier-Stokes)."""

    def __init__(self, mesh, kind):
        self.L = oracle_lib()
        self.mesh = mesh
        self.kind = kind
        self.h = self.L.or_sys_new(mesh.h, kind)
        self.nvars = 1 if kind == 0 else mesh.dim + 1

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_sys_free(self.h)
            self.h = None

    def ndof(self, lev):
        return self.L.or_sys_ndof(self.h, lev)

    def node_dof(self, lev):
        a = np.zeros(self.nvars * self.mesh.ntop, dtype=np.int32)
        self.L.or_sys_node_dof(self.h, lev, a)
        return a

    def bc_preset(self, p):
        self.L.or_sys_bc_preset(self.h, p)

    def set_bc(self, bc0, bc1):
        self.L.or_sys_set_bc(self.h, np.ascontiguousarray(bc0, np.int32), np.ascontiguousarray(bc1, np.int32))

    def bc(self):
        n = self.ndof(self.mesh.nlev - 1)
        b0 = np.zeros(n, np.int32)
        b1 = np.zeros(n, np.int32)
        self.L.or_sys_get_bc(self.h, b0, b1)
        return b0, b1

    def pattern(self, lev):
        n = self.ndof(lev)
        nnz = self.L.or_sys_nnz(self.h, lev)
        rp = np.zeros(n + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        self.L.or_sys_pattern(self.h, lev, rp, col)
        return rp, col

    def prol(self, lev):
        n = self.ndof(lev)
        nnz = self.L.or_sys_prol_nnz(self.h, lev)
        rp = np.zeros(n + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz)
        self.L.or_sys_prol(self.h, lev, rp, col, val)
        return rp, col, val

    def rest(self, lev):
        n = self.ndof(lev)
        nnz = self.L.or_sys_rest_nnz(self.h, lev)
        rp = np.zeros(n + 1, np.int32)
        col = np.zeros(nnz, np.int32)
        val = np.zeros(nnz)
        self.L.or_sys_rest(self.h, lev, rp, col, val)
        return rp, col, val

    def colours(self, lev):
        nitem = self.mesh.nnodes(lev) if self.kind == 0 else (
            self.mesh.nnodes(lev - 1) if lev > 0 else self.mesh.nvert0)
        out = np.zeros(nitem, np.int32)
        nc = C.c_int(0)
        self.L.or_sys_colours(self.h, lev, C.byref(nc), out)
        return nc.value, out

    def assemble(self, lev, mode, phys, xold=None, vel=None, temp=None, qe=None):
        keep = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (xold, vel, temp, qe)]
        self.L.or_sys_assemble(self.h, lev, mode, C.byref(phys), *[_ptr(a) for a in keep])

    def set_turb(self, kold, wold):
        """NS: the kappa, omega fields of the eddy viscosity (kept alive here)."""
        self._turb = [np.ascontiguousarray(a, np.float64) for a in (kold, wold)]
        self.L.or_sys_set_turb(self.h, *[_ptr(a) for a in self._turb])

    def kw_assemble(self, lev, mode, var, phys, vel, kold, wold, dist, nu_wall):
        """Level lev of variable var (0 kappa, 1 omega) of the turbulence template's
        kappa-omega system on this scalar system; dist: this level's element wall
        distances."""
        keep = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (vel, kold, wold, dist)]
        self.L.or_kw_assemble(self.h, lev, mode, var, C.byref(phys), *[_ptr(a) for a in keep], float(nu_wall))

    def ds_assemble(self, lev, mode, direction, dt, u_fsi, d_old):
        """Level lev of the fluid-structure template's displacement direction on this
        scalar system; u_fsi, d_old: [dim][ntop] node fields."""
        keep = [np.ascontiguousarray(a, np.float64) for a in (u_fsi, d_old)]
        self.L.or_ds_assemble(self.h, lev, mode, direction, float(dt), *[_ptr(a) for a in keep])

    def assemble_all(self, phys, xold=None, vel=None, temp=None, qe=None):
        top = self.mesh.nlev - 1
        self.assemble(top, 1, phys, xold, vel, temp, qe)
        for lev in range(top):
            self.assemble(lev, 0, phys, xold, vel, temp, qe)

    def matrix(self, lev):
        v = np.zeros(self.L.or_sys_nnz(self.h, lev))
        self.L.or_sys_get_matrix(self.h, lev, v)
        return v

    def set_matrix(self, lev, v):
        self.L.or_sys_set_matrix(self.h, lev, np.ascontiguousarray(v, np.float64))

    def rhs(self):
        v = np.zeros(self.ndof(self.mesh.nlev - 1))
        self.L.or_sys_get_rhs(self.h, v)
        return v

    def set_rhs(self, v):
        self.L.or_sys_set_rhs(self.h, np.ascontiguousarray(v, np.float64))

    def transpose_all(self):
        self.L.or_sys_transpose_all(self.h)

    def spmv(self, lev, x):
        y = np.zeros(self.ndof(lev))
        self.L.or_spmv(self.h, lev, np.ascontiguousarray(x, np.float64), y)
        return y

    def mg_solve(self, params, x0=None):
        n = self.ndof(self.mesh.nlev - 1)
        x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
        st = OrMgStats()
        self.L.or_mg_solve(self.h, C.byref(params), x, C.byref(st))
        return x, st

    def smooth(self, lev, params, nsweeps, x, b):
        x = np.array(x, dtype=np.float64)
        self.L.or_smooth(self.h, lev, C.byref(params), nsweeps, x, np.ascontiguousarray(b, np.float64))
        return x

    def coarse_solve(self, b):
        x = np.zeros(self.ndof(0))
        rc = self.L.or_coarse_solve(self.h, np.ascontiguousarray(b, np.float64), x)
        if rc:
            raise RuntimeError("singular coarse matrix")
        return x

    def csr(self, lev):
        rp, col = self.pattern(lev)
        return rp, col, self.matrix(lev)


def laspack_available():
    return os.path.exists(os.path.join(_HERE, "_ref", "liblaspack_ref.so"))


class Laspack:
    """The reference's LASPACK kernels (compiled from contrib/laspack/*.c)."""

    def __init__(self):
        global _LP
        if _LP is None:
            path = os.path.join(_HERE, "_ref", "liblaspack_ref.so")
            if not os.path.exists(path):
                raise FileNotFoundError(path)
            L = C.CDLL(path)
            ip = np.ctypeslib.ndpointer(np.int32, flags="C")
            dp = np.ctypeslib.ndpointer(np.float64, flags="C")
            I = C.c_int
            L.lpb_spmv.argtypes = [I, ip, ip, dp, dp, dp]
            L.lpb_spmv_t.argtypes = [I, ip, ip, dp, dp, dp]
            L.lpb_gmres.argtypes = [I, ip, ip, dp, dp, dp, C.c_double, I, I, I, C.POINTER(I),
                                    C.POINTER(C.c_double)]
            L.lpb_sorforw.argtypes = [I, ip, ip, dp, dp, dp, I, C.c_double, C.POINTER(C.c_double)]
            L.lpb_gmres_pc.argtypes = [I, ip, ip, dp, dp, dp, C.c_double, I, I, I, I, C.POINTER(I),
                                       C.POINTER(C.c_double)]
            L.lpb_ilu_apply.argtypes = [I, ip, ip, dp, dp, dp]
            _LP = L
        self.L = _LP

    def spmv(self, rp, col, val, x):
        y = np.zeros(len(rp) - 1)
        self.L.lpb_spmv(len(rp) - 1, rp, col, val, np.ascontiguousarray(x, np.float64), y)
        return y

    def spmv_t(self, rp, col, val, x):
        """A^T x through the reference's Transp_Q and Mul_QV."""
        y = np.zeros(len(rp) - 1)
        self.L.lpb_spmv_t(len(rp) - 1, rp, col, val, np.ascontiguousarray(x, np.float64), y)
        return y

    def gmres(self, rp, col, val, b, x0=None, tol=1e-12, maxit=2000, restart=30, transpose=False, ilu=False):
        """LASPACK GMRESIter (optionally ILU(0)-preconditioned) on A or Transp_Q(A)."""
        n = len(rp) - 1
        x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
        it = C.c_int(0)
        acc = C.c_double(0)
        self.L.lpb_gmres_pc(n, rp, col, val, np.ascontiguousarray(b, np.float64), x, tol, maxit, restart,
                            1 if transpose else 0, 1 if ilu else 0, C.byref(it), C.byref(acc))
        return x, it.value, acc.value

    def ilu_apply(self, rp, col, val, c):
        """ILUPrecond(c): (D + U)^-1 D (D + L)^-1 c with LASPACK's ILU(0) factor of A."""
        y = np.zeros(len(rp) - 1)
        rc = self.L.lpb_ilu_apply(len(rp) - 1, rp, col, val, np.ascontiguousarray(c, np.float64), y)
        if rc:
            raise RuntimeError("LASPACK ILUPrecond failed")
        return y

    def sorforw(self, rp, col, val, b, x0, nsweeps, omega=1.0):
        x = np.array(x0, np.float64)
        acc = C.c_double(0)
        self.L.lpb_sorforw(len(rp) - 1, rp, col, val, np.ascontiguousarray(b, np.float64), x, nsweeps, omega,
                           C.byref(acc))
        return x, acc.value


def set_threads(n):
    """Threads of the oracle's parallel loops (results do not depend on the count)."""
    oracle_lib().or_set_threads(int(n))


def get_threads():
    return int(oracle_lib().or_get_threads())
