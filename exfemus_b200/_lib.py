"""ctypes binding of libexfemus_b200.so (the C ABI declared in include/exfemus_b200.h)."""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libexfemus_b200.so")

EXF_OK = 0
EXF_ERR_ARG = 1
EXF_ERR_CUDA = 2
EXF_ERR_STATE = 3
EXF_ERR_DIVERGED = 4
EXF_ERR_NOT_CONVERGED = 5
EXF_ERR_SINGULAR = 6
EXF_ERR_NOMEM = 7
EXF_ERR_UNSUPPORTED = 8
EXF_ERR_IO = 9

KIND_T = 0
KIND_NS = 1
KIND_K = 2
KIND_W = 3
KIND_DS = 4
BC_HEAT_DIRICHLET = 1
BC_CAVITY = 2
BC_CHANNEL = 3
BC_BOUSS_NS = 4
BC_BOUSS_T = 5
SMOOTH_GS = 0
SMOOTH_VANKA = 1
SMOOTH_GMRES_ILU = 2
PREC_FP64 = 0
PREC_MIXED = 1
VANKA_AUTO = 0
VANKA_TILE = 1
VANKA_ROWS = 2
VANKA_STREAM = 3
VANKA_BULK = 4
STOP_RELRES = 0
STOP_REFERENCE = 1


class ExfMeshDesc(C.Structure):
    _fields_ = [("dim", C.c_int), ("nlev", C.c_int), ("n0", C.c_int * 3), ("box", C.c_double * 6),
                ("device", C.c_int)]


class ExfMeshData(C.Structure):
    _fields_ = [("dim", C.c_int), ("nlev", C.c_int), ("device", C.c_int), ("nnodes", C.c_void_p),
                ("nvert0", C.c_int), ("xyz", C.c_void_p), ("nel", C.c_void_p), ("conn", C.c_void_p),
                ("neigh", C.c_void_p), ("parent", C.c_void_p)]


class ExfMeshCoarse(C.Structure):
    _fields_ = [("dim", C.c_int), ("nlev", C.c_int), ("device", C.c_int), ("nnode0", C.c_int),
                ("nvert0", C.c_int), ("xyz0", C.c_void_p), ("nel0", C.c_int), ("conn0", C.c_void_p)]


class ExfSolnOut(C.Structure):
    _fields_ = [("dir", C.c_char_p), ("basesol", C.c_char_p), ("basemesh", C.c_char_p),
                ("connlin", C.c_char_p), ("ndigits", C.c_int), ("t_step", C.c_int), ("time", C.c_double)]


class ExfNodeFields(C.Structure):
    _fields_ = [("dim", C.c_int), ("nnodes", C.c_int), ("xyz", C.c_void_p), ("nel", C.c_int),
                ("conn", C.c_void_p), ("nvars", C.c_int), ("names", C.POINTER(C.c_char_p)),
                ("order", C.c_void_p), ("vals", C.c_void_p)]


class ExfPhys(C.Structure):
    _fields_ = [("inv_re", C.c_double), ("inv_prdl", C.c_double), ("rho", C.c_double),
                ("rhocp", C.c_double), ("inv_dt", C.c_double), ("penalty", C.c_double),
                ("upwind_ns", C.c_double), ("upwind_t", C.c_double), ("ifr", C.c_double),
                ("dirg", C.c_double * 3), ("buoy", C.c_double), ("traction", C.c_double)]


class ExfMgParams(C.Structure):
    _fields_ = [("eps", C.c_double), ("max_cycles", C.c_int), ("gamma", C.c_int),
                ("nu_pre", C.c_int), ("nu_post", C.c_int), ("double_below_top", C.c_int),
                ("smoother", C.c_int), ("omega", C.c_double), ("corr_damp", C.c_double),
                ("cond_corr", C.c_int), ("reverse_colours", C.c_int), ("precision", C.c_int),
                ("use_graph", C.c_int), ("vanka_kernel", C.c_int), ("stop_test", C.c_int),
                ("fp32_blocks", C.c_int), ("coarse_iters", C.c_int)]


class ExfSolveStats(C.Structure):
    _fields_ = [("cycles", C.c_int), ("converged", C.c_int), ("rel_res", C.c_double),
                ("bnorm", C.c_double), ("seconds", C.c_double), ("hist", C.c_double * 256),
                ("last_acc", C.c_double)]


class ExfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("exfemus_b200 error %d: %s" % (code, msg))
        self.code = code


_L = None

# (name, restype, argtypes) of every exported entry point
_P = C.c_void_p
_I = C.c_int
_IP = C.POINTER(C.c_int)
_DP = C.POINTER(C.c_double)
_LP = C.POINTER(C.c_long)
SIGNATURES = [
    ("exf_last_error", C.c_char_p, []),
    ("exf_version", C.c_char_p, []),
    ("exf_mesh_create", _I, [C.POINTER(ExfMeshDesc), C.POINTER(_P)]),
    ("exf_mesh_destroy", _I, [_P]),
    ("exf_mesh_info", _I, [_P, _I, _IP, _IP, _IP]),
    ("exf_mesh_get_xyz", _I, [_P, _DP]),
    ("exf_mesh_get_conn", _I, [_P, _I, _IP, _IP, _IP]),
    ("exf_sys_create", _I, [_P, _I, C.POINTER(_P)]),
    ("exf_sys_destroy", _I, [_P]),
    ("exf_sys_ndof", _I, [_P, _I, _IP]),
    ("exf_sys_get_node_dof", _I, [_P, _I, _IP]),
    ("exf_sys_bc_preset", _I, [_P, _I]),
    ("exf_sys_set_bc", _I, [_P, _IP, _IP]),
    ("exf_sys_get_bc", _I, [_P, _IP, _IP]),
    ("exf_sys_nnz", _I, [_P, _I, _LP]),
    ("exf_sys_get_pattern", _I, [_P, _I, _IP, _IP]),
    ("exf_sys_get_prol", _I, [_P, _I, _LP, _IP, _IP, _DP]),
    ("exf_sys_get_rest", _I, [_P, _I, _LP, _IP, _IP, _DP]),
    ("exf_sys_get_colours", _I, [_P, _I, _IP, _IP]),
    ("exf_sys_couple", _I, [_P, _P]),
    ("exf_sys_set_wall", _I, [_P, _DP, C.c_double]),
    ("exf_sys_set_ds", _I, [_P, _I, C.c_double, _DP, _DP]),
    ("exf_sys_set_mesh_motion", _I, [_P, _I]),
    ("exf_mesh_wall_dist", _I, [_P, _IP, _DP]),
    ("exf_sys_set_xold", _I, [_P, _DP]),
    ("exf_sys_get_xold", _I, [_P, _DP]),
    ("exf_sys_set_x", _I, [_P, _DP]),
    ("exf_sys_get_x", _I, [_P, _DP]),
    ("exf_sys_xold_update", _I, [_P]),
    ("exf_sys_set_source", _I, [_P, _DP]),
    ("exf_sys_set_rhs", _I, [_P, _DP]),
    ("exf_sys_get_rhs", _I, [_P, _DP]),
    ("exf_gen_mat_rhs", _I, [_P, C.POINTER(ExfPhys), _I, _I]),
    ("exf_assemble_all", _I, [_P, C.POINTER(ExfPhys)]),
    ("exf_get_matrix", _I, [_P, _I, _DP]),
    ("exf_set_matrix", _I, [_P, _I, _DP]),
    ("exf_mg_solve", _I, [_P, C.POINTER(ExfMgParams), C.POINTER(ExfSolveStats)]),
    ("exf_resid", _I, [_P, _I, _DP, _DP, _DP]),
    ("exf_restrict", _I, [_P, _I, _DP, _DP]),
    ("exf_prolong", _I, [_P, _I, _DP, _DP]),
    ("exf_smooth", _I, [_P, _I, C.POINTER(ExfMgParams), _I, _DP, _DP]),
    ("exf_coarse_solve", _I, [_P, _DP, _DP]),
    ("exf_ilu_apply", _I, [_P, _I, _DP, _DP]),
    ("exf_sys_transpose", _I, [_P]),
    ("exf_adjoint_forward", _I, [_P, C.POINTER(ExfPhys), C.POINTER(ExfMgParams), C.POINTER(ExfSolveStats)]),
    ("exf_adjoint_backward", _I, [_P, C.POINTER(ExfPhys), C.POINTER(ExfMgParams), _DP, _DP, _DP,
                                  C.POINTER(ExfSolveStats)]),
    ("exf_time_op", _I, [_P, _I, _I, C.POINTER(ExfMgParams), C.POINTER(ExfPhys), _I, _DP]),
    ("exf_sync", _I, [_P]),
    ("exf_timestep_loop", _I, [C.POINTER(_P), _I, C.POINTER(ExfPhys), C.POINTER(ExfMgParams), _I, _IP, _DP]),
    ("exf_event_record", _I, [_P, _I]),
    ("exf_event_elapsed", _I, [_P, _I, _I, _DP]),
    ("exf_launch_count", C.c_longlong, []),
    ("exf_level_bytes", _I, [_P, _I, _I, _DP, _DP]),
    ("exf_resid_norm_static", _I, [_P, _I, _P, _P, _P, _P]),
    ("exf_mesh_upload", _I, [C.POINTER(ExfMeshData), C.POINTER(_P)]),
    ("exf_mesh_refine_arrays", _I, [C.POINTER(ExfMeshCoarse), C.POINTER(ExfMeshData)]),
    ("exf_mesh_data_free", None, [C.POINTER(ExfMeshData)]),
    ("exf_mesh_refine", _I, [C.POINTER(ExfMeshCoarse), C.POINTER(_P)]),
    ("exf_sys_set_transfer", _I, [_P, _I, _I, _I, _IP, _IP, _IP, _DP]),
    ("exf_sys_get_transfer", _I, [_P, _I, _I, _I, _IP, _LP, _IP, _IP, _DP]),
    ("exf_sys_check_pattern", _I, [_P, _I, _I, _IP, _IP, _IP]),
    ("exf_write_xdmf", _I, [C.POINTER(ExfNodeFields), C.POINTER(ExfSolnOut)]),
    ("exf_print_soln", _I, [C.POINTER(_P), _I, C.POINTER(C.c_char_p), _DP, C.POINTER(ExfSolnOut)]),
    ("exf_write_xdmf_case", _I, [C.POINTER(ExfNodeFields), C.POINTER(ExfSolnOut)]),
    ("exf_print_case", _I, [C.POINTER(_P), _I, C.POINTER(C.c_char_p), _DP, C.POINTER(ExfSolnOut)]),
]


def load():
    """Load the CUDA library; raises if it has not been built (there is no fallback)."""
    global _L
    if _L is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libexfemus_b200.so not built: run python -m exfemus_b200.build")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _L = L
    return _L


def check(rc):
    if rc != EXF_OK:
        msg = load().exf_last_error().decode(errors="replace")
        raise ExfError(rc, msg)
    return rc


def dptr(a):
    return a.ctypes.data_as(_DP)


def iptr(a):
    return a.ctypes.data_as(_IP)
