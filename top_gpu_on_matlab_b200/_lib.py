"""ctypes loader of libtopgpu.so (the package's CUDA library for sm_100a).

The library is built in-tree by ``python -m top_gpu_on_matlab_b200.build``
(or ``make -C top_gpu_on_matlab_b200/csrc``).  Importing this module without
the built library raises ImportError: there is no CPU fallback.
"""
import ctypes as C
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libtopgpu.so"

TOP_OK = 0
TOP_ERR_ARGS = -1
TOP_ERR_TYPE = -2
TOP_ERR_SHAPE = -3
TOP_ERR_CUDA = -4
TOP_ERR_NOT_CONVERGED = -5
TOP_ERR_NAN = -6
TOP_ERR_NOMEM = -7
TOP_ERR_STATE = -8
TOP_F32 = 1
TOP_F64 = 2
TOP_PREC_FP64 = 0
TOP_PREC_MIXED = 1

_ERR_NAMES = {
    TOP_ERR_ARGS: "Args", TOP_ERR_TYPE: "Type", TOP_ERR_SHAPE: "Shape", TOP_ERR_CUDA: "CUDA",
    TOP_ERR_NOT_CONVERGED: "NotConverged", TOP_ERR_NAN: "NaN", TOP_ERR_NOMEM: "NoMem",
    TOP_ERR_STATE: "State",
}


class TopGpuError(RuntimeError):
    """Error raised for a non-zero status of libtopgpu.so.

    ``identifier`` follows MATLAB's mexErrMsgIdAndTxt convention,
    e.g. ``Gathering_inplace:Shape``.
    """

    def __init__(self, status, name, message):
        self.status = status
        self.identifier = "%s:%s" % (name, _ERR_NAMES.get(status, "Error"))
        super().__init__("%s (%d): %s" % (self.identifier, status, message))


class SolverParams(C.Structure):
    _fields_ = [
        ("E0", C.c_double), ("Emin", C.c_double), ("penal", C.c_double),
        ("tol", C.c_double), ("maxIT", C.c_int), ("omega", C.c_double),
        ("precision", C.c_int), ("outerFP32", C.c_int),
    ]


class SensParams(C.Structure):
    _fields_ = [("objective", C.c_int), ("loadCase", C.c_int), ("dof", C.c_int64), ("ft", C.c_int), ("tol", C.c_double)]


class OptParams(C.Structure):
    _fields_ = [("V0", C.c_double), ("rMin", C.c_double), ("nLoop", C.c_int), ("ft", C.c_int)]


class OptRecord(C.Structure):
    _fields_ = [("c", C.c_double), ("vol", C.c_double), ("sharp", C.c_double), ("cons", C.c_double),
                ("change", C.c_double), ("pcgIts", C.c_int), ("msAssemble", C.c_double), ("msSolve", C.c_double),
                ("msOpt", C.c_double), ("msFilter", C.c_double), ("msTotal", C.c_double)]


_vp, _i32p, _i64, _int, _dbl = C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_double

SIGNATURES = {
    "top_last_error": (C.c_char_p, []),
    "top_version": (_int, []),
    "top_gather": (_int, [_vp, _vp, _vp, _int, _i64, _i64, _int, _vp]),
    "top_scatter": (_int, [_vp, _vp, _vp, _i64, _i64, _int, _vp]),
    "top_scatter_accum3": (_int, [_vp, _vp, _i64, _vp, _i64, _int, _vp]),
    "top_assemble_ks_level2": (_int, [_vp] * 8 + [_i64, _int, _i64, _i64, _int, _vp]),
    "top_assemble_ks_level2_noalloc": (_int, [_vp] * 8 + [_i64, _int, _i64, _i64, _int, _vp]),
    "top_assemble_ks_higher": (_int, [_vp] * 4 + [_i64, _int, _i64, _int, _vp]),
    "top_assemble_ks_level2_super": (_int, [_vp] * 8 + [_i64, _int, _i64, _i64, _int, _vp]),
    "top_mesh_create": (_int, [_vp, _int, _int, _int, _int, _dbl, _dbl, _int, _vp]),
    "top_mesh_destroy": (_int, [_vp]),
    "top_mesh_apply_optcase": (_int, [_vp, _int]),
    "top_mesh_apply_bc": (_int, [_vp, _i64, _vp, _int, _vp, _vp, _vp]),
    "top_mesh_create_from_topvoxel": (_int, [C.c_char_p, _int, _dbl, _vp]),
    "top_mesh_info": (_int, [_vp, _vp, _int]),
    "top_mesh_get": (_int, [_vp, _int, C.c_char_p, _vp, _i64, _vp]),
    "top_solver_create": (_int, [_vp, _vp, _vp]),
    "top_solver_destroy": (_int, [_vp]),
    "top_solver_set_stream": (_int, [_vp, _vp]),
    "top_solver_set_modulus": (_int, [_vp, _vp, _int]),
    "top_solver_set_density": (_int, [_vp, _vp, _int]),
    "top_solver_assemble": (_int, [_vp]),
    "top_solver_matvec": (_int, [_vp, _int, _vp, _vp, _int]),
    "top_solver_vcycle": (_int, [_vp, _vp, _vp]),
    "top_solver_restrict": (_int, [_vp, _int, _vp, _vp]),
    "top_solver_interpolate": (_int, [_vp, _int, _vp, _vp]),
    "top_solver_get_diag": (_int, [_vp, _int, _vp]),
    "top_solver_get_ks": (_int, [_vp, _int, _vp]),
    "top_solver_pcg": (_int, [_vp, _int, _vp, _int, _vp, _vp]),
    "top_solver_pcg_rhs": (_int, [_vp, _vp, _vp, _int, _vp, _vp]),
    "top_solver_pcg_all": (_int, [_vp, _vp, _int, _vp, _vp]),
    "top_solver_unit_compliance": (_int, [_vp, _vp, _vp]),
    "top_solver_sizes": (_int, [_vp, _vp]),
    "top_solver_time_kernel": (_int, [_vp, _int, _int, _i64, _vp]),
    "top_solver_filter_setup": (_int, [_vp, _dbl]),
    "top_solver_filter": (_int, [_vp, _vp, _vp, _vp]),
    "top_solver_super_filter_setup": (_int, [_vp, _dbl]),
    "top_solver_super_filter": (_int, [_vp, _vp, _vp, _int]),
    "top_solver_opt_begin": (_int, [_vp, _vp, _vp]),
    "top_solver_set_passive": (_int, [_vp, _vp, _i64]),
    "top_solver_opt_step": (_int, [_vp, _vp]),
    "top_solver_opt_state": (_int, [_vp, _vp, _vp, _vp]),
    "top_solver_opt_case_its": (_int, [_vp, _vp, _int, _vp]),
    "top_solver_get_design": (_int, [_vp, _vp, _vp]),
    "top_solver_set_design": (_int, [_vp, _vp, _vp]),
    "top_solver_launch_count": (_int, [_vp, _vp]),
    "top_solver_set_l0_kernel": (_int, [_vp, _int, _int, _int, _int, _int]),
    "top_solver_get_l0_kernel": (_int, [_vp, _int, _vp]),
    "top_solver_autotune": (_int, [_vp, _int, _i64, _vp, _vp]),
    "top_solver_set_graphs": (_int, [_vp, _int]),
    "top_solver_set_pcg_beta": (_int, [_vp, _int]),
    "top_solver_test_withhold_tile": (_int, [_vp]),
    "top_solver_set_tail_operator": (_int, [_vp, _int, _vp]),
    "top_solver_set_coarse_persistent": (_int, [_vp, _int]),
    "top_solver_sensitivity": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "top_solver_optimize": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
}

_LIB = None


def lib():
    """Load libtopgpu.so (once) and declare its C ABI."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise ImportError(
                "libtopgpu.so is not built (%s); run `make -C top_gpu_on_matlab_b200/csrc` "
                "or __graft_entry__.build()" % LIB_PATH)
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def last_error() -> str:
    msg = lib().top_last_error()
    return msg.decode() if msg else ""


def check(status, name):
    if status != TOP_OK:
        raise TopGpuError(status, name, last_error())
    return status
