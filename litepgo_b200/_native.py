"""ctypes binding of liblpg_b200.so (the C ABI declared in include/litepgo_b200.h).

The CUDA library is the only compute path: if it cannot be loaded, importing this
module raises ImportError. There is no CPU fallback.
"""

import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_lib" / "liblpg_b200.so"

LPG_OK, LPG_EINVAL, LPG_EDOMAIN, LPG_EBUSY, LPG_ENOCONV, LPG_ECUDA, LPG_ELOGIC, LPG_EIO, LPG_ESTOPPED = range(9)
HESSIAN_NONE, HESSIAN_EXACT, HESSIAN_PROJECTED = range(3)
PRECISION_F64, PRECISION_MIXED = 0, 1
MEM_HOST, MEM_DEVICE = 0, 1
LAYOUT_BSR, LAYOUT_CSC = 0, 1

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p
_int = ctypes.c_int
_dbl = ctypes.c_double


class LitepgoError(RuntimeError):
    """A call into the CUDA library failed for a reason other than bad input."""


class NewtonOptionsC(ctypes.Structure):
    _fields_ = [
        ("gradient_tolerance", ctypes.c_double),
        ("max_iterations", ctypes.c_int),
        ("hessian", ctypes.c_int),
        ("max_line_search_steps", ctypes.c_int),
        ("line_search_shrink", ctypes.c_double),
        ("stop_rule", ctypes.c_int),
        ("accept_rule", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("cg_tolerance", ctypes.c_double),
        ("cg_max_iterations", ctypes.c_int),
        ("exact_below", ctypes.c_double),
    ]


class NewtonResultC(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("energy", ctypes.c_double),
        ("gradient_norm", ctypes.c_double),
        ("gradient_norm0", ctypes.c_double),
        ("cg_iterations", ctypes.c_int64),
        ("line_search_evaluations", ctypes.c_int),
        ("seconds", ctypes.c_double),
    ]


class BatchMeshResultC(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("energy", ctypes.c_double),
        ("gradient_norm", ctypes.c_double),
        ("gradient_norm0", ctypes.c_double),
        ("seconds", ctypes.c_double),
    ]


class NewtonStepC(ctypes.Structure):
    _fields_ = [
        ("iteration", ctypes.c_int),
        ("energy", ctypes.c_double),
        ("gradient_norm", ctypes.c_double),
        ("pattern_changed", ctypes.c_int),
        ("diagonal_shifts", ctypes.c_int),
        ("feasible_step", ctypes.c_double),
        ("step", ctypes.c_double),
        ("line_search_evaluations", ctypes.c_int),
        ("gradient_norm_2", ctypes.c_double),
        ("cg_iterations", ctypes.c_int64),
    ]


NEWTON_CALLBACK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.POINTER(NewtonStepC), ctypes.c_void_p)
# (F, rows, want, W, P, A, user) and (F, G, rows, alpha, user): device pointers as integers.
MATERIAL_CALLBACK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)
FEASIBLE_CALLBACK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_double), ctypes.c_void_p)


class NewtonTermsC(ctypes.Structure):
    _fields_ = [
        ("elastic_weight", ctypes.c_double),
        ("a_indptr", _ip),
        ("a_indices", _ip),
        ("a_values", _dp),
        ("constant", ctypes.c_double),
        ("on_iteration", NEWTON_CALLBACK),
        ("user", ctypes.c_void_p),
        ("material", MATERIAL_CALLBACK),
        ("feasible", FEASIBLE_CALLBACK),
        ("material_user", ctypes.c_void_p),
    ]


# (name, restype, argtypes) of every exported entry point, in header order.
SIGNATURES = [
    ("lpg_last_error", ctypes.c_char_p, []),
    ("lpg_abi_version", _int, []),
    ("lpg_build_info", _int, [ctypes.c_char_p, ctypes.c_size_t]),
    ("lpg_mesh_pattern_bsr", _int, [_int, _int, _ip, _i64p, _ip, _ip]),
    ("lpg_mesh_cluster_summary", _int, [_int, _int, _ip, _i64p]),
    ("lpg_fem_create", _int, [_int, _dp, _int, _ip, _dp, _dp, _int, _dp, _int, ctypes.POINTER(_vp)]),
    ("lpg_fem_destroy", _int, [_vp]),
    ("lpg_fem_set_stream", _int, [_vp, _vp]),
    ("lpg_fem_sizes", _int, [_vp, ctypes.POINTER(_int), ctypes.POINTER(_int), ctypes.POINTER(_int), _i64p, _i64p]),
    ("lpg_fem_pattern_bsr", _int, [_vp, _ip, _ip]),
    ("lpg_fem_pattern_csc", _int, [_vp, _ip, _ip]),
    ("lpg_fem_eval", _int, [_vp, _vp, _int, _dp, _vp, _int, _int, _int, _vp, _int]),
    ("lpg_fem_time_eval", _int, [_vp, _vp, _vp, _int, _int, _int, _vp, _int, _int, _dp, _dp]),
    ("lpg_fem_solver_layout", _int, [_vp, _i64p, ctypes.POINTER(_int), _ip, _ip]),
    ("lpg_fem_element_energies", _int, [_vp, _vp, _int, _vp]),
    ("lpg_fem_feasible_step", _int, [_vp, _vp, _vp, _int, _dp]),
    ("lpg_fem_feasible_step_noalloc", _int, [_vp, _vp, _vp, _dp]),
    ("lpg_fem_force_vjp_theta", _int, [_vp, _vp, _vp, _int, _int, _vp]),
    ("lpg_newton_default_options", None, [ctypes.POINTER(NewtonOptionsC)]),
    ("lpg_newton_solve", _int, [_vp, _ip, _int, _vp, _vp, _int, ctypes.POINTER(NewtonOptionsC), _vp,
                                ctypes.POINTER(NewtonResultC)]),
    ("lpg_newton_solve_terms", _int, [_vp, ctypes.POINTER(NewtonTermsC), _ip, _int, _vp, _vp, _int,
                                      ctypes.POINTER(NewtonOptionsC), _vp, ctypes.POINTER(NewtonResultC)]),
    ("lpg_adjoint_solve_terms", _int, [_vp, ctypes.POINTER(NewtonTermsC), _vp, _vp, _ip, _int, _int, _int, _dbl, _vp]),
    ("lpg_batch_newton_solve", _int, [_vp, _int, _ip, _ip, _ip, _int, _vp, _vp, _int, ctypes.POINTER(NewtonOptionsC),
                                      _vp, ctypes.POINTER(BatchMeshResultC), ctypes.POINTER(NewtonResultC)]),
    ("lpg_adjoint_theta", _int, [_vp, _vp, _vp, _ip, _int, _int, _int, _dbl, _int, _vp, _vp]),
    ("lpg_fem_force_vjp_rest", _int, [_vp, _vp, _vp, _int, _vp]),
    ("lpg_adjoint_rest", _int, [_vp, _vp, _vp, _ip, _int, _int, _int, _dbl, _vp, _vp]),
    ("lpg_fem_set_theta", _int, [_vp, _dp, _int]),
    ("lpg_fem_autotune", _int, [_vp]),
    ("lpg_mesh_cluster_summary_cells", _int, [_int, _int, _ip, _int, _i64p]),
    ("lpg_fem_create_hex", _int, [_int, _dp, _int, _ip, _dp, _int, _int, _int, ctypes.POINTER(_vp)]),
    ("lpg_fem_create_hex_hermite", _int, [_int, _dp, _int, _ip, _dp, _int, _int, _int, ctypes.POINTER(_vp)]),
    ("lpg_fem_deformation_gradients", _int, [_vp, _vp, _int, _vp]),
    ("lpg_fem_eval_material", _int, [_vp, _vp, _vp, _vp, _int, _dp, _vp, _int, _int, _int, _vp, _int]),
    ("lpg_fem_set_fp", _int, [_vp, _dp, _int]),
    ("lpg_fem_force_vjp_fp", _int, [_vp, _vp, _vp, _int, _int, _vp]),
    ("lpg_adjoint_fp", _int, [_vp, _vp, _vp, _ip, _int, _int, _int, _dbl, _int, _vp, _vp]),
    ("lpg_read_veg", _int, [ctypes.c_char_p, ctypes.POINTER(_int), ctypes.POINTER(_int), ctypes.POINTER(_int), _dp, _ip]),
    ("lpg_write_veg", _int, [ctypes.c_char_p, _int, _dp, _int, _int, _ip]),
    ("lpg_fem_get_tuning", _int, [_vp, _ip, _dp]),
    ("lpg_fem_set_tuning", _int, [_vp, _ip]),
]

EXPORTED = [name for name, _, _ in SIGNATURES]


def _load():
    if not LIB_PATH.exists():
        raise ImportError(
            f"litepgo_b200: CUDA library {LIB_PATH} is not built; run `python -m litepgo_b200.build` "
            "(there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, restype, argtypes in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    return lib


lib = _load()


def error_message():
    return lib.lpg_last_error().decode(errors="replace")


def check(code):
    """Translates a status into the exception the reference binding raises."""
    if code == LPG_OK:
        return
    msg = error_message()
    if code in (LPG_EINVAL, LPG_EDOMAIN):
        raise ValueError(msg)
    raise LitepgoError(msg)


def build_info():
    buf = ctypes.create_string_buffer(256)
    check(lib.lpg_build_info(buf, 256))
    return buf.value.decode()


def as_f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def dptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def iptr(a):
    return None if a is None else a.ctypes.data_as(_ip)


def vptr(a):
    """void* of a NumPy array or a torch tensor."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(_vp)
