"""ctypes wrapper for the C++ oracle (test infrastructure only; see lpg_oracle.h)."""

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liblpg_oracle.so"

_c_double_p = ctypes.POINTER(ctypes.c_double)
_c_int_p = ctypes.POINTER(ctypes.c_int)


class OracleError(Exception):
    """An oracle call failed; ``code`` mirrors the reference exception class."""

    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


# Reference exception classes by code.
INVALID_ARGUMENT, DOMAIN_ERROR, LOGIC_ERROR = 1, 2, 6


def build(force=False):
    """Compile the oracle with its Makefile (g++ -fopenmp)."""
    sources = [HERE / "lpg_oracle.cpp", HERE / "lpg_oracle.h"]
    if not force and LIB_PATH.exists() and all(LIB_PATH.stat().st_mtime >= s.stat().st_mtime for s in sources):
        return LIB_PATH
    subprocess.run(["make", "-C", str(HERE)], check=True, stdout=subprocess.DEVNULL)
    return LIB_PATH


class NewtonOptions(ctypes.Structure):
    _fields_ = [
        ("gradient_tolerance", ctypes.c_double),
        ("max_iterations", ctypes.c_int),
        ("hessian", ctypes.c_int),
        ("max_line_search_steps", ctypes.c_int),
        ("line_search_shrink", ctypes.c_double),
        ("stop_rule", ctypes.c_int),
        ("accept_rule", ctypes.c_int),
        ("linear_solver", ctypes.c_int),
        ("cg_tolerance", ctypes.c_double),
        ("cg_max_iterations", ctypes.c_int),
    ]


class NewtonResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("iterations", ctypes.c_int),
        ("energy", ctypes.c_double),
        ("gradient_norm", ctypes.c_double),
        ("gradient_norm0", ctypes.c_double),
        ("cg_iterations", ctypes.c_longlong),
        ("line_search_evaluations", ctypes.c_int),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_mesh_nnz.restype = ctypes.c_longlong
        L.orc_mesh_create.argtypes = [ctypes.c_int, _c_double_p, ctypes.c_int, _c_int_p, _c_double_p, _c_double_p,
                                      ctypes.c_int, _c_double_p, ctypes.POINTER(ctypes.c_void_p)]
        L.orc_mesh_destroy.argtypes = [ctypes.c_void_p]
        L.orc_mesh_num_dofs.argtypes = [ctypes.c_void_p]
        L.orc_mesh_nnz.argtypes = [ctypes.c_void_p]
        L.orc_mesh_pattern.argtypes = [ctypes.c_void_p, _c_int_p, _c_int_p]
        L.orc_mesh_eval.argtypes = [ctypes.c_void_p, _c_double_p, _c_double_p, _c_double_p, ctypes.c_int, _c_double_p,
                                    _c_double_p, _c_double_p, _c_double_p]
        L.orc_mesh_feasible_step.argtypes = [ctypes.c_void_p, _c_double_p, _c_double_p, _c_double_p]
        L.orc_mesh_force_vjp_theta.argtypes = [ctypes.c_void_p, _c_double_p, _c_double_p, _c_double_p]
        L.orc_mesh_force_vjp_rest.argtypes = [ctypes.c_void_p, _c_double_p, _c_double_p, _c_double_p]
        L.orc_mesh_force_vjp_fp.argtypes = [ctypes.c_void_p, _c_double_p, _c_double_p, _c_double_p]
        L.orc_newton_solve.argtypes = [ctypes.c_void_p, _c_int_p, ctypes.c_int, _c_double_p, _c_double_p,
                                       ctypes.POINTER(NewtonOptions), _c_double_p, ctypes.POINTER(NewtonResult)]
        L.orc_adjoint_theta.argtypes = [ctypes.c_void_p, _c_double_p, _c_double_p, _c_int_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, _c_double_p, _c_double_p]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _check(code):
    if code != 0:
        raise OracleError(code, lib().orc_last_error().decode())


def _dp(a):
    return None if a is None else a.ctypes.data_as(_c_double_p)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_c_int_p)


def _m3(a):
    """A 3x3 array (row/col indexable) as a column-major contiguous 9-vector."""
    a = np.asarray(a, dtype=np.float64)
    if a.shape == (3, 3):
        return np.ascontiguousarray(a.reshape(3, 3).T.ravel())
    return np.ascontiguousarray(a.ravel())


def set_threads(n):
    lib().orc_set_threads(int(n))


def get_threads():
    return lib().orc_get_threads()


def nh_W(F, Fp, theta):
    out = ctypes.c_double()
    _check(lib().orc_nh_W(_dp(_m3(F)), _dp(_m3(Fp)), _dp(np.asarray(theta, float)), ctypes.byref(out)))
    return out.value


def nh_dW_dF(F, Fp, theta):
    out = np.empty(9)
    _check(lib().orc_nh_dW_dF(_dp(_m3(F)), _dp(_m3(Fp)), _dp(np.asarray(theta, float)), _dp(out)))
    return out.reshape(3, 3).T.copy()  # back to row/col indexing


def nh_d2W_dF2(F, Fp, theta):
    """9x9 tangent over column-major vec(F) (index i + 3 j)."""
    out = np.empty(81)
    _check(lib().orc_nh_d2W_dF2(_dp(_m3(F)), _dp(_m3(Fp)), _dp(np.asarray(theta, float)), _dp(out)))
    return out.reshape(9, 9).T.copy()


def nh_d2W_dF_dtheta(F, Fp, theta):
    out = np.empty(18)
    _check(lib().orc_nh_d2W_dF_dtheta(_dp(_m3(F)), _dp(_m3(Fp)), _dp(np.asarray(theta, float)), _dp(out)))
    return out.reshape(2, 9).T.copy()


def nh_d2W_dF_dFp(F, Fp, theta):
    out = np.empty(81)
    _check(lib().orc_nh_d2W_dF_dFp(_dp(_m3(F)), _dp(_m3(Fp)), _dp(np.asarray(theta, float)), _dp(out)))
    return out.reshape(9, 9).T.copy()


def nh_feasible_step(F, Fp, theta, dF, dFp, dtheta):
    out = ctypes.c_double()
    _check(lib().orc_nh_feasible_step(_dp(_m3(F)), _dp(_m3(Fp)), _dp(np.asarray(theta, float)), _dp(_m3(dF)),
                                      _dp(_m3(dFp)), _dp(np.asarray(dtheta, float)), ctypes.byref(out)))
    return out.value


def positive_det_step(A, dA):
    out = ctypes.c_double()
    _check(lib().orc_positive_det_step(_dp(_m3(A)), _dp(_m3(dA)), ctypes.byref(out)))
    return out.value


def project_psd(H):
    H = np.asarray(H, dtype=np.float64)
    n = H.shape[0]
    src = np.ascontiguousarray(H.T.ravel())
    out = np.empty(n * n)
    _check(lib().orc_project_psd(n, _dp(src), _dp(out)))
    return out.reshape(n, n).T.copy()


class OracleMesh:
    """VolumetricFemEnergy[NeoHookean, TetP1Basis, TetCentroidQuadrature] restated on the CPU."""

    def __init__(self, X, tets, theta, Fp=None, Xe=None):
        X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 3)
        tets = np.ascontiguousarray(tets, dtype=np.int32).reshape(-1, 4)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        per_element = theta.ndim == 2
        self.num_vertices, self.num_tets = X.shape[0], tets.shape[0]
        self._keep = [X, tets, theta]
        if Fp is not None:
            Fp = np.ascontiguousarray(Fp, dtype=np.float64).reshape(-1, 9)
            self._keep.append(Fp)
        if Xe is not None:
            Xe = np.ascontiguousarray(Xe, dtype=np.float64).reshape(-1, 12)
            self._keep.append(Xe)
        handle = ctypes.c_void_p()
        L = lib()
        _check(L.orc_mesh_create(self.num_vertices, _dp(X), self.num_tets, _ip(tets), _dp(Xe), _dp(theta),
                                 1 if per_element else 0, _dp(Fp), ctypes.byref(handle)))
        self._h = handle
        self.num_dofs = L.orc_mesh_num_dofs(self._h)
        self.nnz = int(L.orc_mesh_nnz(self._h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_mesh_destroy(h)
            self._h = None

    def pattern(self):
        outer = np.empty(self.num_dofs + 1, dtype=np.int32)
        inner = np.empty(self.nnz, dtype=np.int32)
        _check(lib().orc_mesh_pattern(self._h, _ip(outer), _ip(inner)))
        return outer, inner

    def eval(self, u, gradient=True, hessian=0, elements=False):
        """Returns (E, grad|None, csc values|None[, (elem_E, elem_g, elem_H)])."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        E = ctypes.c_double()
        g = np.empty(self.num_dofs) if gradient else None
        vals = np.empty(self.nnz) if hessian else None
        eE = np.empty(self.num_tets) if elements else None
        eg = np.empty((self.num_tets, 12)) if elements and gradient else None
        eH = np.empty((self.num_tets, 144)) if elements and hessian else None
        _check(lib().orc_mesh_eval(self._h, _dp(u), ctypes.byref(E), _dp(g), int(hessian), _dp(vals), _dp(eE),
                                   _dp(eg), _dp(eH)))
        if elements:
            if eH is not None:
                eH = eH.reshape(-1, 12, 12).transpose(0, 2, 1).copy()  # column-major -> [e, i, j]
            return E.value, g, vals, (eE, eg, eH)
        return E.value, g, vals

    def hessian_csc(self, u, kind=1):
        import scipy.sparse as sp

        outer, inner = self.pattern()
        _, _, vals = self.eval(u, gradient=False, hessian=kind)
        return sp.csc_matrix((vals, inner, outer), shape=(self.num_dofs, self.num_dofs))

    def feasible_step(self, u, du):
        out = ctypes.c_double()
        _check(lib().orc_mesh_feasible_step(self._h, _dp(np.ascontiguousarray(u, float)),
                                            _dp(np.ascontiguousarray(du, float)), ctypes.byref(out)))
        return out.value

    def force_vjp_theta(self, u, w):
        out = np.empty((self.num_tets, 2))
        _check(lib().orc_mesh_force_vjp_theta(self._h, _dp(np.ascontiguousarray(u, float)),
                                              _dp(np.ascontiguousarray(w, float)), _dp(out)))
        return out

    def force_vjp_fp(self, u, w):
        """(d g / d vec Fp)^T w per element, (T, 9) column-major Fp index."""
        out = np.empty((self.num_tets, 9))
        _check(lib().orc_mesh_force_vjp_fp(self._h, _dp(np.ascontiguousarray(u, float)),
                                           _dp(np.ascontiguousarray(w, float)), _dp(out)))
        return out

    def force_vjp_rest(self, u, w):
        """(d g / d X)^T w over the vertex rest positions (3V)."""
        out = np.empty(self.num_dofs)
        _check(lib().orc_mesh_force_vjp_rest(self._h, _dp(np.ascontiguousarray(u, float)),
                                             _dp(np.ascontiguousarray(w, float)), _dp(out)))
        return out

    def newton(self, fixed, x0, f_ext=None, tol=1e-9, max_iterations=50, hessian=2, max_line_search_steps=30,
               shrink=0.5, stop_rule=0, accept_rule=0, linear_solver=0, cg_tolerance=1e-2, cg_max_iterations=10000):
        fixed = np.ascontiguousarray(fixed, dtype=np.int32)
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        f = None if f_ext is None else np.ascontiguousarray(f_ext, dtype=np.float64)
        opts = NewtonOptions(tol, max_iterations, hessian, max_line_search_steps, shrink, stop_rule, accept_rule,
                             linear_solver, cg_tolerance, cg_max_iterations)
        x = np.empty(self.num_dofs)
        res = NewtonResult()
        _check(lib().orc_newton_solve(self._h, _ip(fixed), len(fixed), _dp(f), _dp(x0), ctypes.byref(opts), _dp(x),
                                      ctypes.byref(res)))
        info = {name: getattr(res, name) for name, _ in NewtonResult._fields_}
        return x, info

    def adjoint_theta(self, u_star, dLdu, fixed, linear_solver=0, cg_tolerance=1e-12):
        fixed = np.ascontiguousarray(fixed, dtype=np.int32)
        out = np.empty((self.num_tets, 2))
        lam = np.empty(self.num_dofs)
        _check(lib().orc_adjoint_theta(self._h, _dp(np.ascontiguousarray(u_star, float)),
                                       _dp(np.ascontiguousarray(dLdu, float)), _ip(fixed), len(fixed),
                                       int(linear_solver), float(cg_tolerance), _dp(out), _dp(lam)))
        return out, lam
