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


class Terms(ctypes.Structure):
    _fields_ = [
        ("elastic_weight", ctypes.c_double),
        ("a_indptr", _c_int_p),
        ("a_indices", _c_int_p),
        ("a_values", _c_double_p),
        ("constant", ctypes.c_double),
    ]


# Fields of one NewtonStep trace record (orc_newton_solve_ex).
TRACE_FIELDS = ("iteration", "energy", "gradient_norm", "diagonal_shifts", "feasible_step", "step",
                "line_search_evaluations")

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
        L.orc_newton_solve_ex.argtypes = [ctypes.c_void_p, ctypes.POINTER(Terms), _c_int_p, ctypes.c_int, _c_double_p,
                                          _c_double_p, ctypes.POINTER(NewtonOptions), _c_double_p,
                                          ctypes.POINTER(NewtonResult), _c_double_p, ctypes.c_int, _c_int_p]
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
               shrink=0.5, stop_rule=0, accept_rule=0, linear_solver=0, cg_tolerance=1e-2, cg_max_iterations=10000,
               elastic_weight=1.0, A=None, constant=0.0, trace=False):
        """Newton over E = w elastic + 1/2 x^T A x - f_ext . x + constant (A a symmetric scipy
        matrix or None). With trace, info["trace"] lists one dict per NewtonStep."""
        fixed = np.ascontiguousarray(fixed, dtype=np.int32)
        x0 = np.ascontiguousarray(x0, dtype=np.float64)
        f = None if f_ext is None else np.ascontiguousarray(f_ext, dtype=np.float64)
        opts = NewtonOptions(tol, max_iterations, hessian, max_line_search_steps, shrink, stop_rule, accept_rule,
                             linear_solver, cg_tolerance, cg_max_iterations)
        x = np.empty(self.num_dofs)
        res = NewtonResult()
        keep = []
        terms = None
        if elastic_weight != 1.0 or A is not None or constant != 0.0:
            terms = Terms(float(elastic_weight), None, None, None, float(constant))
            if A is not None:
                import scipy.sparse as sp

                Ac = sp.csr_matrix(A)
                Ac.sum_duplicates()
                Ac.sort_indices()
                keep = [np.ascontiguousarray(Ac.indptr, dtype=np.int32), np.ascontiguousarray(Ac.indices, dtype=np.int32),
                        np.ascontiguousarray(Ac.data, dtype=np.float64)]
                terms.a_indptr, terms.a_indices, terms.a_values = _ip(keep[0]), _ip(keep[1]), _dp(keep[2])
        cap = max_iterations + 2
        buf = np.zeros((cap, 7))
        count = ctypes.c_int(0)
        _check(lib().orc_newton_solve_ex(self._h, ctypes.byref(terms) if terms is not None else None, _ip(fixed),
                                         len(fixed), _dp(f), _dp(x0), ctypes.byref(opts), _dp(x), ctypes.byref(res),
                                         _dp(buf), cap, ctypes.byref(count)))
        del keep
        info = {name: getattr(res, name) for name, _ in NewtonResult._fields_}
        if trace:
            info["trace"] = [dict(zip(TRACE_FIELDS, row)) for row in buf[:count.value]]
        return x, info

    def adjoint_theta(self, u_star, dLdu, fixed, linear_solver=0, cg_tolerance=1e-12):
        fixed = np.ascontiguousarray(fixed, dtype=np.int32)
        out = np.empty((self.num_tets, 2))
        lam = np.empty(self.num_dofs)
        _check(lib().orc_adjoint_theta(self._h, _dp(np.ascontiguousarray(u_star, float)),
                                       _dp(np.ascontiguousarray(dLdu, float)), _ip(fixed), len(fixed),
                                       int(linear_solver), float(cg_tolerance), _dp(out), _dp(lam)))
        return out, lam


# ---------------------------------------------------------------------------
# Hex Q1 elements (test infrastructure, NumPy): the reference's trilinear HexQ1Basis
# (src/core/fem/basis/3d/hex_q1_basis.hpp: corners (0,0,0), (1,0,0), (1,1,0), (0,1,0), (0,0,1),
# (1,0,1), (1,1,1), (0,1,1) of [0,1]^3) with Gauss-Legendre points on [0,1]^3, last axis fastest
# (src/core/fem/quadrature/3d/gauss_legendre_3d.hpp; 1D rules of
# quadrature/1d/gauss_legendre_1d.hpp), the point weight w_q det J_q
# (fem/integration/volumetric_element.hpp:23-39, det J <= 0 rejected), F = I + sum_a u_a grad N_a^T
# (deformation_gradient_sampling_response.hpp:15-45) and the element sums w B^T vec P,
# w B^T A B (fem/assembly/dof_derivatives.cpp:22-51) with this oracle's NeoHookean W, P, A.
# ---------------------------------------------------------------------------
HEX_CORNERS = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])


def gauss_legendre_01(n):
    """Points and weights of the n-point Gauss-Legendre rule on [0, 1] (n = 2 or 4)."""
    if n == 2:
        return np.array([0.5 - 0.5 / np.sqrt(3.0), 0.5 + 0.5 / np.sqrt(3.0)]), np.array([0.5, 0.5])
    if n == 4:
        outer = np.sqrt((3 + 2 * np.sqrt(6.0 / 5)) / 7)
        inner = np.sqrt((3 - 2 * np.sqrt(6.0 / 5)) / 7)
        wo, wi = (18 - np.sqrt(30.0)) / 72, (18 + np.sqrt(30.0)) / 72
        return (np.array([0.5 * (1 - outer), 0.5 * (1 - inner), 0.5 * (1 + inner), 0.5 * (1 + outer)]),
                np.array([wo, wi, wi, wo]))
    raise ValueError("Gauss-Legendre rule with 2 or 4 points per axis")


def hex_points(n):
    t, w = gauss_legendre_01(n)
    pts, wts = [], []
    for i in range(n):
        for j in range(n):
            for k in range(n):
                pts.append([t[i], t[j], t[k]])
                wts.append(w[i] * w[j] * w[k])
    return np.array(pts), np.array(wts)


def hex_dN_dxi(xi):
    """(8, 3) derivatives of the trilinear basis at xi in [0,1]^3."""
    out = np.empty((8, 3))
    for a, (i, j, k) in enumerate(HEX_CORNERS):
        f = [(1 - xi[d], xi[d]) for d in range(3)]
        df = [(-1.0, 1.0)] * 3
        out[a] = [df[0][i] * f[1][j] * f[2][k], f[0][i] * df[1][j] * f[2][k], f[0][i] * f[1][j] * df[2][k]]
    return out


def hex_eval(X, cells, theta, u, points_per_axis=2, hessian=True, projected=False):
    """E, gradient and dense Hessian (or None) of the hex Q1 neo-Hookean energy (Fp = I); with
    projected, each element's 24x24 Hessian is projected (project_psd) before assembly."""
    X = np.asarray(X, float).reshape(-1, 3)
    cells = np.asarray(cells).reshape(-1, 8)
    U = np.asarray(u, float).reshape(-1, 3)
    T, n = cells.shape[0], X.size
    th = np.broadcast_to(np.asarray(theta, float), (T, 2))
    pts, wts = hex_points(points_per_axis)
    E, g = 0.0, np.zeros(n)
    H = np.zeros((n, n)) if hessian else None
    for e, cell in enumerate(cells):
        dofs = (3 * cell[:, None] + np.arange(3)).ravel()
        ge, He = np.zeros(24), np.zeros((24, 24))
        for xi, wq in zip(pts, wts):
            dN = hex_dN_dxi(xi)
            J = X[cell].T @ dN  # J[i, d] = dX_i / dxi_d
            det = np.linalg.det(J)
            if not det > 0:
                raise ValueError("VolumetricElement3D: invalid reference determinant or volume weight")
            gN = dN @ np.linalg.inv(J)  # rows grad_X N_a
            F = np.eye(3) + U[cell].T @ gN
            w = wq * det
            E += w * nh_W(F, np.eye(3), th[e])
            P = nh_dW_dF(F, np.eye(3), th[e])
            B = np.zeros((9, 24))  # column-major vec(F): r = i + 3 j
            for a in range(8):
                for i in range(3):
                    for j in range(3):
                        B[i + 3 * j, 3 * a + i] = gN[a, j]
            ge += w * B.T @ P.T.ravel()
            if hessian:
                He += w * B.T @ nh_d2W_dF2(F, np.eye(3), th[e]) @ B
        g[dofs] += ge
        if hessian:
            H[np.ix_(dofs, dofs)] += project_psd(He) if projected else He
    return E, g, H


def hex_force_vjp_theta(X, cells, theta, u, w, points_per_axis=2):
    """(d g / d theta)^T w per hex (T, 2) for the hex Q1 neo-Hookean force g (Fp = I): at every
    point w_q d2W/dF dtheta : grad w (VolumetricFemForceMaterialResponse over the hex basis)."""
    X = np.asarray(X, float).reshape(-1, 3)
    cells = np.asarray(cells).reshape(-1, 8)
    U = np.asarray(u, float).reshape(-1, 3)
    Wv = np.asarray(w, float).reshape(-1, 3)
    T = cells.shape[0]
    th = np.broadcast_to(np.asarray(theta, float), (T, 2))
    pts, wts = hex_points(points_per_axis)
    out = np.zeros((T, 2))
    for e, cell in enumerate(cells):
        for xi, wq in zip(pts, wts):
            dN = hex_dN_dxi(xi)
            J = X[cell].T @ dN
            gN = dN @ np.linalg.inv(J)
            F = np.eye(3) + U[cell].T @ gN
            Gw = Wv[cell].T @ gN  # grad w, [i, j]
            D = nh_d2W_dF_dtheta(F, np.eye(3), th[e])  # (9, 2), rows column-major vec(F)
            out[e] += wq * np.linalg.det(J) * (D.T @ Gw.T.ravel())
    return out


# Tricubic Hermite hexes (hex_hermite_basis.hpp, cubic_hermite_basis.hpp): 64 functions, index
# 8 * corner + slot, slot derivative orders below; per vertex 24 physical DOFs (slot-major, 3 per
# slot: u, u_X, u_Y, u_Z, u_XY, u_XZ, u_YZ, u_XYZ), scaled to reference coefficients by
# 1, hx, hy, hz, hx hy, hx hz, hy hz, hx hy hz on an axis-aligned box (basis_dof_transform.hpp:59-148).
HERMITE_ORDERS = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0], [1, 0, 1], [0, 1, 1], [1, 1, 1]])


def cubic_hermite(t):
    """1D cubic Hermite values and t-derivatives ordered u(0), u'(0), u(1), u'(1)."""
    t2, t3 = t * t, t * t * t
    N = np.array([2 * t3 - 3 * t2 + 1, t3 - 2 * t2 + t, -2 * t3 + 3 * t2, t3 - t2])
    dN = np.array([6 * t2 - 6 * t, 3 * t2 - 4 * t + 1, -6 * t2 + 6 * t, 3 * t2 - 2 * t])
    return N, dN


def hex_hermite_N_dN(xi):
    """(64,) values and (64, 3) reference gradients of the tricubic Hermite functions at xi."""
    (x, dx), (y, dy), (z, dz) = (cubic_hermite(c) for c in xi)
    N, dN = np.empty(64), np.empty((64, 3))
    for row in range(64):
        corner, order = HEX_CORNERS[row // 8], HERMITE_ORDERS[row % 8]
        i, j, k = 2 * corner + order
        N[row] = x[i] * y[j] * z[k]
        dN[row] = [dx[i] * y[j] * z[k], x[i] * dy[j] * z[k], x[i] * y[j] * dz[k]]
    return N, dN


def hermite_box(Xc):
    """Edge lengths of an axis-aligned box in corner order (the reference's check: positive lengths,
    normalized corners equal to the unit corners within 1e-12); ValueError otherwise."""
    origin = Xc[0]
    h = np.array([Xc[1, 0] - origin[0], Xc[3, 1] - origin[1], Xc[4, 2] - origin[2]])
    if not np.all(np.isfinite(h)) or np.any(h <= 0):
        raise ValueError("Hermite DOF transform requires positive axis-aligned box dimensions")
    if np.abs((Xc - origin) / h - HEX_CORNERS).max() > 1e-12:
        raise ValueError("Hermite DOF transform requires axis-aligned boxes in Hex corner order")
    return h


def hermite_slot_scales(h):
    return np.array([1, h[0], h[1], h[2], h[0] * h[1], h[0] * h[2], h[1] * h[2], h[0] * h[1] * h[2]])


def hex_hermite_eval(X, cells, theta, u, points_per_axis=2, hessian=True, projected=False):
    """E, gradient and dense Hessian (or None) over the physical DOFs (24 per vertex) of the
    tricubic Hermite neo-Hookean energy on axis-aligned box hexes (Fp = I): reference coefficients
    c = s * d, F = I + sum_b c_b (J^-T dN_b), J = diag(h), and the element gradient and Hessian
    pulled back by the same scales (s g, S H S). With projected, each element's 192 x 192
    Hessian (over its physical DOFs) is projected (project_psd) before assembly, as
    MeshEnergy does for HessianKind::Projected (mesh_energy.cpp:16-27)."""
    X = np.asarray(X, float).reshape(-1, 3)
    cells = np.asarray(cells).reshape(-1, 8)
    D = np.asarray(u, float).reshape(-1, 24)
    T, n = cells.shape[0], D.size
    th = np.broadcast_to(np.asarray(theta, float), (T, 2))
    pts, wts = hex_points(points_per_axis)
    tables = [hex_hermite_N_dN(xi)[1] for xi in pts]
    E, g = 0.0, np.zeros(n)
    H = np.zeros((n, n)) if hessian else None
    for e, cell in enumerate(cells):
        h = hermite_box(X[cell])
        s = np.repeat(np.tile(hermite_slot_scales(h), 8), 3)  # per local DOF, 192
        dofs = (24 * cell[:, None] + np.arange(24)).ravel()
        C = (D[cell].ravel() * s).reshape(64, 3)
        ge, He = np.zeros(192), np.zeros((192, 192))
        for dN, wq in zip(tables, wts):
            gN = dN / h  # rows grad_X N_b (J^-T = diag(1 / h))
            F = np.eye(3) + C.T @ gN
            w = wq * np.prod(h)
            E += w * nh_W(F, np.eye(3), th[e])
            B = np.zeros((9, 192))  # column-major vec(F): r = i + 3 j
            for b in range(64):
                for i in range(3):
                    for j in range(3):
                        B[i + 3 * j, 3 * b + i] = gN[b, j]
            ge += w * B.T @ nh_dW_dF(F, np.eye(3), th[e]).T.ravel()
            if hessian:
                He += w * B.T @ nh_d2W_dF2(F, np.eye(3), th[e]) @ B
        g[dofs] += s * ge
        if hessian:
            Hp = s[:, None] * He * s[None, :]
            H[np.ix_(dofs, dofs)] += project_psd(Hp) if projected else Hp
    return E, g, H


def hex_hermite_force_vjp_theta(X, cells, theta, u, w, points_per_axis=2):
    """(d g / d theta)^T w per Hermite hex (T, 2) over physical DOFs u, w (24 per vertex): at every
    point w_q d2W/dF dtheta : grad w, with grad w = sum_b (s_b w_b) (J^-T dN_b)."""
    X = np.asarray(X, float).reshape(-1, 3)
    cells = np.asarray(cells).reshape(-1, 8)
    D = np.asarray(u, float).reshape(-1, 24)
    Wv = np.asarray(w, float).reshape(-1, 24)
    T = cells.shape[0]
    th = np.broadcast_to(np.asarray(theta, float), (T, 2))
    pts, wts = hex_points(points_per_axis)
    out = np.zeros((T, 2))
    for e, cell in enumerate(cells):
        h = hermite_box(X[cell])
        s = np.repeat(np.tile(hermite_slot_scales(h), 8), 3)
        C = (D[cell].ravel() * s).reshape(64, 3)
        Cw = (Wv[cell].ravel() * s).reshape(64, 3)
        for xi, wq in zip(pts, wts):
            gN = hex_hermite_N_dN(xi)[1] / h
            F = np.eye(3) + C.T @ gN
            Gw = Cw.T @ gN
            Dth = nh_d2W_dF_dtheta(F, np.eye(3), th[e])  # (9, 2), rows column-major vec(F)
            out[e] += wq * np.prod(h) * (Dth.T @ Gw.T.ravel())
    return out


def hex_box(nx, ny=None, nz=None):
    """Structured box of nx*ny*nz unit-spacing-scaled hexes on [0,1]^3 (corner order above)."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    xs, ys, zs = (np.arange(m + 1) / m for m in (nx, ny, nz))
    Z, Y, Xg = np.meshgrid(zs, ys, xs, indexing="ij")
    P = np.stack([Xg.ravel(), Y.ravel(), Z.ravel()], 1)
    idx = lambda i, j, k: i + (nx + 1) * (j + (ny + 1) * k)  # noqa: E731
    cells = [[idx(i + c[0], j + c[1], k + c[2]) for c in HEX_CORNERS]
             for k in range(nz) for j in range(ny) for i in range(nx)]
    return P, np.array(cells, np.int32)
