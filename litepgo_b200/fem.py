"""Volumetric neo-Hookean FEM on the GPU, mirroring litepgo.fem for the TetP1 path.

``VolumetricFemEnergy[NeoHookean, TetP1Basis, TetCentroidQuadrature](displacement_map,
rest_position_fields, Fp, theta, batch_size=256)`` keeps the reference constructor
(src/binding/fem/assembly/volumetric_fem_energy.cpp:41-47; src/python/fem.py:155-233) and
the Energy interface ``eval / eval_value / eval_gradient / eval_hessian / max_feasible_step``
(src/binding/energy/scalar/energy.cpp:26-48). Fields are sampled once at the centroid
(volumetric_fem_energy.hpp:58-63). Hessians are returned as scipy.sparse.csc_matrix with the
reference's pattern (both triangles, sorted rows). All arithmetic runs in the CUDA library;
``batch_size`` is validated and kept for interface compatibility (results do not depend on
it, as the reference's batch-invariance test requires, tests/python/test_fem_batch_size.py).

Arrays are accepted wherever the reference takes per-element Response lists:
rest positions as (V, 3) vertex positions or (T, 4, 3) corners, Fp as (9,) or (T, 9)
column-major, theta as (2,) or (T, 2) [lambda, mu].
"""

import ctypes

import numpy as np

from . import _native as N
from .dof import ConstantDofMap, ElementDofMap, VertexDofMap
from .energy import AffineResponse, Energy, HessianKind

__all__ = [
    "NeoHookean",
    "TetP1Basis",
    "TetCentroidQuadrature",
    "InterpolatedResponse",
    "Template",
    "VolumetricFemEnergy",
    "VolumetricFemForceMaterialResponse",
    "VolumetricFemEnergyTetP1",
    "VolumetricFemForceMaterialResponseTetP1",
    "VolumetricFemForceMaterialResponseHexQ1",
    "VolumetricFemForceRestPositionResponseTetP1",
    "VolumetricFemForceFpResponse",
    "VolumetricFemForceFpResponseTetP1",
    "PyVolumetricMaterial",
    "VolumetricFemEnergyPyMaterialTetP1",
    "HexQ1Basis",
    "HexHermiteBasis",
    "BasisDofTransform",
    "CoefficientInfo",
    "DeformationGradientResponse",
    "GaussLegendre3D",
    "VolumetricFemEnergyHexQ1",
    "VolumetricFemEnergyHexHermite",
    "VolumetricFemEnergyPyMaterialHexQ1",
]


class NeoHookean:
    """W = det(Fp) psi(F Fp^-1), theta = [lambda, mu] (neo_hookean.hpp:9-33)."""

    num_parameters = 2


class CoefficientInfo:
    """Where a basis coefficient lives (basis.hpp's CoefficientInfo): the reference point and the
    derivative order per axis of the functional it interpolates."""

    def __init__(self, point, derivative_orders):
        self.point = np.asarray(point, dtype=np.float64)
        self.derivative_orders = tuple(int(o) for o in derivative_orders)

    def __repr__(self):
        return f"CoefficientInfo(point={self.point.tolist()}, derivative_orders={self.derivative_orders})"


def _check_index(cls, i):
    if not 0 <= int(i) < cls.num_basis_functions:
        raise IndexError(f"{cls.__name__}::coefficient_info: index out of range")
    return int(i)


class TetP1Basis:
    """Linear tetrahedron shape functions (tet_p1_basis.cpp:7-15)."""

    num_basis_functions = 4
    _points = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=np.float64)

    @classmethod
    def coefficient_info(cls, i):
        return CoefficientInfo(cls._points[_check_index(cls, i)], (0, 0, 0))

    @staticmethod
    def eval_N(xi):
        xi = np.asarray(xi, dtype=np.float64)
        return np.array([1 - xi.sum(), xi[0], xi[1], xi[2]])

    @staticmethod
    def eval_dN_dxi(xi):
        return np.array([[-1.0, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]])


class HexQ1Basis:
    """Trilinear hex shape functions on [0,1]^3 (hex_q1_basis.hpp), corners in the order
    (0,0,0), (1,0,0), (1,1,0), (0,1,0), (0,0,1), (1,0,1), (1,1,1), (0,1,1)."""

    num_basis_functions = 8
    corners = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])

    @classmethod
    def coefficient_info(cls, i):
        return CoefficientInfo(cls.corners[_check_index(cls, i)], (0, 0, 0))

    @classmethod
    def eval_N(cls, xi):
        xi = np.asarray(xi, dtype=np.float64)
        f = np.stack([1 - xi, xi])  # f[c, d]
        return np.array([f[i, 0] * f[j, 1] * f[k, 2] for i, j, k in cls.corners])

    @classmethod
    def eval_dN_dxi(cls, xi):
        xi = np.asarray(xi, dtype=np.float64)
        f = np.stack([1 - xi, xi])
        df = np.array([-1.0, 1.0])
        return np.array([[df[i] * f[j, 1] * f[k, 2], f[i, 0] * df[j] * f[k, 2], f[i, 0] * f[j, 1] * df[k]]
                         for i, j, k in cls.corners])


class HexHermiteBasis:
    """Tricubic Hermite functions on [0,1]^3 (hex_hermite_basis.hpp): function 8 corner + slot is
    the product of 1D cubic Hermite factors (u(0), u'(0), u(1), u'(1), cubic_hermite_basis.hpp)
    with index 2 corner_d + order_d per axis; slot derivative orders (0,0,0), (1,0,0), (0,1,0),
    (0,0,1), (1,1,0), (1,0,1), (0,1,1), (1,1,1). A vertex carries 24 physical DOFs (slots u, u_X,
    u_Y, u_Z, u_XY, u_XZ, u_YZ, u_XYZ of 3 components)."""

    num_basis_functions = 64
    dofs_per_vertex = 24
    corners = HexQ1Basis.corners
    orders = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0], [1, 0, 1], [0, 1, 1], [1, 1, 1]])

    @staticmethod
    def _cubic(t):
        t2, t3 = t * t, t * t * t
        return (np.array([2 * t3 - 3 * t2 + 1, t3 - 2 * t2 + t, -2 * t3 + 3 * t2, t3 - t2]),
                np.array([6 * t2 - 6 * t, 3 * t2 - 4 * t + 1, -6 * t2 + 6 * t, 3 * t2 - 2 * t]))

    @classmethod
    def _index(cls, row):
        return 2 * cls.corners[row // 8] + cls.orders[row % 8]

    @classmethod
    def coefficient_info(cls, i):
        i = _check_index(cls, i)
        return CoefficientInfo(cls.corners[i // 8], cls.orders[i % 8])

    @classmethod
    def eval_N(cls, xi):
        (x, _), (y, _), (z, _) = (cls._cubic(float(c)) for c in xi)
        return np.array([x[i] * y[j] * z[k] for i, j, k in (cls._index(r) for r in range(64))])

    @classmethod
    def eval_dN_dxi(cls, xi):
        (x, dx), (y, dy), (z, dz) = (cls._cubic(float(c)) for c in xi)
        return np.array([[dx[i] * y[j] * z[k], x[i] * dy[j] * z[k], x[i] * y[j] * dz[k]]
                         for i, j, k in (cls._index(r) for r in range(64))])


class _GaussLegendre3D:
    """Gauss-Legendre points on [0,1]^3, last axis fastest (gauss_legendre_3d.hpp)."""

    points_per_axis = None

    @classmethod
    def _rule(cls):
        n = cls.points_per_axis
        if n == 2:
            return np.array([0.5 - 0.5 / np.sqrt(3.0), 0.5 + 0.5 / np.sqrt(3.0)]), np.array([0.5, 0.5])
        outer = np.sqrt((3 + 2 * np.sqrt(6.0 / 5)) / 7)
        inner = np.sqrt((3 - 2 * np.sqrt(6.0 / 5)) / 7)
        wo, wi = (18 - np.sqrt(30.0)) / 72, (18 + np.sqrt(30.0)) / 72
        return (np.array([0.5 * (1 - outer), 0.5 * (1 - inner), 0.5 * (1 + inner), 0.5 * (1 + outer)]),
                np.array([wo, wi, wi, wo]))

    @classmethod
    def points(cls):
        t, _ = cls._rule()
        return np.array([[a, b, c] for a in t for b in t for c in t])

    @classmethod
    def weights(cls):
        _, w = cls._rule()
        return np.array([a * b * c for a in w for b in w for c in w])


class GaussLegendre3D_2(_GaussLegendre3D):
    points_per_axis = 2
    num_points = 8


class GaussLegendre3D_4(_GaussLegendre3D):
    points_per_axis = 4
    num_points = 64


GaussLegendre3D_2.__name__ = "GaussLegendre3D[2]"
GaussLegendre3D_4.__name__ = "GaussLegendre3D[4]"


class TetCentroidQuadrature:
    """One point at the centroid, weight 1/6 (tet_centroid_quadrature.hpp:9-23)."""

    num_points = 1

    @staticmethod
    def points():
        return np.full((1, 3), 0.25)

    @staticmethod
    def weights():
        return np.array([1.0 / 6.0])


class _InterpolatedResponseTetP1:
    """xi -> coefficients^T N(xi) (src/core/fem/response/interpolated_response.hpp:13-63)."""

    def __init__(self, coefficients):
        c = np.asarray(coefficients, dtype=np.float64)
        if c.ndim != 2 or c.shape[0] != 4:
            raise ValueError("InterpolatedResponse[TetP1Basis] requires (4, k) coefficients")
        self.coefficients = c.copy()

    @property
    def num_inputs(self):
        return 3

    @property
    def num_outputs(self):
        return self.coefficients.shape[1]

    basis = TetP1Basis

    def eval_value(self, xi):
        return self.coefficients.T @ self.basis.eval_N(xi)

    def eval_jacobian(self, xi):
        """(k, 3): d value / d xi."""
        return self.coefficients.T @ self.basis.eval_dN_dxi(xi)


class _InterpolatedResponseHexQ1(_InterpolatedResponseTetP1):
    """xi -> coefficients^T N(xi) over the trilinear hex basis (8 corner coefficients)."""

    basis = HexQ1Basis

    def __init__(self, coefficients):
        c = np.asarray(coefficients, dtype=np.float64)
        if c.ndim != 2 or c.shape[0] != 8:
            raise ValueError("InterpolatedResponse[HexQ1Basis] requires (8, k) coefficients")
        self.coefficients = c.copy()


class _InterpolatedResponseHexHermite(_InterpolatedResponseTetP1):
    """xi -> coefficients^T N(xi) over the tricubic Hermite basis (64 reference coefficients,
    index 8 corner + slot)."""

    basis = HexHermiteBasis

    def __init__(self, coefficients):
        c = np.asarray(coefficients, dtype=np.float64)
        if c.ndim != 2 or c.shape[0] != 64:
            raise ValueError("InterpolatedResponse[HexHermiteBasis] requires (64, k) coefficients")
        self.coefficients = c.copy()


class DeformationGradientResponse:
    """xi -> vec(F) (column-major) with F = I + (du/dxi)(dX/dxi)^-1 for a displacement field u and a
    rest-position field X over the reference cell (deformation_gradient_response.hpp)."""

    def __init__(self, displacement, rest_position):
        if displacement.num_outputs != 3 or rest_position.num_outputs != 3:
            raise ValueError("DeformationGradientResponse requires three-component fields")
        self.displacement, self.rest_position = displacement, rest_position
        self.num_inputs, self.num_outputs = 3, 9

    def eval_value(self, xi):
        J = self.rest_position.eval_jacobian(xi)
        F = np.eye(3) + self.displacement.eval_jacobian(xi) @ np.linalg.inv(J)
        return F.ravel(order="F")


class _NodalDofTransform:
    """BasisDofTransform for nodal bases (basis_dof_transform.hpp:15-57): 3 DOFs per vertex, the
    coefficients are the DOFs, and the pullback is the identity."""

    dofs_per_vertex = 3
    nodes = None

    def __init__(self, geometry):
        if getattr(geometry, "num_inputs", 3) != 3 or getattr(geometry, "num_outputs", 3) != 3:
            raise ValueError("BasisDofTransform: geometry must map R3 to R3")

    def to_coefficients(self, local):
        a = np.asarray(local, dtype=np.float64)
        if a.shape != (self.nodes, 3) or not np.all(np.isfinite(a)):
            raise ValueError("BasisDofTransform: invalid nodal DOFs")
        return a.copy()

    def pullback(self, gradient=None, hessian=None):
        return (None if gradient is None else np.asarray(gradient, dtype=np.float64).copy(),
                None if hessian is None else np.asarray(hessian, dtype=np.float64).copy())


class _TetP1DofTransform(_NodalDofTransform):
    nodes = 4


class _HexQ1DofTransform(_NodalDofTransform):
    nodes = 8


class _HexHermiteDofTransform:
    """BasisDofTransform<HexHermiteBasis> (basis_dof_transform.hpp:59-148): the geometry must be a
    positive axis-aligned box in corner order (its corners checked to 1e-12); per vertex 24
    physical DOFs (slots u, u_X, u_Y, u_Z, u_XY, u_XZ, u_YZ, u_XYZ) scaled to reference
    coefficients by 1, hx, hy, hz, hx hy, hx hz, hy hz, hx hy hz; the pullback scales a gradient
    (s g) and a Hessian (S H S) by the same factors."""

    dofs_per_vertex = 24

    def __init__(self, geometry):
        if getattr(geometry, "num_inputs", 3) != 3 or getattr(geometry, "num_outputs", 3) != 3:
            raise ValueError("Hermite DOFs require three reference components")
        nodes = np.array([np.asarray(geometry.eval_value(HexQ1Basis.corners[v]), dtype=np.float64)
                          for v in range(8)])
        if nodes.shape != (8, 3) or not np.all(np.isfinite(nodes)):
            raise ValueError("Hermite DOFs require finite three-component reference values")
        origin = nodes[0]
        h = np.array([nodes[1, 0] - origin[0], nodes[3, 1] - origin[1], nodes[4, 2] - origin[2]])
        if not np.all(np.isfinite(h)) or np.any(h <= 0):
            raise ValueError("Hermite DOF transform requires positive axis-aligned box dimensions")
        if np.abs((nodes - origin) / h - HexQ1Basis.corners).max() > 1e-12:
            raise ValueError("Hermite DOF transform requires axis-aligned boxes in Hex corner order")
        slots = np.array([1, h[0], h[1], h[2], h[0] * h[1], h[0] * h[2], h[1] * h[2], h[0] * h[1] * h[2]])
        self.scales = np.tile(np.repeat(slots, 3), 8)

    def to_coefficients(self, local):
        a = np.asarray(local, dtype=np.float64)
        if a.shape != (8, 24) or not np.all(np.isfinite(a)):
            raise ValueError("Hex Hermite requires finite 8x24 physical DOFs")
        return (a.ravel() * self.scales).reshape(64, 3)

    def pullback(self, gradient=None, hessian=None):
        g = None if gradient is None else np.asarray(gradient, dtype=np.float64) * self.scales
        H = None if hessian is None else self.scales[:, None] * np.asarray(hessian, dtype=np.float64) * self.scales
        return g, H


class Template:
    """A template of the reference indexed by argument tuple, e.g. VolumetricFemEnergy[M, B, Q]."""

    def __init__(self, name, instances):
        self.__name__ = name
        self._instances = dict(instances)

    def __getitem__(self, args):
        key = args if isinstance(args, tuple) else (args,)
        factory = getattr(self, "material_factory", None)
        if (factory is not None and len(key) == 3 and isinstance(key[0], type) and
                issubclass(key[0], PyVolumetricMaterial) and key[1:] in _PY_ENERGY_BASES):
            return factory(*key)
        try:
            return self._instances[key]
        except KeyError:
            names = ", ".join(getattr(a, "__name__", repr(a)) for a in key)
            avail = "; ".join(
                f"{self.__name__}[{', '.join(getattr(a, '__name__', repr(a)) for a in k)}]" for k in self._instances)
            raise TypeError(f"{self.__name__}[{names}] is not instantiated; available: {avail}") from None

    @property
    def instances(self):
        return dict(self._instances)

    def __repr__(self):
        return f"<template litepgo_b200.fem.{self.__name__}>"


InterpolatedResponse = Template("InterpolatedResponse", {(TetP1Basis,): _InterpolatedResponseTetP1,
                                                          (HexQ1Basis,): _InterpolatedResponseHexQ1,
                                                          (HexHermiteBasis,): _InterpolatedResponseHexHermite})
BasisDofTransform = Template("BasisDofTransform", {(TetP1Basis,): _TetP1DofTransform,
                                                    (HexQ1Basis,): _HexQ1DofTransform,
                                                    (HexHermiteBasis,): _HexHermiteDofTransform})

_CENTROID = np.full(3, 0.25)


def _sample_fields(fields, count, width, what):
    """Per-element field values at the centroid as a (count, width) array, or (width,) if shared."""
    if fields is None:
        return None
    if isinstance(fields, np.ndarray) or (isinstance(fields, (list, tuple)) and fields and
                                          isinstance(fields[0], (int, float, np.floating))):
        a = np.asarray(fields, dtype=np.float64)
        if a.shape == (width,):
            return a
        if a.shape == (count, width):
            return np.ascontiguousarray(a)
        raise ValueError(f"VolumetricFemEnergy: {what} must have shape ({width},) or ({count}, {width})")
    fields = list(fields)
    if len(fields) != count:
        raise ValueError("VolumetricFemEnergy: incompatible map or response counts")
    out = np.empty((count, width))
    cache = {}
    for e, f in enumerate(fields):
        if f is None or getattr(f, "num_inputs", 3) != 3 or getattr(f, "num_outputs", width) != width:
            raise ValueError("VolumetricFemEnergy: incompatible spatial responses")
        key = id(f)
        if key not in cache:
            cache[key] = np.asarray(f.eval_value(_CENTROID), dtype=np.float64)
        out[e] = cache[key]
    if len(cache) == 1:
        return out[0].copy()
    return out


def _hex_rest_positions(fields, cells, num_vertices):
    """Vertex rest positions (V, 3) of a hex mesh from a (V, 3) array or from per-element fields
    with (8, 3) corner coefficients (InterpolatedResponse[HexQ1Basis]); per-element corners must
    agree at shared vertices (the hex path keeps one position per vertex)."""
    if isinstance(fields, np.ndarray) or (isinstance(fields, (list, tuple)) and fields and
                                          not hasattr(fields[0], "coefficients")):
        X = np.asarray(fields, dtype=np.float64)
        if X.size != 3 * num_vertices:
            raise ValueError("VolumetricFemEnergy: rest positions must be (V, 3)")
        return np.ascontiguousarray(X.reshape(-1, 3))
    fields = list(fields)
    if len(fields) != cells.shape[0]:
        raise ValueError("VolumetricFemEnergy: incompatible map or response counts")
    X = np.full((num_vertices, 3), np.nan)
    for e, f in enumerate(fields):
        c = np.asarray(getattr(f, "coefficients", None), dtype=np.float64)
        if c.shape != (8, 3):
            raise ValueError("VolumetricFemEnergy: hex rest fields need (8, 3) corner coefficients")
        for a in range(8):
            v = cells[e, a]
            if np.all(np.isnan(X[v])):
                X[v] = c[a]
            elif not np.array_equal(X[v], c[a]):
                raise ValueError("VolumetricFemEnergy: per-element hex rest fields must agree at shared vertices")
    if np.any(np.isnan(X)):
        raise ValueError("VolumetricFemEnergy: a vertex of no element has no rest position")
    return X


def _sample_fields_hex(fields, count, width, what, points):
    """Per-element values of fields that must be constant over each hex: arrays as in
    _sample_fields; spatial responses are evaluated at every quadrature point and must agree to
    1e-12 (the hex path keeps theta and Fp per element)."""
    if fields is None or isinstance(fields, np.ndarray) or (isinstance(fields, (list, tuple)) and fields and
                                                            isinstance(fields[0], (int, float, np.floating))):
        return _sample_fields(fields, count, width, what)
    fields = list(fields)
    if len(fields) != count:
        raise ValueError("VolumetricFemEnergy: incompatible map or response counts")
    out = np.empty((count, width))
    cache = {}
    for e, f in enumerate(fields):
        if f is None or getattr(f, "num_inputs", 3) != 3 or getattr(f, "num_outputs", width) != width:
            raise ValueError("VolumetricFemEnergy: incompatible spatial responses")
        if id(f) not in cache:
            vals = np.array([np.asarray(f.eval_value(xi), dtype=np.float64) for xi in points])
            if np.abs(vals - vals[0]).max() > 1e-12 * max(1.0, np.abs(vals).max()):
                raise ValueError(f"VolumetricFemEnergy: hex meshes take element-constant {what} fields")
            cache[id(f)] = vals[0]
        out[e] = cache[id(f)]
    if len(cache) == 1:
        return out[0].copy()
    return out


def _rest_geometry(fields, num_vertices, count):
    """(X, Xe): vertex positions (V, 3) or per-element corners (T, 12)."""
    if isinstance(fields, np.ndarray):
        a = np.asarray(fields, dtype=np.float64)
        if a.shape == (num_vertices, 3) or (a.ndim == 1 and a.size == 3 * num_vertices):
            return np.ascontiguousarray(a.reshape(-1, 3)), None
        if a.shape == (count, 4, 3) or a.shape == (count, 12):
            return None, np.ascontiguousarray(a.reshape(count, 12))
        raise ValueError("VolumetricFemEnergy: rest positions must be (V, 3) or (T, 4, 3)")
    fields = list(fields)
    if len(fields) != count:
        raise ValueError("VolumetricFemEnergy: incompatible map or response counts")
    Xe = np.empty((count, 12))
    for e, f in enumerate(fields):
        c = getattr(f, "coefficients", None)
        if c is None or np.shape(c) != (4, 3):
            raise ValueError("VolumetricFemEnergy: incompatible displacement basis")
        Xe[e] = np.asarray(c, dtype=np.float64).ravel()
    return None, Xe


def _device_index():
    try:
        import torch

        if torch.cuda.is_available():
            return torch.cuda.current_device()
    except ImportError:  # pragma: no cover - torch is part of the image
        pass
    return 0


class _Input:
    """A vector argument as (pointer, memory flag), keeping NumPy copies alive."""

    def __init__(self, x, n, name="x", check_finite=True):
        self.tensor = None
        if hasattr(x, "is_cuda") and x.is_cuda:
            import torch

            if x.dtype != torch.float64 or x.ndim != 1 or x.numel() != n:
                raise ValueError(f"Energy: {name} must be a one-dimensional float64 tensor with num_dofs entries")
            self.tensor = x.contiguous()
            self.ptr, self.mem = N.vptr(self.tensor), N.MEM_DEVICE
            self.array = None
        else:
            if hasattr(x, "detach"):
                x = x.detach().cpu().numpy()
            a = np.ascontiguousarray(x, dtype=np.float64)
            if a.ndim != 1 or a.size != n or (check_finite and not np.all(np.isfinite(a))):
                raise ValueError(f"Energy::eval: {name} must have num_dofs finite entries")
            self.array = a
            self.ptr, self.mem = N.vptr(a), N.MEM_HOST


class VolumetricFemEnergyTetP1(Energy):
    """VolumetricFemEnergy[NeoHookean, TetP1Basis, TetCentroidQuadrature] on one GPU."""

    def __init__(self, displacement_map, rest_position_fields, Fp, theta, batch_size=256):
        if isinstance(batch_size, bool) or int(batch_size) <= 0:
            raise ValueError("MeshEnergy: invalid batch size")
        if not isinstance(displacement_map, VertexDofMap) or displacement_map.dofs_per_vertex != 3:
            raise ValueError("VolumetricFemEnergy: incompatible map or response counts")
        self.batch_size = int(batch_size)
        T = displacement_map.num_elements
        V = displacement_map.num_vertices
        X, Xe = _rest_geometry(rest_position_fields, V, T)
        th = _sample_fields(theta, T, 2, "theta")
        if th is None:
            raise ValueError("VolumetricFemEnergy: incompatible spatial responses")
        fp = _sample_fields(Fp, T, 9, "Fp")
        if fp is not None:
            eye = np.eye(3).ravel()
            if (fp.ndim == 1 and np.array_equal(fp, eye)) or (fp.ndim == 2 and np.all(fp == eye)):
                fp = None  # identity plastic field: the record carries no Fp^-1
            elif fp.ndim == 1:
                fp = np.ascontiguousarray(np.broadcast_to(fp, (T, 9)))
        self._init(V, displacement_map.cells, X, Xe, th, fp)
        self.map = displacement_map

    @classmethod
    def from_arrays(cls, X, tets, theta, Fp=None, batch_size=256):
        """Builds the energy from rest positions (V, 3), cells (T, 4) and theta (2,) or (T, 2)."""
        from .mesh import TetTopology

        X = np.asarray(X, dtype=np.float64).reshape(-1, 3)
        topo = TetTopology(X.shape[0], tets)
        return cls(VertexDofMap(topo, 3), X, Fp, theta, batch_size)

    def _init(self, V, cells, X, Xe, theta, Fp):
        self._h = None
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        T = cells.shape[0]
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        per_element = 1 if theta.ndim == 2 else 0
        if Fp is not None:
            Fp = np.ascontiguousarray(Fp, dtype=np.float64).reshape(T, 9)
        if X is None and Xe is None:
            raise ValueError("VolumetricFemEnergy: missing rest positions")
        h = ctypes.c_void_p()
        self.device = _device_index()
        N.check(N.lib.lpg_fem_create(V, N.dptr(X), T, N.iptr(cells), N.dptr(Xe), N.dptr(theta), per_element,
                                     N.dptr(Fp), self.device, ctypes.byref(h)))
        self._h = h
        self._theta = theta
        V_, T_, n_ = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        nnzb, nnz = ctypes.c_int64(), ctypes.c_int64()
        N.check(N.lib.lpg_fem_sizes(h, ctypes.byref(V_), ctypes.byref(T_), ctypes.byref(n_), ctypes.byref(nnzb),
                                    ctypes.byref(nnz)))
        self.num_vertices, self.num_elements, self.num_dofs = V_.value, T_.value, n_.value
        self.nnzb, self.nnz = nnzb.value, nnz.value
        self._csc = None
        self._bsr = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and N is not None and getattr(N, "lib", None) is not None:
            N.lib.lpg_fem_destroy(h)
            self._h = None

    def set_theta(self, theta):
        """Replaces [lambda, mu] ((2,) or (num_elements, 2)) in place, keeping the plan and the
        rest geometry (no reference counterpart: the reference builds a new energy)."""
        th = np.ascontiguousarray(theta, dtype=np.float64)
        if th.shape not in ((2,), (self.num_elements, 2)):
            raise ValueError("VolumetricFemEnergy: theta must have shape (2,) or (num_elements, 2)")
        N.check(N.lib.lpg_fem_set_theta(self._h, N.dptr(th), 1 if th.ndim == 2 else 0))
        self._theta = th

    def set_fp(self, Fp):
        """Replaces the plastic field in place: (9,) shared or (num_elements, 9) per element,
        column-major vec(Fp); None (or the identity) removes it. Plan, rest geometry and theta
        are kept (no reference counterpart: the reference builds a new energy)."""
        if Fp is None:
            N.check(N.lib.lpg_fem_set_fp(self._h, None, 0))
            return
        fp = np.ascontiguousarray(Fp, dtype=np.float64)
        if fp.shape not in ((9,), (self.num_elements, 9)):
            raise ValueError("VolumetricFemEnergy: Fp must have shape (9,) or (num_elements, 9)")
        eye = np.eye(3).ravel()
        if np.all(fp.reshape(-1, 9) == eye):
            N.check(N.lib.lpg_fem_set_fp(self._h, None, 0))
            return
        N.check(N.lib.lpg_fem_set_fp(self._h, N.dptr(fp), 1 if fp.ndim == 2 else 0))

    # ---- autotuned launch variants (no reference counterpart) ----
    TUNING_KEYS = ("assembly_f64", "assembly_f32", "spmv_f64", "spmv_f32", "clamp_f64", "clamp_f32")

    def tuning(self):
        """The launch variants the autotuner chose for this mesh and the mean ms per launch it
        measured: {"choice": {key: variant}, "ms": {key: [ms per variant, NaN if not timed]}}.
        Variants differ in register budget and unrolling only, never in results."""
        choice = np.zeros(6, dtype=np.int32)
        ms = np.zeros(18)
        N.check(N.lib.lpg_fem_get_tuning(self._h, N.iptr(choice), N.dptr(ms)))
        fam = {"assembly": 0, "spmv": 1, "clamp": 2}
        out_ms = {}
        for key in self.TUNING_KEYS:
            f, p = key.rsplit("_", 1)
            base = 6 * fam[f] + 3 * (0 if p == "f64" else 1)
            out_ms[key] = [float(v) for v in ms[base:base + 3]]
        return {"choice": dict(zip(self.TUNING_KEYS, (int(c) for c in choice))), "ms": out_ms}

    def autotune(self):
        """Times every launch variant on this mesh again and keeps the fastest."""
        N.check(N.lib.lpg_fem_autotune(self._h))
        return self.tuning()

    def set_tuning(self, **choice):
        """Forces variants by key (see TUNING_KEYS), e.g. set_tuning(spmv_f32=1)."""
        vals = np.full(6, -1, dtype=np.int32)
        for k, v in choice.items():
            if k not in self.TUNING_KEYS:
                raise ValueError(f"unknown tuning key {k!r}")
            vals[self.TUNING_KEYS.index(k)] = int(v)
        N.check(N.lib.lpg_fem_set_tuning(self._h, N.iptr(vals)))

    @property
    def handle(self):
        return self._h

    # ---- patterns ----
    def pattern_csc(self):
        if self._csc is None:
            outer = np.empty(self.num_dofs + 1, dtype=np.int32)
            inner = np.empty(self.nnz, dtype=np.int32)
            N.check(N.lib.lpg_fem_pattern_csc(self._h, N.iptr(outer), N.iptr(inner)))
            self._csc = (outer, inner)
        return self._csc

    def pattern_bsr(self):
        if self._bsr is None:
            row_ptr = np.empty(self.num_dofs // 3 + 1, dtype=np.int32)  # one block row per 3 DOFs
            col_idx = np.empty(self.nnzb, dtype=np.int32)
            N.check(N.lib.lpg_fem_pattern_bsr(self._h, N.iptr(row_ptr), N.iptr(col_idx)))
            self._bsr = (row_ptr, col_idx)
        return self._bsr

    # ---- Energy interface ----
    def _set_stream_for(self, *inputs):
        """Device inputs: run on torch's current stream so their producers are ordered first."""
        if any(i is not None and i.mem == N.MEM_DEVICE for i in inputs):
            import torch

            N.check(N.lib.lpg_fem_set_stream(self._h, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        else:
            N.check(N.lib.lpg_fem_set_stream(self._h, None))

    def eval(self, x, gradient=False, hessian=None, precision="f64"):
        """(value, gradient or None, csc_matrix or None) in one assembly."""
        import scipy.sparse as sp

        kind = _hessian_kind(hessian)
        prec = _precision(precision)
        xi = _Input(x, self.num_dofs)
        self._set_stream_for(xi)
        E = ctypes.c_double()
        g = np.empty(self.num_dofs) if gradient else None
        vals = np.empty(self.nnz, dtype=np.float64 if prec == N.PRECISION_F64 else np.float32) if kind else None
        N.check(N.lib.lpg_fem_eval(self._h, xi.ptr, N.MEM_HOST if xi.mem == N.MEM_HOST else N.MEM_DEVICE,
                                   ctypes.byref(E), N.vptr(g) if xi.mem == N.MEM_HOST else None, kind, prec,
                                   N.LAYOUT_CSC, N.vptr(vals), N.MEM_HOST))
        if g is not None and xi.mem == N.MEM_DEVICE:
            g = self.eval_device(xi.tensor, gradient=True)[1].cpu().numpy()
        H = None
        if kind:
            outer, inner = self.pattern_csc()
            H = sp.csc_matrix((vals.astype(np.float64, copy=False), inner, outer), shape=(self.num_dofs,) * 2)
        return E.value, g, H

    def eval_value(self, x):
        return self.eval(x)[0]

    def eval_gradient(self, x):
        return self.eval(x, gradient=True)[1]

    def eval_hessian(self, x, kind=HessianKind.Exact):
        return self.eval(x, hessian=kind)[2]

    def max_feasible_step(self, x, dx):
        xi = _Input(x, self.num_dofs, "x")
        di = _Input(dx, self.num_dofs, "dx")
        if xi.mem != di.mem:
            raise ValueError("max_feasible_step: x and dx must live on the same device")
        self._set_stream_for(xi, di)
        a = ctypes.c_double()
        N.check(N.lib.lpg_fem_feasible_step(self._h, xi.ptr, di.ptr, xi.mem, ctypes.byref(a)))
        return a.value

    def element_energies(self, x):
        xi = _Input(x, self.num_dofs)
        out = np.empty(self.num_elements)
        self._set_stream_for(xi)
        if xi.mem == N.MEM_DEVICE:
            import torch

            t = torch.empty(self.num_elements, dtype=torch.float64, device=xi.tensor.device)
            N.check(N.lib.lpg_fem_element_energies(self._h, xi.ptr, N.MEM_DEVICE, N.vptr(t)))
            return t
        N.check(N.lib.lpg_fem_element_energies(self._h, xi.ptr, N.MEM_HOST, N.vptr(out)))
        return out

    # ---- device-resident evaluation ----
    def eval_device(self, u, gradient=True, hessian=None, precision="f64", layout="bsr", grad_out=None,
                    hess_out=None):
        """Energy (float), gradient and Hessian values as CUDA tensors, without host copies.

        ``u`` is a CUDA float64 tensor of num_dofs entries. The Hessian values come in
        block-CSR order (nnzb blocks of 3x3, row-major) or the reference's CSC order.
        """
        import torch

        kind = _hessian_kind(hessian)
        prec = _precision(precision)
        lay = N.LAYOUT_BSR if layout == "bsr" else N.LAYOUT_CSC
        xi = _Input(u, self.num_dofs)
        if xi.mem != N.MEM_DEVICE:
            raise ValueError("eval_device requires a CUDA tensor")
        dev = xi.tensor.device
        g = None
        if gradient:
            g = grad_out if grad_out is not None else torch.empty(self.num_dofs, dtype=torch.float64, device=dev)
        H = None
        if kind:
            dt = torch.float64 if prec == N.PRECISION_F64 else torch.float32
            H = hess_out if hess_out is not None else torch.empty(self.nnz, dtype=dt, device=dev)
        self._set_stream_for(xi)
        E = ctypes.c_double()
        N.check(N.lib.lpg_fem_eval(self._h, xi.ptr, N.MEM_DEVICE, ctypes.byref(E), N.vptr(g), kind, prec, lay,
                                   N.vptr(H), N.MEM_DEVICE))
        return E.value, g, H


def _hessian_kind(hessian):
    if hessian is None or hessian is False:
        return N.HESSIAN_NONE
    k = int(hessian)
    if k not in (N.HESSIAN_EXACT, N.HESSIAN_PROJECTED):
        raise ValueError("Energy: invalid Hessian kind")
    return k


def _precision(p):
    if p in ("f64", "fp64", N.PRECISION_F64):
        return N.PRECISION_F64
    if p in ("mixed", "fp32", N.PRECISION_MIXED):
        return N.PRECISION_MIXED
    raise ValueError("precision must be 'f64' or 'mixed'")


class VolumetricFemForceMaterialResponseTetP1:
    """Force response p -> g(u; p) at a fixed displacement, differentiated in theta.

    Mirrors VolumetricFemForceMaterialResponse[NeoHookean, TetP1Basis, TetCentroidQuadrature]
    (src/core/fem/assembly/volumetric_fem_force_material_response.hpp; binding
    src/binding/detail/fem_helpers.hpp:76-98). ConstantDofMap shares one [lambda, mu];
    ElementDofMap gives each element its own block.
    """

    _energy_cls = VolumetricFemEnergyTetP1

    def __init__(self, parameter_map, displacement_map, rest_position_fields, displacement, Fp, batch_size=256):
        if isinstance(batch_size, bool) or int(batch_size) <= 0:
            raise ValueError("VolumetricFemForceResponse: incompatible element count or batch size")
        if not isinstance(parameter_map, (ConstantDofMap, ElementDofMap)):
            raise TypeError("parameter_map must be a ConstantDofMap or an ElementDofMap")
        width = parameter_map.num_dofs if isinstance(parameter_map, ConstantDofMap) else parameter_map.dofs_per_element
        if parameter_map.num_elements != displacement_map.num_elements:
            raise ValueError("VolumetricFemForceResponse: incompatible element count or batch size")
        if width != 2:
            raise ValueError("VolumetricFemForceResponse: invalid parameter count")
        self.per_element = isinstance(parameter_map, ElementDofMap)
        self.parameter_map = parameter_map
        u = np.ascontiguousarray(displacement, dtype=np.float64)
        if u.size != displacement_map.num_dofs or not np.all(np.isfinite(u)):
            raise ValueError("VolumetricFemForceResponse: incompatible map, displacement or responses")
        # theta does not enter d g / d theta (P is linear in theta); any valid value builds the mesh.
        self._energy = self._energy_cls(displacement_map, rest_position_fields, Fp, np.array([1.0, 1.0]))
        self.displacement = u
        self.num_inputs = parameter_map.num_dofs
        self.num_outputs = displacement_map.num_dofs

    def _check_p(self, p):
        p = np.asarray(p, dtype=np.float64).ravel()
        if p.size != self.num_inputs:
            raise ValueError("Response: p must have num_inputs entries")
        th = p.reshape(-1, 2)
        if not np.all(np.isfinite(th)) or np.any(th[:, 0] < 0) or np.any(th[:, 1] <= 0):
            raise ValueError("NeoHookean requires finite lambda >= 0 and mu > 0")
        return p

    def eval_vjp(self, p, w):
        """(d g / d theta)^T w: (2,) for a ConstantDofMap, (2 T,) for an ElementDofMap."""
        self._check_p(p)
        wv = np.ascontiguousarray(w, dtype=np.float64)
        if wv.size != self.num_outputs:
            raise ValueError("Response: weights must have num_outputs entries")
        T = self._energy.num_elements
        out = np.empty(2 * T if self.per_element else 2)
        N.check(N.lib.lpg_fem_force_vjp_theta(self._energy.handle, N.vptr(self.displacement), N.vptr(wv), N.MEM_HOST,
                                              1 if self.per_element else 0, N.vptr(out)))
        return out


class VolumetricFemForceRestPositionResponseTetP1:
    """Force response X -> g(u; X) in the vertex rest positions at a fixed displacement.

    No reference counterpart: the reference differentiates its force response in theta
    (VolumetricFemForceMaterialResponse) and Fp only. ``eval_vjp(X, w)`` returns
    (dg/dX)^T w (num_dofs values) with X the (V, 3) rest positions, flattened; used as the
    ``make_response`` of a StaticEquilibriumResponse over rest positions. Needs vertex rest
    positions and no plastic field.
    """

    def __init__(self, displacement_map, displacement, theta):
        if not isinstance(displacement_map, VertexDofMap) or displacement_map.dofs_per_vertex != 3:
            raise ValueError("VolumetricFemForceResponse: incompatible map, displacement or responses")
        u = np.ascontiguousarray(displacement, dtype=np.float64)
        if u.size != displacement_map.num_dofs or not np.all(np.isfinite(u)):
            raise ValueError("VolumetricFemForceResponse: incompatible map, displacement or responses")
        self.map = displacement_map
        self.theta = np.ascontiguousarray(theta, dtype=np.float64)
        self.displacement = u
        self.num_inputs = self.num_outputs = displacement_map.num_dofs
        self._energy = None
        self._X = None

    def _energy_at(self, X):
        X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 3)
        if X.shape[0] != self.map.num_vertices or not np.all(np.isfinite(X)):
            raise ValueError("Response: p must hold num_vertices finite rest positions")
        if self._energy is None or not np.array_equal(X, self._X):
            self._energy = VolumetricFemEnergyTetP1(self.map, X, None, self.theta)
            self._X = X.copy()
        return self._energy

    def eval_vjp(self, X, w):
        """(dg/dX)^T w at the rest positions X (num_dofs values)."""
        e = self._energy_at(X)
        wv = np.ascontiguousarray(w, dtype=np.float64)
        if wv.size != self.num_outputs:
            raise ValueError("Response: weights must have num_outputs entries")
        out = np.empty(self.num_inputs)
        N.check(N.lib.lpg_fem_set_stream(e.handle, None))
        N.check(N.lib.lpg_fem_force_vjp_rest(e.handle, N.vptr(self.displacement), N.vptr(wv), N.MEM_HOST, N.vptr(out)))
        return out


class VolumetricFemForceFpResponseTetP1:
    """Force response Fp -> g(u; Fp) at a fixed displacement and theta, differentiated in the
    plastic field.

    Mirrors VolumetricFemForceFpResponse[NeoHookean, TetP1Basis, TetCentroidQuadrature]
    (src/core/fem/assembly/volumetric_fem_force_fp_response.hpp:8-10; binding
    src/binding/fem/assembly/volumetric_fem_force_fp_response.cpp): input column-major vec(Fp),
    one block shared (ConstantDofMap, 9 inputs) or one per element (ElementDofMap, 9 per
    element). ``eval_value(p)`` is the elastic force (the energy gradient) with Fp = p,
    ``eval_vjp(p, w)`` is (dg/dFp)^T w.
    """

    def __init__(self, parameter_map, displacement_map, rest_position_fields, displacement, theta, batch_size=256):
        if isinstance(batch_size, bool) or int(batch_size) <= 0:
            raise ValueError("VolumetricFemForceResponse: incompatible element count or batch size")
        if not isinstance(parameter_map, (ConstantDofMap, ElementDofMap)):
            raise TypeError("parameter_map must be a ConstantDofMap or an ElementDofMap")
        width = parameter_map.num_dofs if isinstance(parameter_map, ConstantDofMap) else parameter_map.dofs_per_element
        if parameter_map.num_elements != displacement_map.num_elements:
            raise ValueError("VolumetricFemForceResponse: incompatible element count or batch size")
        if width != 9:
            raise ValueError("VolumetricFemForceResponse: invalid parameter count")
        self.per_element = isinstance(parameter_map, ElementDofMap)
        self.parameter_map = parameter_map
        u = np.ascontiguousarray(displacement, dtype=np.float64)
        if u.size != displacement_map.num_dofs or not np.all(np.isfinite(u)):
            raise ValueError("VolumetricFemForceResponse: incompatible map, displacement or responses")
        self._energy = VolumetricFemEnergyTetP1(displacement_map, rest_position_fields, None, theta)
        self.displacement = u
        self.num_inputs = parameter_map.num_dofs
        self.num_outputs = displacement_map.num_dofs
        self._fp = None

    def _set(self, p):
        p = np.asarray(p, dtype=np.float64).ravel()
        if p.size != self.num_inputs:
            raise ValueError("Response: p must have num_inputs entries")
        if not np.all(np.isfinite(p)):
            raise ValueError("MultiplicativeKinematics requires finite F and Fp")
        if self._fp is None or not np.array_equal(self._fp, p):
            self._energy.set_fp(p.reshape(-1, 9) if self.per_element else p)
            self._fp = p.copy()
        return p

    def eval_value(self, p):
        """The elastic force g(u; Fp = p) (num_outputs values)."""
        self._set(p)
        return self._energy.eval_gradient(self.displacement)

    def eval_vjp(self, p, w):
        """(d g / d Fp)^T w: (9,) for a ConstantDofMap, (9 T,) for an ElementDofMap."""
        self._set(p)
        wv = np.ascontiguousarray(w, dtype=np.float64)
        if wv.size != self.num_outputs:
            raise ValueError("Response: weights must have num_outputs entries")
        T = self._energy.num_elements
        out = np.empty(9 * T if self.per_element else 9)
        N.check(N.lib.lpg_fem_set_stream(self._energy.handle, None))
        N.check(N.lib.lpg_fem_force_vjp_fp(self._energy.handle, N.vptr(self.displacement), N.vptr(wv), N.MEM_HOST,
                                           1 if self.per_element else 0, N.vptr(out)))
        return out


class VolumetricFemEnergyHexQ1(VolumetricFemEnergyTetP1):
    """VolumetricFemEnergy[NeoHookean, HexQ1Basis, GaussLegendre3D[n]] on one GPU (the class
    variable ``points_per_axis`` is set by the template). The rest positions are vertex positions
    (V, 3); no plastic field. The Energy interface is the tet energy's, with the Exact and the
    Projected Hessian (each element's 24x24 Hessian projected to PSD); set_theta, the theta force
    response and the theta adjoint work as for tets."""

    points_per_axis = 2
    _dofs_per_vertex = 3  # DOFs per mesh vertex (24 for Hermite)
    _create = "lpg_fem_create_hex"

    def __init__(self, displacement_map, rest_position_fields, Fp, theta, batch_size=256):
        if isinstance(batch_size, bool) or int(batch_size) <= 0:
            raise ValueError("MeshEnergy: invalid batch size")
        if not isinstance(displacement_map, VertexDofMap) or displacement_map.dofs_per_vertex != self._dofs_per_vertex:
            raise ValueError("VolumetricFemEnergy: incompatible map or response counts")
        cells = np.ascontiguousarray(displacement_map.cells, dtype=np.int32)
        if cells.ndim != 2 or cells.shape[1] != 8:
            raise ValueError("VolumetricFemEnergy: HexQ1Basis needs 8 vertices per cell")
        points = (GaussLegendre3D_2 if self.points_per_axis == 2 else GaussLegendre3D_4).points()
        fp = _sample_fields_hex(Fp, cells.shape[0], 9, "Fp", points)
        if fp is not None and not np.all(np.asarray(fp).reshape(-1, 9) == np.eye(3).ravel()):
            raise ValueError("VolumetricFemEnergy: hex meshes take no plastic field here")
        X = _hex_rest_positions(rest_position_fields, cells, displacement_map.num_vertices)
        th = _sample_fields_hex(theta, cells.shape[0], 2, "theta", points)
        if th is None:
            raise ValueError("VolumetricFemEnergy: incompatible spatial responses")
        self.batch_size = int(batch_size)
        self._h = None
        th = np.ascontiguousarray(th, dtype=np.float64)
        h = ctypes.c_void_p()
        self.device = _device_index()
        N.check(getattr(N.lib, self._create)(X.shape[0], N.dptr(X), cells.shape[0], N.iptr(cells), N.dptr(th),
                                             1 if th.ndim == 2 else 0, int(self.points_per_axis), self.device,
                                             ctypes.byref(h)))
        self._h = h
        self._theta = th
        V_, T_, n_ = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        nnzb, nnz = ctypes.c_int64(), ctypes.c_int64()
        N.check(N.lib.lpg_fem_sizes(h, ctypes.byref(V_), ctypes.byref(T_), ctypes.byref(n_), ctypes.byref(nnzb),
                                    ctypes.byref(nnz)))
        # The plan's block rows are (vertex, 3-DOF group): one per vertex, 8 per Hermite vertex.
        self.num_vertices, self.num_elements, self.num_dofs = X.shape[0], T_.value, n_.value
        self.nnzb, self.nnz = nnzb.value, nnz.value
        self._csc = None
        self._bsr = None
        self.map = displacement_map

    @classmethod
    def from_arrays(cls, X, cells, theta, Fp=None, batch_size=256):
        from .mesh import HexTopology

        X = np.asarray(X, dtype=np.float64).reshape(-1, 3)
        topo = HexTopology(X.shape[0], cells)
        return cls(VertexDofMap(topo, cls._dofs_per_vertex), X, Fp, theta, batch_size)


class VolumetricFemEnergyHexQ1GL4(VolumetricFemEnergyHexQ1):
    points_per_axis = 4


class VolumetricFemEnergyHexHermite(VolumetricFemEnergyHexQ1):
    """VolumetricFemEnergy[NeoHookean, HexHermiteBasis, GaussLegendre3D[n]] on one GPU: rest
    positions (V, 3) of axis-aligned box cells in corner order (ValueError otherwise), 24 physical
    DOFs per vertex (VertexDofMap(topology, 24)), the reference's DOF scaling by the box edges.
    The Exact Hessian only (a projected request raises ValueError): run Newton with
    hessian=Exact. set_theta, the theta force response and the theta adjoint work; Python
    materials are tet/Q1 only."""

    _dofs_per_vertex = 24
    _create = "lpg_fem_create_hex_hermite"


class VolumetricFemEnergyHexHermiteGL4(VolumetricFemEnergyHexHermite):
    points_per_axis = 4


class VolumetricFemForceMaterialResponseHexHermite(VolumetricFemForceMaterialResponseTetP1):
    """VolumetricFemForceMaterialResponse[NeoHookean, HexHermiteBasis, GaussLegendre3D[2]]: the
    force's VJP in theta over the 24 physical DOFs per vertex (VertexDofMap(topology, 24));
    usable as the make_response of a StaticEquilibriumResponse."""

    _energy_cls = VolumetricFemEnergyHexHermite


class VolumetricFemForceMaterialResponseHexHermiteGL4(VolumetricFemForceMaterialResponseTetP1):
    _energy_cls = VolumetricFemEnergyHexHermiteGL4


class VolumetricFemForceMaterialResponseHexQ1(VolumetricFemForceMaterialResponseTetP1):
    """VolumetricFemForceMaterialResponse[NeoHookean, HexQ1Basis, GaussLegendre3D[2]]: the
    force's VJP in theta summed over the quadrature points of each hex (vertex rest positions
    (V, 3), no plastic field); usable as the make_response of a StaticEquilibriumResponse."""

    _energy_cls = VolumetricFemEnergyHexQ1


class VolumetricFemForceMaterialResponseHexQ1GL4(VolumetricFemForceMaterialResponseTetP1):
    _energy_cls = VolumetricFemEnergyHexQ1GL4


class PyVolumetricMaterial:
    """Base class for volumetric materials written in Python (the reference's
    PyVolumetricMaterial, src/python/fem.py:59-109): subclass it and put the subclass in the
    Material slot of VolumetricFemEnergy[Material, TetP1Basis, TetCentroidQuadrature].

    Required: ``num_parameters`` (the width k of theta) and
    ``eval(F, Fp, theta, *, outputs) -> dict`` returning at least the requested entries of
    ``W`` (N,), ``dW_dF`` (N,3,3) with [n,i,j] = dW/dF_ij and ``d2W_dF2`` (N,3,3,3,3) with
    [n,i,j,k,l] = d2W/dF_ij dF_kl. Unlike the reference, whose batches are CPU NumPy arrays, F,
    Fp and theta arrive here as CUDA float64 tensors of the whole mesh (one row per element), so
    a torch material runs on the GPU; NumPy arrays are accepted as return values too. Energies
    request ("W",), ("W", "dW_dF") or ("W", "dW_dF", "d2W_dF2"). Optional
    ``eval_feasible_step(F, Fp, theta, dF) -> (N,)``: a bound in [0, 1] keeping each element
    feasible along F + t dF; without it the step keeps det F > 0. Non-finite returned values
    reject the evaluation (ValueError, as a native domain error)."""

    num_parameters = None
    eval_feasible_step = None

    @staticmethod
    def eval(F, Fp, theta, *, outputs):
        raise NotImplementedError("PyVolumetricMaterial subclasses must implement eval")


def _cuda_f64(a, shape, device):
    import torch

    t = torch.as_tensor(a, dtype=torch.float64, device=device)
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"PyVolumetricMaterial.eval returned shape {tuple(t.shape)}, expected {tuple(shape)}")
    return t.contiguous()


class VolumetricFemEnergyPyMaterialTetP1(Energy):
    """VolumetricFemEnergy[Material, TetP1Basis, TetCentroidQuadrature] for a
    PyVolumetricMaterial subclass ``material`` (set by the template), on one GPU: the library
    exports every element's deformation gradient, the material evaluates W and its derivatives
    on the device, and the library integrates (E = sum vol W, g_a = vol P grad N_a) and assembles
    the Hessian (vol B^T A B, Exact or per-element eigenvalue clamp) as for the native material."""

    material = None
    _geometry_cls = VolumetricFemEnergyTetP1  # the native handle carrying the rest geometry

    def __init__(self, displacement_map, rest_position_fields, Fp, theta, batch_size=256):
        import torch

        mat = self.material
        if mat is None or not isinstance(mat.num_parameters, int) or mat.num_parameters < 0:
            raise ValueError("PyVolumetricMaterial: num_parameters must be a non-negative int")
        if isinstance(batch_size, bool) or int(batch_size) <= 0:
            raise ValueError("MeshEnergy: invalid batch size")
        T = displacement_map.num_elements
        k = mat.num_parameters
        per = getattr(self._geometry_cls, "points_per_axis", None)
        if per is None:
            sample = _sample_fields
        else:  # hexes: element-constant fields, checked at every quadrature point
            points = (GaussLegendre3D_2 if per == 2 else GaussLegendre3D_4).points()
            sample = lambda f, c, w, what: _sample_fields_hex(f, c, w, what, points)  # noqa: E731
        th = sample(theta, T, k, "theta") if k > 0 else np.zeros((T, 0))
        if th is None:
            raise ValueError("VolumetricFemEnergy: incompatible spatial responses")
        fp = sample(Fp, T, 9, "Fp")
        fp = np.tile(np.eye(3).ravel(), (T, 1)) if fp is None else np.array(np.broadcast_to(fp, (T, 9)))
        # The geometry handle: the native records carry only rest geometry here.
        self._geo = self._geometry_cls(displacement_map, rest_position_fields, None, np.array([1.0, 1.0]),
                                       batch_size)
        self.map = displacement_map
        self.num_vertices, self.num_elements, self.num_dofs = (self._geo.num_vertices, self._geo.num_elements,
                                                               self._geo.num_dofs)
        self.nnzb, self.nnz = self._geo.nnzb, self._geo.nnz
        self.device = torch.device("cuda", self._geo.device)
        # Material rows: one per element (tets) or per quadrature point (hexes, element-major);
        # Fp and theta are per element, the same at each of its points.
        per = getattr(self._geo, "points_per_axis", None)
        self._points = 1 if per is None else per ** 3
        self._rows = T * self._points
        # Fp column-major vec -> (T, 3, 3) matrices.
        self._Fp = torch.as_tensor(np.ascontiguousarray(fp, dtype=np.float64).reshape(T, 3, 3).transpose(0, 2, 1),
                                   device=self.device).repeat_interleave(self._points, dim=0).contiguous()
        self._theta = torch.as_tensor(np.array(np.broadcast_to(th, (T, k)), dtype=np.float64),
                                      device=self.device).repeat_interleave(self._points, dim=0).contiguous()

    @property
    def handle(self):
        return self._geo.handle

    def pattern_csc(self):
        return self._geo.pattern_csc()

    def pattern_bsr(self):
        return self._geo.pattern_bsr()

    def _u(self, x):
        import torch

        if isinstance(x, torch.Tensor):
            u = x.detach().to(device=self.device, dtype=torch.float64).contiguous()
        else:
            u = torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device=self.device)
        if u.numel() != self.num_dofs:
            raise ValueError("Energy: x must have num_dofs finite entries")
        return u

    def deformation_gradients(self, x):
        """CUDA tensor of F = I + grad u: (T, 3, 3) per element for tets, (T n^3, 3, 3) per
        quadrature point (element-major) for hexes."""
        import torch

        u = self._u(x)
        F = torch.empty((self._rows, 3, 3), dtype=torch.float64, device=self.device)
        N.check(N.lib.lpg_fem_set_stream(self.handle, ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)))
        N.check(N.lib.lpg_fem_deformation_gradients(self.handle, N.vptr(u), N.MEM_DEVICE, N.vptr(F)))
        return F

    def _material(self, F, outputs):
        out = self.material.eval(F, self._Fp, self._theta, outputs=outputs)
        T = self._rows
        shapes = {"W": (T,), "dW_dF": (T, 3, 3), "d2W_dF2": (T, 3, 3, 3, 3)}
        return [_cuda_f64(out[name], shapes[name], self.device) for name in outputs]

    def eval_device(self, x, gradient=True, hessian=None, precision="f64", layout="bsr"):
        """Energy (float), gradient and Hessian values as CUDA tensors (block-CSR or CSC order)."""
        import torch

        kind = _hessian_kind(hessian)
        prec = _precision(precision)
        lay = N.LAYOUT_BSR if layout == "bsr" else N.LAYOUT_CSC
        F = self.deformation_gradients(x)
        outputs = ("W",) + (("dW_dF",) if gradient else ()) + (("d2W_dF2",) if kind else ())
        vals = self._material(F, outputs)
        W = vals[0]
        P = vals[1] if gradient else None
        A = vals[-1] if kind else None
        g = torch.empty(self.num_dofs, dtype=torch.float64, device=self.device) if gradient else None
        H = None
        if kind:
            dt = torch.float64 if prec == N.PRECISION_F64 else torch.float32
            H = torch.empty(self.nnz, dtype=dt, device=self.device)
        E = ctypes.c_double()
        N.check(N.lib.lpg_fem_set_stream(self.handle, ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)))
        N.check(N.lib.lpg_fem_eval_material(self.handle, N.vptr(W), N.vptr(P), N.vptr(A), N.MEM_DEVICE,
                                            ctypes.byref(E), N.vptr(g), kind, prec, lay, N.vptr(H), N.MEM_DEVICE))
        return E.value, g, H

    def eval(self, x, gradient=False, hessian=None, precision="f64"):
        """(value, gradient or None, csc_matrix or None), like the native energy."""
        import scipy.sparse as sp

        E, g, H = self.eval_device(x, gradient=gradient, hessian=hessian, precision=precision, layout="csc")
        gh = g.cpu().numpy() if g is not None else None
        Hs = None
        if H is not None:
            outer, inner = self.pattern_csc()
            Hs = sp.csc_matrix((H.double().cpu().numpy(), inner, outer), shape=(self.num_dofs,) * 2)
        return E, gh, Hs

    def eval_value(self, x):
        return self.eval(x)[0]

    def eval_gradient(self, x):
        return self.eval(x, gradient=True)[1]

    def eval_hessian(self, x, kind=HessianKind.Exact):
        return self.eval(x, hessian=kind)[2]

    def max_feasible_step(self, x, dx):
        """The material's bound when it has eval_feasible_step (min over elements, in [0, 1]);
        otherwise the largest step keeping det F > 0 (the native feasible step)."""
        import torch

        if self.material.eval_feasible_step is None:
            u = self._u(x)
            du = self._u(dx)
            a = ctypes.c_double()
            N.check(N.lib.lpg_fem_set_stream(self.handle, None))
            N.check(N.lib.lpg_fem_feasible_step(self.handle, N.vptr(u), N.vptr(du), N.MEM_DEVICE, ctypes.byref(a)))
            return a.value
        F = self.deformation_gradients(x)
        dF = self.deformation_gradients(dx) - torch.eye(3, dtype=torch.float64, device=self.device)
        bound = _cuda_f64(self.material.eval_feasible_step(F, self._Fp, self._theta, dF), (self._rows,),
                          self.device)
        if not bool(torch.all(torch.isfinite(bound))):
            raise ValueError("PyVolumetricMaterial.eval_feasible_step returned non-finite values")
        return float(torch.clamp(bound, 0.0, 1.0).min()) if self.num_elements else 1.0


class VolumetricFemEnergyPyMaterialHexQ1(VolumetricFemEnergyPyMaterialTetP1):
    """VolumetricFemEnergy[Material, HexQ1Basis, GaussLegendre3D[2]] for a PyVolumetricMaterial:
    the library exports F at every quadrature point, the material evaluates W, dW/dF and
    d2W/dF2 there (one row per point, element-major; theta and Fp per element, repeated over its
    points), and the library integrates E = sum_q w_q W, g_a = sum_q w_q P grad N_a and
    H = sum_q w_q B_q^T A_q B_q per hex and assembles them as the native hex energy (Exact, or
    each element's 24x24 Hessian projected to PSD)."""

    _geometry_cls = VolumetricFemEnergyHexQ1


class VolumetricFemEnergyPyMaterialHexQ1GL4(VolumetricFemEnergyPyMaterialHexQ1):
    _geometry_cls = VolumetricFemEnergyHexQ1GL4


class VolumetricFemForceMaterialResponsePyTetP1:
    """VolumetricFemForceMaterialResponse[Material, TetP1Basis, TetCentroidQuadrature] for a
    PyVolumetricMaterial subclass ``material`` (set by the template; the reference's binding,
    src/binding/detail/fem_helpers.hpp:76-98, with a Python material in the Material slot): the
    force g(u; p) at a fixed displacement as a response of the material parameters, ConstantDofMap
    (one theta for every element) or ElementDofMap (one per element). Its VJP is
    (dg/dtheta_e)^T w = vol_e (d2W/dF dtheta) : grad w_e, with the material's d2W_dF_dtheta at every
    element's F (one material row per element, on the GPU) and grad w_e = F(w) - I from the library."""

    material = None

    def __init__(self, parameter_map, displacement_map, rest_position_fields, displacement, Fp, batch_size=256):
        import torch

        mat = self.material
        k = getattr(mat, "num_parameters", None)
        if mat is None or not isinstance(k, int) or k <= 0:
            raise ValueError("PyVolumetricMaterial: num_parameters must be a positive int for a material response")
        if isinstance(batch_size, bool) or int(batch_size) <= 0:
            raise ValueError("VolumetricFemForceResponse: incompatible element count or batch size")
        if not isinstance(parameter_map, (ConstantDofMap, ElementDofMap)):
            raise TypeError("parameter_map must be a ConstantDofMap or an ElementDofMap")
        width = parameter_map.num_dofs if isinstance(parameter_map, ConstantDofMap) else parameter_map.dofs_per_element
        if parameter_map.num_elements != displacement_map.num_elements:
            raise ValueError("VolumetricFemForceResponse: incompatible element count or batch size")
        if width != k:
            raise ValueError("VolumetricFemForceResponse: invalid parameter count")
        self.per_element = isinstance(parameter_map, ElementDofMap)
        T, V = displacement_map.num_elements, displacement_map.num_vertices
        u = np.ascontiguousarray(displacement, dtype=np.float64)
        if u.size != displacement_map.num_dofs or not np.all(np.isfinite(u)):
            raise ValueError("VolumetricFemForceResponse: incompatible map, displacement or responses")
        # The parameters enter through the material only; any value builds the energy's geometry.
        self._energy = _py_energy_class(mat)(displacement_map, rest_position_fields, Fp, np.ones(k), batch_size)
        X, Xe = _rest_geometry(rest_position_fields, V, T)
        corners = Xe.reshape(T, 4, 3) if Xe is not None else X[displacement_map.cells]
        D = corners[:, 1:] - corners[:, :1]
        vol = np.einsum("ij,ij->i", D[:, 0], np.cross(D[:, 1], D[:, 2])) / 6.0
        self._vol = torch.as_tensor(vol, device=self._energy.device)
        self._F = self._energy.deformation_gradients(u)
        self._k, self._T = k, T
        self.displacement = u
        self.num_inputs = parameter_map.num_dofs
        self.num_outputs = displacement_map.num_dofs

    def eval_vjp(self, p, w):
        """(d g / d p)^T w: (k,) for a ConstantDofMap, (k T,) for an ElementDofMap."""
        import torch

        p = np.asarray(p, dtype=np.float64).ravel()
        if p.size != self.num_inputs or not np.all(np.isfinite(p)):
            raise ValueError("Response: p must have num_inputs finite entries")
        wv = np.ascontiguousarray(w, dtype=np.float64)
        if wv.size != self.num_outputs:
            raise ValueError("Response: weights must have num_outputs entries")
        T, k, dev = self._T, self._k, self._energy.device
        th = p.reshape(T, k) if self.per_element else np.broadcast_to(p, (T, k))
        theta = torch.as_tensor(np.ascontiguousarray(th), device=dev)
        Gw = self._energy.deformation_gradients(wv) - torch.eye(3, dtype=torch.float64, device=dev)
        out = self.material.eval(self._F, self._energy._Fp, theta, outputs=("dW_dF", "d2W_dF_dtheta"))
        Dt = _cuda_f64(out["d2W_dF_dtheta"], (T, 3, 3, k), dev)
        per = self._vol[:, None] * torch.einsum("nija,nij->na", Dt, Gw)
        if not bool(torch.all(torch.isfinite(per))):
            raise ValueError("PyVolumetricMaterial.eval returned non-finite values")
        return (per.reshape(-1) if self.per_element else per.sum(0)).cpu().numpy()


def _py_response_class(material, basis=TetP1Basis, quadrature=TetCentroidQuadrature):
    if (basis, quadrature) != (TetP1Basis, TetCentroidQuadrature):
        raise TypeError("VolumetricFemForceMaterialResponse of a Python material is instantiated for "
                        "TetP1Basis, TetCentroidQuadrature")
    return type(f"VolumetricFemForceMaterialResponse[{material.__name__}, {basis.__name__}, {quadrature.__name__}]",
                (VolumetricFemForceMaterialResponsePyTetP1,), {"material": material})


_PY_ENERGY_BASES = {(TetP1Basis, TetCentroidQuadrature): VolumetricFemEnergyPyMaterialTetP1,
                    (HexQ1Basis, GaussLegendre3D_2): VolumetricFemEnergyPyMaterialHexQ1,
                    (HexQ1Basis, GaussLegendre3D_4): VolumetricFemEnergyPyMaterialHexQ1GL4}


def _py_energy_class(material, basis=TetP1Basis, quadrature=TetCentroidQuadrature):
    base = _PY_ENERGY_BASES[(basis, quadrature)]
    return type(f"VolumetricFemEnergy[{material.__name__}, {basis.__name__}, {quadrature.__name__}]", (base,),
                {"material": material})


GaussLegendre3D = Template("GaussLegendre3D", {(2,): GaussLegendre3D_2, (4,): GaussLegendre3D_4})
VolumetricFemEnergy = Template("VolumetricFemEnergy",
                               {(NeoHookean, TetP1Basis, TetCentroidQuadrature): VolumetricFemEnergyTetP1,
                                (NeoHookean, HexQ1Basis, GaussLegendre3D_2): VolumetricFemEnergyHexQ1,
                                (NeoHookean, HexQ1Basis, GaussLegendre3D_4): VolumetricFemEnergyHexQ1GL4,
                                (NeoHookean, HexHermiteBasis, GaussLegendre3D_2): VolumetricFemEnergyHexHermite,
                                (NeoHookean, HexHermiteBasis, GaussLegendre3D_4): VolumetricFemEnergyHexHermiteGL4})
VolumetricFemEnergy.material_factory = _py_energy_class
VolumetricFemForceMaterialResponse = Template(
    "VolumetricFemForceMaterialResponse",
    {(NeoHookean, TetP1Basis, TetCentroidQuadrature): VolumetricFemForceMaterialResponseTetP1,
     (NeoHookean, HexQ1Basis, GaussLegendre3D_2): VolumetricFemForceMaterialResponseHexQ1,
     (NeoHookean, HexQ1Basis, GaussLegendre3D_4): VolumetricFemForceMaterialResponseHexQ1GL4,
     (NeoHookean, HexHermiteBasis, GaussLegendre3D_2): VolumetricFemForceMaterialResponseHexHermite,
     (NeoHookean, HexHermiteBasis, GaussLegendre3D_4): VolumetricFemForceMaterialResponseHexHermiteGL4})
VolumetricFemForceMaterialResponse.material_factory = _py_response_class
VolumetricFemForceFpResponse = Template(
    "VolumetricFemForceFpResponse",
    {(NeoHookean, TetP1Basis, TetCentroidQuadrature): VolumetricFemForceFpResponseTetP1})

# A constant field helper matching the reference tests' constant_fields(value, count).
def constant_fields(value, count):
    v = np.asarray(value, dtype=np.float64).ravel()
    return [AffineResponse(np.zeros((v.size, 3)), v)] * count
