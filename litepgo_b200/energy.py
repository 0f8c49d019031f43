"""Energy interface pieces of litepgo.energy used by the volumetric FEM path.

HessianKind: src/core/energy/scalar/energy.hpp:6-13.
AffineResponse (constant / affine material fields): src/core/energy/response/affine_response.hpp.
QuadraticEnergy as a linear load E = b . x (A must be zero on this path):
src/core/energy/scalar/quadratic_energy.hpp:10-20.
WeightedSumEnergy (elastic + load): src/core/energy/scalar/weighted_sum_energy.hpp:16-47.
"""

import enum

import numpy as np

__all__ = ["HessianKind", "Energy", "AffineResponse", "QuadraticEnergy", "WeightedSumEnergy"]


class HessianKind(enum.IntEnum):
    Exact = 1
    Projected = 2


class Energy:
    """Marker base of the energies of this package (evaluated by the CUDA library)."""

    num_dofs = 0


class AffineResponse:
    """x -> A @ x + offset, used here as a (usually constant) per-element material field."""

    def __init__(self, A, offset=None):
        import scipy.sparse as sp

        A = A.toarray() if sp.issparse(A) else np.asarray(A, dtype=np.float64)
        if A.ndim != 2:
            raise ValueError("AffineResponse requires a 2-D matrix")
        self.A = np.ascontiguousarray(A, dtype=np.float64)
        off = np.zeros(self.A.shape[0]) if offset is None or np.size(offset) == 0 else np.asarray(offset, np.float64)
        if off.shape != (self.A.shape[0],):
            raise ValueError("AffineResponse: offset size must equal the number of outputs")
        self.offset = off.copy()

    @property
    def num_inputs(self):
        return self.A.shape[1]

    @property
    def num_outputs(self):
        return self.A.shape[0]

    def eval_value(self, x):
        return self.A @ np.asarray(x, dtype=np.float64) + self.offset


class QuadraticEnergy(Energy):
    """E(x) = 1/2 x^T A x + b^T x. The GPU Newton path supports A = 0 (a linear load)."""

    def __init__(self, A, b=None):
        import scipy.sparse as sp

        A = sp.csc_matrix(A)
        if A.shape[0] != A.shape[1]:
            raise ValueError("QuadraticEnergy requires a square matrix")
        self.A = A
        self.num_dofs = A.shape[0]
        self.b = np.zeros(self.num_dofs) if b is None or np.size(b) == 0 else np.asarray(b, np.float64).ravel()
        if self.b.size != self.num_dofs:
            raise ValueError("QuadraticEnergy: b size must equal num_dofs")

    @property
    def is_linear(self):
        return self.A.nnz == 0 or not np.any(self.A.data)

    def eval(self, x, gradient=False, hessian=None):
        """(1/2 x^T A x + b^T x, A x + b, A) on the host (quadratic_energy.hpp:10-20)."""
        if hasattr(x, "detach"):
            x = x.detach().cpu().numpy()
        x = np.asarray(x, dtype=np.float64).ravel()
        if x.size != self.num_dofs or not np.all(np.isfinite(x)):
            raise ValueError("Energy::eval: x must have num_dofs finite entries")
        Ax = self.A @ x
        value = 0.5 * float(x @ Ax) + float(self.b @ x)
        return value, (Ax + self.b if gradient else None), (self.A.copy() if hessian else None)

    def eval_value(self, x):
        return self.eval(x)[0]

    def eval_gradient(self, x):
        return self.eval(x, gradient=True)[1]


class WeightedSumEnergy(Energy):
    """E(x) = sum_i w_i E_i(x) over terms with the same DOFs (a list of (energy, weight))."""

    def __init__(self, terms):
        terms = [(t, 1.0) if isinstance(t, Energy) else (t[0], float(t[1])) for t in terms]
        if not terms:
            raise ValueError("WeightedSumEnergy requires at least one term")
        n = terms[0][0].num_dofs
        for e, w in terms:
            if e.num_dofs != n:
                raise ValueError("WeightedSumEnergy terms must share num_dofs")
            if not np.isfinite(w) or w == 0:
                raise ValueError("WeightedSumEnergy weights must be finite and nonzero")
        self.terms = terms
        self.num_dofs = n

    def split(self):
        """(fem_energy, load f_ext) with E = fem(x) - f_ext . x; raises ValueError otherwise."""
        from .fem import VolumetricFemEnergyTetP1

        fem, b = None, np.zeros(self.num_dofs)
        for e, w in self.terms:
            if isinstance(e, VolumetricFemEnergyTetP1):
                if fem is not None or w != 1.0:
                    raise ValueError("WeightedSumEnergy: one elastic term with weight 1 is supported on the GPU path")
                fem = e
            elif isinstance(e, QuadraticEnergy) and e.is_linear:
                b += w * e.b
            else:
                raise ValueError("WeightedSumEnergy: only an elastic term plus linear loads are supported on the GPU path")
        if fem is None:
            raise ValueError("WeightedSumEnergy: no VolumetricFemEnergy term")
        return fem, -b

    def eval(self, x, gradient=False, hessian=None):
        fem, f = self.split()
        value, g, H = fem.eval(x, gradient=gradient, hessian=hessian)
        xv = np.asarray(x, dtype=np.float64)
        value -= float(f @ xv)
        if g is not None:
            g = g - f
        return value, g, H

    def eval_value(self, x):
        return self.eval(x)[0]

    def eval_gradient(self, x):
        return self.eval(x, gradient=True)[1]

    def eval_hessian(self, x, kind=HessianKind.Exact):
        return self.eval(x, hessian=kind)[2]

    def max_feasible_step(self, x, dx):
        fem, _ = self.split()
        return fem.max_feasible_step(x, dx)
