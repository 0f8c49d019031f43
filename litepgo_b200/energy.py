"""Energy interface pieces of litepgo.energy used by the volumetric FEM path.

HessianKind: src/core/energy/scalar/energy.hpp:6-13.
AffineResponse (constant / affine material fields): src/core/energy/response/affine_response.hpp.
QuadraticEnergy E = 1/2 x^T A x + b . x: src/core/energy/scalar/quadratic_energy.hpp:10-20.
VertexPullingEnergy (zero-rest-length springs): src/core/energy/scalar/vertex_pulling_energy.hpp.
WeightedSumEnergy (one elastic term plus quadratic terms, any weights):
src/core/energy/scalar/weighted_sum_energy.hpp:16-47.
"""

import enum

import numpy as np

__all__ = ["HessianKind", "Energy", "AffineResponse", "QuadraticEnergy", "VertexPullingEnergy", "WeightedSumEnergy"]


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
    """E(x) = 1/2 x^T A x + b^T x (quadratic_energy.hpp:10-20). On the GPU Newton path A must be
    symmetric and couple only DOFs of vertices that share an element (springs, penalties and
    loads on a mesh)."""

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

    def quadratic_form(self):
        """(A, b, c) with E(x) = 1/2 x^T A x + b^T x + c."""
        return self.A, self.b, 0.0

    def max_feasible_step(self, x, dx):
        return 1.0


class VertexPullingEnergy(Energy):
    """Zero-rest-length springs pulling vertices toward targets (the reference's
    VertexPullingEnergy, src/core/energy/scalar/vertex_pulling_energy.hpp; binding
    src/binding/energy/scalar/vertex_pulling_energy.cpp): E(x) = k/2 sum_i |x[d_i] - t_i|^2 with
    d_i vertex i's three position DOFs and t_i its target row. Its Hessian is the constant
    diagonal k on the pulled DOFs (both Hessian kinds)."""

    def __init__(self, num_dofs, position_dofs, targets, stiffness):
        import scipy.sparse as sp

        num_dofs = int(num_dofs)
        dofs = np.asarray(position_dofs, dtype=np.int64).reshape(-1, 3)
        t = np.asarray(targets, dtype=np.float64)
        if num_dofs < 0:
            raise ValueError("VertexPullingEnergy requires a non-negative DOF count")
        flat = np.sort(dofs.ravel())
        if flat.size and (flat[0] < 0 or flat[-1] >= num_dofs):
            raise ValueError("VertexPullingEnergy position DOFs must be in [0, num_dofs)")
        if flat.size and np.any(flat[1:] == flat[:-1]):
            raise ValueError("VertexPullingEnergy position DOFs must be distinct")
        if t.size != dofs.size or t.ndim > 2 or (t.ndim == 2 and t.shape[1] != 3):
            raise ValueError("VertexPullingEnergy requires one target row per pulled vertex")
        if not np.all(np.isfinite(t)):
            raise ValueError("VertexPullingEnergy requires three finite target entries per pulled vertex")
        stiffness = float(stiffness)
        if not np.isfinite(stiffness) or stiffness <= 0.0:
            raise ValueError("VertexPullingEnergy requires a finite positive stiffness")
        self.num_dofs = num_dofs
        self.position_dofs = dofs.astype(np.int32)
        self.targets = t.reshape(-1, 3).copy()
        self.stiffness = stiffness
        d = self.position_dofs.ravel()
        self._A = sp.csr_matrix((np.full(d.size, stiffness), (d, d)), shape=(num_dofs, num_dofs))
        self._b = np.zeros(num_dofs)
        self._b[d] = -stiffness * self.targets.ravel()
        self._c = 0.5 * stiffness * float(self.targets.ravel() @ self.targets.ravel())

    def eval(self, x, gradient=False, hessian=None):
        if hasattr(x, "detach"):
            x = x.detach().cpu().numpy()
        x = np.asarray(x, dtype=np.float64).ravel()
        if x.size != self.num_dofs or not np.all(np.isfinite(x)):
            raise ValueError("Energy::eval: x must have num_dofs finite entries")
        d = self.position_dofs.ravel()
        gap = x[d] - self.targets.ravel()
        value = 0.5 * self.stiffness * float(gap @ gap)
        g = None
        if gradient:
            g = np.zeros(self.num_dofs)
            g[d] = self.stiffness * gap
        return value, g, (self._A.tocsc() if hessian else None)

    def eval_value(self, x):
        return self.eval(x)[0]

    def eval_gradient(self, x):
        return self.eval(x, gradient=True)[1]

    def eval_hessian(self, x, kind=HessianKind.Exact):
        return self.eval(x, hessian=kind)[2]

    def quadratic_form(self):
        """(A, b, c) with E(x) = 1/2 x^T A x + b^T x + c."""
        return self._A, self._b, self._c

    def max_feasible_step(self, x, dx):
        return 1.0


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

    def potential(self):
        """The sum as (fem_energy, elastic weight, A or None, f_ext, c) with
        E(x) = w fem(x) + 1/2 x^T A x - f_ext . x + c: one elastic term of any nonzero weight
        plus QuadraticEnergy / VertexPullingEnergy terms (their weighted A, b and constants
        summed). Raises ValueError for other terms."""
        import scipy.sparse as sp

        from .fem import VolumetricFemEnergyPyMaterialTetP1, VolumetricFemEnergyTetP1

        fem, wf, A, b, c = None, 1.0, None, np.zeros(self.num_dofs), 0.0
        for e, w in self.terms:
            if isinstance(e, (VolumetricFemEnergyTetP1, VolumetricFemEnergyPyMaterialTetP1)):
                if fem is not None:
                    raise ValueError("WeightedSumEnergy: one elastic term is supported on the GPU path")
                fem, wf = e, w
            elif isinstance(e, (QuadraticEnergy, VertexPullingEnergy)):
                Ae, be, ce = e.quadratic_form()
                if Ae.nnz and np.any(Ae.data):
                    A = w * sp.csr_matrix(Ae) if A is None else A + w * sp.csr_matrix(Ae)
                b += w * be
                c += w * ce
            else:
                raise ValueError("WeightedSumEnergy: only an elastic term plus quadratic terms (QuadraticEnergy, "
                                 "VertexPullingEnergy) are supported on the GPU path")
        if fem is None:
            raise ValueError("WeightedSumEnergy: no VolumetricFemEnergy term")
        return fem, wf, (None if A is None else sp.csr_matrix(A)), -b, c

    def split(self):
        """(fem_energy, load f_ext) with E = fem(x) - f_ext . x; raises ValueError when the sum
        has a weighted elastic term, a non-zero quadratic matrix or a constant."""
        fem, w, A, f, c = self.potential()
        if w != 1.0 or A is not None or c != 0.0:
            raise ValueError("WeightedSumEnergy: this sum is more than an elastic term plus linear loads")
        return fem, f

    def eval(self, x, gradient=False, hessian=None):
        fem, w, A, f, c = self.potential()
        value, g, H = fem.eval(x, gradient=gradient, hessian=hessian)
        xv = np.asarray(x.detach().cpu().numpy() if hasattr(x, "detach") else x, dtype=np.float64)
        value = w * value - float(f @ xv) + c
        if A is not None:
            Ax = A @ xv
            value += 0.5 * float(xv @ Ax)
        if g is not None:
            g = w * g - f
            if A is not None:
                g = g + Ax
        if H is not None:
            H = w * H
            if A is not None:
                H = (H + A).tocsc()
        return value, g, H

    def eval_value(self, x):
        return self.eval(x)[0]

    def eval_gradient(self, x):
        return self.eval(x, gradient=True)[1]

    def eval_hessian(self, x, kind=HessianKind.Exact):
        return self.eval(x, hessian=kind)[2]

    def max_feasible_step(self, x, dx):
        fem = self.potential()[0]
        return fem.max_feasible_step(x, dx)
