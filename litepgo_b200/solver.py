"""Nonlinear solvers mirroring litepgo.solver for the volumetric FEM path.

newton_solve(energy, fixed, x0, options, solver=None, on_iteration=None) keeps the binding's
signature (src/binding/solver/newton.cpp:62-82) and the semantics of newton.cpp:112-183;
the direct sparse solver is replaced by block-Jacobi PCG on the GPU block-CSR Hessian, so
``solver`` must be None. NewtonOptions keeps the reference fields and defaults
(src/core/solver/newton.hpp:13-20) and adds the GPU linear-solve controls.

StaticEquilibriumResponse(num_parameters, fixed, initial, options, make_energy,
make_response) mirrors src/core/solver/static_equilibrium_response.hpp:15-32: p -> u*(p)
from the same initial state on every call; eval_vjp solves the adjoint with the EXACT
Hessian and returns -(dg/dtheta)^T lambda (static_equilibrium_response.cpp:43-88).
"""

import ctypes
import enum

import numpy as np

from . import _native as N
from .energy import HessianKind, WeightedSumEnergy

__all__ = ["NewtonOptions", "NewtonStatus", "NewtonResult", "NewtonStep", "newton_solve", "batch_newton_solve",
           "StaticEquilibriumResponse"]


class NewtonStatus(enum.IntEnum):
    Converged = 0
    MaxIterations = 1
    StepTooSmall = 2
    NoDescentDirection = 3


class NewtonOptions:
    """Options of newton_solve.

    Reference fields: gradient_tolerance (required), max_iterations=50,
    hessian=HessianKind.Projected, max_line_search_steps=30, line_search_shrink=0.5.
    GPU additions: stop_rule ("max_abs": max |g_free| <= tol, the reference rule; "relative":
    ||g_free||_2 <= tol ||g_free(x0)||_2), accept_rule ("noise": the reference's decrease
    within 16 eps; "armijo": sufficient decrease c = 1e-4 plus that noise), precision
    ("f64" or "mixed": FP32 Hessian and PCG, FP64 energy and residual), cg_tolerance (cap of
    the PCG forcing term), cg_max_iterations, and exact_below (0 = off: once the gradient norm
    falls to exact_below times its initial value, the Exact Hessian replaces ``hessian``).
    """

    def __init__(self, gradient_tolerance=float("nan"), max_iterations=50, hessian=HessianKind.Projected,
                 max_line_search_steps=30, line_search_shrink=0.5, stop_rule="max_abs", accept_rule="noise",
                 precision="f64", cg_tolerance=1e-2, cg_max_iterations=20000, exact_below=0.0):
        self.gradient_tolerance = gradient_tolerance
        self.max_iterations = max_iterations
        self.hessian = hessian
        self.max_line_search_steps = max_line_search_steps
        self.line_search_shrink = line_search_shrink
        self.stop_rule = stop_rule
        self.accept_rule = accept_rule
        self.precision = precision
        self.cg_tolerance = cg_tolerance
        self.cg_max_iterations = cg_max_iterations
        self.exact_below = exact_below

    def to_c(self):
        o = N.NewtonOptionsC()
        o.gradient_tolerance = float(self.gradient_tolerance)
        o.max_iterations = int(self.max_iterations)
        o.hessian = int(self.hessian)
        o.max_line_search_steps = int(self.max_line_search_steps)
        o.line_search_shrink = float(self.line_search_shrink)
        o.stop_rule = {"max_abs": 0, "relative": 1}[self.stop_rule]
        o.accept_rule = {"noise": 0, "armijo": 1}[self.accept_rule]
        o.precision = N.PRECISION_F64 if self.precision == "f64" else N.PRECISION_MIXED
        o.cg_tolerance = float(self.cg_tolerance)
        o.cg_max_iterations = int(self.cg_max_iterations)
        o.exact_below = float(self.exact_below)
        return o


class NewtonResult:
    def __init__(self, status, x, energy, gradient_norm, iterations, gradient_norm0=0.0, cg_iterations=0,
                 line_search_evaluations=0, seconds=0.0):
        self.status = NewtonStatus(status)
        self.x = x
        self.energy = energy
        self.gradient_norm = gradient_norm
        self.iterations = iterations
        self.gradient_norm0 = gradient_norm0
        self.cg_iterations = cg_iterations
        self.line_search_evaluations = line_search_evaluations
        self.seconds = seconds

    def __repr__(self):
        return (f"NewtonResult(status={self.status.name}, iterations={self.iterations}, energy={self.energy:.6e}, "
                f"gradient_norm={self.gradient_norm:.3e}, cg_iterations={self.cg_iterations})")


class NewtonStep:
    """What one iteration did (newton.hpp:34-44; binding src/binding/solver/newton.cpp:42-50),
    passed to newton_solve's on_iteration: iteration, energy, gradient_norm (max-norm over the
    free DOFs), pattern_changed, diagonal_shifts, feasible_step, step, line_search_evaluations;
    plus gradient_norm_2 (2-norm) and cg_iterations (PCG iterations of the step), which the
    reference does not report."""

    __slots__ = ("iteration", "energy", "gradient_norm", "pattern_changed", "diagonal_shifts", "feasible_step", "step",
                 "line_search_evaluations", "gradient_norm_2", "cg_iterations")

    def __init__(self, c):
        self.iteration = int(c.iteration)
        self.energy = float(c.energy)
        self.gradient_norm = float(c.gradient_norm)
        self.pattern_changed = bool(c.pattern_changed)
        self.diagonal_shifts = int(c.diagonal_shifts)
        self.feasible_step = float(c.feasible_step)
        self.step = float(c.step)
        self.line_search_evaluations = int(c.line_search_evaluations)
        self.gradient_norm_2 = float(c.gradient_norm_2)
        self.cg_iterations = int(c.cg_iterations)

    def __repr__(self):
        return (f"NewtonStep(iteration={self.iteration}, energy={self.energy:.6e}, gradient_norm={self.gradient_norm:.3e}, "
                f"diagonal_shifts={self.diagonal_shifts}, step={self.step:.3g}, "
                f"line_search_evaluations={self.line_search_evaluations})")


def _split_energy(energy):
    """(fem, elastic weight, A or None, f_ext or None, constant) of a potential; fem is a native
    or a Python-material VolumetricFemEnergy."""
    from .fem import VolumetricFemEnergyPyMaterialTetP1, VolumetricFemEnergyTetP1

    if isinstance(energy, (VolumetricFemEnergyTetP1, VolumetricFemEnergyPyMaterialTetP1)):
        return energy, 1.0, None, None, 0.0
    if isinstance(energy, WeightedSumEnergy):
        fem, w, A, f, c = energy.potential()
        return fem, w, A, (f if np.any(f) else None), c
    raise TypeError("newton_solve: energy must be a VolumetricFemEnergy or a WeightedSumEnergy of one plus quadratic "
                    "terms")


class _DeviceArray:
    """A float64 device buffer of the library as a torch-importable array (zero copy)."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _view(ptr, shape, device):
    import torch

    return torch.as_tensor(_DeviceArray(ptr, shape), device=device)


def _material_callbacks(fem, t, keep, box):
    """The material and feasible-step callbacks of a Python-material energy (PyVolumetricMaterial
    or TorchVolumetricMaterial): the library hands over F at every material row and takes W, P
    and A back in its own device buffers."""
    import torch

    dev = fem.device

    def material(Fp, rows, want, Wp, Pp, Ap, _user):
        try:
            F = _view(Fp, (rows, 3, 3), dev)
            outputs = ("W",) + (("dW_dF",) if want >= 1 else ()) + (("d2W_dF2",) if want >= 2 else ())
            vals = fem._material(F, outputs)
            _view(Wp, (rows,), dev).copy_(vals[0])
            if want >= 1:
                _view(Pp, (rows, 3, 3), dev).copy_(vals[1])
            if want >= 2:
                _view(Ap, (rows, 3, 3, 3, 3), dev).copy_(vals[2])
            return 0
        except BaseException as exc:  # re-raised after the solve returns
            box.append(exc)
            return 1

    cb = N.MATERIAL_CALLBACK(material)
    keep.append(cb)
    t.material = cb
    if fem.material.eval_feasible_step is not None:
        from .fem import _cuda_f64

        def feasible(Fp, Gp, rows, alpha, _user):
            try:
                F = _view(Fp, (rows, 3, 3), dev)
                dF = _view(Gp, (rows, 3, 3), dev) - torch.eye(3, dtype=torch.float64, device=dev)
                bound = _cuda_f64(fem.material.eval_feasible_step(F, fem._Fp, fem._theta, dF), (rows,), dev)
                if not bool(torch.all(torch.isfinite(bound))):
                    raise ValueError("PyVolumetricMaterial.eval_feasible_step returned non-finite values")
                alpha[0] = float(torch.clamp(bound, 0.0, 1.0).min()) if rows else 1.0
                return 0
            except BaseException as exc:
                box.append(exc)
                return 1

        fcb = N.FEASIBLE_CALLBACK(feasible)
        keep.append(fcb)
        t.feasible = fcb


def _terms(w, A, c, on_iteration, fem=None):
    """lpg_newton_terms for a weighted sum, an optional callback and a Python material (None when
    none is needed). Returns (terms, keep-alive list, error box): an exception raised by a
    callback stops the solve (LPG_ESTOPPED) and is re-raised by the caller from the box."""
    from .fem import VolumetricFemEnergyPyMaterialTetP1

    is_material = isinstance(fem, VolumetricFemEnergyPyMaterialTetP1)
    if w == 1.0 and A is None and c == 0.0 and on_iteration is None and not is_material:
        return None, [], None
    keep, box = [], []
    t = N.NewtonTermsC()
    t.elastic_weight = float(w)
    t.constant = float(c)
    if A is not None:
        A = A.tocsr()
        A.sum_duplicates()
        ptr = np.ascontiguousarray(A.indptr, dtype=np.int32)
        idx = np.ascontiguousarray(A.indices, dtype=np.int32)
        val = np.ascontiguousarray(A.data, dtype=np.float64)
        keep += [ptr, idx, val]
        t.a_indptr, t.a_indices, t.a_values = N.iptr(ptr), N.iptr(idx), N.dptr(val)
    if on_iteration is not None:
        def trampoline(step_ptr, _user):
            try:
                on_iteration(NewtonStep(step_ptr.contents))
                return 0
            except BaseException as exc:  # re-raised after the solve returns
                box.append(exc)
                return 1

        cb = N.NEWTON_CALLBACK(trampoline)
        keep.append(cb)
        t.on_iteration = cb
    if is_material:
        _material_callbacks(fem, t, keep, box)
    return t, keep, box


def newton_solve(energy, fixed, x0, options, solver=None, on_iteration=None):
    """Minimises energy over the free DOFs of ``fixed`` from x0 on the GPU. ``energy`` is a
    VolumetricFemEnergy or a WeightedSumEnergy of one plus QuadraticEnergy /
    VertexPullingEnergy terms; on_iteration(NewtonStep) is called as the reference calls it."""
    if solver is not None:
        raise ValueError("newton_solve: the GPU path solves with block-Jacobi PCG; pass solver=None")
    fem, w, A, f, c = _split_energy(energy)
    n = fem.num_dofs
    if fixed.num_dofs != n:
        raise ValueError("newton_solve: energy, fixed DOFs, and x0 must have the same DOF count")
    is_dev = hasattr(x0, "is_cuda") and x0.is_cuda
    if is_dev:
        import torch

        x0t = x0.detach().contiguous()
        if x0t.dtype != torch.float64 or x0t.numel() != n:
            raise ValueError("newton_solve: energy, fixed DOFs, and x0 must have the same DOF count")
        xo = torch.empty_like(x0t)
        ft = None if f is None else torch.as_tensor(f, device=x0t.device)
        N.check(N.lib.lpg_fem_set_stream(fem.handle, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        ptrs = (N.vptr(ft), N.vptr(x0t), N.vptr(xo), N.MEM_DEVICE)
    else:
        x0a = np.ascontiguousarray(x0, dtype=np.float64)
        if x0a.size != n:
            raise ValueError("newton_solve: energy, fixed DOFs, and x0 must have the same DOF count")
        xo = np.empty(n)
        fa = None if f is None else np.ascontiguousarray(f)
        N.check(N.lib.lpg_fem_set_stream(fem.handle, None))
        ptrs = (N.vptr(fa), N.vptr(x0a), N.vptr(xo), N.MEM_HOST)
    fixed_arr = np.ascontiguousarray(fixed.fixed_dofs, dtype=np.int32)
    res = N.NewtonResultC()
    opts = options.to_c()
    terms, keep, box = _terms(w, A, c, on_iteration, fem)
    if terms is not None and terms.material:
        # The material runs on torch's current stream: the library's work goes on the same one.
        import torch

        N.check(N.lib.lpg_fem_set_stream(fem.handle, ctypes.c_void_p(torch.cuda.current_stream(fem.device).cuda_stream)))
    if terms is None:
        N.check(N.lib.lpg_newton_solve(fem.handle, N.iptr(fixed_arr), int(fixed_arr.size), ptrs[0], ptrs[1], ptrs[3],
                                       ctypes.byref(opts), ptrs[2], ctypes.byref(res)))
    else:
        code = N.lib.lpg_newton_solve_terms(fem.handle, ctypes.byref(terms), N.iptr(fixed_arr), int(fixed_arr.size),
                                            ptrs[0], ptrs[1], ptrs[3], ctypes.byref(opts), ptrs[2], ctypes.byref(res))
        if code == N.LPG_ESTOPPED and box:
            raise box[0]
        N.check(code)
    del keep
    return NewtonResult(res.status, xo, res.energy, res.gradient_norm, res.iterations, res.gradient_norm0,
                        res.cg_iterations, res.line_search_evaluations, res.seconds)


def batch_newton_solve(energy, mesh_vertex_offsets, mesh_element_offsets, fixed, x0, options):
    """newton_solve of many independent meshes held in one energy (no reference counterpart).

    ``energy`` is one VolumetricFemEnergy (plus linear loads) over the meshes' disjoint union,
    the meshes being contiguous vertex ranges ``mesh_vertex_offsets`` and element ranges
    ``mesh_element_offsets`` (num_meshes + 1 entries each, see ``mesh.concatenate``). Every
    mesh has its own stop test, PCG, feasible step and line search; the element and SpMV work
    runs once over all of them. Returns (x, per_mesh, total): x over the union, per_mesh a list
    of NewtonResult-like records (status, iterations, energy, gradient_norm, gradient_norm0,
    seconds = time from the call's start to the iteration that ended the mesh), total the
    whole call's NewtonResult.
    """
    fem, w, A, f, c = _split_energy(energy)
    if w != 1.0 or A is not None or c != 0.0:
        raise ValueError("batch_newton_solve: the energy must be the elastic term plus linear loads")
    n = fem.num_dofs
    voff = np.ascontiguousarray(mesh_vertex_offsets, dtype=np.int32)
    eoff = np.ascontiguousarray(mesh_element_offsets, dtype=np.int32)
    if voff.ndim != 1 or eoff.shape != voff.shape or voff.size < 2:
        raise ValueError("batch_newton_solve: mesh offsets must be two arrays of num_meshes + 1 entries")
    M = voff.size - 1
    if fixed.num_dofs != n:
        raise ValueError("newton_solve: energy, fixed DOFs, and x0 must have the same DOF count")
    is_dev = hasattr(x0, "is_cuda") and x0.is_cuda
    if is_dev:
        import torch

        x0t = x0.detach().contiguous()
        if x0t.dtype != torch.float64 or x0t.numel() != n:
            raise ValueError("newton_solve: energy, fixed DOFs, and x0 must have the same DOF count")
        xo = torch.empty_like(x0t)
        ft = None if f is None else torch.as_tensor(f, device=x0t.device)
        N.check(N.lib.lpg_fem_set_stream(fem.handle, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        ptrs = (N.vptr(ft), N.vptr(x0t), N.vptr(xo), N.MEM_DEVICE)
    else:
        x0a = np.ascontiguousarray(x0, dtype=np.float64)
        if x0a.size != n:
            raise ValueError("newton_solve: energy, fixed DOFs, and x0 must have the same DOF count")
        xo = np.empty(n)
        fa = None if f is None else np.ascontiguousarray(f)
        N.check(N.lib.lpg_fem_set_stream(fem.handle, None))
        ptrs = (N.vptr(fa), N.vptr(x0a), N.vptr(xo), N.MEM_HOST)
    fixed_arr = np.ascontiguousarray(fixed.fixed_dofs, dtype=np.int32)
    per = (N.BatchMeshResultC * M)()
    res = N.NewtonResultC()
    opts = options.to_c()
    N.check(N.lib.lpg_batch_newton_solve(fem.handle, M, N.iptr(voff), N.iptr(eoff), N.iptr(fixed_arr),
                                         int(fixed_arr.size), ptrs[0], ptrs[1], ptrs[3], ctypes.byref(opts), ptrs[2],
                                         per, ctypes.byref(res)))
    meshes = [NewtonResult(p.status, None, p.energy, p.gradient_norm, p.iterations, p.gradient_norm0, 0, 0, p.seconds)
              for p in per]
    total = NewtonResult(res.status, xo, res.energy, res.gradient_norm, res.iterations, res.gradient_norm0,
                         res.cg_iterations, res.line_search_evaluations, res.seconds)
    return xo, meshes, total


class StaticEquilibriumResponse:
    """p -> equilibrium displacement; eval_vjp by one adjoint solve on the GPU."""

    def __init__(self, num_parameters, fixed, initial, options, make_energy, make_response, precision="f64",
                 adjoint_tolerance=1e-10):
        initial = np.asarray(initial, dtype=np.float64)
        o = options
        if (int(num_parameters) <= 0 or initial.size != fixed.num_dofs or not np.all(np.isfinite(initial))
                or make_energy is None or make_response is None or not np.isfinite(o.gradient_tolerance)
                or o.gradient_tolerance < 0 or o.max_iterations < 0 or o.max_line_search_steps < 1
                or not (0 < o.line_search_shrink < 1)):
            raise ValueError("StaticEquilibriumResponse: invalid initial state, options or callbacks")
        self.num_inputs = int(num_parameters)
        self.num_outputs = fixed.num_dofs
        self.fixed = fixed
        self.initial = initial.copy()
        self.options = options
        self.make_energy = make_energy
        self.make_response = make_response
        self.precision = precision
        self.adjoint_tolerance = adjoint_tolerance
        self._last = None  # (p, potential, x) of the last solve, reused for the same p

    def _solve(self, p):
        p = np.asarray(p, dtype=np.float64).ravel()
        if p.size != self.num_inputs or not np.all(np.isfinite(p)):
            raise ValueError("Response: p must have num_inputs finite entries")
        if self._last is not None and np.array_equal(self._last[0], p):
            return self._last
        potential = self.make_energy(p)
        if potential is None or potential.num_dofs != self.num_outputs:
            raise ValueError("StaticEquilibriumResponse: incompatible energy")
        result = newton_solve(potential, self.fixed, self.initial, self.options)
        if result.status != NewtonStatus.Converged:
            raise ValueError("StaticEquilibriumResponse: equilibrium did not converge")
        self._last = (p.copy(), potential, np.array(result.x, copy=True))
        return self._last

    def eval_value(self, p):
        return self._solve(p)[2]

    def eval_vjp(self, p, w):
        p, potential, x = self._solve(p)
        w = np.ascontiguousarray(w, dtype=np.float64)
        if w.size != self.num_outputs:
            raise ValueError("Response: weights must have num_outputs entries")
        if self.fixed.num_free == 0:
            return np.zeros(self.num_inputs)
        force = self.make_response(x)
        if force is None or force.num_inputs != self.num_inputs or force.num_outputs != self.num_outputs:
            raise ValueError("StaticEquilibriumResponse: incompatible force response")
        fem, wf, A, _, c = _split_energy(potential)
        fixed_arr = np.ascontiguousarray(self.fixed.fixed_dofs, dtype=np.int32)
        prec = N.PRECISION_F64 if self.precision == "f64" else N.PRECISION_MIXED
        from .fem import VolumetricFemEnergyPyMaterialTetP1, VolumetricFemForceMaterialResponsePyTetP1

        if (wf != 1.0 or A is not None or isinstance(fem, VolumetricFemEnergyPyMaterialTetP1)
                or isinstance(force, VolumetricFemForceMaterialResponsePyTetP1)):
            # The general form (static_equilibrium_response.cpp:43-88): lambda from the potential's
            # Exact Hessian at x (a Python material evaluated through its callback), then
            # -(dg/dp)^T lambda from the caller's force response.
            terms, keep, box = _terms(wf, A, c, None, fem)
            if terms is not None and terms.material:
                import torch

                N.check(N.lib.lpg_fem_set_stream(fem.handle,
                                                 ctypes.c_void_p(torch.cuda.current_stream(fem.device).cuda_stream)))
            else:
                N.check(N.lib.lpg_fem_set_stream(fem.handle, None))
            lam = np.empty(self.num_outputs)
            code = N.lib.lpg_adjoint_solve_terms(fem.handle, ctypes.byref(terms) if terms is not None else None,
                                                 N.vptr(np.ascontiguousarray(x)), N.vptr(w), N.iptr(fixed_arr),
                                                 int(fixed_arr.size), N.MEM_HOST, prec, float(self.adjoint_tolerance),
                                                 N.vptr(lam))
            if code == N.LPG_ESTOPPED and box:
                raise box[0]
            N.check(code)
            del keep
            return -np.asarray(force.eval_vjp(p, lam), dtype=np.float64)
        from .fem import VolumetricFemForceFpResponseTetP1, VolumetricFemForceRestPositionResponseTetP1

        if isinstance(force, VolumetricFemForceFpResponseTetP1):
            T = fem.num_elements
            out = np.empty(9 * T if force.per_element else 9)
            N.check(N.lib.lpg_fem_set_stream(fem.handle, None))
            N.check(N.lib.lpg_adjoint_fp(fem.handle, N.vptr(x), N.vptr(w), N.iptr(fixed_arr), int(fixed_arr.size),
                                         N.MEM_HOST, prec, float(self.adjoint_tolerance),
                                         1 if force.per_element else 0, N.vptr(out), None))
            return out
        if isinstance(force, VolumetricFemForceRestPositionResponseTetP1):
            out = np.empty(self.num_inputs)
            N.check(N.lib.lpg_fem_set_stream(fem.handle, None))
            N.check(N.lib.lpg_adjoint_rest(fem.handle, N.vptr(x), N.vptr(w), N.iptr(fixed_arr), int(fixed_arr.size),
                                           N.MEM_HOST, prec, float(self.adjoint_tolerance), N.vptr(out), None))
            return out
        T = fem.num_elements
        out = np.empty(2 * T if force.per_element else 2)
        N.check(N.lib.lpg_fem_set_stream(fem.handle, None))
        N.check(N.lib.lpg_adjoint_theta(fem.handle, N.vptr(x), N.vptr(w), N.iptr(fixed_arr), int(fixed_arr.size),
                                        N.MEM_HOST, prec, float(self.adjoint_tolerance),
                                        1 if force.per_element else 0, N.vptr(out), None))
        return out
