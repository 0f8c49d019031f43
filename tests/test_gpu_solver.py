"""GPU Newton and adjoint against the CPU oracle (direct LDL^T solves) and finite differences."""

import numpy as np
import pytest

import oracle
from conftest import TWO_TET_CELLS, TWO_TET_THETA, TWO_TET_X, rel_err
from litepgo_b200 import dof, energy, fem, mesh, solver, workloads

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def total_energy(w):
    e = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    load = energy.QuadraticEnergy(np.zeros((w["X"].size, w["X"].size)), -w["f"])
    return e, energy.WeightedSumEnergy([(e, 1.0), (load, 1.0)])


# volumetric_fem_energy_tet_p1_gtest.cpp:153-169 on the GPU path.
def test_two_tet_newton_relax():
    e = fem.VolumetricFemEnergyTetP1.from_arrays(TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA)
    u = np.zeros(15)
    u[11], u[14] = 0.3, -0.2
    initial = e.eval_value(u)
    res = solver.newton_solve(e, dof.DofReduction(15, range(9)), u, solver.NewtonOptions(gradient_tolerance=1e-9))
    assert res.status == solver.NewtonStatus.Converged
    assert res.iterations > 0 and res.energy < initial
    assert abs(res.energy) < 1e-12
    assert np.all(res.x[:9] == 0)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_gravity_newton_matches_oracle(precision):
    w = workloads.gravity_box(4, seed=0)
    fem_e, total = total_energy(w)
    fixed = dof.DofReduction(w["X"].size, w["fixed"])
    opts = solver.NewtonOptions(gradient_tolerance=1e-8, stop_rule="relative", accept_rule="armijo",
                                precision=precision, max_iterations=100)
    res = solver.newton_solve(total, fixed, w["u0"], opts)
    assert res.status == solver.NewtonStatus.Converged, res
    orc = oracle.OracleMesh(w["X"], w["tets"], w["theta"])
    xr, info = orc.newton(w["fixed"], w["u0"], f_ext=w["f"], tol=1e-10, hessian=2, stop_rule=1, accept_rule=1,
                          linear_solver=0, max_iterations=100)
    assert info["status"] == 0
    assert rel_err(res.x, xr) <= 1e-6
    # Independent check of convergence with the oracle's gradient.
    _, g, _ = orc.eval(res.x, True, 0)
    g = g - w["f"]
    free = fixed.free_dofs
    assert np.linalg.norm(g[free]) <= 1.5e-8 * res.gradient_norm0
    assert np.all(res.x[w["fixed"]] == 0)


def test_reference_stop_rule_and_statuses():
    w = workloads.gravity_box(3, seed=1)
    _, total = total_energy(w)
    fixed = dof.DofReduction(w["X"].size, w["fixed"])
    res = solver.newton_solve(total, fixed, w["u0"], solver.NewtonOptions(gradient_tolerance=1e-6))
    assert res.status == solver.NewtonStatus.Converged
    orc = oracle.OracleMesh(w["X"], w["tets"], w["theta"])
    _, g, _ = orc.eval(res.x, True, 0)
    assert np.abs((g - w["f"])[fixed.free_dofs]).max() <= 1e-6
    res0 = solver.newton_solve(total, fixed, w["u0"], solver.NewtonOptions(gradient_tolerance=1e-6, max_iterations=0))
    assert res0.status == solver.NewtonStatus.MaxIterations and res0.iterations == 0
    with pytest.raises(ValueError, match="gradient_tolerance"):
        solver.newton_solve(total, fixed, w["u0"], solver.NewtonOptions())
    with pytest.raises(ValueError, match="line_search_shrink"):
        solver.newton_solve(total, fixed, w["u0"], solver.NewtonOptions(gradient_tolerance=1, line_search_shrink=1))
    with pytest.raises(ValueError, match="solver=None"):
        solver.newton_solve(total, fixed, w["u0"], solver.NewtonOptions(gradient_tolerance=1), solver=object())


def test_all_fixed_returns_initial_state():
    e = fem.VolumetricFemEnergyTetP1.from_arrays(TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA)
    u = 0.01 * TWO_TET_X.ravel()
    res = solver.newton_solve(e, dof.DofReduction(15, range(15)), u, solver.NewtonOptions(gradient_tolerance=1e-9))
    assert res.status == solver.NewtonStatus.Converged
    np.testing.assert_array_equal(res.x, u)


def _equilibrium(w, theta_flat, opts):
    topo = mesh.TetTopology(w["X"].shape[0], w["tets"])
    vm = dof.VertexDofMap(topo, 3)
    fixed = dof.DofReduction(w["X"].size, w["fixed"])
    Energy = fem.VolumetricFemEnergy[fem.NeoHookean, fem.TetP1Basis, fem.TetCentroidQuadrature]
    Force = fem.VolumetricFemForceMaterialResponse[fem.NeoHookean, fem.TetP1Basis, fem.TetCentroidQuadrature]
    load = energy.QuadraticEnergy(np.zeros((w["X"].size,) * 2), -w["f"])

    def make_energy(p):
        return energy.WeightedSumEnergy([(Energy(vm, w["X"], None, p.reshape(-1, 2)), 1.0), (load, 1.0)])

    def make_response(u):
        return Force(dof.ElementDofMap(topo, 2), vm, w["X"], u, None)

    return solver.StaticEquilibriumResponse(theta_flat.size, fixed, w["u0"], opts, make_energy, make_response)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_adjoint_matches_oracle_and_finite_differences(precision):
    w = workloads.gravity_box(3, seed=2)
    theta = w["theta"].ravel().copy()
    # The finite differences below resolve 1e-6 of a derivative only if every equilibrium is
    # solved to near round-off: the Exact Hessian takes over at 1e-3 of the initial gradient, so
    # the last Newton steps converge quadratically past the 1e-12 stopping bound (with the
    # projected Hessian alone they converge linearly and stop just below it).
    opts = solver.NewtonOptions(gradient_tolerance=1e-12, stop_rule="relative", accept_rule="armijo",
                                max_iterations=100, cg_tolerance=1e-3, exact_below=1e-3)
    eq = _equilibrium(w, theta, opts)
    eq.precision = precision
    rng = np.random.default_rng(0)
    x_t = eq.eval_value(theta) + 0.01 * rng.standard_normal(w["X"].size)
    x = eq.eval_value(theta)
    dLdx = 2 * (x - x_t)
    grad = eq.eval_vjp(theta, dLdx)
    # Oracle adjoint with a direct solve at the same equilibrium.
    orc = oracle.OracleMesh(w["X"], w["tets"], w["theta"])
    ref, _ = orc.adjoint_theta(x, dLdx, w["fixed"], linear_solver=0)
    assert rel_err(grad, ref.ravel()) <= (1e-9 if precision == "f64" else 1e-6)
    loss = lambda p: float(np.sum((eq.eval_value(p) - x_t) ** 2))  # noqa: E731
    for k in range(3):
        v = rng.standard_normal(theta.size) * theta
        # Five-point stencil at h = 1e-4 (truncation O(h^4)); the equilibria's residual noise
        # is divided by 12 h instead of the 2 h of a central difference at 1e-5.
        h = 1e-4
        fd = (8 * (loss(theta + h * v) - loss(theta - h * v)) - (loss(theta + 2 * h * v) - loss(theta - 2 * h * v))) / (12 * h)
        assert abs(grad @ v - fd) <= 1e-6 * abs(fd) + 1e-12


def test_adjoint_all_fixed_is_zero():
    w = workloads.gravity_box(2, seed=0)
    w = dict(w, fixed=np.arange(w["X"].size, dtype=np.int32))
    eq = _equilibrium(w, w["theta"].ravel(), solver.NewtonOptions(gradient_tolerance=1e-10))
    np.testing.assert_array_equal(eq.eval_value(w["theta"].ravel()), w["u0"])
    np.testing.assert_array_equal(eq.eval_vjp(w["theta"].ravel(), np.ones(w["X"].size)), 0)


def test_exact_below_switch_converges_from_a_rough_state():
    """NewtonOptions.exact_below (not in the reference): projected Hessian until the gradient
    has dropped by the given factor, then the Exact one; on a noisy compressed box it reaches
    the same equilibrium as the projected-only Newton, in fewer iterations."""
    import torch

    w = workloads.compressed_box(8, seed=0)
    X = w["X"]
    e = fem.VolumetricFemEnergyTetP1.from_arrays(X, w["tets"], w["theta"])
    tb = np.flatnonzero((X[:, 2] == 0.0) | (X[:, 2] == 1.0))
    fixed = dof.DofReduction(X.size, (3 * tb[:, None] + np.arange(3)).ravel())
    u = torch.as_tensor(w["u"], device="cuda")
    res = {}
    for name, below in (("projected", 0.0), ("hybrid", 1e-3)):
        o = solver.NewtonOptions(gradient_tolerance=1e-9, stop_rule="relative", accept_rule="armijo",
                                 max_iterations=200, exact_below=below)
        res[name] = solver.newton_solve(e, fixed, u, o)
        assert res[name].status == solver.NewtonStatus.Converged
    assert res["hybrid"].iterations < res["projected"].iterations
    d = (res["hybrid"].x - res["projected"].x).abs().max().item()
    assert d <= 1e-6 * max(1.0, res["projected"].x.abs().max().item())
    with pytest.raises(ValueError, match="exact_below"):
        solver.newton_solve(e, fixed, u, solver.NewtonOptions(gradient_tolerance=1e-9, exact_below=-1.0))
