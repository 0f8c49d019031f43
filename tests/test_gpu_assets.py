"""The reference's own mesh assets through the GPU path (tests/golden/assets.npz, made from the
reference's assets/box-tet.veg and assets/bunny-tet.veg by tests/golden/make_assets.py):

- E, gradient and the Exact and Projected CSC Hessian against the oracle (pattern bit for bit,
  values 1e-12 / 1e-11 max-norm relative) on deformed states of both meshes;
- the feasible step against the oracle;
- a gravity equilibrium of the bunny (its lowest vertices fixed) by Newton on the GPU, checked
  with the oracle's gradient and against the oracle's own Newton solution;
- the reference's corner-pull example on box-tet (examples/fem/equilibrium/tet_p1_corner_pull.py):
  VertexPullingEnergy springs at the eight bounding-box corners, no fixed DOF, default options
  with gradient_tolerance 1e-8, against the oracle's Newton with the same springs.
"""

from pathlib import Path

import numpy as np
import pytest

import oracle
from conftest import rel_err
from litepgo_b200 import dof, energy, fem, solver, workloads

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ASSETS = np.load(Path(__file__).resolve().parent / "golden" / "assets.npz")


def mesh_of(name):
    return ASSETS[name + "_X"], ASSETS[name + "_cells"]


def deformed_state(X, tets, seed, scale):
    rng = np.random.default_rng(seed)
    ext = np.ptp(X, axis=0).max()
    A = np.eye(3) + 0.05 * rng.standard_normal((3, 3))
    u = (X @ A.T - X + scale * ext * rng.standard_normal(X.shape)).ravel()
    assert np.all(workloads.det_F(X, tets, u) > 0)
    return u


@pytest.mark.parametrize("name,scale", [("box_tet", 2e-3), ("bunny_tet", 2e-4)])
def test_asset_energy_against_oracle(name, scale):
    X, tets = mesh_of(name)
    rng = np.random.default_rng(1)
    mu = np.exp(rng.uniform(np.log(1e3), np.log(1e5), tets.shape[0]))
    theta = np.stack([workloads.lame(mu, 0.4)[0], mu], axis=1)
    u = deformed_state(X, tets, 2, scale)
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta)
    orc = oracle.OracleMesh(X, tets, theta)
    outer, inner = gpu.pattern_csc()
    oo, oi = orc.pattern()
    assert np.array_equal(outer, oo) and np.array_equal(inner, oi)
    E, g, H = gpu.eval(u, gradient=True, hessian=energy.HessianKind.Exact)
    Er, gr, vr = orc.eval(u, True, 1)
    assert abs(E - Er) <= 1e-12 * abs(Er)
    assert rel_err(g, gr) <= 1e-12
    assert rel_err(H.data, vr) <= 1e-12
    _, _, Hp = gpu.eval(u, hessian=energy.HessianKind.Projected)
    _, _, vp = orc.eval(u, False, 2)
    assert rel_err(Hp.data, vp) <= 1e-11
    du = np.random.default_rng(3).standard_normal(u.size) * np.ptp(X)
    assert abs(gpu.max_feasible_step(u, du) - orc.feasible_step(u, du)) <= 1e-12


def test_bunny_gravity_equilibrium():
    X, tets = mesh_of("bunny_tet")
    theta = np.array([1.4e5, 3.4e4])
    zmin = X[:, 1].min()
    base = np.flatnonzero(X[:, 1] <= zmin + 0.05 * np.ptp(X[:, 1]))
    fixed = (3 * base[:, None] + np.arange(3)).ravel().astype(np.int32)
    f = workloads.gravity_load(X, tets, rho=1000.0, g=(0.0, -9.8, 0.0))
    n = X.size
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta)
    import scipy.sparse as sp

    total = energy.WeightedSumEnergy([(gpu, 1.0), (energy.QuadraticEnergy(sp.csc_matrix((n, n)), -f), 1.0)])
    opts = solver.NewtonOptions(gradient_tolerance=1e-10, stop_rule="relative", cg_tolerance=1e-3)
    r = solver.newton_solve(total, dof.DofReduction(n, fixed), np.zeros(n), opts)
    assert r.status == solver.NewtonStatus.Converged, r
    orc = oracle.OracleMesh(X, tets, theta)
    _, go, _ = orc.eval(r.x, True, 0)
    free = np.setdiff1d(np.arange(n), fixed)
    assert np.linalg.norm((go - f)[free]) <= 1.5e-10 * r.gradient_norm0
    # The oracle's PCG restatement (its sparse LDL^T takes many minutes at 18.5k DOFs).
    xo, info = orc.newton(fixed, np.zeros(n), f_ext=f, tol=1e-10, stop_rule=1, linear_solver=1, cg_tolerance=1e-3)
    assert info["status"] == 0
    assert rel_err(r.x, xo) <= 1e-8
    assert np.all(r.x[fixed] == 0.0)


def corner_pull_problem():
    """The reference example's potential on box-tet: theta = [2, 3], springs of stiffness 1 from
    the eight bounding-box corners to a copy of the box stretched by 0.3 about its minimum."""
    X, tets = mesh_of("box_tet")
    lower, upper = X.min(axis=0), X.max(axis=0)
    tol = (upper - lower).max() * 1e-8
    near = (np.abs(X - lower) <= tol) | (np.abs(X - upper) <= tol)
    corners = np.flatnonzero(near.all(axis=1))
    assert corners.size == 8
    dofs = (3 * corners[:, None] + np.arange(3)).astype(np.int32)
    targets = 0.3 * (X[corners] - lower)
    return X, tets, dofs, targets


def test_corner_pull_example_against_oracle():
    X, tets, dofs, targets = corner_pull_problem()
    n = X.size
    elastic = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, np.array([2.0, 3.0]))
    pulling = energy.VertexPullingEnergy(n, dofs, targets, 1.0)
    potential = energy.WeightedSumEnergy([(elastic, 1.0), (pulling, 1.0)])
    steps = []
    opts = solver.NewtonOptions(gradient_tolerance=1e-8, cg_tolerance=1e-12)
    r = solver.newton_solve(potential, dof.DofReduction(n, []), np.zeros(n), opts, on_iteration=steps.append)
    assert r.status == solver.NewtonStatus.Converged, r
    A, b, c = pulling.quadratic_form()
    orc = oracle.OracleMesh(X, tets, np.array([2.0, 3.0]))
    xo, info = orc.newton(np.zeros(0, np.int32), np.zeros(n), f_ext=-b, tol=1e-8, A=A, constant=c, trace=True)
    assert info["status"] == 0
    assert rel_err(r.x, xo) <= 1e-7
    assert abs(r.energy - info["energy"]) <= 1e-10 * abs(info["energy"])
    # The corners reach their anchors up to the balance of spring and elastic forces.
    gap = np.linalg.norm(r.x.reshape(-1, 3)[dofs[:, 0] // 3] - targets, axis=1).max()
    assert gap < 0.3 * np.ptp(X)
    # One NewtonStep per iteration, as the oracle's trace (the reference's report points).
    trace = info["trace"]
    assert len(steps) == len(trace) == r.iterations + 1
    for s, t in zip(steps, trace):
        assert s.iteration == int(t["iteration"])
        assert abs(s.energy - t["energy"]) <= 1e-9 * max(abs(t["energy"]), 1.0)
        assert s.diagonal_shifts == int(t["diagonal_shifts"])
        assert s.line_search_evaluations == int(t["line_search_evaluations"])
        assert abs(s.step - t["step"]) <= 1e-9 and abs(s.feasible_step - t["feasible_step"]) <= 1e-9
    assert steps[0].pattern_changed and not any(s.pattern_changed for s in steps[1:])
    assert steps[-1].step == 0.0 and steps[-1].gradient_norm <= 1e-8
