"""Tricubic Hermite hexes on the GPU path (VolumetricFemEnergy[NeoHookean, HexHermiteBasis,
GaussLegendre3D[n]]): energy, gradient and Exact Hessian over the 24 physical DOFs per vertex
against the Hermite oracle (the two-box fixture of the reference's hex force test and a
structured box), the feasible step, the construction checks, Newton with the Exact Hessian, and
the theta force response and adjoint."""

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from conftest import rel_err
from litepgo_b200 import dof, energy, fem, mesh, solver
from test_oracle_hermite import HERMITE_CELLS, HERMITE_THETA, HERMITE_X, hermite_state

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

Exact, Projected = energy.HessianKind.Exact, energy.HessianKind.Projected


def hermite_energy(X, cells, theta, n=2):
    cls = fem.VolumetricFemEnergy[fem.NeoHookean, fem.HexHermiteBasis, fem.GaussLegendre3D[n]]
    return cls.from_arrays(X, cells, theta)


@pytest.mark.parametrize("n", [2, 4])
@pytest.mark.parametrize("scale,e_tol", [(0.05, 1e-12), (0.002, 1e-10)])
def test_two_box_fixture_matches_the_oracle(n, scale, e_tol):
    """At the reference test's scale (0.002) W is second order in strains whose terms are first
    order, so the energy carries ~1/strain times the round-off of F (different summation orders
    of the 64 nodes): its tolerance is wider there; gradient and Hessian keep 1e-12."""
    x = hermite_state(scale)
    gpu = hermite_energy(HERMITE_X, HERMITE_CELLS, HERMITE_THETA, n)
    assert gpu.num_dofs == 24 * 12
    E, g, H = gpu.eval(x, gradient=True, hessian=Exact)
    Er, gr, Hr = oracle.hex_hermite_eval(HERMITE_X, HERMITE_CELLS, HERMITE_THETA, x, points_per_axis=n)
    assert abs(E - Er) <= e_tol * abs(Er)
    assert rel_err(g, gr) <= 1e-12
    assert rel_err(H.toarray(), Hr) <= 1e-12
    D = (H - H.T).tocsc()
    D.eliminate_zeros()
    assert D.nnz == 0  # bitwise symmetric
    _, _, H32 = gpu.eval(x, hessian=Exact, precision="mixed")
    assert rel_err(H32.toarray(), Hr) <= 1e-6
    assert abs(gpu.element_energies(x).sum() - E) <= e_tol * abs(E)


def test_structured_box_and_feasible_step():
    X, cells = mesh.make_hex_box(3, 2, 2)
    rng = np.random.default_rng(4)
    T = cells.shape[0]
    mu = np.exp(rng.uniform(np.log(1e3), np.log(1e5), T))
    theta = np.column_stack([3 * mu, mu])
    u = 0.02 * rng.standard_normal(24 * X.shape[0])  # det F >= 0.78 at every point
    gpu = hermite_energy(X, cells, theta)
    E, g, H = gpu.eval(u, gradient=True, hessian=Exact)
    Er, gr, Hr = oracle.hex_hermite_eval(X, cells, theta, u)
    assert abs(E - Er) <= 1e-12 * abs(Er)
    assert rel_err(g, gr) <= 1e-12
    assert rel_err(H.toarray(), Hr) <= 1e-12
    # The feasible step: the reference's positive-determinant step at every point, minimum.
    du = 0.3 * rng.standard_normal(u.size)
    pts, _ = oracle.hex_points(2)
    U, dU = u.reshape(-1, 24), du.reshape(-1, 24)
    ref = 1.0
    for cell in cells:
        h = oracle.hermite_box(X[cell])
        s = np.repeat(np.tile([1, h[0], h[1], h[2], h[0] * h[1], h[0] * h[2], h[1] * h[2], np.prod(h)], 8), 3)
        C, dC = (U[cell].ravel() * s).reshape(64, 3), (dU[cell].ravel() * s).reshape(64, 3)
        for xi in pts:
            gN = oracle.hex_hermite_N_dN(xi)[1] / h
            ref = min(ref, oracle.positive_det_step(np.eye(3) + C.T @ gN, dC.T @ gN))
    assert ref < 1.0
    assert abs(gpu.max_feasible_step(u, du) - ref) <= 1e-12


def test_construction_and_unsupported_requests():
    gpu = hermite_energy(HERMITE_X, HERMITE_CELLS, HERMITE_THETA)
    corners = oracle.HEX_CORNERS.astype(float)
    cell = np.arange(8, dtype=np.int32)[None]
    hermite_energy(corners, cell, HERMITE_THETA)
    sheared = corners.copy()
    sheared[:, 0] += 0.2 * sheared[:, 1]
    with pytest.raises(ValueError, match="axis-aligned"):
        hermite_energy(sheared, cell, HERMITE_THETA)
    with pytest.raises(ValueError):
        hermite_energy(corners, np.array([[1, 0, 3, 2, 5, 4, 7, 6]], dtype=np.int32), HERMITE_THETA)
    topo = mesh.HexTopology(12, HERMITE_CELLS)
    with pytest.raises(ValueError):  # the Q1 map width
        fem.VolumetricFemEnergy[fem.NeoHookean, fem.HexHermiteBasis, fem.GaussLegendre3D[2]](
            dof.VertexDofMap(topo, 3), HERMITE_X, None, HERMITE_THETA)
    Resp = fem.VolumetricFemForceMaterialResponseHexQ1  # the Q1 response rejects the Hermite map width
    with pytest.raises(ValueError):
        Resp(dof.ConstantDofMap(topo, 2), dof.VertexDofMap(topo, 24), HERMITE_X, hermite_state(), None)
    th = np.tile([3.0, 4.0], (2, 1))
    gpu.set_theta(th)
    assert gpu.eval(hermite_state())[0] == hermite_energy(HERMITE_X, HERMITE_CELLS, th).eval(hermite_state())[0]


def test_hermite_newton_exact_hessian():
    """A 3x2x2 Hermite box (4 points per axis: 2 leave zero-energy modes in the tricubic field)
    with its x = 0 vertices held (all 24 DOFs) and a load on the value slots: Newton with the
    Exact Hessian converges, and the oracle's free gradient equals the load."""
    X, cells = mesh.make_hex_box(3, 2, 2)
    n = 24 * X.shape[0]
    theta = np.array([1.4e5, 3.4e4])
    gpu = hermite_energy(X, cells, theta, 4)
    rng = np.random.default_rng(8)
    f = np.zeros(n)
    value = (24 * np.arange(X.shape[0])[:, None] + np.arange(3)).ravel()
    f[value] = 50.0 * rng.standard_normal(value.size)
    fixed = (24 * np.flatnonzero(X[:, 0] == 0)[:, None] + np.arange(24)).ravel()
    f[fixed] = 0
    total = energy.WeightedSumEnergy([(gpu, 1.0), (energy.QuadraticEnergy(sp.csc_matrix((n, n)), -f), 1.0)])
    opts = solver.NewtonOptions(gradient_tolerance=1e-10, stop_rule="relative", accept_rule="armijo",
                                precision="f64", max_iterations=50, cg_tolerance=1e-4, hessian=Exact)
    r = solver.newton_solve(total, dof.DofReduction(n, fixed), np.zeros(n), opts)
    assert r.status.name == "Converged"
    _, g, _ = oracle.hex_hermite_eval(X, cells, theta, np.asarray(r.x), points_per_axis=4, hessian=False)
    free = np.setdiff1d(np.arange(n), fixed)
    assert np.abs((g - f)[free]).max() <= 1e-7 * np.abs(f).max()


@pytest.mark.parametrize("n", [2, 4])
def test_hermite_theta_vjp(n):
    """The Hermite force's theta VJP over physical DOFs against the oracle, per element and summed."""
    x = hermite_state(0.05)
    w = np.cos(np.arange(x.size) + 0.7)
    topo = mesh.HexTopology(12, HERMITE_CELLS)
    Resp = fem.VolumetricFemForceMaterialResponse[fem.NeoHookean, fem.HexHermiteBasis, fem.GaussLegendre3D[n]]
    ref = oracle.hex_hermite_force_vjp_theta(HERMITE_X, HERMITE_CELLS, [1.0, 1.0], x, w, points_per_axis=n)
    per = Resp(dof.ElementDofMap(topo, 2), dof.VertexDofMap(topo, 24), HERMITE_X, x, None)
    assert rel_err(per.eval_vjp(np.tile(HERMITE_THETA, 2), w).reshape(2, 2), ref) <= 1e-12
    shared = Resp(dof.ConstantDofMap(topo, 2), dof.VertexDofMap(topo, 24), HERMITE_X, x, None)
    assert rel_err(shared.eval_vjp(HERMITE_THETA, w), ref.sum(0)) <= 1e-12


def test_hermite_theta_adjoint_matches_finite_differences():
    """Per-element [lambda, mu] of a 2x2x1 box of unit Hermite cells (4 points per axis) as a torch
    leaf, loss |x*(theta) - x_t|^2, with the bottom vertices and every vertex's mixed-derivative
    slots held (the free Hessian's condition is then ~1e3, not ~1e7) and a downward load on the
    value slots: the adjoint gradient against five-point differences (step 1e-4 relative to
    theta) along 6 seeded directions, to 1e-6."""
    from litepgo_b200 import torch as bridge

    X, cells = mesh.make_hex_box(2, 2, 1)
    X = X * np.array([2.0, 2.0, 1.0])
    n, T = 24 * X.shape[0], cells.shape[0]
    rng = np.random.default_rng(3)
    mu = 3e4 * (1 + 0.5 * rng.random(T))
    theta0 = np.column_stack([4 * mu, mu])
    f = np.zeros(n)
    value = (24 * np.arange(X.shape[0])[:, None] + np.arange(3)).ravel()
    f[value] = -2e3 * (value % 3 == 2)
    base = (24 * np.flatnonzero(X[:, 2] == 0)[:, None] + np.arange(24)).ravel()
    mixed = (24 * np.arange(X.shape[0])[:, None] + np.arange(12, 24)).ravel()
    fixed = np.union1d(base, mixed)
    f[fixed] = 0
    load = energy.QuadraticEnergy(sp.csc_matrix((n, n)), -f)
    shared = hermite_energy(X, cells, theta0, 4)
    topo = mesh.HexTopology(X.shape[0], cells)
    Resp = fem.VolumetricFemForceMaterialResponse[fem.NeoHookean, fem.HexHermiteBasis, fem.GaussLegendre3D[4]]

    def make_energy(p):
        shared.set_theta(p.reshape(T, 2))
        return energy.WeightedSumEnergy([(shared, 1.0), (load, 1.0)])

    def make_response(u):
        return Resp(dof.ElementDofMap(topo, 2), dof.VertexDofMap(topo, 24), X, u, None)

    opts = solver.NewtonOptions(gradient_tolerance=1e-12 * np.abs(f).max(), stop_rule="max_abs", accept_rule="noise",
                                max_iterations=100, cg_tolerance=1e-3, hessian=Exact)
    model = solver.StaticEquilibriumResponse(2 * T, dof.DofReduction(n, fixed), np.zeros(n), opts, make_energy,
                                             make_response)
    x_target = model.eval_value((theta0 * (1 + 0.2 * rng.standard_normal(theta0.shape))).ravel())
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    loss = ((bridge.response(model, theta.reshape(-1)) - torch.as_tensor(x_target)) ** 2).sum()
    loss.backward()
    grad = theta.grad.numpy().ravel()
    th0 = theta0.ravel()
    warm = solver.StaticEquilibriumResponse(2 * T, dof.DofReduction(n, fixed), model.eval_value(th0), opts,
                                            make_energy, make_response)

    def L(q):
        return float(np.sum((warm.eval_value(q) - x_target) ** 2))

    h = 1e-4
    for _ in range(6):
        d = rng.standard_normal(2 * T) * th0
        fd = (8 * (L(th0 + h * d) - L(th0 - h * d)) - (L(th0 + 2 * h * d) - L(th0 - 2 * h * d))) / (12 * h)
        assert abs(grad @ d - fd) <= 1e-6 * abs(fd)


def expanded_hermite_state(X, scale, noise, seed):
    """The affine field u = scale X in physical Hermite DOFs (value slot scale X, u_X, u_Y, u_Z the
    columns of scale I, mixed slots zero) plus seeded noise on every DOF."""
    V = X.shape[0]
    D = np.zeros((V, 8, 3))
    D[:, 0] = scale * X
    for k in range(3):
        D[:, 1 + k, k] = scale
    return D.ravel() + noise * np.random.default_rng(seed).standard_normal(24 * V)


@pytest.mark.parametrize("precision,tol", [("f64", 1e-11), ("mixed", 1e-6)])
def test_projected_hessian_matches_the_oracle(precision, tol):
    """HessianKind.Projected on Hermite hexes: every element's 192 x 192 Hessian clamped to PSD
    (the reference's per-element eigenvalue clamp) where its tangents are indefinite; here a
    uniform expansion with lambda / mu = 10 makes them so."""
    X, cells = mesh.make_hex_box(3, 2, 2)
    theta = np.array([10.0, 1.0])
    u = expanded_hermite_state(X, 0.5, 1e-3, 3)
    gpu = hermite_energy(X, cells, theta)
    _, _, Hp = gpu.eval(u, hessian=Projected, precision=precision)
    _, _, He = gpu.eval(u, hessian=Exact)
    _, _, Hr = oracle.hex_hermite_eval(X, cells, theta, u, projected=True)
    assert rel_err(Hp.toarray(), Hr) <= tol
    assert rel_err(He.toarray(), Hr) > 1e-3  # the clamp changed the matrix
    # Semi-definite up to the rounding of the stored values (FP32 records in mixed precision).
    assert np.linalg.eigvalsh(Hp.toarray()).min() >= -10 * tol * np.abs(Hr).max()
    D = (Hp - Hp.T).tocsc()
    D.eliminate_zeros()
    assert D.nnz == 0  # bitwise symmetric


def test_hermite_corner_pull_example():
    """The reference's examples/fem/equilibrium/hex_hermite_corner_pull.py on its own box-hex.veg:
    tricubic Hermite hexes with GaussLegendre3D[4], theta = [2, 3], springs pulling the value
    slots of the eight bounding-box corners to a copy of the box stretched by 0.3, no fixed DOF,
    default NewtonOptions (Projected Hessian) with gradient_tolerance 1e-8. The oracle's gradient
    of the same potential at the result meets the tolerance."""
    from pathlib import Path

    assets = np.load(Path(__file__).resolve().parent / "golden" / "assets.npz")
    X, cells = assets["box_hex_X"], assets["box_hex_cells"]
    theta = np.array([2.0, 3.0])
    elastic = hermite_energy(X, cells, theta, 4)
    n = elastic.num_dofs
    lower, upper = X.min(axis=0), X.max(axis=0)
    tol = (upper - lower).max() * 1e-8
    near = (np.abs(X - lower) <= tol) | (np.abs(X - upper) <= tol)
    corners = np.flatnonzero(near.all(axis=1))
    assert corners.size == 8
    pulled = (24 * corners[:, None] + np.arange(3)).astype(np.int32)
    targets = 0.3 * (X[corners] - lower)
    pulling = energy.VertexPullingEnergy(n, pulled, targets, 1.0)
    potential = energy.WeightedSumEnergy([(elastic, 1.0), (pulling, 1.0)])
    steps = []
    r = solver.newton_solve(potential, dof.DofReduction(n, []), np.zeros(n),
                            solver.NewtonOptions(gradient_tolerance=1e-8), on_iteration=steps.append)
    assert r.status == solver.NewtonStatus.Converged, r
    assert any(s.diagonal_shifts == 0 for s in steps) and steps[-1].gradient_norm <= 1e-8
    _, g, _ = oracle.hex_hermite_eval(X, cells, theta, np.asarray(r.x), points_per_axis=4, hessian=False)
    g = g + pulling.eval_gradient(r.x)
    assert np.abs(g).max() <= 1e-8 + 1e-12 * np.abs(pulling.eval_gradient(np.zeros(n))).max()
