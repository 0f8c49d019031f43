"""Hex Q1 meshes on the GPU path (VolumetricFemEnergy[NeoHookean, HexQ1Basis, GaussLegendre3D[n]]):
energy, gradient and Exact Hessian against the hex oracle (the reference's two-hex fixture and a
hex box), the Projected Hessian (per-element eigen-projection) against the oracle's, the solvers'
layout through Newton, the feasible step, and the construction checks."""

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from conftest import rel_err
from litepgo_b200 import dof, energy, fem, mesh, solver
from test_oracle_hex import HEX_CELLS, HEX_THETA, HEX_X, hex_states

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

Exact, Projected = energy.HessianKind.Exact, energy.HessianKind.Projected


def hex_energy(X, cells, theta, n=2):
    cls = fem.VolumetricFemEnergy[fem.NeoHookean, fem.HexQ1Basis, fem.GaussLegendre3D[n]]
    return cls.from_arrays(X, cells, theta)


@pytest.mark.parametrize("state", [0, 1, 2])
def test_two_hex_fixture_matches_the_oracle(state):
    x = hex_states()[state]
    gpu = hex_energy(HEX_X, HEX_CELLS, HEX_THETA)
    E, g, H = gpu.eval(x, gradient=True, hessian=Exact)
    Er, gr, Hr = oracle.hex_eval(HEX_X, HEX_CELLS, HEX_THETA, x)
    assert abs(E - Er) <= 1e-12 * max(abs(Er), 1e-300) + 1e-15
    assert rel_err(g, gr) <= 1e-12 or np.abs(gr).max() == 0
    assert rel_err(H.toarray(), Hr) <= 1e-12
    D = (H - H.T).tocsc()
    D.eliminate_zeros()
    assert D.nnz == 0  # bitwise symmetric


@pytest.mark.parametrize("n", [2, 4])
def test_hex_box_matches_the_oracle(n):
    X, cells = oracle.hex_box(3, 3, 2)
    rng = np.random.default_rng(n)
    T = cells.shape[0]
    mu = np.exp(rng.uniform(np.log(1e3), np.log(1e5), T))
    nu = rng.uniform(0.30, 0.45, T)
    theta = np.stack([2 * mu * nu / (1 - 2 * nu), mu], 1)
    A = np.eye(3) + 0.1 * rng.standard_normal((3, 3))
    u = (X @ A.T - X + 1e-3 * rng.standard_normal(X.shape)).ravel()
    gpu = hex_energy(X, cells, theta, n)
    E, g, H = gpu.eval(u, gradient=True, hessian=Exact)
    Er, gr, Hr = oracle.hex_eval(X, cells, theta, u, points_per_axis=n)
    assert abs(E - Er) <= 1e-12 * abs(Er)
    assert rel_err(g, gr) <= 1e-12
    assert rel_err(H.toarray(), Hr) <= 1e-12
    _, _, H32 = gpu.eval(u, hessian=Exact, precision="mixed")
    assert rel_err(H32.toarray(), Hr) <= 1e-6
    # The element energies sum to the energy; the feasible step is the minimum over every point.
    assert abs(gpu.element_energies(u).sum() - E) <= 1e-12 * abs(E)
    du = rng.standard_normal(u.size)
    pts, _ = oracle.hex_points(n)
    ref = 1.0
    U, dU = u.reshape(-1, 3), du.reshape(-1, 3)
    for cell in cells:
        for xi in pts:
            dN = oracle.hex_dN_dxi(xi)
            gN = dN @ np.linalg.inv(X[cell].T @ dN)
            F = np.eye(3) + U[cell].T @ gN
            dF = dU[cell].T @ gN
            ref = min(ref, oracle.positive_det_step(F, dF))
    assert abs(gpu.max_feasible_step(u, du) - ref) <= 1e-12


@pytest.mark.parametrize("state", [0, 1, 2])
def test_two_hex_projected_hessian(state):
    """HessianKind::Projected on the reference's two-hex fixture: elements already PSD keep
    their Hessian up to the eigen-iteration's rounding."""
    x = hex_states()[state]
    gpu = hex_energy(HEX_X, HEX_CELLS, HEX_THETA)
    E, g, H = gpu.eval(x, gradient=True, hessian=Projected)
    Er, gr, Hr = oracle.hex_eval(HEX_X, HEX_CELLS, HEX_THETA, x, projected=True)
    assert abs(E - Er) <= 1e-12 * max(abs(Er), 1e-300) + 1e-15
    assert rel_err(H.toarray(), Hr) <= 1e-11
    D = (H - H.T).tocsc()
    D.eliminate_zeros()
    assert D.nnz == 0


def test_compressed_hex_box_projected_hessian():
    """A compressed hex box whose every element Hessian is indefinite (checked on the CPU):
    the projected Hessian matches the oracle's per-element eigen-projection in FP64 and mixed
    precision, is PSD, bitwise symmetric, and differs from the Exact one."""
    X, cells = oracle.hex_box(3, 3, 2)
    rng = np.random.default_rng(11)
    T = cells.shape[0]
    mu = np.exp(rng.uniform(np.log(1e3), np.log(1e5), T))
    nu = rng.uniform(0.30, 0.45, T)
    theta = np.stack([2 * mu * nu / (1 - 2 * nu), mu], 1)
    A = np.diag([1.0, 1.0, 0.45]) + 0.05 * rng.standard_normal((3, 3))
    u = (X @ A.T - X + 5e-3 * rng.standard_normal(X.shape)).ravel()
    _, _, He = oracle.hex_eval(X, cells, theta, u)
    _, _, Hr = oracle.hex_eval(X, cells, theta, u, projected=True)
    assert rel_err(Hr, He) > 0.1
    gpu = hex_energy(X, cells, theta)
    _, _, H = gpu.eval(u, hessian=Projected)
    assert rel_err(H.toarray(), Hr) <= 1e-11
    D = (H - H.T).tocsc()
    D.eliminate_zeros()
    assert D.nnz == 0
    assert np.linalg.eigvalsh(H.toarray()).min() >= -1e-10 * np.abs(Hr).max()
    _, _, H32 = gpu.eval(u, hessian=Projected, precision="mixed")
    assert rel_err(H32.toarray(), Hr) <= 1e-6


def test_projected_hessian_half_at_rest():
    """The lower layer of a hex box compressed to half its height, the upper layer at rest: the
    upper elements pass the per-point semi-definiteness pre-test (their Hessian is kept), the
    lower ones are indefinite and eigen-projected, in one launch."""
    X, cells = oracle.hex_box(3, 3, 2)
    theta = np.array([1.4e5, 3.4e4])
    u = np.zeros_like(X)
    u[:, 2] = -0.5 * np.minimum(X[:, 2], 0.5)
    u = u.ravel()
    _, _, He = oracle.hex_eval(X, cells, theta, u)
    _, _, Hr = oracle.hex_eval(X, cells, theta, u, projected=True)
    assert rel_err(Hr, He) > 0.05
    gpu = hex_energy(X, cells, theta)
    for precision, tol in (("f64", 1e-11), ("mixed", 1e-6)):
        _, _, H = gpu.eval(u, hessian=Projected, precision=precision)
        assert rel_err(H.toarray(), Hr) <= tol


def test_construction_errors():
    gpu = hex_energy(HEX_X, HEX_CELLS, HEX_THETA)
    assert gpu.eval(hex_states()[1])[0] > 0
    for scale in (0.0, -1.0, 1e200):
        with pytest.raises(ValueError):
            hex_energy(scale * HEX_X, HEX_CELLS, HEX_THETA)
    bad = HEX_X.copy()
    bad[0, 0] = np.nan
    with pytest.raises(ValueError):
        hex_energy(bad, HEX_CELLS, HEX_THETA)
    with pytest.raises(TypeError):
        fem.GaussLegendre3D[3]


@pytest.mark.parametrize("precision,hessian", [("f64", Exact), ("mixed", Exact), ("f64", Projected),
                                               ("mixed", Projected)])
def test_hex_newton_under_gravity(precision, hessian):
    """A 4x4x4 hex box with its bottom face held under gravity (rho 1000): Newton with the Exact
    or the (default) Projected Hessian reaches the relative tolerance and the oracle's free
    gradient vanishes there."""
    X, cells = oracle.hex_box(4)
    n = X.size
    theta = np.array([1.4e5, 3.4e4])
    gpu = hex_energy(X, cells, theta)
    # Consistent load: f_a = -rho g sum_q w_q det J_q N_a(xi_q) (z component).
    pts, wts = oracle.hex_points(2)
    f = np.zeros(n)
    for cell in cells:
        for xi, wq in zip(pts, wts):
            dN = oracle.hex_dN_dxi(xi)
            det = np.linalg.det(X[cell].T @ dN)
            Nq = fem.HexQ1Basis.eval_N(xi)
            f[3 * cell + 2] += -9.8 * 1000 * wq * det * Nq
    fixed = np.flatnonzero(np.repeat(X[:, 2] == 0, 3))
    total = energy.WeightedSumEnergy([(gpu, 1.0), (energy.QuadraticEnergy(sp.csc_matrix((n, n)), -f), 1.0)])
    opts = solver.NewtonOptions(gradient_tolerance=1e-10, stop_rule="relative", accept_rule="armijo",
                                precision=precision, max_iterations=50, cg_tolerance=1e-3, hessian=hessian)
    r = solver.newton_solve(total, dof.DofReduction(n, fixed), np.zeros(n), opts)
    assert r.status.name == "Converged"
    x = np.asarray(r.x)
    _, g, _ = oracle.hex_eval(X, cells, theta, x, hessian=False)
    free = np.setdiff1d(np.arange(n), fixed)
    assert np.abs((g - f)[free]).max() <= 1e-7 * np.abs(f).max()


def test_hex_theta_vjp_and_set_theta():
    """The hex force's theta VJP (VolumetricFemForceMaterialResponse over HexQ1Basis) against
    the oracle per element and summed; set_theta against a freshly built energy (bitwise)."""
    from litepgo_b200 import dof

    X, cells = oracle.hex_box(3, 3, 2)
    rng = np.random.default_rng(5)
    T = cells.shape[0]
    A = np.eye(3) + 0.1 * rng.standard_normal((3, 3))
    u = (X @ A.T - X + 1e-3 * rng.standard_normal(X.shape)).ravel()
    w = rng.standard_normal(u.size)
    topo = mesh.HexTopology(X.shape[0], cells)
    ref = oracle.hex_force_vjp_theta(X, cells, np.array([1.0, 1.0]), u, w)
    for cls, n in ((fem.VolumetricFemForceMaterialResponse[fem.NeoHookean, fem.HexQ1Basis, fem.GaussLegendre3D[2]], 2),
                   (fem.VolumetricFemForceMaterialResponse[fem.NeoHookean, fem.HexQ1Basis, fem.GaussLegendre3D[4]], 4)):
        r = oracle.hex_force_vjp_theta(X, cells, np.array([1.0, 1.0]), u, w, points_per_axis=n) if n == 4 else ref
        per = cls(dof.ElementDofMap(topo, 2), dof.VertexDofMap(topo, 3), X, u, None)
        got = per.eval_vjp(np.tile([1e5, 3e4], T), w).reshape(T, 2)
        assert rel_err(got, r) <= 1e-12
        shared = cls(dof.ConstantDofMap(topo, 2), dof.VertexDofMap(topo, 3), X, u, None)
        assert rel_err(shared.eval_vjp(np.array([1e5, 3e4]), w), r.sum(0)) <= 1e-12
    th = np.column_stack([np.full(T, 1.2e5), 3e4 * (1 + 0.3 * rng.random(T))])
    e = hex_energy(X, cells, np.array([1.4e5, 3.4e4]))
    e.set_theta(th)
    E1, g1, H1 = e.eval(u, gradient=True, hessian=Exact)
    E2, g2, H2 = hex_energy(X, cells, th).eval(u, gradient=True, hessian=Exact)
    assert E1 == E2 and np.array_equal(g1, g2) and np.array_equal(H1.data, H2.data)


def test_hex_theta_adjoint_matches_finite_differences():
    """Per-element [lambda, mu] of a 5x5x5 hex box under gravity (bottom face held) as a torch
    leaf, loss |x*(theta) - x_t|^2: the adjoint gradient against five-point differences of the
    loss (step 1e-4 relative to theta) along 8 seeded directions, to 1e-6."""
    from litepgo_b200 import dof
    from litepgo_b200 import torch as bridge

    X, cells = oracle.hex_box(5)
    n, T = X.size, cells.shape[0]
    rng = np.random.default_rng(3)
    mu = 3e4 * (1 + 0.5 * rng.random(T))
    theta0 = np.column_stack([4 * mu, mu])
    pts, wts = oracle.hex_points(2)
    f = np.zeros(n)
    for cell in cells:
        for xi, wq in zip(pts, wts):
            dN = oracle.hex_dN_dxi(xi)
            f[3 * cell + 2] += -9.8 * 1000 * wq * np.linalg.det(X[cell].T @ dN) * fem.HexQ1Basis.eval_N(xi)
    fixed = np.flatnonzero(np.repeat(X[:, 2] == 0, 3))
    load = energy.QuadraticEnergy(sp.csc_matrix((n, n)), -f)
    shared = hex_energy(X, cells, theta0)
    topo = mesh.HexTopology(X.shape[0], cells)
    Resp = fem.VolumetricFemForceMaterialResponse[fem.NeoHookean, fem.HexQ1Basis, fem.GaussLegendre3D[2]]

    def make_energy(p):
        shared.set_theta(p.reshape(T, 2))
        return energy.WeightedSumEnergy([(shared, 1.0), (load, 1.0)])

    def make_response(u):
        return Resp(dof.ElementDofMap(topo, 2), dof.VertexDofMap(topo, 3), X, u, None)

    opts = solver.NewtonOptions(gradient_tolerance=1e-12 * np.abs(f).max(), stop_rule="max_abs", accept_rule="noise",
                                max_iterations=100, cg_tolerance=1e-3)
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
    for _ in range(8):
        d = rng.standard_normal(2 * T) * th0
        fd = (8 * (L(th0 + h * d) - L(th0 - h * d)) - (L(th0 + 2 * h * d) - L(th0 - 2 * h * d))) / (12 * h)
        assert abs(grad @ d - fd) <= 1e-6 * abs(fd)
