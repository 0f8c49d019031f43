"""An unstructured mesh through VEG into the GPU path: a Delaunay ball (irregular valence, no
structured ordering, so the solvers' borrowed blocks are scattered reads) read back from a VEG
file, evaluated against the oracle and solved by Newton in both precisions."""

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from conftest import rel_err
from litepgo_b200 import dof, energy, fem, mesh, solver

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

Exact, Projected = energy.HessianKind.Exact, energy.HessianKind.Projected


@pytest.fixture(scope="module")
def ball(tmp_path_factory):
    X, tets = mesh.delaunay_ball(3000, seed=5)
    path = tmp_path_factory.mktemp("veg") / "ball.veg"
    mesh.write_veg(path, mesh.TetMesh(X, tets))
    data = mesh.read_veg(path)
    rng = np.random.default_rng(2)
    T = data.cells.shape[0]
    mu = np.exp(rng.uniform(np.log(1e4), np.log(1e5), T))
    nu = rng.uniform(0.30, 0.45, T)
    theta = np.stack([2 * mu * nu / (1 - 2 * nu), mu], 1)
    A = np.eye(3) + 0.05 * rng.standard_normal((3, 3))
    # Noise 3e-5 of the unit radius: the ball's smallest tets are ~1e-3 of the mean volume, so
    # larger noise inverts some (det F in [0.75, 0.95] here).
    u = (data.positions @ A.T - data.positions + 3e-5 * rng.standard_normal(data.positions.shape)).ravel()
    x = data.positions + u.reshape(-1, 3)
    D, D0 = x[data.cells[:, 1:]] - x[data.cells[:, :1]], data.positions[data.cells[:, 1:]] - data.positions[data.cells[:, :1]]
    assert np.all(np.linalg.det(D) / np.linalg.det(D0) > 0.5)
    return data, theta, u


def test_unstructured_parity_with_oracle(ball):
    data, theta, u = ball
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(data.positions, data.cells, theta)
    orc = oracle.OracleMesh(data.positions, data.cells, theta)
    E, g, H = gpu.eval(u, gradient=True, hessian=Exact)
    Er, gr, vr = orc.eval(u, True, 1)
    assert abs(E - Er) <= 1e-12 * abs(Er)
    assert rel_err(g, gr) <= 1e-12
    assert rel_err(H.data, vr) <= 1e-12
    _, _, Hp = gpu.eval(u, hessian=Projected)
    _, _, vp = orc.eval(u, False, 2)
    assert rel_err(Hp.data, vp) <= 1e-11
    E32, g32, H32 = gpu.eval(u, gradient=True, hessian=Exact, precision="mixed")
    assert abs(E32 - Er) <= 2e-6 * abs(Er)
    assert rel_err(g32, gr) <= 2e-5
    assert rel_err(H32.data, vr) <= 1e-5


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_unstructured_newton(ball, precision):
    """Gravity on the ball with its lowest vertices held: Newton in the upper-triangle solver
    layout (scattered transposed blocks) reaches the relative tolerance, and both precisions
    reach the same equilibrium."""
    data, theta, _ = ball
    X, tets = data.positions, data.cells
    n = X.size
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta)
    D = X[tets[:, 1:]] - X[tets[:, :1]]
    vol = np.einsum("ij,ij->i", D[:, 0], np.cross(D[:, 1], D[:, 2])) / 6
    f = np.zeros(n)
    np.add.at(f, 3 * tets.ravel() + 2, np.repeat(-9.8 * 100 * vol / 4, 4))  # rho = 100: strains ~0.1
    low = np.flatnonzero(X[:, 2] < X[:, 2].min() + 0.3)
    fixed_dofs = (3 * low[:, None] + np.arange(3)).ravel()
    total = energy.WeightedSumEnergy([(gpu, 1.0), (energy.QuadraticEnergy(sp.csc_matrix((n, n)), -f), 1.0)])
    opts = solver.NewtonOptions(gradient_tolerance=1e-9, stop_rule="relative", accept_rule="armijo",
                                precision=precision, max_iterations=60, cg_tolerance=1e-2, exact_below=1e-3)
    r = solver.newton_solve(total, dof.DofReduction(n, fixed_dofs), np.zeros(n), opts)
    assert r.status.name == "Converged"
    x = np.asarray(r.x)
    ref = solver.newton_solve(total, dof.DofReduction(n, fixed_dofs), np.zeros(n),
                              solver.NewtonOptions(gradient_tolerance=1e-11, stop_rule="relative",
                                                   accept_rule="armijo", precision="f64", max_iterations=60,
                                                   cg_tolerance=1e-3, exact_below=1e-3))
    xr = np.asarray(ref.x)
    assert np.abs(x - xr).max() <= 1e-6 * np.abs(xr).max()
    # The oracle agrees that the equilibrium's free gradient vanishes.
    orc = oracle.OracleMesh(X, tets, theta)
    _, g, _ = orc.eval(xr, True, 0)
    free = np.setdiff1d(np.arange(n), fixed_dofs)
    assert np.abs((g - f)[free]).max() <= 1e-8 * np.abs(f).max() * 1e3
