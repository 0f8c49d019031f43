"""Python/Torch materials on the GPU path (the reference's PyVolumetricMaterial and
TorchVolumetricMaterial): the library exports F per element, the material evaluates W and its
derivatives on the device, the library integrates and assembles. A torch neo-Hookean must
reproduce the native NeoHookean energy; a torch St. Venant-Kirchhoff material is checked against
a dense NumPy assembly of vol B^T vec P and vol B^T A B from the same material on the CPU. The
same on hex meshes (HexQ1Basis, GaussLegendre3D[n]), with one material row per quadrature point."""

import numpy as np
import pytest

from conftest import rel_err
from litepgo_b200 import dof, energy, fem, mesh, workloads

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from litepgo_b200.torch import TorchVolumetricMaterial  # noqa: E402

Exact, Projected = energy.HessianKind.Exact, energy.HessianKind.Projected


class TorchNeoHookean(TorchVolumetricMaterial):
    num_parameters = 2

    @staticmethod
    def W(F, Fp, theta):
        lam, mu = theta[:, 0], theta[:, 1]
        L = torch.log(torch.linalg.det(F))
        return 0.5 * mu * ((F * F).sum((1, 2)) - 3) - mu * L + 0.5 * lam * L * L


class TorchStVK(TorchVolumetricMaterial):
    num_parameters = 2

    @staticmethod
    def W(F, Fp, theta):
        lam, mu = theta[:, 0], theta[:, 1]
        I = torch.eye(3, dtype=F.dtype, device=F.device)
        E = 0.5 * (F.transpose(1, 2) @ F - I)
        tr = E.diagonal(dim1=1, dim2=2).sum(1)
        return mu * (E * E).sum((1, 2)) + 0.5 * lam * tr * tr


def build(material, w):
    topo = mesh.TetTopology(w["X"].shape[0], w["tets"])
    cls = fem.VolumetricFemEnergy[material, fem.TetP1Basis, fem.TetCentroidQuadrature]
    return cls(dof.VertexDofMap(topo, 3), w["X"], None, w["theta"])


def test_torch_neo_hookean_matches_the_native_energy():
    w = workloads.deformed_box(6, seed=3)
    native = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    py = build(TorchNeoHookean, w)
    u = w["u"]
    H_exact = None
    for hk, tol in ((Exact, 1e-12), (Projected, 1e-11)):
        E0, g0, H0 = native.eval(u, gradient=True, hessian=hk)
        E1, g1, H1 = py.eval(u, gradient=True, hessian=hk)
        assert abs(E1 - E0) <= 1e-12 * abs(E0)
        assert rel_err(g1, g0) <= 1e-12
        assert rel_err(H1.data, H0.data) <= tol
        if hk == Exact:
            H_exact = H0
    # Mixed precision: FP32 blocks from the same FP64 material outputs.
    _, _, H32 = py.eval(u, hessian=Exact, precision="mixed")
    assert rel_err(H32.data, H_exact.data) <= 1e-5
    # The default feasible step is the native one (det F > 0).
    du = 0.5 * np.random.default_rng(1).standard_normal(u.size)
    assert py.max_feasible_step(u, du) == native.max_feasible_step(u, du)


def dense_reference(material, X, tets, theta, u):
    """E, g and dense H of sum_e vol [W, B^T vec P, B^T A B] with the material on the CPU."""
    T, n = tets.shape[0], X.size
    U = u.reshape(-1, 3)
    Fs, vols, grads = [], [], []
    for cell in tets:
        Dm = np.stack([X[cell[k + 1]] - X[cell[0]] for k in range(3)], 1)
        Dmi = np.linalg.inv(Dm)
        gN = np.vstack([-Dmi.sum(0), Dmi])  # rows grad N_a
        Fs.append(np.eye(3) + (U[cell[1:]] - U[cell[0]]).T @ Dmi)
        vols.append(np.linalg.det(Dm) / 6)
        grads.append(gN)
    F = torch.tensor(np.array(Fs))
    out = material.eval(F, torch.eye(3, dtype=torch.float64).expand(T, 3, 3),
                        torch.tensor(np.broadcast_to(theta, (T, 2)).copy()), outputs=("W", "dW_dF", "d2W_dF2"))
    W, P, A = out["W"].numpy(), out["dW_dF"].numpy(), out["d2W_dF2"].numpy()
    E, g, H = 0.0, np.zeros(n), np.zeros((n, n))
    for e, cell in enumerate(tets):
        vol, gN = vols[e], grads[e]
        E += vol * W[e]
        dofs = (3 * cell[:, None] + np.arange(3)).ravel()
        # dF_ij / du_(a,k) = delta_ik gN[a, j]
        Bm = np.zeros((9, 12))
        for a in range(4):
            for i in range(3):
                for j in range(3):
                    Bm[3 * i + j, 3 * a + i] = gN[a, j]
        g[dofs] += vol * Bm.T @ P[e].ravel()
        H[np.ix_(dofs, dofs)] += vol * Bm.T @ A[e].reshape(9, 9) @ Bm
    return E, g, H


def test_torch_stvk_matches_a_dense_assembly():
    w = workloads.deformed_box(3, seed=5)
    X, tets = w["X"], w["tets"]
    theta = np.array([1.4e5, 3.4e4])
    w2 = dict(w, theta=theta)
    py = build(TorchStVK, w2)
    u = w["u"]
    E, g, H = py.eval(u, gradient=True, hessian=Exact)
    Er, gr, Hr = dense_reference(TorchStVK, X, tets, theta, u)
    assert abs(E - Er) <= 1e-12 * abs(Er)
    assert rel_err(g, gr) <= 1e-12
    assert rel_err(H.toarray(), Hr) <= 1e-12
    # Projected: positive semi-definite and equal to the Exact one where that already is.
    _, _, Hp = py.eval(u, hessian=Projected)
    x = np.random.default_rng(2).standard_normal(u.size)
    assert x @ (Hp @ x) >= -1e-10 * np.abs(Hp.data).max() * (x @ x)


def test_non_finite_material_outputs_are_rejected():
    class Broken(TorchVolumetricMaterial):
        num_parameters = 0

        @staticmethod
        def W(F, Fp, theta):
            return torch.log(F[:, 0, 0] - 10.0)  # NaN at these states

    w = workloads.deformed_box(2, seed=0)
    topo = mesh.TetTopology(w["X"].shape[0], w["tets"])
    e = fem.VolumetricFemEnergy[Broken, fem.TetP1Basis, fem.TetCentroidQuadrature](
        dof.VertexDofMap(topo, 3), w["X"], None, None)
    with pytest.raises(ValueError):
        e.eval(w["u"], gradient=True)

    class Bounded(TorchNeoHookean):
        @staticmethod
        def eval_feasible_step(F, Fp, theta, dF):
            return torch.full((F.shape[0],), 0.5, dtype=F.dtype, device=F.device)

    b = build(Bounded, w)
    assert b.max_feasible_step(w["u"], np.ones(w["u"].size)) == 0.5


def hex_build(material, X, cells, theta, n=2):
    topo = mesh.HexTopology(X.shape[0], cells)
    cls = fem.VolumetricFemEnergy[material, fem.HexQ1Basis, fem.GaussLegendre3D[n]]
    return cls(dof.VertexDofMap(topo, 3), X, None, theta)


def hex_state():
    """A 3x3x2 hex box, per-element theta, compressed to 0.6 in z with noise (det F >= 0.55 at
    every point; the projection changes the Hessian by 16 % of its largest entry)."""
    import oracle

    X, cells = oracle.hex_box(3, 3, 2)
    rng = np.random.default_rng(7)
    T = cells.shape[0]
    theta = np.column_stack([1.4e5 * (1 + 0.2 * rng.random(T)), 3.4e4 * (1 + 0.2 * rng.random(T))])
    A = np.diag([1.0, 1.0, 0.6]) + 0.05 * rng.standard_normal((3, 3))
    u = (X @ A.T - X + 2e-3 * rng.standard_normal(X.shape)).ravel()
    return X, cells, theta, u


@pytest.mark.parametrize("n", [2, 4])
def test_torch_neo_hookean_on_hexes_matches_the_native_energy(n):
    """VolumetricFemEnergy[TorchNeoHookean, HexQ1Basis, GaussLegendre3D[n]]: F exported at every
    quadrature point, the torch material's W, P, A integrated per hex — equal to the native hex
    energy (Exact and Projected), in FP64 and mixed precision, with the native feasible step."""
    X, cells, theta, u = hex_state()
    native = fem.VolumetricFemEnergy[fem.NeoHookean, fem.HexQ1Basis, fem.GaussLegendre3D[n]].from_arrays(X, cells, theta)
    py = hex_build(TorchNeoHookean, X, cells, theta, n)
    assert py.deformation_gradients(u).shape == (cells.shape[0] * n ** 3, 3, 3)
    H_exact = None
    for hk, tol in ((Exact, 1e-12), (Projected, 1e-11)):
        E0, g0, H0 = native.eval(u, gradient=True, hessian=hk)
        E1, g1, H1 = py.eval(u, gradient=True, hessian=hk)
        assert abs(E1 - E0) <= 1e-12 * abs(E0)
        assert rel_err(g1, g0) <= 1e-12
        assert rel_err(H1.toarray(), H0.toarray()) <= tol
        if hk == Exact:
            H_exact = H0
    _, _, H32 = py.eval(u, hessian=Exact, precision="mixed")
    assert rel_err(H32.toarray(), H_exact.toarray()) <= 1e-6
    du = 0.5 * np.random.default_rng(1).standard_normal(u.size)
    assert py.max_feasible_step(u, du) == native.max_feasible_step(u, du)


def test_torch_stvk_on_hexes_matches_a_dense_assembly():
    """A torch St. Venant-Kirchhoff material on hexes against sum_q w_q [W, B^T vec P, B^T A B]
    assembled densely on the CPU from the same material at the same points."""
    import oracle

    X, cells, _, u = hex_state()
    theta = np.array([1.4e5, 3.4e4])
    pts, wts = oracle.hex_points(2)
    U = u.reshape(-1, 3)
    Fs, ws, gNs = [], [], []
    for cell in cells:
        for xi, wq in zip(pts, wts):
            dN = oracle.hex_dN_dxi(xi)
            J = X[cell].T @ dN
            gN = dN @ np.linalg.inv(J)
            Fs.append(np.eye(3) + U[cell].T @ gN)
            ws.append(wq * np.linalg.det(J))
            gNs.append(gN)
    R = len(Fs)
    out = TorchStVK.eval(torch.tensor(np.array(Fs)), torch.eye(3, dtype=torch.float64).expand(R, 3, 3),
                         torch.tensor(np.broadcast_to(theta, (R, 2)).copy()), outputs=("W", "dW_dF", "d2W_dF2"))
    W, P, A = out["W"].numpy(), out["dW_dF"].numpy(), out["d2W_dF2"].numpy()
    Er, gr, Hr = 0.0, np.zeros(X.size), np.zeros((X.size, X.size))
    r = 0
    for cell in cells:
        dofs = (3 * cell[:, None] + np.arange(3)).ravel()
        for _ in range(len(pts)):
            Bm = np.zeros((9, 24))
            for a in range(8):
                for i in range(3):
                    for j in range(3):
                        Bm[3 * i + j, 3 * a + i] = gNs[r][a, j]
            Er += ws[r] * W[r]
            gr[dofs] += ws[r] * Bm.T @ P[r].ravel()
            Hr[np.ix_(dofs, dofs)] += ws[r] * Bm.T @ A[r].reshape(9, 9) @ Bm
            r += 1
    py = hex_build(TorchStVK, X, cells, theta)
    E, g, H = py.eval(u, gradient=True, hessian=Exact)
    assert abs(E - Er) <= 1e-12 * abs(Er)
    assert rel_err(g, gr) <= 1e-12
    assert rel_err(H.toarray(), Hr) <= 1e-12


def test_newton_over_a_torch_material_matches_the_native_solve():
    """The reference runs newton_solve on a TorchVolumetricMaterial energy
    (examples/fem/fitting/torch_neohookean.py:112-113): a torch neo-Hookean gravity equilibrium
    (projected Hessian, Exact near the end) matches the native one, with the same step records;
    an exception in the material stops the solve and propagates."""
    import scipy.sparse as sp

    from litepgo_b200 import solver

    g = workloads.gravity_box(4, seed=0)
    n = g["X"].size
    load = energy.QuadraticEnergy(sp.csc_matrix((n, n)), -g["f"])
    native = fem.VolumetricFemEnergyTetP1.from_arrays(g["X"], g["tets"], g["theta"])
    py = build(TorchNeoHookean, {"X": g["X"], "tets": g["tets"], "theta": g["theta"]})
    opts = solver.NewtonOptions(gradient_tolerance=1e-10, stop_rule="relative", cg_tolerance=1e-8)
    fixed = dof.DofReduction(n, g["fixed"])
    steps_n, steps_p = [], []
    rn = solver.newton_solve(energy.WeightedSumEnergy([(native, 1.0), (load, 1.0)]), fixed, np.zeros(n), opts,
                             on_iteration=steps_n.append)
    rp = solver.newton_solve(energy.WeightedSumEnergy([(py, 1.0), (load, 1.0)]), fixed, np.zeros(n), opts,
                             on_iteration=steps_p.append)
    assert rn.status == rp.status == solver.NewtonStatus.Converged
    assert rel_err(rp.x, rn.x) <= 1e-8
    # The two evaluate the same energy with different summation orders, so the last step that
    # crosses the 1e-10 stopping bound may come one iteration apart.
    assert abs(rp.iterations - rn.iterations) <= 1 and abs(len(steps_p) - len(steps_n)) <= 1
    for a, b in zip(steps_p, steps_n):
        assert abs(a.energy - b.energy) <= 1e-9 * abs(b.energy) + 1e-300
    # A device start works too; a failing material stops the solve with its own exception.
    rd = solver.newton_solve(energy.WeightedSumEnergy([(py, 1.0), (load, 1.0)]), fixed,
                             torch.zeros(n, dtype=torch.float64, device="cuda"), opts)
    assert rel_err(rd.x.cpu().numpy(), rn.x) <= 1e-8

    class Broken(TorchNeoHookean):
        @staticmethod
        def W(F, Fp, theta):
            raise RuntimeError("material failed")

    bad = build(Broken, {"X": g["X"], "tets": g["tets"], "theta": g["theta"]})
    with pytest.raises(RuntimeError, match="material failed"):
        solver.newton_solve(bad, fixed, np.zeros(n), opts)


def test_static_equilibrium_response_over_a_torch_material():
    """The reference's neural equilibrium fit pattern (examples/fem/fitting/neural_equilibrium_fit.py):
    StaticEquilibriumResponse over a TorchVolumetricMaterial energy with
    VolumetricFemForceMaterialResponse[material, ...]. Its value and VJP equal those of the native
    neo-Hookean response with the same theta (the adjoint through the material's Exact Hessian and
    d2W/dF dtheta against lpg_adjoint_theta), and the VJP matches central differences."""
    import scipy.sparse as sp

    from litepgo_b200 import solver

    g = workloads.gravity_box(2, seed=0)
    X, tets, f = g["X"], g["tets"], g["f"]
    n, T = X.size, tets.shape[0]
    topo = mesh.TetTopology(X.shape[0], tets)
    dmap = dof.VertexDofMap(topo, 3)
    pmap = dof.ConstantDofMap(topo, 2)
    # Ten times gravity: a large sag (0.3 of the box) at a stable equilibrium (the oracle's Exact
    # stiffness there has smallest eigenvalue 1.2e3; at 50 times the box collapses to an unstable one).
    load = energy.QuadraticEnergy(sp.csc_matrix((n, n)), -10.0 * f)
    fixed = dof.DofReduction(n, g["fixed"])
    opts = solver.NewtonOptions(gradient_tolerance=1e-10, stop_rule="relative", max_iterations=100, cg_tolerance=1e-8)

    def make(material):
        key = (material, fem.TetP1Basis, fem.TetCentroidQuadrature)

        def make_energy(p):
            return energy.WeightedSumEnergy([(fem.VolumetricFemEnergy[key](dmap, X, None, np.asarray(p)), 1.0),
                                             (load, 1.0)])

        def make_response(u):
            return fem.VolumetricFemForceMaterialResponse[key](pmap, dmap, X, u, None)

        return solver.StaticEquilibriumResponse(2, fixed, np.zeros(n), opts, make_energy, make_response)

    p0 = np.array([1.4e5, 3.4e4])
    torch_model, native_model = make(TorchNeoHookean), make(fem.NeoHookean)
    xt, xn = torch_model.eval_value(p0), native_model.eval_value(p0)
    assert rel_err(xt, xn) <= 1e-9
    w = np.random.default_rng(3).standard_normal(n)
    vt, vn = torch_model.eval_vjp(p0, w), native_model.eval_vjp(p0, w)
    assert rel_err(vt, vn) <= 1e-8
    d = np.array([0.3, -0.7]) * p0
    h = 1e-4
    fd = (w @ torch_model.eval_value(p0 + h * d) - w @ torch_model.eval_value(p0 - h * d)) / (2 * h)
    assert abs(vt @ d - fd) <= 1e-5 * abs(fd)
