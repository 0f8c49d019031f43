"""TorchVolumetricMaterial (src/python/torch.py:72-94 of the reference): derivatives by autograd,
checked on the CPU against the oracle's closed-form neo-Hookean W, dW/dF and d2W/dF2
(NeoHookean, neo_hookean.cpp:33-86)."""

import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")
from litepgo_b200 import fem  # noqa: E402
from litepgo_b200.torch import TorchVolumetricMaterial  # noqa: E402


class TorchNeoHookean(TorchVolumetricMaterial):
    num_parameters = 2

    @staticmethod
    def W(F, Fp, theta):
        lam, mu = theta[:, 0], theta[:, 1]
        L = torch.log(torch.linalg.det(F))
        return 0.5 * mu * ((F * F).sum((1, 2)) - 3) - mu * L + 0.5 * lam * L * L


def test_torch_neo_hookean_derivatives_match_the_oracle():
    rng = np.random.default_rng(0)
    n = 6
    F = torch.tensor(np.eye(3) + 0.2 * rng.standard_normal((n, 3, 3)))
    theta = torch.tensor(np.stack([rng.uniform(1e3, 1e5, n), rng.uniform(1e3, 1e5, n)], 1))
    Fp = torch.eye(3, dtype=torch.float64).expand(n, 3, 3)
    out = TorchNeoHookean.eval(F, Fp, theta, outputs=("W", "dW_dF", "d2W_dF2"))
    assert out["W"].shape == (n,) and out["dW_dF"].shape == (n, 3, 3) and out["d2W_dF2"].shape == (n, 3, 3, 3, 3)
    for k in range(n):
        Fk, th = F[k].numpy(), theta[k].numpy()
        W = oracle.nh_W(Fk, np.eye(3), th)
        P = oracle.nh_dW_dF(Fk, np.eye(3), th)
        D = oracle.nh_d2W_dF2(Fk, np.eye(3), th)  # column-major vec indices i + 3 j
        A = out["d2W_dF2"][k].numpy()
        Acol = np.empty((9, 9))
        for i in range(3):
            for j in range(3):
                for kk in range(3):
                    for ll in range(3):
                        Acol[i + 3 * j, kk + 3 * ll] = A[i, j, kk, ll]
        assert abs(out["W"][k].item() - W) <= 1e-12 * abs(W) + 1e-9
        np.testing.assert_allclose(out["dW_dF"][k].numpy(), P, rtol=1e-12, atol=1e-12 * np.abs(P).max())
        np.testing.assert_allclose(Acol, D, rtol=1e-12, atol=1e-12 * np.abs(D).max())


def test_requested_outputs_only_and_shape_checks():
    F = torch.eye(3, dtype=torch.float64).expand(2, 3, 3).clone()
    th = torch.tensor([[1.0, 1.0], [1.0, 1.0]])
    out = TorchNeoHookean.eval(F, F, th, outputs=("W",))
    assert set(out) == {"W"} and torch.all(out["W"].abs() < 1e-12)

    class Bad(TorchVolumetricMaterial):
        num_parameters = 0

        @staticmethod
        def W(F, Fp, theta):
            return F.sum()

    with pytest.raises(ValueError):
        Bad.eval(F, F, th[:, :0], outputs=("W",))
    # The template accepts a Python material in the Material slot.
    cls = fem.VolumetricFemEnergy[TorchNeoHookean, fem.TetP1Basis, fem.TetCentroidQuadrature]
    assert issubclass(cls, fem.VolumetricFemEnergyPyMaterialTetP1) and cls.material is TorchNeoHookean
    with pytest.raises(TypeError):
        fem.VolumetricFemEnergy[int, fem.TetP1Basis, fem.TetCentroidQuadrature]


def test_quadrature_and_basis_templates():
    """The hex templates as the reference's tests/python/test_fem.py:21-30 names them."""
    cls = fem.VolumetricFemEnergy[fem.NeoHookean, fem.HexQ1Basis, fem.GaussLegendre3D[2]]
    assert cls.points_per_axis == 2
    assert fem.GaussLegendre3D[4].num_points == 64
    assert abs(fem.GaussLegendre3D[2].weights().sum() - 1.0) < 1e-15
    with pytest.raises(TypeError, match=r"available: .*GaussLegendre3D\[2\]"):
        fem.GaussLegendre3D[3]
    with pytest.raises(TypeError):
        fem.VolumetricFemEnergy[fem.NeoHookean, fem.TetP1Basis, fem.GaussLegendre3D[2]]


def test_hermite_and_hex_templates():
    """Every (material, basis, quadrature) the hex rows instantiate, as the reference binds them
    (src/binding/detail/fem_helpers.hpp:112-118), and the Hermite basis mirror."""
    import oracle

    for n in (2, 4):
        Q = fem.GaussLegendre3D[n]
        herm = fem.VolumetricFemEnergy[fem.NeoHookean, fem.HexHermiteBasis, Q]
        assert herm.points_per_axis == n and herm._dofs_per_vertex == 24
        resp = fem.VolumetricFemForceMaterialResponse[fem.NeoHookean, fem.HexQ1Basis, Q]
        assert resp._energy_cls.points_per_axis == n
        mat = fem.VolumetricFemEnergy[TorchNeoHookean, fem.HexQ1Basis, Q]
        assert mat.material is TorchNeoHookean and mat._geometry_cls.points_per_axis == n
    with pytest.raises(TypeError):
        fem.VolumetricFemEnergy[fem.NeoHookean, fem.HexHermiteBasis, fem.TetCentroidQuadrature]
    with pytest.raises(TypeError):  # no Python materials over the Hermite basis
        fem.VolumetricFemEnergy[TorchNeoHookean, fem.HexHermiteBasis, fem.GaussLegendre3D[2]]
    rng = np.random.default_rng(0)
    for xi in rng.random((5, 3)):
        N0, dN0 = oracle.hex_hermite_N_dN(xi)
        np.testing.assert_allclose(fem.HexHermiteBasis.eval_N(xi), N0, rtol=0, atol=1e-15)
        np.testing.assert_allclose(fem.HexHermiteBasis.eval_dN_dxi(xi), dN0, rtol=0, atol=1e-14)
        # The value functions alone sum to one (the reference's tests/python/test_fem.py:43).
        assert abs(fem.HexHermiteBasis.eval_N(xi)[0::8].sum() - 1.0) < 1e-14


def test_hex_fields_as_the_reference_builds_them():
    """Reference-style hex inputs (its examples/fem/equilibrium/hex_hermite_corner_pull.py): per-element
    InterpolatedResponse[HexQ1Basis] rest fields become vertex positions, constant AffineResponse
    theta and Fp fields become per-element values; inconsistent corners and varying fields raise."""
    from litepgo_b200 import mesh
    from litepgo_b200.energy import AffineResponse

    X, cells = mesh.make_hex_box(2, 1, 1)
    Field = fem.InterpolatedResponse[fem.HexQ1Basis]
    fields = [Field(X[c]) for c in cells]
    np.testing.assert_allclose(fields[0].eval_value(np.full(3, 0.5)), X[cells[0]].mean(0), atol=1e-15)
    np.testing.assert_array_equal(fem._hex_rest_positions(fields, cells, X.shape[0]), X)
    bad = [Field(X[cells[0]]), Field(X[cells[1]] + [0, 0, 1e-9])]
    with pytest.raises(ValueError, match="agree"):
        fem._hex_rest_positions(bad, cells, X.shape[0])
    pts = fem.GaussLegendre3D[2].points()
    theta_field = AffineResponse(np.zeros((2, 3)), np.array([2.0, 3.0]))
    np.testing.assert_array_equal(fem._sample_fields_hex([theta_field] * 2, 2, 2, "theta", pts), [2.0, 3.0])
    varying = AffineResponse(np.array([[1.0, 0, 0], [0, 0, 0]]), np.array([2.0, 3.0]))
    with pytest.raises(ValueError, match="element-constant"):
        fem._sample_fields_hex([varying] * 2, 2, 2, "theta", pts)
    # Interpolated theta from equal nodal values is constant (the reference's test_fem.py:247-257).
    q1 = Field(np.tile([2.0, 3.0], (8, 1)))
    np.testing.assert_allclose(fem._sample_fields_hex([q1] * 2, 2, 2, "theta", pts), [2.0, 3.0], atol=1e-15)


def test_basis_dof_transform_and_deformation_gradient():
    """The Hermite DOF convention through the basis utilities (the reference's
    tests/python/test_fem.py:472-496 scenario): on an axis-aligned box, an affine displacement's
    physical slots (u, u_X, u_Y, u_Z, zero mixed derivatives) interpolate to F = I + A at interior
    points, and the pullback scales by 1, hx, hy, hz, hx hy, hx hz, hy hz, hx hy hz."""
    size, origin = np.array([2.0, 1.0, 3.0]), np.array([0.5, -1.0, 2.0])
    X_nodes = origin + size * np.array([fem.HexQ1Basis.coefficient_info(v).point for v in range(8)])
    X_field = fem.InterpolatedResponse[fem.HexQ1Basis](X_nodes)
    transform = fem.BasisDofTransform[fem.HexHermiteBasis](X_field)
    assert transform.dofs_per_vertex == 24
    A = np.array([[0.1, -0.2, 0.05], [0.3, 0.0, -0.1], [0.02, 0.15, 0.2]])
    local = np.hstack([X_nodes @ A.T, np.tile(A.T.ravel(), (8, 1)), np.zeros((8, 12))])
    u_field = fem.InterpolatedResponse[fem.HexHermiteBasis](transform.to_coefficients(local))
    F = fem.DeformationGradientResponse(u_field, X_field)
    for xi in ([0.2, 0.7, 0.4], [0.9, 0.1, 0.5]):
        np.testing.assert_allclose(F.eval_value(np.array(xi)), (np.eye(3) + A).ravel(order="F"), atol=1e-13)
    gradient, hessian = transform.pullback(gradient=np.ones(192))
    assert hessian is None
    hx, hy, hz = size
    slots = np.array([1, hx, hy, hz, hx * hy, hx * hz, hy * hz, hx * hy * hz])
    np.testing.assert_allclose(gradient, np.tile(np.repeat(slots, 3), 8))
    _, H = transform.pullback(hessian=np.ones((192, 192)))
    np.testing.assert_allclose(H, np.outer(np.tile(np.repeat(slots, 3), 8), np.tile(np.repeat(slots, 3), 8)))
    nodal = fem.BasisDofTransform[fem.HexQ1Basis](X_field)
    assert nodal.dofs_per_vertex == 3
    np.testing.assert_array_equal(nodal.to_coefficients(X_nodes), X_nodes)
    sheared = X_nodes.copy()
    sheared[:, 0] += 0.2 * sheared[:, 1]
    with pytest.raises(ValueError):
        fem.BasisDofTransform[fem.HexHermiteBasis](fem.InterpolatedResponse[fem.HexQ1Basis](sheared))
    info = fem.HexHermiteBasis.coefficient_info(8 * 6 + 7)
    assert info.point.tolist() == [1, 1, 1] and info.derivative_orders == (1, 1, 1)
    with pytest.raises(IndexError):
        fem.HexHermiteBasis.coefficient_info(64)
