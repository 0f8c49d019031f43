"""The oracle's tricubic Hermite hex energy (HexHermiteBasis with GaussLegendre3D, physical DOFs
scaled by BasisDofTransform<HexHermiteBasis>), pinned by the basis's interpolation property
(each function's own corner functional is 1, every other one 0), an affine patch test on two
boxes of different sizes sharing a face (F = A at every point, E = W(A) x volume), finite
differences of the energy and gradient, and the reference's geometry check (sheared boxes
rejected, tests/python/test_hex_force_response.py:60-75)."""

import numpy as np
import pytest

import oracle

# Two axis-aligned boxes sharing the face x = 1.7 (sizes 1.7 x 0.8 x 1.2 and 1.0 x 0.8 x 1.2).
HERMITE_X = np.array([[0, 0, 0], [1.7, 0, 0], [1.7, 0.8, 0], [0, 0.8, 0], [0, 0, 1.2], [1.7, 0, 1.2], [1.7, 0.8, 1.2],
                      [0, 0.8, 1.2], [2.7, 0, 0], [2.7, 0.8, 0], [2.7, 0, 1.2], [2.7, 0.8, 1.2]]) + [2.0, -0.3, 0.4]
HERMITE_CELLS = np.array([[0, 1, 2, 3, 4, 5, 6, 7], [1, 8, 9, 2, 5, 10, 11, 6]], dtype=np.int32)
HERMITE_THETA = np.array([2.0, 3.0])


def hermite_state(scale=0.002):
    return scale * np.sin(np.arange(24 * 12) + 0.3)


def test_interpolation_property():
    eps = 1e-5
    for c, corner in enumerate(oracle.HEX_CORNERS.astype(float)):
        N, dN = oracle.hex_hermite_N_dN(corner)
        np.testing.assert_allclose(N, np.eye(64)[8 * c], atol=1e-14)
        for d in range(3):
            np.testing.assert_allclose(dN[:, d], np.eye(64)[8 * c + 1 + d], atol=1e-14)
        # Mixed slots 4..7: xy, xz, yz, xyz, by central differences of the reference gradient.
        def mixed(i, j):
            ep = np.zeros(3)
            ep[j] = eps
            return (oracle.hex_hermite_N_dN(corner + ep)[1][:, i] - oracle.hex_hermite_N_dN(corner - ep)[1][:, i]) / (2 * eps)
        for slot, (i, j) in zip((4, 5, 6), ((0, 1), (0, 2), (1, 2))):
            np.testing.assert_allclose(mixed(i, j), np.eye(64)[8 * c + slot], atol=1e-8)


def test_affine_patch():
    A = np.eye(3) + 0.1 * np.array([[1, 2, 0], [0, 1, 3], [1, 0, 2.0]])
    L = A - np.eye(3)
    D = np.zeros((12, 24))
    D[:, 0:3] = HERMITE_X @ L.T
    for d in range(3):
        D[:, 3 * (1 + d):3 * (2 + d)] = L[:, d]
    E, _, _ = oracle.hex_hermite_eval(HERMITE_X, HERMITE_CELLS, HERMITE_THETA, D.ravel(), hessian=False)
    vol = 1.7 * 0.8 * 1.2 + 1.0 * 0.8 * 1.2
    assert E == pytest.approx(oracle.nh_W(A, np.eye(3), HERMITE_THETA) * vol, rel=1e-13)


@pytest.mark.parametrize("n", [2, 4])
def test_finite_differences(n):
    x = hermite_state()
    E, g, H = oracle.hex_hermite_eval(HERMITE_X, HERMITE_CELLS, HERMITE_THETA, x, points_per_axis=n)
    assert np.array_equal(H, H.T) or np.abs(H - H.T).max() <= 1e-12 * np.abs(H).max()
    rng = np.random.default_rng(n)
    h = 1e-5
    for _ in range(4):
        d = rng.standard_normal(x.size)
        Ep = oracle.hex_hermite_eval(HERMITE_X, HERMITE_CELLS, HERMITE_THETA, x + h * d, n, hessian=False)
        Em = oracle.hex_hermite_eval(HERMITE_X, HERMITE_CELLS, HERMITE_THETA, x - h * d, n, hessian=False)
        assert abs((Ep[0] - Em[0]) / (2 * h) - g @ d) <= 1e-7 * (1 + abs(g @ d))
        np.testing.assert_allclose((Ep[1] - Em[1]) / (2 * h), H @ d, rtol=0, atol=1e-6 * np.abs(H @ d).max())


def test_sheared_geometry_is_rejected():
    X = oracle.HEX_CORNERS.astype(float)
    oracle.hermite_box(X)
    sheared = X.copy()
    sheared[:, 0] += 0.2 * sheared[:, 1]
    with pytest.raises(ValueError):
        oracle.hermite_box(sheared)
    with pytest.raises(ValueError):
        oracle.hermite_box(X[[1, 0, 3, 2, 5, 4, 7, 6]])


def test_theta_vjp_matches_finite_differences():
    """The oracle's Hermite theta VJP per element against central differences of w . g(u; theta)
    in each element's [lambda, mu] (g is linear in theta)."""
    x = hermite_state(0.05)
    w = np.cos(np.arange(x.size) + 0.7)
    theta = np.array([[2.0, 3.0], [5.0, 1.5]])
    vjp = oracle.hex_hermite_force_vjp_theta(HERMITE_X, HERMITE_CELLS, theta, x, w)
    h = 1e-3
    for e in range(2):
        for c in range(2):
            tp, tm = theta.copy(), theta.copy()
            tp[e, c] += h
            tm[e, c] -= h
            gp = oracle.hex_hermite_eval(HERMITE_X, HERMITE_CELLS, tp, x, hessian=False)[1]
            gm = oracle.hex_hermite_eval(HERMITE_X, HERMITE_CELLS, tm, x, hessian=False)[1]
            fd = w @ (gp - gm) / (2 * h)
            assert abs(vjp[e, c] - fd) <= 1e-9 * (1 + abs(fd))


@pytest.mark.parametrize("kind", ["q1", "hermite"])
def test_theta_vjp_reproduces_the_force(kind):
    """g is linear in theta, so w . g(u; theta) = sum_e theta_e . vjp_e(w) (the reference's
    tests/python/test_material_force_response.py: the force response equals the energy gradient)."""
    theta = np.array([[2.0, 3.0], [5.0, 1.5]])
    if kind == "q1":
        from test_oracle_hex import HEX_CELLS, HEX_X, hex_states

        X, cells, x = HEX_X, HEX_CELLS, hex_states()[2]
        g = oracle.hex_eval(X, cells, theta, x, hessian=False)[1]
        vjp = oracle.hex_force_vjp_theta(X, cells, theta, x, g)
    else:
        X, cells, x = HERMITE_X, HERMITE_CELLS, hermite_state(0.05)
        g = oracle.hex_hermite_eval(X, cells, theta, x, hessian=False)[1]
        vjp = oracle.hex_hermite_force_vjp_theta(X, cells, theta, x, g)
    assert abs((vjp * theta).sum() - g @ g) <= 1e-12 * (g @ g)
