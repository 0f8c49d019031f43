"""The oracle's hex Q1 neo-Hookean energy (HexQ1Basis, GaussLegendre3D), pinned by the
reference's own hex test (tests/cpp/fem/assembly/volumetric_fem_energy_hex_q1_gtest.cpp:24-98:
two hexes of widths 1 and 2 sharing a face, theta = [2, 3], three states, finite differences of
the gradient and Hessian with h in {1e-3, 3e-4, 1e-4} to 10 h^2 + 1e-9, and a mixed second
difference of the scalar energy), plus a patch test: an affine displacement gives F = A at every
point and E = W(A) x volume."""

import numpy as np
import pytest

import oracle

HEX_X = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1],
                  [3, 0, 0], [3, 1, 0], [3, 0, 1], [3, 1, 1]], dtype=float)
HEX_CELLS = np.array([[0, 1, 2, 3, 4, 5, 6, 7], [1, 8, 9, 2, 5, 10, 11, 6]], dtype=np.int32)
HEX_THETA = np.array([2.0, 3.0])


def hex_states():
    x1 = 0.1 * HEX_X.ravel()
    x2 = x1 + 0.02 * np.sin(np.arange(x1.size) + 0.3)
    return [np.zeros(x1.size), x1, x2]


@pytest.mark.parametrize("state", [0, 1, 2])
def test_two_hex_finite_differences(state):
    x = hex_states()[state]
    E, g, H = oracle.hex_eval(HEX_X, HEX_CELLS, HEX_THETA, x)
    assert np.linalg.norm(H - H.T) < 1e-12 * (1 + np.linalg.norm(H))
    f = lambda y: oracle.hex_eval(HEX_X, HEX_CELLS, HEX_THETA, y, hessian=False)  # noqa: E731
    d = np.sin(np.arange(x.size) + 0.5)
    v = np.cos(np.arange(x.size) + 0.2)
    d, v = d / np.linalg.norm(d), v / np.linalg.norm(v)
    for h in (1e-3, 3e-4, 1e-4):
        fd_g, fd_h = np.zeros(x.size), np.zeros((x.size, x.size))
        for j in range(x.size):
            p, m = x.copy(), x.copy()
            p[j] += h
            m[j] -= h
            Ep, gp, _ = f(p)
            Em, gm, _ = f(m)
            fd_g[j] = (Ep - Em) / (2 * h)
            fd_h[:, j] = (gp - gm) / (2 * h)
        assert np.linalg.norm(g - fd_g) / (1 + np.linalg.norm(g)) < 10 * h * h + 1e-9
        assert np.linalg.norm(H - fd_h) / (1 + np.linalg.norm(H)) < 10 * h * h + 1e-9
        mixed = (f(x + h * d + h * v)[0] - f(x + h * d - h * v)[0] - f(x - h * d + h * v)[0] +
                 f(x - h * d - h * v)[0]) / (4 * h * h)
        assert abs(d @ H @ v - mixed) <= (10 * h * h + 1e-7) * (1 + np.linalg.norm(H))


@pytest.mark.parametrize("n", [2, 4])
def test_patch_test_and_quadrature(n):
    rng = np.random.default_rng(4)
    A = np.eye(3) + 0.1 * rng.standard_normal((3, 3))
    u = (HEX_X @ A.T - HEX_X).ravel()
    E, _, _ = oracle.hex_eval(HEX_X, HEX_CELLS, HEX_THETA, u, points_per_axis=n, hessian=False)
    volume = 1.0 + 2.0
    assert abs(E - volume * oracle.nh_W(A, np.eye(3), HEX_THETA)) <= 1e-12 * abs(E)
    _, w = oracle.hex_points(n)
    assert abs(w.sum() - 1.0) < 1e-15


@pytest.mark.parametrize("scale", [0.0, -1.0])
def test_invalid_geometry_is_rejected(scale):
    with pytest.raises(ValueError):
        oracle.hex_eval(scale * HEX_X, HEX_CELLS, HEX_THETA, np.zeros(HEX_X.size))


@pytest.mark.parametrize("state", [1, 2])
def test_hex_theta_vjp_matches_finite_differences(state):
    """The oracle's hex theta VJP (per element) against central differences of w . g(u; theta)
    in each element's own [lambda, mu] (g is linear in theta, so the difference is exact up to
    rounding)."""
    x = hex_states()[state]
    w = np.cos(np.arange(x.size) + 0.7)
    theta = np.array([[2.0, 3.0], [5.0, 1.5]])
    vjp = oracle.hex_force_vjp_theta(HEX_X, HEX_CELLS, theta, x, w)
    h = 1e-3
    for e in range(2):
        for c in range(2):
            tp, tm = theta.copy(), theta.copy()
            tp[e, c] += h
            tm[e, c] -= h
            gp = oracle.hex_eval(HEX_X, HEX_CELLS, tp, x, hessian=False)[1]
            gm = oracle.hex_eval(HEX_X, HEX_CELLS, tm, x, hessian=False)[1]
            fd = w @ (gp - gm) / (2 * h)
            assert abs(vjp[e, c] - fd) <= 1e-9 * (1 + abs(fd))
