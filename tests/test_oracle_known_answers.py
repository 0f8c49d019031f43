"""Pins the CPU oracle to the reference's own known-answer tests.

Each test restates one case of the reference's GoogleTest suites for this path, with its
constants and tolerances:
  tests/cpp/fem/material/volumetric/neo_hookean_gtest.cpp
  tests/cpp/fem/kinematics/positive_det_feasible_step_gtest.cpp
"""

import numpy as np
import pytest

import oracle
from conftest import rotation

I = np.eye(3)
Z = np.zeros((3, 3))
INF, NAN = float("inf"), float("nan")


def raises(code, fn, *args):
    with pytest.raises(oracle.OracleError) as e:
        fn(*args)
    assert e.value.code == code, str(e.value)


INVALID, DOMAIN = oracle.oracle.INVALID_ARGUMENT, oracle.oracle.DOMAIN_ERROR


# neo_hookean_gtest.cpp:15-33
def test_mixed_parameter_derivative_dilation_and_shear():
    theta = np.array([0.0, 3.0])
    p, stretch = 1.3, 1.25
    dil = oracle.nh_d2W_dF_dtheta(p * stretch * I, p * I, theta)
    expected = np.zeros((9, 2))
    for i in range(3):
        expected[4 * i, 0] = p * p * 3 * np.log(stretch) / stretch
        expected[4 * i, 1] = p * p * (stretch - 1 / stretch)
    assert np.linalg.norm(dil - expected) <= 1e-13 * np.linalg.norm(expected)
    F = I.copy()
    F[0, 1] = 0.4
    expected = np.zeros((9, 2))
    expected[3, 1] = 0.4
    expected[1, 1] = 0.4
    assert np.linalg.norm(oracle.nh_d2W_dF_dtheta(F, I, theta) - expected) <= 1e-14 * np.linalg.norm(expected)
    assert np.linalg.norm(oracle.nh_d2W_dF_dtheta(p * I, p * I, theta)) < 1e-13


# neo_hookean_gtest.cpp:35-52
def test_mixed_derivative_reconstructs_stress_with_plastic_state():
    F = np.array([[1.2, .3, -.1], [.1, .9, .2], [-.05, .1, 1.1]])
    Fp = np.array([[1.3, .2, .1], [0, .9, -.1], [.1, .2, 1.2]])
    R = rotation(0.7, [1, 2, 3])
    B = oracle.nh_d2W_dF_dtheta(F, Fp, [2, 3])
    for theta in ([0, 1], [5, .7], [2, 3]):
        P = oracle.nh_dW_dF(F, Fp, theta)
        Pv = P.T.ravel()
        assert np.linalg.norm(B @ np.array(theta, float) - Pv) <= 1e-13 * np.linalg.norm(Pv)
        assert np.linalg.norm(B - oracle.nh_d2W_dF_dtheta(F, Fp, theta)) == 0
    rotated = oracle.nh_d2W_dF_dtheta(R @ F, Fp, [2, 3])
    for c in range(2):
        expected = (R @ B[:, c].reshape(3, 3).T).T.ravel()
        assert np.linalg.norm(rotated[:, c] - expected) <= 1e-13 * np.linalg.norm(expected)


# neo_hookean_gtest.cpp:54-72
def test_mixed_derivative_rejects_invalid_inputs_and_overflow():
    for bad in ([-1, 3], [2, 0], [2, INF]):
        raises(INVALID, oracle.nh_d2W_dF_dtheta, I, I, bad)
    bad = I.copy()
    bad[0, 0] = NAN
    raises(INVALID, oracle.nh_d2W_dF_dtheta, bad, I, [2, 3])
    raises(INVALID, oracle.nh_d2W_dF_dtheta, I, bad, [2, 3])
    raises(DOMAIN, oracle.nh_d2W_dF_dtheta, -I, I, [2, 3])
    raises(DOMAIN, oracle.nh_d2W_dF_dtheta, I, Z, [2, 3])
    Fp = I.copy()
    Fp[1, 1] = Fp[2, 2] = 1e150
    F = Fp.copy()
    F[0, 0] = 1e-20
    raises(DOMAIN, oracle.nh_d2W_dF_dtheta, F, Fp, [2, 3])


# neo_hookean_gtest.cpp:74-91
def test_overflowing_values_or_derivatives_are_domain_errors():
    F = I.copy()
    F[0, 0] = 1e155
    raises(DOMAIN, oracle.nh_W, F, I, [2, 3])
    F = I.copy()
    F[0, 0] = 2
    assert np.isfinite(oracle.nh_W(F, I, [0, 1e308]))
    raises(DOMAIN, oracle.nh_dW_dF, F, I, [0, 1e308])
    assert oracle.nh_W(I, I, [0, 1e308]) == 0
    assert np.all(np.isfinite(oracle.nh_dW_dF(I, I, [0, 1e308])))
    raises(DOMAIN, oracle.nh_d2W_dF2, I, I, [0, 1e308])


# neo_hookean_gtest.cpp:93-110
def test_stress_free_and_linear_elastic_tangent():
    theta = [2.0, 3.0]
    Fp = np.array([[1.3, 0.2, 0.1], [0.0, 0.9, -0.1], [0.1, 0.2, 1.2]])
    R = rotation(0.7, [1, 2, 3])
    for F in (Fp, R @ Fp):
        assert abs(oracle.nh_W(F, Fp, theta)) < 1e-13
        assert np.linalg.norm(oracle.nh_dW_dF(F, Fp, theta)) < 1e-13
    H = oracle.nh_d2W_dF2(I, I, theta)
    for j in range(9):
        D = np.zeros(9)
        D[j] = 1
        Dm = D.reshape(3, 3).T  # column-major index j -> matrix
        expected = theta[1] * (Dm + Dm.T) + theta[0] * np.trace(Dm) * I
        assert np.linalg.norm(H[:, j] - expected.T.ravel()) < 1e-13


# neo_hookean_gtest.cpp:112-126
def test_analytic_dilation_and_objectivity():
    theta = [2.0, 3.0]
    s, p = 1.25, 1.3
    L = 3 * np.log(s)
    psi = 1.5 * theta[1] * (s * s - 1) - theta[1] * L + 0.5 * theta[0] * L * L
    assert abs(oracle.nh_W(s * p * I, p * I, theta) - p ** 3 * psi) < 1e-13
    expectedP = p * p * (theta[1] * s + (theta[0] * L - theta[1]) / s) * I
    P = oracle.nh_dW_dF(s * p * I, p * I, theta)
    assert np.linalg.norm(P - expectedP) <= 1e-13 * np.linalg.norm(expectedP)
    F = np.array([[1.2, 0.2, 0.1], [-0.1, 0.8, 0.3], [0.2, 0.1, 1.1]])
    R = rotation(0.6, [2, -1, 3])
    assert abs(oracle.nh_W(R @ F, p * I, theta) - oracle.nh_W(F, p * I, theta)) < 1e-13
    a, b = oracle.nh_dW_dF(R @ F, p * I, theta), R @ oracle.nh_dW_dF(F, p * I, theta)
    assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(b)


# neo_hookean_gtest.cpp:128-179
@pytest.mark.parametrize("sample", range(12))
def test_full_gradient_and_hessian_finite_differences(sample):
    j = np.arange(9)
    Fp = (0.12 * np.sin(1.7 * (j + 1) * (sample + 1))).reshape(3, 3).T
    Fe = (0.15 * np.cos(0.8 * (j + 1) * (sample + 2))).reshape(3, 3).T
    Fp += (0.8 + 0.06 * sample) * I
    Fe += (0.7 + 0.05 * sample) * I
    F = Fe @ Fp
    assert np.linalg.det(Fp) > 0 and np.linalg.det(Fe) > 0
    theta = [0.5 * sample, 0.7 + sample]
    P = oracle.nh_dW_dF(F, Fp, theta)
    H = oracle.nh_d2W_dF2(F, Fp, theta)
    assert np.linalg.norm(H - H.T) < 1e-12 * (1 + np.linalg.norm(H))
    Fv = F.T.ravel()
    for h in (1e-3, 3e-4, 1e-4):
        fdP = np.zeros(9)
        fdH = np.zeros((9, 9))
        for k in range(9):
            plus, minus = Fv.copy(), Fv.copy()
            plus[k] += h
            minus[k] -= h
            Fpl, Fmi = plus.reshape(3, 3).T, minus.reshape(3, 3).T
            fdP[k] = (oracle.nh_W(Fpl, Fp, theta) - oracle.nh_W(Fmi, Fp, theta)) / (2 * h)
            fdH[:, k] = ((oracle.nh_dW_dF(Fpl, Fp, theta) - oracle.nh_dW_dF(Fmi, Fp, theta)) / (2 * h)).T.ravel()
        Pv = P.T.ravel()
        assert np.linalg.norm(Pv - fdP) / (1 + np.linalg.norm(Pv)) < 20 * h * h + 1e-9
        assert np.linalg.norm(H - fdH) / (1 + np.linalg.norm(H)) < 20 * h * h + 1e-9
    U = np.array([[1, 2, -1], [0, 1, 3], [-2, 0, 1]], float)
    Vm = np.array([[0, 1, 2], [-1, 3, 0], [1, -2, 1]], float)
    U /= np.linalg.norm(U)
    Vm /= np.linalg.norm(Vm)
    h = 2e-4
    W = lambda A: oracle.nh_W(A, Fp, theta)  # noqa: E731
    fd = (W(F + h * U + h * Vm) - W(F + h * U - h * Vm) - W(F - h * U + h * Vm) + W(F - h * U - h * Vm)) / (4 * h * h)
    exact = U.T.ravel() @ H @ Vm.T.ravel()
    assert abs(fd - exact) < 2e-6 * (1 + np.linalg.norm(H))


# neo_hookean_gtest.cpp:181-210
def test_rejects_invalid_states_and_parameters_in_every_entry_point():
    fns = (oracle.nh_W, oracle.nh_dW_dF, oracle.nh_d2W_dF2, oracle.nh_d2W_dF_dtheta)
    for x in (0.0, -1.0):
        bad = I.copy()
        bad[0, 0] = x
        for fn in fns:
            raises(DOMAIN, fn, bad, I, [2, 3])
            raises(DOMAIN, fn, I, bad, [2, 3])
    for bad in ([-1, 3], [2, 0], [2, -1], [NAN, 3], [2, INF]):
        for fn in fns:
            raises(INVALID, fn, I, I, bad)
    bad = I.copy()
    bad[0, 0] = NAN
    for fn in fns:
        raises(INVALID, fn, bad, I, [2, 3])


# neo_hookean_gtest.cpp:212-226
def test_feasible_step_limits_total_and_plastic_gradients():
    dF = np.diag([-4.0, -4, 0])
    dFp = np.diag([-8.0, 0, 0])
    for plastic in (False, True):
        alpha = oracle.nh_feasible_step(I, I, [2, 3], dF, dFp if plastic else Z, [0, 0])
        assert abs(alpha - (0.1125 if plastic else 0.225)) < 1e-6
        for i in range(101):
            t = alpha * i / 100
            assert np.isfinite(oracle.nh_W(I + t * dF, I + t * (dFp if plastic else Z), [2, 3]))


# neo_hookean_gtest.cpp:228-246
def test_feasible_step_keeps_parameters_in_domain():
    assert abs(oracle.nh_feasible_step(I, I, [2, 3], Z, Z, [-8, 0]) - 0.225) < 1e-14
    assert abs(oracle.nh_feasible_step(I, I, [2, 3], Z, Z, [0, -12]) - 0.225) < 1e-14
    assert oracle.nh_feasible_step(I, I, [0, 3], Z, Z, [-1, 0]) == 0
    assert oracle.nh_feasible_step(I, I, [0, 3], Z, Z, [1, 1]) == 1
    alpha = oracle.nh_feasible_step(I, I, [1e308, 3], Z, Z, [1e308, 0])
    assert 0 < alpha < 1
    assert np.isfinite(oracle.nh_W(I, I, [1e308 + alpha * 1e308, 3]))


# neo_hookean_gtest.cpp:248-263
def test_feasible_step_rejects_malformed_directions_and_infeasible_starts():
    raises(DOMAIN, oracle.nh_feasible_step, -I, I, [2, 3], Z, Z, [0, 0])
    raises(DOMAIN, oracle.nh_feasible_step, I, Z, [2, 3], Z, Z, [0, 0])
    raises(INVALID, oracle.nh_feasible_step, I, I, [-1, 3], Z, Z, [0, 0])
    bad = Z.copy()
    bad[0, 0] = INF
    raises(INVALID, oracle.nh_feasible_step, I, I, [2, 3], Z, bad, [0, 0])
    raises(INVALID, oracle.nh_feasible_step, I, I, [2, 3], Z, Z, [0, NAN])


# neo_hookean_gtest.cpp:270-279
def test_plastic_mixed_derivative_rest_and_dilation():
    theta = [2.0, 3.0]
    A = oracle.nh_d2W_dF_dFp(I, I, theta)
    B = -oracle.nh_d2W_dF2(I, I, theta)
    assert np.linalg.norm(A - B) <= 1e-14 * np.linalg.norm(B)
    a, b = 1.3, 0.8
    M = oracle.nh_d2W_dF_dFp(a * I, b * I, theta)
    d = I.T.ravel()
    expected = theta[1] * a + b * b / a * (9 * theta[0] * np.log(a / b) - 3 * theta[1] - 3 * theta[0])
    assert np.linalg.norm(M @ d - expected * d) <= 1e-13 * np.linalg.norm(expected * d)


# neo_hookean_gtest.cpp:283-304
def test_plastic_mixed_derivative_matches_stress_perturbations():
    F = np.array([[1.2, .2, -.1], [.05, .9, .1], [.02, -.04, 1.1]])
    Fp = np.array([[.9, -.1, .03], [.04, 1.2, .08], [-.02, .05, 1.1]])
    theta = [2.0, 3.0]
    B = oracle.nh_d2W_dF_dFp(F, Fp, theta)
    Fpv = Fp.T.ravel()
    for c in range(9):
        plus, minus = Fpv.copy(), Fpv.copy()
        plus[c] += 1e-6
        minus[c] -= 1e-6
        dP = (oracle.nh_dW_dF(F, plus.reshape(3, 3).T, theta) - oracle.nh_dW_dF(F, minus.reshape(3, 3).T, theta)) / 2e-6
        assert np.linalg.norm(B[:, c] - dP.T.ravel()) <= 1e-8 * max(np.linalg.norm(dP), 1e-300)
    raises(DOMAIN, oracle.nh_d2W_dF_dFp, F, Z, theta)
    raises(DOMAIN, oracle.nh_d2W_dF_dFp, -F, Fp, theta)
    raises(INVALID, oracle.nh_d2W_dF_dFp, F, Fp, [2, 0])
    bad = Fp.copy()
    bad[0, 0] = NAN
    raises(INVALID, oracle.nh_d2W_dF_dFp, F, bad, theta)
    raises(DOMAIN, oracle.nh_d2W_dF_dFp, I, I, [0, 1e308])


def _check_segment(A, dA, alpha):
    assert 0 <= alpha <= 1
    for i in range(101):
        d = np.linalg.det(A + (alpha * i / 100) * dA)
        assert d > 0 and np.isfinite(d)


# positive_det_feasible_step_gtest.cpp:24-36
def test_positive_det_full_step_directions():
    shear = Z.copy()
    shear[0, 1] = 10
    rot = Z.copy()
    rot[0, 1], rot[1, 0] = -4, 4
    for dA in (Z, I, shear, rot):
        assert oracle.positive_det_step(I, dA) == 1
        _check_segment(I, dA, 1)


# positive_det_feasible_step_gtest.cpp:38-54
def test_positive_det_linear_quadratic_cubic():
    for diag in ([-4, 0, 0], [-4, -2, 0], [-4, -2, -1]):
        dA = np.diag(np.array(diag, float))
        alpha = oracle.positive_det_step(I, dA)
        assert abs(alpha - 0.225) < 1e-12
        _check_segment(I, dA, alpha)
    assert oracle.positive_det_step(I, -0.5 * I) == 1
    cyclic = np.array([[0, 1, 0], [0, 0, 1], [-8, 0, 0]], float)
    alpha = oracle.positive_det_step(I, cyclic)
    assert abs(alpha - 0.45) < 1e-12
    _check_segment(I, cyclic, alpha)


# positive_det_feasible_step_gtest.cpp:56-68
def test_positive_det_double_and_triple_roots():
    for diag in ([-4, -4, 0], [-4, -4, 1], [-4, -4, -4]):
        dA = np.diag(np.array(diag, float))
        alpha = oracle.positive_det_step(I, dA)
        assert abs(alpha - 0.225) < 2e-5 and alpha < 0.25
        _check_segment(I, dA, alpha)


# positive_det_feasible_step_gtest.cpp:70-88
def test_positive_det_scaling_and_basis_invariance():
    R = rotation(0.7, [1, 2, 3])
    B = np.array([[1.2, 0.2, -0.1], [0.1, 0.9, 0.2], [0.02, -0.1, 1.1]])
    D = np.diag([-4.0, -2, 1])
    for scale in (1e-50, 0.1, 1.0, 10.0, 1e50):
        A, dA = scale * R @ B, scale * R @ D @ B
        alpha = oracle.positive_det_step(A, dA)
        assert abs(alpha - 0.225) < 1e-12
        _check_segment(A, dA, alpha)
    extreme = Z.copy()
    extreme[0, 0] = -1e200
    tiny = oracle.positive_det_step(I, extreme)
    assert abs(tiny / 9e-201 - 1) < 1e-12
    assert oracle.positive_det_step(I, 1e300 * I) == 0


# positive_det_feasible_step_gtest.cpp:90-100
def test_positive_det_rejects_invalid_starts():
    raises(DOMAIN, oracle.positive_det_step, Z, I)
    raises(DOMAIN, oracle.positive_det_step, -I, Z)
    raises(DOMAIN, oracle.positive_det_step, 1e200 * I, Z)
    for v in (INF, NAN):
        bad = I.copy()
        bad[0, 0] = v
        raises(INVALID, oracle.positive_det_step, bad, Z)
        raises(INVALID, oracle.positive_det_step, I, bad)


def test_psd_projection_clamps_negative_eigenvalues():
    rng = np.random.default_rng(3)
    Q, _ = np.linalg.qr(rng.standard_normal((12, 12)))
    lam = np.linspace(-3, 5, 12)
    H = Q @ np.diag(lam) @ Q.T
    P = oracle.project_psd(H)
    expected = Q @ np.diag(np.maximum(lam, 0)) @ Q.T
    assert np.linalg.norm(P - expected) < 1e-12 * np.linalg.norm(expected)
