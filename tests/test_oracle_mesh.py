"""Mesh-level known answers of the reference, reproduced on the CPU oracle.

tests/cpp/fem/assembly/volumetric_fem_energy_tet_p1_gtest.cpp (two-tet mesh),
tests/cpp/solver/static_equilibrium_response_gtest.cpp:14-88 (single-tet equilibrium),
tests/python/test_fem_batch_size.py (bitwise invariance of the assembled Hessian).
"""

import numpy as np
import pytest

import oracle
from conftest import TWO_TET_CELLS, TWO_TET_THETA, TWO_TET_X, two_tet_states
from litepgo_b200 import workloads


def two_tet_mesh():
    return oracle.OracleMesh(TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA)


def dense_hessian(m, u, kind=1):
    return m.hessian_csc(u, kind).toarray()


# volumetric_fem_energy_tet_p1_gtest.cpp:51-115
@pytest.mark.parametrize("state", [0, 1, 2])
def test_two_tet_energy_gradient_hessian(state):
    m = two_tet_mesh()
    x = two_tet_states()[state]
    E, g, _ = m.eval(x)
    H = dense_hessian(m, x)
    assert np.linalg.norm(H - H.T) < 1e-12 * (1 + np.linalg.norm(H))
    expected = 0.0
    for cell in TWO_TET_CELLS:
        Dm = np.stack([TWO_TET_X[cell[c + 1]] - TWO_TET_X[cell[0]] for c in range(3)], axis=1)
        U = x.reshape(-1, 3)
        Du = np.stack([U[cell[c + 1]] - U[cell[0]] for c in range(3)], axis=1)
        expected += np.linalg.det(Dm) / 6 * oracle.nh_W(np.eye(3) + Du @ np.linalg.inv(Dm), np.eye(3), TWO_TET_THETA)
    assert abs(E - expected) < 1e-13
    for h in (1e-3, 3e-4, 1e-4):
        fd_g = np.zeros(x.size)
        fd_h = np.zeros((x.size, x.size))
        for j in range(x.size):
            p, q = x.copy(), x.copy()
            p[j] += h
            q[j] -= h
            Ep, gp, _ = m.eval(p)
            Eq, gq, _ = m.eval(q)
            fd_g[j] = (Ep - Eq) / (2 * h)
            fd_h[:, j] = (gp - gq) / (2 * h)
        assert np.linalg.norm(g - fd_g) / (1 + np.linalg.norm(g)) < 10 * h * h + 1e-9
        assert np.linalg.norm(H - fd_h) / (1 + np.linalg.norm(H)) < 10 * h * h + 1e-9


# volumetric_fem_energy_tet_p1_gtest.cpp:117-130
def test_two_tet_construction_rejects_invalid_geometry():
    for scale in (0.0, -1.0, 1e200):
        with pytest.raises(oracle.OracleError) as e:
            oracle.OracleMesh(scale * TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA)
        assert e.value.code == oracle.oracle.INVALID_ARGUMENT
    for bad in (np.nan, np.inf, -np.inf):
        X = TWO_TET_X.copy()
        X[0, 0] = bad
        with pytest.raises(oracle.OracleError) as e:
            oracle.OracleMesh(X, TWO_TET_CELLS, TWO_TET_THETA)
        assert e.value.code == oracle.oracle.INVALID_ARGUMENT


# volumetric_fem_energy_tet_p1_gtest.cpp:132-151
def test_two_tet_feasible_step():
    m = two_tet_mesh()
    X = TWO_TET_X.ravel()
    zero = np.zeros_like(X)
    assert m.feasible_step(zero, zero) == 1
    assert m.feasible_step(zero, 0.1 * X) == 1
    d = zero.copy()
    d[0::3] = -4 * X[0::3]
    d[1::3] = -4 * X[1::3]
    alpha = m.feasible_step(zero, d)
    assert abs(alpha - 0.225) < 1e-6
    for i in range(21):
        assert np.isfinite(m.eval(alpha * i / 20 * d, gradient=False)[0])
    d = zero.copy()
    d[14] = 16
    assert abs(m.feasible_step(zero, d) - 0.1125) < 1e-12
    with pytest.raises(oracle.OracleError) as e:
        m.feasible_step(-X, zero)
    assert e.value.code == oracle.oracle.DOMAIN_ERROR


# volumetric_fem_energy_tet_p1_gtest.cpp:153-169
def test_two_tet_newton_relaxes_free_vertices():
    m = two_tet_mesh()
    u = np.zeros(15)
    u[11] = 0.3
    u[14] = -0.2
    initial = m.eval(u, gradient=False)[0]
    x, info = m.newton(np.arange(9), u, tol=1e-9, hessian=2)
    assert info["status"] == 0
    assert info["iterations"] > 0
    assert info["energy"] < initial
    assert abs(info["energy"]) < 1e-12
    assert np.all(x[:9] == 0)


# volumetric_fem_energy_tet_p1_gtest.cpp:196-248 (per-element fields) restated with arrays:
# the energy of a mesh with per-element theta / Fp equals the sum of one-element meshes.
def test_per_element_fields_sum_over_elements():
    theta = np.array([[2.5, 3.5], [5.0, 7.0]])
    Fp = np.stack([(1.0 + 0.015 * k) * np.eye(3) for k in (0, 10)]).reshape(2, 9)
    both = oracle.OracleMesh(TWO_TET_X, TWO_TET_CELLS, theta, Fp=Fp)
    u = 0.03 * TWO_TET_X.ravel()
    parts = [oracle.OracleMesh(TWO_TET_X, TWO_TET_CELLS[e:e + 1], theta[e:e + 1], Fp=Fp[e:e + 1]) for e in (0, 1)]
    Eb, gb, _ = both.eval(u)
    Es = sum(p.eval(u)[0] for p in parts)
    gs = sum(p.eval(u)[1] for p in parts)
    assert abs(Eb - Es) < 1e-12
    assert np.allclose(gb, gs, rtol=1e-12, atol=1e-14)
    Hb = dense_hessian(both, u)
    Hs = sum(dense_hessian(p, u) for p in parts)
    assert np.allclose(Hb, Hs, rtol=1e-12, atol=1e-12)
    d = -2 * TWO_TET_X.ravel()
    assert both.feasible_step(u, d) == min(p.feasible_step(u, d) for p in parts)


# tests/python/test_fem_batch_size.py:7-21: the assembled Hessian is bitwise identical across
# thread counts (the oracle has no batch size; its element loop is thread-parallel).
def test_hessian_bitwise_thread_invariant():
    w = workloads.deformed_box(4, seed=1)
    m = oracle.OracleMesh(w["X"], w["tets"], w["theta"])
    oracle.set_threads(1)
    a = m.eval(w["u"], True, 2)
    oracle.set_threads(4)
    b = m.eval(w["u"], True, 2)
    oracle.set_threads(0)
    assert a[0] == b[0]
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[2], b[2])


# static_equilibrium_response_gtest.cpp:14-88: single-tet equilibrium with theta = (2, 3);
# the adjoint VJP matches central differences of re-solves.
def test_equilibrium_adjoint_matches_resolve_fd():
    X = np.array([[0, 0, 0], [1.2, 0, 0], [0, .8, 0], [0, 0, 1.5]], float)
    cells = np.array([[0, 1, 2, 3]], np.int32)
    Fp = np.eye(3)
    Fp[0, 1] = .08
    Fp[2, 2] = 1.1
    Fpv = Fp.T.ravel()[None, :]
    fixed = np.arange(9)
    initial = np.zeros(12)
    initial[3] = .15
    initial[7] = -.04

    def solve(p):
        m = oracle.OracleMesh(X, cells, np.asarray(p, float), Fp=Fpv)
        x, info = m.newton(fixed, initial, tol=1e-12, max_iterations=100, hessian=2)
        assert info["status"] == 0
        return m, x

    p = np.array([2.0, 3.0])
    m, u = solve(p)
    w = np.linspace(-.8, 1.1, 12)
    jtw, _ = m.adjoint_theta(u, w, fixed)
    jtw = jtw.sum(axis=0)
    v = np.array([.4, -.7])
    eps = 1e-4
    jv = (solve(p + eps * v)[1] - solve(p - eps * v)[1]) / (2 * eps)
    assert abs(w @ jv - v @ jtw) < 1e-8 * (1 + abs(w @ jv))
    for h in (1e-3, 1e-4):
        for c in range(2):
            e = np.zeros(2)
            e[c] = h
            col = (solve(p + e)[1] - solve(p - e)[1]) / (2 * h)
            assert abs(w @ col - jtw[c]) < 2e-7 * (1 + abs(jtw[c]))
    assert np.all(u[:9] == initial[:9])


def _rest_fd(X, cells, theta, u, w, h=1e-6):
    """Central finite differences of w . g(u; X) in every rest coordinate."""
    out = np.empty(X.size)
    for k in range(X.size):
        Xp, Xm = X.copy().ravel(), X.copy().ravel()
        Xp[k] += h
        Xm[k] -= h
        gp = oracle.OracleMesh(Xp.reshape(-1, 3), cells, theta).eval(u, True, 0)[1]
        gm = oracle.OracleMesh(Xm.reshape(-1, 3), cells, theta).eval(u, True, 0)[1]
        out[k] = (w @ gp - w @ gm) / (2 * h)
    return out


@pytest.mark.parametrize("state", [1, 2])
def test_rest_position_vjp_matches_finite_differences(state):
    """The rest-position force VJP has no reference counterpart: its oracle restatement is
    pinned against central differences of the oracle's own force."""
    u = two_tet_states()[state]
    w = np.sin(np.arange(u.size) + 0.7)
    m = two_tet_mesh()
    got = m.force_vjp_rest(u, w)
    fd = _rest_fd(TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA, u, w)
    assert np.max(np.abs(got - fd)) <= 1e-6 * max(1.0, np.max(np.abs(fd)))


def test_rest_position_vjp_box_per_element_theta():
    w_ = workloads.deformed_box(2, seed=4)
    X, cells, theta, u = w_["X"], w_["tets"], w_["theta"], w_["u"]
    rng = np.random.default_rng(3)
    th = np.column_stack([theta[0] * (1 + 0.3 * rng.random(cells.shape[0])), theta[1] * (1 + 0.3 * rng.random(cells.shape[0]))])
    w = rng.standard_normal(u.size)
    got = oracle.OracleMesh(X, cells, th).force_vjp_rest(u, w)
    fd = np.empty(X.size)
    h = 1e-6
    for k in range(X.size):
        Xp, Xm = X.copy().ravel(), X.copy().ravel()
        Xp[k] += h
        Xm[k] -= h
        gp = oracle.OracleMesh(Xp.reshape(-1, 3), cells, th).eval(u, True, 0)[1]
        gm = oracle.OracleMesh(Xm.reshape(-1, 3), cells, th).eval(u, True, 0)[1]
        fd[k] = (w @ gp - w @ gm) / (2 * h)
    assert np.max(np.abs(got - fd)) <= 1e-6 * np.max(np.abs(fd))
