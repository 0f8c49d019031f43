"""The oracle's plastic force sensitivity (VolumetricFemForceFpResponse, src/core/fem/assembly/
volumetric_fem_force_fp_response.hpp with NeoHookean::eval_d2W_dF_dFp, neo_hookean.cpp:103-128),
pinned by central finite differences of the oracle force in Fp, as the reference's
tests/python/test_fp_force_response.py checks its Jacobian columns (rtol 1e-7)."""

import numpy as np

import oracle
from conftest import TWO_TET_CELLS, TWO_TET_THETA, TWO_TET_X, two_tet_states


def plastic_field(T, seed):
    rng = np.random.default_rng(seed)
    return np.stack([(np.eye(3) + 0.1 * rng.standard_normal((3, 3))).T.ravel() for _ in range(T)])


def test_fp_vjp_matches_finite_differences_of_the_force():
    X, cells, theta = TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA
    T = cells.shape[0]
    Fp = plastic_field(T, 1)
    x = two_tet_states()[1]
    w = np.random.default_rng(2).standard_normal(X.size)
    vjp = oracle.OracleMesh(X, cells, theta, Fp=Fp).force_vjp_fp(x, w)
    h = 1e-6
    for e in range(T):
        for c in range(9):
            Fpp, Fpm = Fp.copy(), Fp.copy()
            Fpp[e, c] += h
            Fpm[e, c] -= h
            gp = oracle.OracleMesh(X, cells, theta, Fp=Fpp).eval(x, True, 0)[1]
            gm = oracle.OracleMesh(X, cells, theta, Fp=Fpm).eval(x, True, 0)[1]
            fd = w @ (gp - gm) / (2 * h)
            assert abs(vjp[e, c] - fd) <= 1e-7 * abs(fd) + 1e-9 * np.abs(vjp).max()


def test_fp_vjp_at_identity_matches_the_closed_form():
    """At Fp = I, dP/dFp_c = tr(E_c) P - A : (F E_c) - P E_c^T (the reference's formula with
    Fp^-1 = I); contracted with B w this is the oracle's per-element VJP."""
    X, cells, theta = TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA
    x = two_tet_states()[2]
    w = np.random.default_rng(4).standard_normal(X.size)
    vjp = oracle.OracleMesh(X, cells, theta, Fp=np.tile(np.eye(3).ravel(), (2, 1))).force_vjp_fp(x, w)
    for e, cell in enumerate(cells):
        Dm = np.stack([X[cell[k + 1]] - X[cell[0]] for k in range(3)], 1)
        Dmi = np.linalg.inv(Dm)
        gradN = np.vstack([-Dmi.sum(0), Dmi])  # rows grad N_a
        U = x.reshape(-1, 3)[cell]
        F = np.eye(3) + (U[1:] - U[0]).T @ Dmi
        Gw = w.reshape(-1, 3)[cell].T @ gradN
        D = oracle.nh_d2W_dF_dFp(F, np.eye(3), theta)
        vol = np.linalg.det(Dm) / 6
        ref = vol * D.T @ Gw.T.ravel()
        np.testing.assert_allclose(vjp[e], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
