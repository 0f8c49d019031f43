"""The element projection of the projected Hessian for hex meshes (litepgo_b200/csrc/lpg_psd.h,
the parallel-ordered cyclic Jacobi method the GPU runs one warp per element), compiled for the
host and checked against the oracle's eigensolver projection (mesh_energy.cpp:16-27) on random
indefinite matrices, hex element Hessians, singular and degenerate cases."""

import ctypes
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT

_dp = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def psd(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    out = tmp_path_factory.mktemp("psd") / "libpsd.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", str(ROOT / "litepgo_b200" / "csrc"),
                    str(ROOT / "tests" / "psd_jacobi_host.cpp"), "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    lib.psd_project.argtypes = [ctypes.c_int, _dp, _dp, _dp]
    lib.psd_round_pairs.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.psd_semidefinite9.argtypes = [_dp, ctypes.c_double]
    lib.psd_semidefinite9f.argtypes = [ctypes.POINTER(ctypes.c_float), ctypes.c_float]
    lib.clamp9_host.argtypes = [ctypes.c_int, _dp, _dp]

    def run(H):
        H = np.ascontiguousarray(H, dtype=np.float64)
        n = H.shape[0]
        out, eig = np.empty((n, n)), np.empty(n)
        sweeps = lib.psd_project(n, H.ctypes.data_as(_dp), out.ctypes.data_as(_dp), eig.ctypes.data_as(_dp))
        assert sweeps >= 0
        return out, np.sort(eig), sweeps

    run.lib = lib
    return run


def check(run, H, tol=1e-13):
    P, eig, sweeps = run(H)
    ref = oracle.project_psd(H)
    scale = max(np.linalg.norm(H), 1e-300)
    assert np.array_equal(P, P.T)  # bitwise symmetric
    assert np.linalg.norm(P - ref) <= tol * scale
    assert np.abs(eig - np.linalg.eigvalsh(H)).max() <= tol * scale
    assert sweeps <= 15
    return P, sweeps


def test_round_robin_covers_every_pair_once(psd):
    seen = set()
    for r in range(23):
        pairs = np.empty(24, np.int32)
        psd.lib.psd_round_pairs(r, pairs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        p, q = pairs[0::2], pairs[1::2]
        assert np.all(p < q) and sorted(np.concatenate([p, q]).tolist()) == list(range(24))
        seen.update(zip(p.tolist(), q.tolist()))
    assert len(seen) == 24 * 23 // 2


@pytest.mark.parametrize("n", [2, 8, 24])
def test_random_indefinite(psd, n):
    rng = np.random.default_rng(n)
    for scale in (1e-8, 1.0, 1e7):
        A = rng.standard_normal((n, n))
        check(psd, scale * (A + A.T))


def test_hex_element_hessians(psd):
    """The 24x24 Hessians of one hex at rest (PSD, singular: rigid translations), stretched, and
    compressed (indefinite): projected like the oracle, PSD ones left as they are."""
    X, cells = oracle.hex_box(1)
    rng = np.random.default_rng(4)
    theta = np.array([1.4e5, 3.4e4])
    for A, noise in ((np.eye(3), 0.0), (np.diag([1.3, 0.9, 1.1]), 0.02), (np.diag([1.0, 1.0, 0.35]), 0.05)):
        u = (X @ A.T - X + noise * rng.standard_normal(X.shape)).ravel()
        _, _, H = oracle.hex_eval(X, cells, theta, u)
        P, _ = check(psd, H)
        if np.linalg.eigvalsh(H).min() >= 0:
            assert np.linalg.norm(P - H) <= 1e-13 * np.linalg.norm(H)
    assert np.linalg.eigvalsh(H).min() < -1e-3 * np.abs(np.linalg.eigvalsh(H)).max()  # the last one was indefinite


def test_degenerate_spectra(psd):
    rng = np.random.default_rng(7)
    Q, _ = np.linalg.qr(rng.standard_normal((24, 24)))
    lam = np.repeat([-2.0, 0.0, 1.0, 3.0], 6)  # repeated eigenvalues, a zero block
    M = (Q * lam) @ Q.T
    check(psd, 0.5 * (M + M.T))  # exactly symmetric, as the element records are
    P, sweeps = check(psd, np.zeros((24, 24)))
    assert sweeps == 0 and not P.any()
    D = np.diag(np.linspace(-1, 1, 24))
    P, sweeps = check(psd, D)
    assert sweeps == 0 and np.array_equal(P, np.maximum(D, 0))
    low = rng.standard_normal((24, 3))
    check(psd, low @ low.T)  # rank 3, PSD


def nh_tangent_rowmajor(F, lam, mu):
    """A(3i+j, 3k+l) = mu d_ik d_jl + lam G_ij G_kl - p G_il G_kj, G = F^-T, p = lam log J - mu:
    the closed form the hex pre-test forms at each quadrature point."""
    G = np.linalg.inv(F).T
    p = lam * np.log(np.linalg.det(F)) - mu
    A = mu * np.eye(9) + lam * np.outer(G.ravel(), G.ravel())
    A -= p * np.einsum("il,kj->ijkl", G, G).reshape(9, 9)
    return A


@pytest.mark.parametrize("stretch", [1.0, 1.1, 0.9, 0.6, 1.6])
def test_tangent_closed_form_and_semidefinite_test(psd, stretch):
    """The closed-form tangent equals the oracle's d2W/dF2 (column-major vec there), and the LDL^T
    test (tol 64 eps max|diag|, the tet projection pass's) agrees with the eigenvalues' sign:
    at rest the tangent is singular semi-definite (rotation modes) and passes."""
    lam, mu = 1.4e5, 3.4e4
    rng = np.random.default_rng(int(stretch * 10))
    F = np.diag([1.0, 1.0, stretch]) + (0.0 if stretch == 1.0 else 0.03) * rng.standard_normal((3, 3))
    A = nh_tangent_rowmajor(F, lam, mu)
    perm = np.array([i + 3 * j for i in range(3) for j in range(3)])  # row-major r -> column-major index
    Ao = oracle.nh_d2W_dF2(F, np.eye(3), [lam, mu])[np.ix_(perm, perm)]
    assert np.abs(A - Ao).max() <= 1e-12 * np.abs(Ao).max()
    A = np.ascontiguousarray(A)
    tol = 64 * np.finfo(float).eps * np.abs(np.diag(A)).max()
    ev = np.linalg.eigvalsh(A)
    got = psd.lib.psd_semidefinite9(A.ctypes.data_as(_dp), ctypes.c_double(tol))
    if ev.min() >= 0 or ev.min() > -tol:
        assert got == 1
    elif ev.min() < -1e3 * tol:
        assert got == 0


def test_semidefinite_test_edge_cases(psd):
    lib = psd.lib
    rng = np.random.default_rng(3)
    Q, _ = np.linalg.qr(rng.standard_normal((9, 9)))

    def run(lam):
        A = np.ascontiguousarray((Q * lam) @ Q.T)
        return lib.psd_semidefinite9(A.ctypes.data_as(_dp), 64 * np.finfo(float).eps * np.abs(np.diag(A)).max())

    assert run(np.linspace(0.1, 2, 9)) == 1
    assert run(np.r_[np.zeros(3), np.linspace(0.1, 2, 6)]) == 1       # singular semi-definite
    assert run(np.r_[-1e-6, np.linspace(0.1, 2, 8)]) == 0              # a small negative eigenvalue
    assert run(np.r_[-1.0, np.zeros(2), np.linspace(0.1, 2, 6)]) == 0
    assert run(np.zeros(9)) == 1


def test_semidefinite_test_in_fp32(psd):
    """The FP32 instantiation (tol 64 eps_f max|diag|): semi-definite and singular semi-definite
    matrices pass, a clearly negative eigenvalue fails."""
    lib = psd.lib
    fp = ctypes.POINTER(ctypes.c_float)
    rng = np.random.default_rng(5)
    Q, _ = np.linalg.qr(rng.standard_normal((9, 9)))

    def run(lam):
        A = np.ascontiguousarray(((Q * lam) @ Q.T).astype(np.float32))
        A = np.ascontiguousarray(0.5 * (A + A.T))
        tol = np.float32(64 * np.finfo(np.float32).eps * np.abs(np.diag(A)).max())
        return lib.psd_semidefinite9f(A.ctypes.data_as(fp), tol)

    assert run(np.linspace(0.1, 2, 9)) == 1
    assert run(np.r_[np.zeros(3), np.linspace(0.1, 2, 6)]) == 1
    assert run(np.r_[-1e-2, np.linspace(0.1, 2, 8)]) == 0



def clamp9(psd, M, fp32):
    M = np.ascontiguousarray(M, dtype=np.float64)
    out = np.empty((9, 9))
    psd.lib.clamp9_host(1 if fp32 else 0, M.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
    return out


@pytest.mark.parametrize("fp32,tol", [(False, 1e-13), (True, 2e-6)])
def test_tet_tangent_clamp_matches_the_oracle(psd, fp32, tol):
    """The tet tangent's 9x9 clamp (lpg_clamp9.h, run by clamp_kernel) against the oracle's
    eigensolver projection, on indefinite neo-Hookean tangents and random symmetric matrices."""
    rng = np.random.default_rng(21)
    mats = [nh_tangent_rowmajor(np.diag([1.0, 1.0, s]) + 0.03 * rng.standard_normal((3, 3)), 1.4e5, 3.4e4)
            for s in (0.6, 1.6, 0.35)]
    mats += [(lambda B: 0.5 * (B + B.T))(rng.standard_normal((9, 9)) * 10.0 ** k) for k in (-6, 0, 6)]
    for M in mats:
        M = np.asarray(M, dtype=np.float32 if fp32 else np.float64).astype(np.float64)
        ref = oracle.project_psd(M)
        P = clamp9(psd, M, fp32)
        assert np.all(np.isfinite(P))
        assert np.linalg.norm(P - ref) <= tol * np.linalg.norm(M)


@pytest.mark.parametrize("fp32", [False, True])
def test_tet_tangent_clamp_with_an_underflowing_rotation(psd, fp32):
    """Two equal diagonal entries coupled by an off-diagonal entry so small (1e-30 of the largest)
    that d^2 + (2 a_pq)^2 underflows in FP32: the pair is left unrotated instead of producing a
    NaN, and the clamp still matches the oracle's."""
    M = np.diag([1.0, -0.5, 0.25, 0.25, 2.0, -1.0, 0.5, 3.0, 0.75])
    M[2, 3] = M[3, 2] = 1e-30
    M[0, 4] = M[4, 0] = 0.1
    P = clamp9(psd, M, fp32)
    assert np.all(np.isfinite(P))
    assert np.linalg.norm(P - oracle.project_psd(M)) <= (2e-6 if fp32 else 1e-13) * np.linalg.norm(M)
