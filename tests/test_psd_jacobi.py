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
    check(psd, (Q * lam) @ Q.T)
    P, sweeps = check(psd, np.zeros((24, 24)))
    assert sweeps == 0 and not P.any()
    D = np.diag(np.linspace(-1, 1, 24))
    P, sweeps = check(psd, D)
    assert sweeps == 0 and np.array_equal(P, np.maximum(D, 0))
    low = rng.standard_normal((24, 3))
    check(psd, low @ low.T)  # rank 3, PSD
