"""The tet assembly kernel's plan-driven work (tet_cluster_kernel, litepgo_b200/csrc/lpg_assemble.cu)
replayed on the host: tests/tet_assembly_host.cpp builds the library's own cluster plan
(litepgo_b200/csrc/lpg_plan.cpp, compiled with g++) and runs the element, item and copy passes
the kernel runs, in FP64, into BSR and CSC values. Compared with the oracle's assembly
(mesh_energy.cpp's per-column CSC sums), this checks every staging position, transpose flag and
contributor list of the plan on structured boxes, a shuffled numbering, a Delaunay ball and the
reference's bunny, without a GPU."""

import ctypes
import shutil
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from conftest import ROOT, corner_chain, rel_err
from litepgo_b200 import mesh

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
THETA = np.array([1.4e5, 3.4e4])


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    csrc = ROOT / "litepgo_b200" / "csrc"
    out = tmp_path_factory.mktemp("tetplan") / "libtetplan.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", str(csrc), "-I", "/usr/local/cuda/include",
                    str(ROOT / "tests" / "tet_assembly_host.cpp"), str(csrc / "lpg_plan.cpp"), "-o", str(out)],
                   check=True)
    lib = ctypes.CDLL(str(out))
    lib.tet_assemble.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _ip, _dp, _dp, ctypes.c_int, _dp, _dp, _dp,
                                 ctypes.c_char_p, ctypes.c_int]

    def run(X, tets, theta, u, nnz, layout):
        X = np.ascontiguousarray(X, np.float64)
        tets = np.ascontiguousarray(tets, np.int32)
        theta = np.ascontiguousarray(np.broadcast_to(theta, (tets.shape[0], 2)), np.float64)
        u = np.ascontiguousarray(u, np.float64)
        E, g, vals = ctypes.c_double(), np.full(u.size, np.nan), np.full(nnz, np.nan)
        err = ctypes.create_string_buffer(256)
        rc = lib.tet_assemble(X.shape[0], X.ctypes.data_as(_dp), tets.shape[0], tets.ctypes.data_as(_ip),
                              theta.ctypes.data_as(_dp), u.ctypes.data_as(_dp), layout, ctypes.byref(E),
                              g.ctypes.data_as(_dp), vals.ctypes.data_as(_dp), err, 256)
        assert rc == 0, err.value.decode()
        return E.value, g, vals

    return run


def deformed(X, seed, noise=0.01):
    rng = np.random.default_rng(seed)
    A = np.eye(3) + 0.05 * rng.standard_normal((3, 3))
    return (X @ A.T - X + noise * rng.standard_normal(X.shape)).ravel()


def check(host, X, tets, theta, u):
    orc = oracle.OracleMesh(X, tets, theta)
    Er, gr, vr = orc.eval(u, True, 1)
    E, g, vals = host(X, tets, theta, u, orc.nnz, 1)
    assert abs(E - Er) <= 1e-12 * abs(Er)
    assert rel_err(g, gr) <= 1e-12
    assert not np.isnan(vals).any()
    assert rel_err(vals, vr) <= 1e-12
    # BSR: the same values block by block; the matrix is bitwise symmetric.
    outer, inner = orc.pattern()
    _, _, bsr = host(X, tets, theta, u, orc.nnz, 0)
    Hc = sp.csc_matrix((vals, inner, outer), shape=(orc.num_dofs,) * 2)
    assert (Hc != Hc.T).nnz == 0
    assert np.array_equal(np.sort(bsr), np.sort(vals))


@pytest.mark.parametrize("n", [1, 3, 8, 14])
def test_box(host, n):
    """Boxes from one cube (a single cluster) to 14^3 (many clusters, boundary edges both ways)."""
    X, tets = mesh.make_box(n)
    check(host, X, tets, THETA, deformed(X, n, 0.03 / n))


def test_shuffled_numbering_and_per_element_theta(host):
    """A 6x5x7 box with randomly permuted vertices and elements: cluster rows are no longer
    contiguous and edge orientations flip; per-element theta."""
    X, tets = mesh.make_box(6, 5, 7)
    rng = np.random.default_rng(11)
    perm = rng.permutation(X.shape[0])
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    X, tets = X[perm], inv[tets][rng.permutation(tets.shape[0])]
    theta = np.stack([rng.uniform(5e4, 2e5, tets.shape[0]), rng.uniform(1e4, 5e4, tets.shape[0])], 1)
    check(host, X, tets, theta, deformed(X, 3, 0.01))


def test_delaunay_ball(host):
    X, tets = mesh.delaunay_ball(1500, seed=9)
    check(host, X, tets, THETA, deformed(X, 4, 1e-5))


def test_corner_chain_full_clusters(host):
    """Clusters of 64 owned rows (the limit): the diagonal items are summed by lane pairs there
    and by lane quads in the smaller clusters."""
    X, tets = corner_chain(200)
    check(host, X, tets, THETA, deformed(X, 6, 0.01))


def test_bunny_asset(host):
    d = np.load(ROOT / "tests" / "golden" / "assets.npz")
    X, tets = d["bunny_tet_X"], d["bunny_tet_cells"]
    h = np.cbrt(np.abs(np.linalg.det(X[tets[:, 1:]] - X[tets[:, :1]])).mean())
    check(host, X, tets, THETA, deformed(X, 5, 0.02 * h))
