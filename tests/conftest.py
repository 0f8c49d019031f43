import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a); run with -m gpu")


def rotation(angle, axis):
    """Rotation matrix of `angle` about `axis` (Rodrigues)."""
    a = np.asarray(axis, dtype=float)
    a = a / np.linalg.norm(a)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(angle) * K + (1 - np.cos(angle)) * K @ K


def colmajor(m):
    """Column-major vec of a 3x3 (index i + 3 j), the reference's Eigen layout."""
    return np.asarray(m, dtype=float).T.ravel()


# The reference's two-tet fixture (tests/cpp/fem/assembly/volumetric_fem_energy_tet_p1_gtest.cpp:26-49):
# two positively oriented tets sharing a face, volumes 1/6 and 1/3, theta = [2, 3], Fp = I.
TWO_TET_X = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.3, 0.2, -2]], dtype=float)
TWO_TET_CELLS = np.array([[0, 1, 2, 3], [0, 2, 1, 4]], dtype=np.int32)
TWO_TET_THETA = np.array([2.0, 3.0])


@pytest.fixture
def two_tet():
    return TWO_TET_X.copy(), TWO_TET_CELLS.copy(), TWO_TET_THETA.copy()


def two_tet_states():
    """States u in {0, 0.1 X, 0.1 X + 0.02 sin(j + 0.3)} of the reference FD test (:55-62)."""
    X = TWO_TET_X.ravel()
    out = []
    for state in (0, 1, 2):
        x = 0.1 * X
        if state == 0:
            x = np.zeros_like(X)
        if state == 2:
            x = x + 0.02 * np.sin(np.arange(X.size) + 0.3)
        out.append(x)
    return out


def rel_err(a, b):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    scale = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(a - b)) / scale)


def corner_chain(k):
    """k tets in a chain sharing only corner vertices: tet i = (a_i, b_i, c_i, a_i+1). Every vertex
    has 4 or 7 Hessian blocks in its row, so the tet assembly's clusters reach their 64-row limit
    (the diagonal items then fall back from four lanes to two)."""
    a = np.stack([2.0 * np.arange(k + 1), np.zeros(k + 1), np.zeros(k + 1)], 1)
    i = np.arange(k)
    b = np.stack([2.0 * i + 1, np.ones(k), np.zeros(k)], 1)
    c = np.stack([2.0 * i + 1, np.full(k, 0.5), np.full(k, 0.9)], 1)
    X = np.concatenate([a, b, c])
    tets = np.stack([i, k + 1 + i, 2 * k + 1 + i, i + 1], 1).astype(np.int32)
    neg = np.linalg.det(X[tets[:, 1:]] - X[tets[:, :1]]) < 0
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()
    return X, tets
