"""Seeded synthetic workloads on structured five-tet boxes.

Every workload is generated from numpy.random.default_rng(seed); there is no dataset.

- deformed_box: n^3 cubes, uniform mu = 3.4e4, lambda = 1.4e5, deformed positions
  x = A X + 0.01 N(0, 1) with A = I + 0.1 N(0, 1) (3x3), u = x - X. Seeds whose state
  inverts an element (det F <= 0) are skipped; the seed used is returned.
- gravity_box: n^3 cubes, per-element mu log-uniform in [1e3, 1e5] and Poisson ratio
  nu ~ U[0.30, 0.45] (lambda = 2 mu nu / (1 - 2 nu)), bottom face z = 0 fixed,
  gravity (0, 0, -9.8) with density 1000 lumped as f_a = rho g vol_e / 4 (exact for P1).
- adjoint_box: n^3 cubes with per-element [lambda, mu] = [1.4e5, 3.4e4] (the parameters of
  an adjoint fit), bottom face fixed, gravity as above, and target parameters whose mu is
  perturbed to mu (1 + 0.2 N(0, 1)) (clipped below at 0.05 mu).
- batch_boxes: independent boxes with cube counts per axis drawn from U{4..24} (spacing 1/16),
  each with its own affine state A = I + 0.1 N(0, 1) (u0 = (A - I) X), uniform
  [lambda, mu] = [1.4e5, 3.4e4], its bottom face fixed at u0 and gravity as above; returned as
  one union (mesh.concatenate) with per-mesh offsets.
- compressed_box: 0.6x axial compression along z plus per-vertex noise 0.05 h N(0, 1)
  (h = 1/n), resampled until every element has det F in [0.2, 3.0].
"""

import numpy as np

from .mesh import make_box

__all__ = ["deformed_box", "gravity_box", "adjoint_box", "batch_boxes", "compressed_box", "lame", "gravity_load", "det_F"]


def lame(mu, nu):
    """(lambda, mu) from shear modulus and Poisson ratio."""
    return 2.0 * mu * nu / (1.0 - 2.0 * nu), mu


def det_F(X, tets, u):
    """det F per element for displacement u (V*3)."""
    U = np.asarray(u).reshape(-1, 3)
    Dm = np.stack([X[tets[:, c + 1]] - X[tets[:, 0]] for c in range(3)], axis=2)
    Ds = np.stack([(X + U)[tets[:, c + 1]] - (X + U)[tets[:, 0]] for c in range(3)], axis=2)
    return np.linalg.det(Ds) / np.linalg.det(Dm)


def element_volumes(X, tets):
    D = X[tets[:, 1:]] - X[tets[:, :1]]
    return np.einsum("ij,ij->i", D[:, 0], np.cross(D[:, 1], D[:, 2])) / 6.0


def gravity_load(X, tets, rho=1000.0, g=(0.0, 0.0, -9.8)):
    """Consistent P1 body-force vector f (V*3): f_a = sum_e rho g vol_e / 4."""
    vol = element_volumes(X, tets)
    f = np.zeros((X.shape[0], 3))
    for a in range(4):
        np.add.at(f, tets[:, a], np.outer(rho * vol / 4.0, np.asarray(g)))
    return f.ravel()


def deformed_box(n=10, seed=0, mu=3.4e4, lam=1.4e5):
    X, tets = make_box(n)
    s = seed
    while True:
        rng = np.random.default_rng(s)
        A = np.eye(3) + 0.1 * rng.standard_normal((3, 3))
        x = X @ A.T + 0.01 * rng.standard_normal(X.shape)
        u = (x - X).ravel()
        if np.all(det_F(X, tets, u) > 0):
            break
        s += 1
    theta = np.array([lam, mu])
    return dict(X=X, tets=tets, u=u, theta=theta, seed=s, n=n)


def gravity_box(n=64, seed=0, rho=1000.0):
    X, tets = make_box(n)
    rng = np.random.default_rng(seed)
    T = tets.shape[0]
    mu = np.exp(rng.uniform(np.log(1e3), np.log(1e5), T))
    nu = rng.uniform(0.30, 0.45, T)
    lam, mu = lame(mu, nu)
    theta = np.ascontiguousarray(np.stack([lam, mu], axis=1))
    bottom = np.flatnonzero(X[:, 2] == 0.0)
    fixed = (3 * bottom[:, None] + np.arange(3)).ravel().astype(np.int32)
    f = gravity_load(X, tets, rho)
    return dict(X=X, tets=tets, theta=theta, fixed=fixed, f=f, u0=np.zeros(X.size), seed=seed, n=n)


def adjoint_box(n=32, seed=0, mu=3.4e4, lam=1.4e5, rho=1000.0):
    X, tets = make_box(n)
    rng = np.random.default_rng(seed)
    T = tets.shape[0]
    theta = np.tile(np.array([lam, mu]), (T, 1))
    target = theta.copy()
    target[:, 1] = mu * np.maximum(1.0 + 0.2 * rng.standard_normal(T), 0.05)
    bottom = np.flatnonzero(X[:, 2] == 0.0)
    fixed = (3 * bottom[:, None] + np.arange(3)).ravel().astype(np.int32)
    return dict(X=X, tets=tets, theta=theta, target_theta=target, fixed=fixed, f=gravity_load(X, tets, rho),
                u0=np.zeros(X.size), seed=seed, n=n)


def batch_boxes(count=256, seed=0, lo=4, hi=24, mu=3.4e4, lam=1.4e5, rho=1000.0):
    from .mesh import concatenate

    rng = np.random.default_rng(seed)
    meshes, u0, fixed, f, dims = [], [], [], [], []
    base = 0
    for _ in range(count):
        nx, ny, nz = (int(v) for v in rng.integers(lo, hi + 1, 3))
        X, tets = make_box(nx, ny, nz, size=(nx / 16, ny / 16, nz / 16))
        A = np.eye(3) + 0.1 * rng.standard_normal((3, 3))
        meshes.append((X, tets))
        u0.append((X @ A.T - X).ravel())
        bottom = np.flatnonzero(X[:, 2] == 0.0)
        fixed.append(base * 3 + (3 * bottom[:, None] + np.arange(3)).ravel())
        f.append(gravity_load(X, tets, rho))
        dims.append((nx, ny, nz))
        base += X.shape[0]
    X, tets, voff, eoff = concatenate(meshes)
    return dict(X=X, tets=tets, vertex_offsets=voff, element_offsets=eoff, u0=np.concatenate(u0),
                fixed=np.concatenate(fixed).astype(np.int32), f=np.concatenate(f), theta=np.array([lam, mu]),
                dims=dims, seed=seed)


def compressed_box(n=128, seed=0, mu=3.4e4, lam=1.4e5):
    X, tets = make_box(n)
    h = 1.0 / n
    s = seed
    while True:
        rng = np.random.default_rng(s)
        x = X.copy()
        x[:, 2] *= 0.6
        x += 0.05 * h * rng.standard_normal(X.shape)
        u = (x - X).ravel()
        d = det_F(X, tets, u)
        if d.min() >= 0.2 and d.max() <= 3.0:
            break
        s += 1
    return dict(X=X, tets=tets, u=u, theta=np.array([lam, mu]), seed=s, n=n)
