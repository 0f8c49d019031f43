"""Size-independent properties at the 64^3-cube workload size (1,310,720 tets).

At this size the oracle only checks per-element energies; the assembled results are
checked through properties: bitwise symmetry, gradient and Hessian-vector products against
central differences of the GPU energy/gradient, and FP32 against FP64.
"""

import numpy as np
import pytest

import oracle
from conftest import rel_err
from litepgo_b200 import energy, fem, mesh, workloads

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def big():
    n = 64
    X, tets = mesh.make_box(n)
    g = workloads.gravity_box(n, seed=0)
    rng = np.random.default_rng(11)
    A = np.eye(3) + 0.1 * rng.standard_normal((3, 3))
    u = (X @ A.T - X + 0.001 * rng.standard_normal(X.shape)).ravel()
    assert np.all(workloads.det_F(X, tets, u) > 0)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, g["theta"])
    return X, tets, g["theta"], u, e


def test_fullsize_counts_and_symmetry(big):
    X, tets, theta, u, e = big
    assert (e.num_vertices, e.num_elements, e.nnzb) == mesh.box_counts(64)
    ut = torch.as_tensor(u, device="cuda")
    _, _, Hc = e.eval_device(ut, gradient=False, hessian=energy.HessianKind.Exact, layout="csc")
    import scipy.sparse as sp

    outer, inner = e.pattern_csc()
    H = sp.csc_matrix((Hc.cpu().numpy(), inner, outer), shape=(e.num_dofs,) * 2)
    D = (H - H.T).tocsc()
    D.eliminate_zeros()
    assert D.nnz == 0


def test_fullsize_derivatives_against_differences(big):
    X, tets, theta, u, e = big
    ut = torch.as_tensor(u, device="cuda")
    E, g, Hb = e.eval_device(ut, gradient=True, hessian=energy.HessianKind.Exact)
    rng = np.random.default_rng(12)
    d = torch.as_tensor(1e-3 * rng.standard_normal(u.size), device="cuda")
    h = 1e-4
    Ep = e.eval_device(ut + h * d, gradient=True)
    Em = e.eval_device(ut - h * d, gradient=True)
    fd = (Ep[0] - Em[0]) / (2 * h)
    assert abs(fd - float(g @ d)) <= 1e-6 * abs(fd)
    # Hessian-vector product from the block-CSR values.
    row_ptr, col_idx = e.pattern_bsr()
    import scipy.sparse as sp

    K = sp.bsr_matrix((Hb.cpu().numpy().reshape(-1, 3, 3), col_idx, row_ptr), shape=(e.num_dofs,) * 2)
    Kd = K @ d.cpu().numpy()
    fdg = ((Ep[1] - Em[1]) / (2 * h)).cpu().numpy()
    assert rel_err(Kd, fdg) <= 1e-6


def test_fullsize_element_energies_and_mixed_precision(big):
    X, tets, theta, u, e = big
    orc = oracle.OracleMesh(X, tets, theta)
    _, _, _, (eEr, _, _) = orc.eval(u, False, 0, elements=True)
    assert rel_err(e.element_energies(u), eEr) <= 1e-12
    ut = torch.as_tensor(u, device="cuda")
    E64, g64, H64 = e.eval_device(ut, gradient=True, hessian=energy.HessianKind.Exact)
    E32, g32, H32 = e.eval_device(ut, gradient=True, hessian=energy.HessianKind.Exact, precision="mixed")
    assert abs(E32 - E64) <= 1e-5 * abs(E64)
    assert rel_err(g32.cpu().numpy(), g64.cpu().numpy()) <= 1e-4
    assert rel_err(H32.double().cpu().numpy(), H64.cpu().numpy()) <= 1e-5
