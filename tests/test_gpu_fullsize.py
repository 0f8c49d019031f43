"""The benchmarked 64^3-cube workload (1,310,720 tets) against the oracle, in full.

The mesh, Lamé field and state are those of the bench's evaluation step. Compared with the
oracle's assembly (the reference's EnergyAssembler restated):
  - the scalar CSC pattern, bit for bit;
  - E, the gradient and the Exact CSC Hessian in FP64 (max-norm relative 1e-12);
  - the Projected Hessian in FP64 (1e-11);
  - the mixed-precision results at their stated bounds;
  - the config-2 Newton equilibrium of both precisions, re-evaluated with the oracle's
    gradient (free relative residual <= 1.5e-8).
Size-independent properties (bitwise symmetry, derivatives against central differences of
the GPU's own energy) are kept beside them.
"""

import numpy as np
import pytest

import oracle
from conftest import rel_err
from litepgo_b200 import dof, energy, fem, mesh, solver, workloads

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


@pytest.fixture(scope="module")
def orc(big):
    X, tets, theta, _, _ = big
    return oracle.OracleMesh(X, tets, theta)


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


def test_fullsize_exact_against_oracle(big, orc):
    """Bench workload: pattern bit-exact, E, gradient and Exact Hessian to 1e-12 (FP64)."""
    X, tets, theta, u, e = big
    outer, inner = e.pattern_csc()
    o_outer, o_inner = orc.pattern()
    assert np.array_equal(outer, o_outer) and np.array_equal(inner, o_inner)
    ut = torch.as_tensor(u, device="cuda")
    E, g, Hc = e.eval_device(ut, gradient=True, hessian=energy.HessianKind.Exact, layout="csc")
    Er, gr, vr = orc.eval(u, True, 1)
    errs = {"energy": abs(E - Er) / abs(Er), "gradient": rel_err(g.cpu().numpy(), gr),
            "hessian": rel_err(Hc.cpu().numpy(), vr)}
    print("FP64 vs oracle at 64^3:", errs)
    assert errs["energy"] <= 1e-12 and errs["gradient"] <= 1e-12 and errs["hessian"] <= 1e-12


def test_fullsize_projected_against_oracle(big, orc):
    """Bench workload: Projected Hessian (per-element eigenvalue clamp) to 1e-11 (FP64)."""
    X, tets, theta, u, e = big
    ut = torch.as_tensor(u, device="cuda")
    _, _, Hc = e.eval_device(ut, gradient=False, hessian=energy.HessianKind.Projected, layout="csc")
    _, _, vr = orc.eval(u, False, 2)
    err = rel_err(Hc.cpu().numpy(), vr)
    print("FP64 projected vs oracle at 64^3:", err)
    assert err <= 1e-11


def test_fullsize_mixed_against_oracle(big, orc):
    """Mixed precision (FP32 element arithmetic and Hessian, FP64 energy sum and gradient
    output) at its stated bounds: energy 1e-6, gradient 1e-4, Exact Hessian 1e-5."""
    X, tets, theta, u, e = big
    ut = torch.as_tensor(u, device="cuda")
    E32, g32, H32 = e.eval_device(ut, gradient=True, hessian=energy.HessianKind.Exact, precision="mixed",
                                  layout="csc")
    Er, gr, vr = orc.eval(u, True, 1)
    errs = {"energy": abs(E32 - Er) / abs(Er), "gradient": rel_err(g32.cpu().numpy(), gr),
            "hessian": rel_err(H32.double().cpu().numpy(), vr)}
    print("mixed vs oracle at 64^3:", errs)
    assert errs["energy"] <= 1e-6 and errs["gradient"] <= 1e-4 and errs["hessian"] <= 1e-5


def test_fullsize_element_energies(big, orc):
    X, tets, theta, u, e = big
    _, _, _, (eEr, _, _) = orc.eval(u, False, 0, elements=True)
    assert rel_err(e.element_energies(u), eEr) <= 1e-12


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
    row_ptr, col_idx = e.pattern_bsr()
    import scipy.sparse as sp

    K = sp.bsr_matrix((Hb.cpu().numpy().reshape(-1, 3, 3), col_idx, row_ptr), shape=(e.num_dofs,) * 2)
    Kd = K @ d.cpu().numpy()
    fdg = ((Ep[1] - Em[1]) / (2 * h)).cpu().numpy()
    assert rel_err(Kd, fdg) <= 1e-6


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_fullsize_newton_equilibrium_against_oracle(precision):
    """Config 2: the gravity box Newton solve of the bench (relative gradient 1e-8, Armijo),
    its equilibrium re-evaluated with the oracle's gradient."""
    import scipy.sparse as sp

    g = workloads.gravity_box(64, seed=0)
    n = g["X"].size
    e = fem.VolumetricFemEnergyTetP1.from_arrays(g["X"], g["tets"], g["theta"])
    total = energy.WeightedSumEnergy([(e, 1.0), (energy.QuadraticEnergy(sp.csc_matrix((n, n)), -g["f"]), 1.0)])
    opts = solver.NewtonOptions(gradient_tolerance=1e-8, stop_rule="relative", accept_rule="armijo",
                                precision=precision, max_iterations=100, cg_tolerance=1e-2, cg_max_iterations=20000)
    x0 = torch.zeros(n, dtype=torch.float64, device="cuda")
    r = solver.newton_solve(total, dof.DofReduction(n, g["fixed"]), x0, opts)
    assert r.status == solver.NewtonStatus.Converged, r
    x = r.x.cpu().numpy() if hasattr(r.x, "cpu") else np.asarray(r.x)
    o = oracle.OracleMesh(g["X"], g["tets"], g["theta"])
    _, go, _ = o.eval(x, True, 0)
    free = np.setdiff1d(np.arange(n), g["fixed"])
    res = np.linalg.norm((go - g["f"])[free])
    print(f"{precision}: Newton {r.iterations} iterations, oracle residual {res / r.gradient_norm0:.3e} relative")
    assert res <= 1.5e-8 * r.gradient_norm0
    assert np.all(x[g["fixed"]] == 0.0)
