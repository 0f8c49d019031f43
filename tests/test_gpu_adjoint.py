"""Torch bridge on the GPU path and the adjoint sensitivities.

- litepgo_b200.torch.energy on CPU and CUDA tensors against Energy.eval (bitwise);
- set_theta against a freshly built energy (bitwise);
- the rest-position force VJP against the oracle (1e-12 relative) and the rest-position
  adjoint against central finite differences;
- the per-element Lame adjoint of a 32^3 box through torch.autograd against central finite
  differences along 20 seeded directions (steps relative to theta): 1e-6 relative at step
  1e-4, and within the solves' round-off noise at step 1e-6; and against the oracle's
  equilibrium gradient at the same equilibrium (1e-7 max-norm relative).
"""

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from conftest import TWO_TET_CELLS, TWO_TET_THETA, TWO_TET_X, two_tet_states
from litepgo_b200 import dof, energy, fem, mesh, solver, workloads

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
from litepgo_b200 import torch as bridge  # noqa: E402


def _fem(X, tets, theta):
    return fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta)


def test_torch_energy_matches_eval_on_cpu_and_cuda():
    w = workloads.deformed_box(4, seed=2)
    e = _fem(w["X"], w["tets"], w["theta"])
    E, g, _ = e.eval(w["u"], gradient=True)
    for device in ("cpu", "cuda"):
        x = torch.tensor(w["u"], dtype=torch.float64, device=device, requires_grad=True)
        value = bridge.energy(e, x)
        assert value.device.type == device and value.item() == E
        value.backward()
        assert np.array_equal(x.grad.cpu().numpy(), g)


@pytest.mark.parametrize("device", ["cpu", "cuda"])
def test_torch_energy_gradcheck_two_tet(device):
    e = _fem(TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA)
    x = torch.tensor(two_tet_states()[2], dtype=torch.float64, device=device, requires_grad=True)
    assert torch.autograd.gradcheck(lambda x: bridge.energy(e, x), (x,), eps=1e-6, atol=1e-8, rtol=1e-6)


def test_torch_weighted_sum_energy_on_cuda():
    w = workloads.deformed_box(3, seed=5)
    e = _fem(w["X"], w["tets"], w["theta"])
    f = np.sin(np.arange(w["u"].size))
    total = energy.WeightedSumEnergy([(e, 1.0), (energy.QuadraticEnergy(sp.csc_matrix((f.size, f.size)), -f), 1.0)])
    x = torch.tensor(w["u"], dtype=torch.float64, device="cuda", requires_grad=True)
    value = bridge.energy(total, x)
    value.backward()
    E, g, _ = e.eval(w["u"], gradient=True)
    assert abs(value.item() - (E - f @ w["u"])) <= 1e-12 * abs(E)
    np.testing.assert_allclose(x.grad.cpu().numpy(), g - f, rtol=0, atol=1e-12 * np.abs(g).max())


def test_set_theta_matches_a_new_energy():
    w = workloads.deformed_box(4, seed=1)
    T = w["tets"].shape[0]
    th = np.column_stack([np.full(T, 1.2e5), 3e4 * (1 + 0.3 * np.random.default_rng(0).random(T))])
    e = _fem(w["X"], w["tets"], w["theta"])
    e.set_theta(th)
    E1, g1, H1 = e.eval(w["u"], gradient=True, hessian=energy.HessianKind.Exact)
    E2, g2, H2 = _fem(w["X"], w["tets"], th).eval(w["u"], gradient=True, hessian=energy.HessianKind.Exact)
    assert E1 == E2 and np.array_equal(g1, g2) and np.array_equal(H1.data, H2.data)
    with pytest.raises(ValueError):
        e.set_theta(np.ones(3))


def test_rest_position_vjp_parity():
    w = workloads.deformed_box(4, seed=3)
    T = w["tets"].shape[0]
    th = np.column_stack([np.full(T, 1.4e5), 3.4e4 * (1 + 0.5 * np.random.default_rng(1).random(T))])
    wv = np.random.default_rng(2).standard_normal(w["u"].size)
    topo = mesh.TetTopology(w["X"].shape[0], w["tets"])
    resp = fem.VolumetricFemForceRestPositionResponseTetP1(dof.VertexDofMap(topo, 3), w["u"], th)
    got = resp.eval_vjp(w["X"].ravel(), wv)
    ref = oracle.OracleMesh(w["X"], w["tets"], th).force_vjp_rest(w["u"], wv)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    plastic = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], th, Fp=np.diag([1.1, 1.0, 1.0]).ravel())
    from litepgo_b200 import _native as N

    with pytest.raises(ValueError, match="plastic"):
        N.check(N.lib.lpg_fem_force_vjp_rest(plastic.handle, N.vptr(w["u"]), N.vptr(wv), N.MEM_HOST,
                                             N.vptr(np.empty(w["u"].size))))


def _options():
    return solver.NewtonOptions(gradient_tolerance=1e-12, stop_rule="relative", accept_rule="noise",
                                max_iterations=100, cg_tolerance=1e-3)


def test_rest_position_adjoint_matches_finite_differences():
    g = workloads.gravity_box(4, seed=3)
    X, tets, theta, f, fixed = g["X"], g["tets"], g["theta"], g["f"], g["fixed"]
    n = X.size
    load = energy.QuadraticEnergy(sp.csc_matrix((n, n)), -f)
    topo = mesh.TetTopology(X.shape[0], tets)
    dmap = dof.VertexDofMap(topo, 3)
    model = solver.StaticEquilibriumResponse(
        n, dof.DofReduction(n, fixed), np.zeros(n), _options(),
        lambda p: energy.WeightedSumEnergy([(_fem(p.reshape(-1, 3), tets, theta), 1.0), (load, 1.0)]),
        lambda u: fem.VolumetricFemForceRestPositionResponseTetP1(dmap, u, theta))
    rng = np.random.default_rng(7)
    target = model.eval_value(X.ravel()) + 1e-3 * rng.standard_normal(n)
    p = torch.tensor(X.ravel(), dtype=torch.float64, requires_grad=True)
    loss = ((bridge.response(model, p) - torch.as_tensor(target)) ** 2).sum()
    loss.backward()
    grad = p.grad.numpy()
    h = 1e-6 / g["n"]

    def L(q):
        return float(np.sum((model.eval_value(q) - target) ** 2))

    for _ in range(3):
        d = rng.standard_normal(n)
        fd = (L(X.ravel() + h * d) - L(X.ravel() - h * d)) / (2 * h)
        assert abs(grad @ d - fd) <= 1e-6 * abs(fd)


def test_theta_adjoint_32cube_matches_finite_differences():
    """Per-element [lambda, mu] as a torch leaf, loss |x*(theta) - x_t|^2 (32^3 box)."""
    g = workloads.adjoint_box(32, seed=0)
    X, tets, fixed, f = g["X"], g["tets"], g["fixed"], g["f"]
    n, T = X.size, tets.shape[0]
    load = energy.QuadraticEnergy(sp.csc_matrix((n, n)), -f)
    shared = _fem(X, tets, g["theta"])
    topo = mesh.TetTopology(X.shape[0], tets)

    def make_energy(p):
        shared.set_theta(p.reshape(T, 2))
        return energy.WeightedSumEnergy([(shared, 1.0), (load, 1.0)])

    def make_response(u):
        return fem.VolumetricFemForceMaterialResponseTetP1(dof.ElementDofMap(topo, 2), dof.VertexDofMap(topo, 3), X, u,
                                                          np.eye(3).ravel())

    # Max-norm stop 1e-12 |f|_max, about 4x the round-off floor of the FP64 gradient: the
    # finite-difference solves start from x*(theta) and end at that floor, so the difference of
    # two solves is not swamped by their stopping residuals.
    opts = solver.NewtonOptions(gradient_tolerance=1e-12 * np.abs(f).max(), stop_rule="max_abs", accept_rule="noise",
                                max_iterations=100, cg_tolerance=1e-3)
    model = solver.StaticEquilibriumResponse(2 * T, dof.DofReduction(n, fixed), np.zeros(n), opts, make_energy,
                                             make_response)
    x_target = model.eval_value(g["target_theta"].ravel())
    theta = torch.tensor(g["theta"], dtype=torch.float64, requires_grad=True)
    loss = ((bridge.response(model, theta.reshape(-1)) - torch.as_tensor(x_target)) ** 2).sum()
    loss.backward()
    grad = theta.grad.numpy().ravel()
    th0 = g["theta"].ravel()
    warm = solver.StaticEquilibriumResponse(2 * T, dof.DofReduction(n, fixed), model.eval_value(th0), opts,
                                            make_energy, make_response)

    def L(q):
        return float(np.sum((warm.eval_value(q) - x_target) ** 2))

    # The difference of two equilibrium solves carries their FP64 round-off (the gradient's
    # floor, about 2.5e-13 |f|_max here), which divided by 2h dominates the central difference
    # at small steps: its error falls as 1/h (about 1e-4 at h = 1e-7, 1e-5 at 1e-6, 1e-6 at
    # 1e-5) down to 1e-7 at h = 1e-4. So the 1e-6 agreement is asserted at h = 1e-4 with the
    # fourth-order five-point difference (truncation O(h^4)), and the h = 1e-6 central
    # difference at its noise bound.
    rng = np.random.default_rng(20)
    errs = {1e-6: [], 1e-4: []}
    for _ in range(20):
        d = rng.standard_normal(2 * T) * th0
        h = 1e-6
        fd = (L(th0 + h * d) - L(th0 - h * d)) / (2 * h)
        errs[h].append(abs(grad @ d - fd) / abs(fd))
        h = 1e-4
        fd = (8 * (L(th0 + h * d) - L(th0 - h * d)) - (L(th0 + 2 * h * d) - L(th0 - 2 * h * d))) / (12 * h)
        errs[h].append(abs(grad @ d - fd) / abs(fd))
    print("adjoint vs central differences, max relative error per step:", {h: max(v) for h, v in errs.items()})
    assert max(errs[1e-4]) <= 1e-6, errs
    assert max(errs[1e-6]) <= 2e-4, errs
    # The reference's own equilibrium gradient (StaticEquilibriumResponse's adjoint,
    # static_equilibrium_response.cpp:43-88, restated by the oracle) at the same equilibrium
    # x*(theta0) with dL/du = 2 (x* - x_target): per-element [d/dlambda, d/dmu]. The oracle solves
    # K lambda = dL/du with its block-Jacobi PCG to 1e-12 (its envelope LDL^T does not fit 32^3).
    x_star = model.eval_value(th0)
    orc = oracle.OracleMesh(X, tets, g["theta"])
    dtheta, _ = orc.adjoint_theta(x_star, 2.0 * (x_star - x_target), fixed, linear_solver=1, cg_tolerance=1e-12)
    err = float(np.max(np.abs(grad - dtheta.ravel())) / np.max(np.abs(dtheta)))
    print("adjoint vs the oracle's equilibrium gradient at 32^3:", err)
    assert err <= 1e-7
