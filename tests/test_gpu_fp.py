"""The plastic field on the GPU path: lpg_fem_set_fp, the Fp force sensitivity
(VolumetricFemForceFpResponse, tests/python/test_fp_force_response.py of the reference) and the
equilibrium adjoint in Fp, against the oracle and finite differences."""

import numpy as np
import pytest

import oracle
from conftest import rel_err
from litepgo_b200 import dof, energy, fem, mesh, solver, workloads

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

Exact, Projected = energy.HessianKind.Exact, energy.HessianKind.Projected


def plastic_field(T, seed, scale=0.08):
    rng = np.random.default_rng(seed)
    return np.stack([(np.eye(3) + scale * rng.standard_normal((3, 3))).T.ravel() for _ in range(T)])


@pytest.fixture(scope="module")
def box():
    w = workloads.deformed_box(5, seed=4)
    Fp = plastic_field(w["tets"].shape[0], 7)
    return w, Fp


def test_set_fp_equals_a_handle_built_with_fp(box):
    w, Fp = box
    built = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"], Fp=Fp)
    later = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    plain = later.eval(w["u"], gradient=True, hessian=Exact)
    later.set_fp(Fp)
    for prec in ("f64", "mixed"):
        a = built.eval(w["u"], gradient=True, hessian=Exact, precision=prec)
        b = later.eval(w["u"], gradient=True, hessian=Exact, precision=prec)
        assert a[0] == b[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[2].data, b[2].data)
    orc = oracle.OracleMesh(w["X"], w["tets"], w["theta"], Fp=Fp)
    E, g, H = later.eval(w["u"], gradient=True, hessian=Exact)
    Er, gr, vr = orc.eval(w["u"], True, 1)
    assert abs(E - Er) <= 1e-12 * abs(Er) and rel_err(g, gr) <= 1e-12 and rel_err(H.data, vr) <= 1e-12
    later.set_fp(None)
    back = later.eval(w["u"], gradient=True, hessian=Exact)
    assert back[0] == plain[0] and np.array_equal(back[1], plain[1]) and np.array_equal(back[2].data, plain[2].data)
    with pytest.raises(ValueError):
        later.set_fp(np.zeros(9))  # det Fp = 0
    with pytest.raises(ValueError):
        later.set_fp(np.full(9, np.nan))


@pytest.mark.parametrize("per_element", [True, False])
def test_fp_vjp_matches_oracle(box, per_element):
    w, Fp = box
    topo = mesh.TetTopology(w["X"].shape[0], w["tets"])
    vm = dof.VertexDofMap(topo, 3)
    T = w["tets"].shape[0]
    pmap = dof.ElementDofMap(topo, 9) if per_element else dof.ConstantDofMap(topo, 9)
    p = Fp.ravel() if per_element else Fp[0]
    Fp_all = Fp if per_element else np.tile(Fp[0], (T, 1))
    resp = fem.VolumetricFemForceFpResponse[fem.NeoHookean, fem.TetP1Basis, fem.TetCentroidQuadrature](
        pmap, vm, w["X"], w["u"], w["theta"])
    wv = np.random.default_rng(8).standard_normal(w["X"].size)
    got = resp.eval_vjp(p, wv)
    ref = oracle.OracleMesh(w["X"], w["tets"], w["theta"], Fp=Fp_all).force_vjp_fp(w["u"], wv)
    ref = ref.ravel() if per_element else ref.sum(0)
    assert rel_err(got, ref) <= 1e-12
    # The value is the energy gradient with that Fp (test_fp_force_energy_jacobian_and_recovery).
    gr = oracle.OracleMesh(w["X"], w["tets"], w["theta"], Fp=Fp_all).eval(w["u"], True, 0)[1]
    assert rel_err(resp.eval_value(p), gr) <= 1e-12


def test_fp_vjp_matches_finite_differences_of_the_gpu_force(box):
    w, Fp = box
    topo = mesh.TetTopology(w["X"].shape[0], w["tets"])
    resp = fem.VolumetricFemForceFpResponseTetP1(dof.ElementDofMap(topo, 9), dof.VertexDofMap(topo, 3), w["X"],
                                                 w["u"], w["theta"])
    rng = np.random.default_rng(9)
    wv = rng.standard_normal(w["X"].size)
    p = Fp.ravel()
    vjp = resp.eval_vjp(p, wv)
    for _ in range(4):
        d = rng.standard_normal(p.size)
        h = 1e-6
        fd = wv @ (resp.eval_value(p + h * d) - resp.eval_value(p - h * d)) / (2 * h)
        assert abs(vjp @ d - fd) <= 1e-7 * abs(fd) + 1e-9 * np.abs(vjp).sum()
    # A shared Fp is the sum of the per-element blocks (the reference's ConstantDofMap check).
    shared = fem.VolumetricFemForceFpResponseTetP1(dof.ConstantDofMap(topo, 9), dof.VertexDofMap(topo, 3), w["X"],
                                                   w["u"], w["theta"])
    rep = np.tile(Fp[0], w["tets"].shape[0])
    np.testing.assert_allclose(shared.eval_vjp(Fp[0], wv), resp.eval_vjp(rep, wv).reshape(-1, 9).sum(0),
                               rtol=1e-12, atol=1e-12 * np.abs(vjp).max())


def test_equilibrium_adjoint_in_fp_matches_finite_differences():
    g = workloads.gravity_box(3, seed=2)
    X, tets = g["X"], g["tets"]
    T, n = tets.shape[0], X.size
    topo = mesh.TetTopology(X.shape[0], tets)
    vm = dof.VertexDofMap(topo, 3)
    fixed = dof.DofReduction(n, g["fixed"])
    load = energy.QuadraticEnergy(np.zeros((n, n)), -g["f"])
    opts = solver.NewtonOptions(gradient_tolerance=1e-12, stop_rule="relative", accept_rule="armijo",
                                max_iterations=100, cg_tolerance=1e-3, exact_below=1e-3)
    Energy = fem.VolumetricFemEnergy[fem.NeoHookean, fem.TetP1Basis, fem.TetCentroidQuadrature]
    Force = fem.VolumetricFemForceFpResponse[fem.NeoHookean, fem.TetP1Basis, fem.TetCentroidQuadrature]

    def make_energy(p):
        return energy.WeightedSumEnergy([(Energy(vm, X, p.reshape(-1, 9), g["theta"]), 1.0), (load, 1.0)])

    def make_response(u):
        return Force(dof.ElementDofMap(topo, 9), vm, X, u, g["theta"])

    eq = solver.StaticEquilibriumResponse(9 * T, fixed, g["u0"], opts, make_energy, make_response)
    p0 = plastic_field(T, 3, scale=0.03).ravel()
    rng = np.random.default_rng(5)
    x_t = eq.eval_value(p0) + 0.01 * rng.standard_normal(n)
    loss = lambda p: float(np.sum((eq.eval_value(p) - x_t) ** 2))  # noqa: E731
    grad = eq.eval_vjp(p0, 2 * (eq.eval_value(p0) - x_t))
    for _ in range(2):
        d = rng.standard_normal(p0.size) * 0.05
        h = 1e-4
        fd = (8 * (loss(p0 + h * d) - loss(p0 - h * d)) - (loss(p0 + 2 * h * d) - loss(p0 - 2 * h * d))) / (12 * h)
        assert abs(grad @ d - fd) <= 1e-6 * abs(fd) + 1e-12
