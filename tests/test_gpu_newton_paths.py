"""Newton's other paths on the GPU (the reference's newton_gtest.cpp cases that a mesh energy can
reach), its per-iteration records, weighted-sum potentials, and the error statuses of the
solver entry points. Every failure is made on the host: options, loads and states, never a
fault.

- iteration limit (ReportsTheIterationLimit): status MaxIterations, x unchanged, one record;
- cg_max_iterations bounds every PCG solve of the step records;
- diagonal shifts on an indefinite Exact Hessian: a start where the direct solve's direction
  is an ascent direction (its gradient along the most negative curvature direction); the GPU's
  PCG takes the reference's shift loop like the oracle's PCG restatement does, step by step;
- a free vertex in no element (a zero Jacobi pivot): finite, converged, the vertex unchanged;
- a weighted-sum potential (elastic weight 2.5, a quadratic penalty along mesh edges, a load and
  a constant) against the oracle's Newton over the same sum;
- a quadratic term outside the elastic pattern, and an exception raised by on_iteration;
- the adjoint of an indefinite stiffness: LPG_EDOMAIN, not a wrong gradient;
- two threads on one handle: LPG_EBUSY (the reference's BusyScope).
"""

import threading

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from conftest import rel_err
from litepgo_b200 import _native as N
from litepgo_b200 import dof, energy, fem, mesh, solver, workloads

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def gravity(n=2):
    g = workloads.gravity_box(n, seed=0)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(g["X"], g["tets"], g["theta"])
    N_ = g["X"].size
    load = energy.QuadraticEnergy(sp.csc_matrix((N_, N_)), -g["f"])
    return g, e, energy.WeightedSumEnergy([(e, 1.0), (load, 1.0)])


def test_iteration_limit_reports_one_step():
    g, e, total = gravity()
    n = g["X"].size
    x0 = np.zeros(n)
    steps = []
    r = solver.newton_solve(total, dof.DofReduction(n, g["fixed"]), x0,
                            solver.NewtonOptions(gradient_tolerance=1e-10, max_iterations=0), on_iteration=steps.append)
    assert r.status == solver.NewtonStatus.MaxIterations and r.iterations == 0
    assert np.array_equal(r.x, x0)
    assert len(steps) == 1 and steps[0].iteration == 0 and steps[0].step == 0.0 and steps[0].pattern_changed
    Er = oracle.OracleMesh(g["X"], g["tets"], g["theta"]).eval(x0, False, 0)[0]
    assert abs(steps[0].energy - Er) <= 1e-12 * max(abs(Er), 1.0)


def test_cg_max_iterations_bounds_every_solve():
    g, e, total = gravity(3)
    n = g["X"].size
    steps = []
    opts = solver.NewtonOptions(gradient_tolerance=1e-12, stop_rule="relative", max_iterations=3, cg_max_iterations=2,
                                cg_tolerance=1e-12)
    r = solver.newton_solve(total, dof.DofReduction(n, g["fixed"]), np.zeros(n), opts, on_iteration=steps.append)
    assert r.status == solver.NewtonStatus.MaxIterations and r.iterations == 3
    assert len(steps) == 4
    for s in steps[:-1]:
        assert 0 < s.cg_iterations <= 2 * (s.diagonal_shifts + 1)
    assert r.cg_iterations == sum(s.cg_iterations for s in steps)
    assert all(np.isfinite(s.energy) for s in steps)


def indefinite_start():
    """lambda = 10, mu = 1, u = 0.5 X (det F = 3.375): the Exact Hessian has negative
    eigenvalues; the load makes the free gradient at u0 0.1 times the most negative curvature
    direction, so the direct solve's Newton direction is an ascent direction there."""
    X, tets = mesh.make_box(2)
    n = X.size
    bottom = np.flatnonzero(X[:, 2] == 0)
    fixed = (3 * bottom[:, None] + np.arange(3)).ravel().astype(np.int32)
    free = np.setdiff1d(np.arange(n), fixed)
    theta = np.array([10.0, 1.0])
    orc = oracle.OracleMesh(X, tets, theta)
    u0 = 0.5 * X.ravel()
    _, g0, _ = orc.eval(u0, True, 0)
    K = orc.hessian_csc(u0, kind=1).toarray()[np.ix_(free, free)]
    w, V = np.linalg.eigh(K)
    assert w[0] < 0
    v = np.zeros(n)
    v[free] = V[:, 0]
    return X, tets, theta, fixed, u0, g0 - 0.1 * v, orc


def test_indefinite_exact_hessian_shift_loop_matches_the_oracle_pcg():
    X, tets, theta, fixed, u0, f, orc = indefinite_start()
    n = X.size
    e = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta)
    total = energy.WeightedSumEnergy([(e, 1.0), (energy.QuadraticEnergy(sp.csc_matrix((n, n)), -f), 1.0)])
    steps = []
    opts = solver.NewtonOptions(gradient_tolerance=1e-9, stop_rule="relative", hessian=energy.HessianKind.Exact,
                                cg_tolerance=1e-12)
    r = solver.newton_solve(total, dof.DofReduction(n, fixed), u0, opts, on_iteration=steps.append)
    xo, info = orc.newton(fixed, u0, f_ext=f, tol=1e-9, stop_rule=1, hessian=1, linear_solver=1, cg_tolerance=1e-12,
                          trace=True)
    xd, infod = orc.newton(fixed, u0, f_ext=f, tol=1e-9, stop_rule=1, hessian=1, linear_solver=0, trace=True)
    assert infod["trace"][0]["diagonal_shifts"] > 0  # the direct solve needs the shifts here
    assert r.status == solver.NewtonStatus.Converged and info["status"] == 0
    assert steps[0].diagonal_shifts == int(info["trace"][0]["diagonal_shifts"])
    assert rel_err(r.x, xo) <= 1e-6
    # The direct solve's shifted first steps (9, 9, 8, 7 shifts) lead this non-convex energy to
    # another equilibrium, of higher energy (-14.89 against -17.37).
    assert infod["status"] == 0 and infod["energy"] > r.energy + 1.0


def test_free_vertex_in_no_element_is_a_zero_pivot():
    g = workloads.gravity_box(2, seed=0)
    X = np.vstack([g["X"], [[2.0, 2.0, 2.0]]])  # one vertex no element references
    n = X.size
    e = fem.VolumetricFemEnergyTetP1.from_arrays(X, g["tets"], g["theta"])
    f = np.concatenate([g["f"], np.zeros(3)])
    total = energy.WeightedSumEnergy([(e, 1.0), (energy.QuadraticEnergy(sp.csc_matrix((n, n)), -f), 1.0)])
    x0 = np.zeros(n)
    x0[-3:] = [0.1, -0.2, 0.3]
    r = solver.newton_solve(total, dof.DofReduction(n, g["fixed"]), x0,
                            solver.NewtonOptions(gradient_tolerance=1e-10, stop_rule="relative"))
    assert r.status == solver.NewtonStatus.Converged and np.all(np.isfinite(r.x))
    assert np.array_equal(r.x[-3:], x0[-3:])
    orc = oracle.OracleMesh(g["X"], g["tets"], g["theta"])
    xo, info = orc.newton(g["fixed"], np.zeros(g["X"].size), f_ext=g["f"], tol=1e-10, stop_rule=1)
    assert rel_err(r.x[:-3], xo) <= 1e-7


def edge_penalty(X, tets, k):
    """k/2 sum over mesh edges of |x_i - x_j|^2: A = k (L kron I3) with L the edge graph Laplacian."""
    V = X.shape[0]
    pairs = set()
    for t in tets:
        for a in range(4):
            for b in range(a + 1, 4):
                pairs.add((min(t[a], t[b]), max(t[a], t[b])))
    i, j = np.array(sorted(pairs)).T
    L = sp.coo_matrix((np.ones(i.size), (i, j)), shape=(V, V))
    L = L + L.T
    L = sp.diags(np.asarray(L.sum(axis=1)).ravel()) - L
    return k * sp.kron(L, sp.eye(3)).tocsr()


def test_weighted_sum_potential_against_the_oracle():
    g = workloads.gravity_box(3, seed=0)
    X, tets, theta, fixed, f = g["X"], g["tets"], g["theta"], g["fixed"], g["f"]
    n = X.size
    A = edge_penalty(X, tets, 50.0)
    b = -3.0 * f
    e = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta)
    total = energy.WeightedSumEnergy([(e, 2.5), (energy.QuadraticEnergy(A, b), 1.0),
                                      (energy.QuadraticEnergy(sp.csc_matrix((n, n)), -f), 2.0)])
    steps = []
    x0 = np.zeros(n)
    opts = solver.NewtonOptions(gradient_tolerance=1e-10, stop_rule="relative", cg_tolerance=1e-12)
    r = solver.newton_solve(total, dof.DofReduction(n, fixed), x0, opts, on_iteration=steps.append)
    assert r.status == solver.NewtonStatus.Converged, r
    orc = oracle.OracleMesh(X, tets, theta)
    xo, info = orc.newton(fixed, x0, f_ext=-(b - 2.0 * f), tol=1e-10, stop_rule=1, elastic_weight=2.5, A=A, trace=True)
    assert info["status"] == 0
    assert rel_err(r.x, xo) <= 1e-8
    assert abs(r.energy - info["energy"]) <= 1e-10 * abs(info["energy"])
    assert len(steps) == len(info["trace"])
    # The potential's own host evaluation agrees with the solver's energy.
    assert abs(total.eval_value(r.x) - r.energy) <= 1e-10 * abs(r.energy)


def test_quadratic_outside_the_pattern_and_callback_errors():
    g, e, total = gravity(2)
    n = g["X"].size
    far = sp.csr_matrix(([1.0, 1.0], ([0, n - 1], [n - 1, 0])), shape=(n, n))  # vertices 0 and V-1 share no element
    bad = energy.WeightedSumEnergy([(e, 1.0), (energy.QuadraticEnergy(far), 1.0)])
    opts = solver.NewtonOptions(gradient_tolerance=1e-10)
    with pytest.raises(ValueError, match="pattern"):
        solver.newton_solve(bad, dof.DofReduction(n, g["fixed"]), np.zeros(n), opts)

    class Stop(Exception):
        pass

    def stop_at_one(step):
        if step.iteration == 1:
            raise Stop("stop here")

    with pytest.raises(Stop):
        solver.newton_solve(total, dof.DofReduction(n, g["fixed"]), np.zeros(n), opts, on_iteration=stop_at_one)
    # The handle stays usable: the same solve on it and on a fresh handle gives the same result,
    # bit for bit (the solve is deterministic, so any state the aborted solve left behind would
    # show). The 1e-10 max-abs test sits at this box's round-off floor (element energies ~1e3
    # summing to |E| ~ 190 under the 16 eps accept rule), so only a loose bound is asserted on
    # the gradient itself.
    r = solver.newton_solve(total, dof.DofReduction(n, g["fixed"]), np.zeros(n), opts)
    _, _, fresh = gravity(2)
    r2 = solver.newton_solve(fresh, dof.DofReduction(n, g["fixed"]), np.zeros(n), opts)
    assert (r.status, r.iterations, r.cg_iterations) == (r2.status, r2.iterations, r2.cg_iterations)
    assert r.energy == r2.energy and np.array_equal(r.x, r2.x)
    assert r.gradient_norm <= 1e-6


def test_adjoint_of_an_indefinite_stiffness_is_a_domain_error():
    X, tets, theta, fixed, u0, f, orc = indefinite_start()
    e = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta)
    n = X.size
    out = np.empty(2)
    w = np.random.default_rng(0).standard_normal(n)
    code = N.lib.lpg_adjoint_theta(e.handle, N.vptr(np.ascontiguousarray(u0)), N.vptr(w), N.iptr(fixed),
                                   int(fixed.size), N.MEM_HOST, N.PRECISION_F64, 1e-10, 0, N.vptr(out), None)
    assert code == N.LPG_EDOMAIN, N.error_message()
    assert "indefinite" in N.error_message() or "singular" in N.error_message()
    # The oracle's PCG restatement rejects the same system with the same error class (its direct
    # solve, like the reference's LDL^T, factors the indefinite matrix).
    with pytest.raises(oracle.OracleError) as err:
        orc.adjoint_theta(u0, w, fixed, linear_solver=1, cg_tolerance=1e-10)
    assert err.value.code == oracle.DOMAIN_ERROR


def test_two_threads_on_one_handle_get_busy():
    import time

    g = workloads.gravity_box(48, seed=0)
    n = g["X"].size
    e = fem.VolumetricFemEnergyTetP1.from_arrays(g["X"], g["tets"], g["theta"])
    total = energy.WeightedSumEnergy([(e, 1.0), (energy.QuadraticEnergy(sp.csc_matrix((n, n)), -g["f"]), 1.0)])
    opts = solver.NewtonOptions(gradient_tolerance=1e-10, stop_rule="relative", cg_tolerance=1e-4)
    done = threading.Event()
    errors = []

    def solve():
        try:
            solver.newton_solve(total, dof.DofReduction(n, g["fixed"]), np.zeros(n), opts)
        except Exception as exc:  # noqa: BLE001
            errors.append(exc)
        finally:
            done.set()

    th = threading.Thread(target=solve)
    th.start()
    time.sleep(0.3)  # let the solve take the handle first
    busy = 0
    u = np.zeros(n)
    while not done.is_set():
        try:
            e.eval_value(u)
        except N.LitepgoError as exc:
            assert "in use" in str(exc)
            busy += 1
    th.join()
    assert not errors and busy > 0
    assert np.isfinite(e.eval_value(u))  # free again
