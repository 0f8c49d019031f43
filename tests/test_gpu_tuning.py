"""The autotuner: every launch variant it can choose computes bitwise the same results.

The Exact-Hessian assembly, the PCG SpMV and the eigenvalue clamp each come in variants that
differ in register budget and unrolling only. The handle times them at creation and keeps the
fastest; forcing each variant in turn must not change one bit of an evaluation or of a
Newton solve (which runs the projected Hessian's clamp, the PCG SpMV and the assembly).
"""

import itertools
import math

import numpy as np
import pytest
import scipy.sparse as sp

from litepgo_b200 import _native as N
from litepgo_b200 import dof, energy, fem, solver, workloads

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

Exact, Projected = energy.HessianKind.Exact, energy.HessianKind.Projected
VARIANTS = {"assembly_f64": 3, "assembly_f32": 3, "spmv_f64": 3, "spmv_f32": 3, "clamp_f64": 1, "clamp_f32": 2}


def test_tuning_report_is_complete():
    w = workloads.deformed_box(6, seed=1)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    t = e.tuning()
    for key, n in VARIANTS.items():
        assert 0 <= t["choice"][key] < n
        ms = t["ms"][key]
        assert len(ms) == 3 and all(math.isnan(v) for v in ms[n:])
        if n == 1:  # nothing to choose, nothing timed
            assert t["choice"][key] == 0 and math.isnan(ms[0])
            continue
        timed = ms[:n]
        assert all(math.isfinite(v) and v > 0 for v in timed), (key, ms)
        assert t["choice"][key] == int(np.argmin(timed))
    t2 = e.autotune()
    assert set(t2["choice"]) == set(VARIANTS)
    with pytest.raises(ValueError):
        e.set_tuning(spmv_f32=3)
    with pytest.raises(ValueError):
        e.set_tuning(clamp_f64=1)


def _evals(e, u):
    out = []
    for prec in ("f64", "mixed"):
        for hk in (Exact, Projected):
            E, g, H = e.eval(u, gradient=True, hessian=hk, precision=prec)
            out.append((E, g.copy(), H.data.copy()))
    return out


def test_assembly_and_clamp_variants_are_bitwise_identical():
    w = workloads.deformed_box(8, seed=3)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    u = w["u"]  # deformed: part of the elements need the clamp
    ref = None
    for a64, a32, c32 in itertools.product(range(3), range(3), range(2)):
        e.set_tuning(assembly_f64=a64, assembly_f32=a32, clamp_f32=c32)
        got = _evals(e, u)
        if ref is None:
            ref = got
            continue
        for (E0, g0, H0), (E1, g1, H1) in zip(ref, got):
            assert E0 == E1 and np.array_equal(g0, g1) and np.array_equal(H0, H1)


@pytest.mark.parametrize("precision", ["mixed", "f64"])
def test_newton_is_bitwise_identical_across_spmv_and_clamp_variants(precision):
    g = workloads.gravity_box(6, seed=0)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(g["X"], g["tets"], g["theta"])
    n = g["X"].size
    total = energy.WeightedSumEnergy([(e, 1.0), (energy.QuadraticEnergy(sp.csc_matrix((n, n)), -g["f"]), 1.0)])
    fixed = dof.DofReduction(n, g["fixed"])
    opts = solver.NewtonOptions(gradient_tolerance=1e-8, stop_rule="relative", accept_rule="armijo",
                                precision=precision, max_iterations=50, cg_tolerance=1e-2)
    x0 = np.zeros(n)
    ref = None
    key = "f64" if precision == "f64" else "f32"
    for sv, cv in itertools.product(range(3), range(VARIANTS["clamp_" + key])):
        e.set_tuning(**{"spmv_" + key: sv, "clamp_" + key: cv})
        r = solver.newton_solve(total, fixed, x0, opts)
        x = np.asarray(r.x.cpu() if hasattr(r.x, "cpu") else r.x)
        if ref is None:
            ref = (x, r.iterations, int(r.cg_iterations))
            assert r.status.name == "Converged"
            continue
        assert np.array_equal(x, ref[0]) and r.iterations == ref[1] and int(r.cg_iterations) == ref[2]
