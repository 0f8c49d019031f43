"""Golden fixtures (tests/golden/, written by tests/golden/make_golden.py from the oracle).

CPU: the oracle still reproduces them (1e-14 relative: a regression pin of the oracle).
GPU: the CUDA path through the C ABI matches them (FP64: 1e-12 relative, max-norm; the
projected Hessian 1e-11, its eigenvalue clamp being an iterative method on both sides).
"""

from pathlib import Path

import numpy as np
import pytest

import oracle
from litepgo_b200 import energy, fem

GOLDEN = Path(__file__).resolve().parent / "golden"


def load(name):
    return dict(np.load(GOLDEN / name))


def probe(n):
    return np.sin(np.arange(n) + 0.5)


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)) if b.size else 0.0


@pytest.mark.parametrize("name", ["two_tet.npz", "box3.npz"])
def test_oracle_reproduces_full_fixtures(name):
    d = load(name)
    m = oracle.OracleMesh(d["X"], d["tets"], d["theta"])
    outer, inner = m.pattern()
    assert np.array_equal(outer, d["outer"]) and np.array_equal(inner, d["inner"])
    for k, u in enumerate(d["u"]):
        E, g, H1 = m.eval(u, True, 1)
        _, _, H2 = m.eval(u, False, 2)
        assert abs(E - d["E"][k]) <= 1e-14 * max(abs(d["E"][k]), 1e-300)
        assert rel(g, d["g"][k]) <= 1e-14
        assert rel(H1, d["H_exact"][k]) <= 1e-14
        assert rel(H2, d["H_projected"][k]) <= 1e-13


def test_oracle_reproduces_box10_fixture():
    from litepgo_b200 import workloads

    d = load("box10.npz")
    w = workloads.deformed_box(10, seed=0)
    assert int(d["seed"]) == w["seed"] and np.array_equal(d["u"], w["u"])
    m = oracle.OracleMesh(w["X"], w["tets"], w["theta"])
    E, g, H, (eE, _, _) = m.eval(w["u"], True, 1, elements=True)
    assert abs(E - d["E"]) <= 1e-14 * abs(d["E"])
    assert rel(g, d["g"]) <= 1e-14 and rel(eE, d["elem_E"]) <= 1e-14
    assert rel(m.hessian_csc(w["u"], 1) @ probe(w["u"].size), d["H_w"]) <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["two_tet.npz", "box3.npz"])
def test_gpu_matches_full_fixtures(name):
    d = load(name)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(d["X"], d["tets"], d["theta"])
    outer, inner = e.pattern_csc()
    assert np.array_equal(outer, d["outer"]) and np.array_equal(inner, d["inner"])
    for k, u in enumerate(d["u"]):
        E, g, H1 = e.eval(u, gradient=True, hessian=energy.HessianKind.Exact)
        _, _, H2 = e.eval(u, hessian=energy.HessianKind.Projected)
        assert abs(E - d["E"][k]) <= 1e-12 * max(abs(d["E"][k]), 1e-300)
        assert rel(g, d["g"][k]) <= 1e-12
        assert rel(H1.data, d["H_exact"][k]) <= 1e-12
        assert rel(H2.data, d["H_projected"][k]) <= 1e-11


@pytest.mark.gpu
def test_gpu_matches_box10_fixture():
    from litepgo_b200 import workloads

    d = load("box10.npz")
    w = workloads.deformed_box(10, seed=0)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    E, g, H = e.eval(w["u"], gradient=True, hessian=energy.HessianKind.Exact)
    assert abs(E - d["E"]) <= 1e-12 * abs(d["E"])
    assert rel(g, d["g"]) <= 1e-12
    assert rel(e.element_energies(w["u"]), d["elem_E"]) <= 1e-12
    assert rel(H @ probe(w["u"].size), d["H_w"]) <= 1e-12
    assert abs(np.sqrt(np.sum(H.data ** 2)) - d["H_fro"]) <= 1e-12 * d["H_fro"]
