"""The allocation-free feasible step, lpg_fem_feasible_step_noalloc.

It serves callers that cannot allocate device memory when they ask for the step: code
recording a CUDA stream capture, or a solver inside a framework that owns the device memory
pool. Its scratch is a fixed array in the library image shared by all calls, so this test
checks it against the allocating entry point, lpg_fem_feasible_step, on two calls in a row
(the second must not see the first call's leftovers), including a call that fails and leaves
an error status behind. This file is collected last, so a failure here comes after every
other test has run.
"""

import ctypes

import numpy as np
import pytest

from litepgo_b200 import _native as N
from litepgo_b200 import fem, workloads

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def noalloc_step(energy, u, du):
    out = ctypes.c_double()
    N.check(N.lib.lpg_fem_feasible_step_noalloc(energy.handle, N.vptr(u), N.vptr(du), ctypes.byref(out)))
    return out.value


def test_noalloc_feasible_step_matches_allocating_entry_point():
    w = workloads.deformed_box(6, seed=3)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    u = torch.as_tensor(w["u"], device="cuda")
    rng = np.random.default_rng(8)
    for scale in (2.0, 0.3):  # two calls in a row, with different results
        du = torch.as_tensor(scale * rng.standard_normal(e.num_dofs), device="cuda")
        expected = e.max_feasible_step(u, du)
        got = noalloc_step(e, u, du)
        assert abs(got - expected) <= 1e-12 * max(expected, 1e-300)
    assert got > 0


def test_noalloc_feasible_step_clears_the_previous_status():
    w = workloads.deformed_box(4, seed=1)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    bad = torch.as_tensor(-3 * w["X"].ravel(), device="cuda")  # inverted elements: det F < 0
    du = torch.as_tensor(np.random.default_rng(9).standard_normal(e.num_dofs), device="cuda")
    with pytest.raises(ValueError, match="det"):
        noalloc_step(e, bad, du)
    u = torch.as_tensor(w["u"], device="cuda")
    for _ in range(2):
        expected = e.max_feasible_step(u, du)
        assert abs(noalloc_step(e, u, du) - expected) <= 1e-12 * max(expected, 1e-300)
