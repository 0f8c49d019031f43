"""The allocation-free feasible step, lpg_fem_feasible_step_noalloc.

It serves callers that must not allocate device memory when they ask for the step: a solver
inside a framework that owns the device memory pool, where a library cudaMalloc mid-step
fragments or exceeds that pool's budget. Its scratch is a fixed array in the library image
shared by all calls, so this test checks it against the allocating entry point,
lpg_fem_feasible_step, on two calls in a row (the second must not see the first call's
leftovers) on tet, hex and Hermite handles, including a call that fails and leaves an error
status behind; that a first call on a fresh handle makes no device allocation (the library's
allocation count in lpg_build_info does not move); and that host pointers are refused before
any launch. This file is collected last, so a failure here comes after every other test has
run.
"""

import ctypes
import re

import numpy as np
import pytest

from litepgo_b200 import _native as N
from litepgo_b200 import fem, mesh, workloads

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def noalloc_step(energy, u, du):
    out = ctypes.c_double()
    N.check(N.lib.lpg_fem_feasible_step_noalloc(energy.handle, N.vptr(u), N.vptr(du), ctypes.byref(out)))
    return out.value


def device_allocations():
    return int(re.search(r"device allocations (\d+)", N.build_info()).group(1))


def check_two_calls(e, u, rng, scales=(2.0, 0.3)):
    u = torch.as_tensor(u, device="cuda")
    got = None
    for scale in scales:  # two calls in a row, with different results
        du = torch.as_tensor(scale * rng.standard_normal(e.num_dofs), device="cuda")
        expected = e.max_feasible_step(u, du)
        got = noalloc_step(e, u, du)
        assert abs(got - expected) <= 1e-12 * max(expected, 1e-300)
    return got


def test_noalloc_feasible_step_matches_allocating_entry_point():
    w = workloads.deformed_box(6, seed=3)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    assert check_two_calls(e, w["u"], np.random.default_rng(8)) > 0


def test_noalloc_feasible_step_on_hex_and_hermite_handles():
    rng = np.random.default_rng(10)
    X, cells = mesh.make_hex_box(3, 2, 2)
    theta = np.array([1.4e5, 3.4e4])
    q1 = fem.VolumetricFemEnergy[fem.NeoHookean, fem.HexQ1Basis, fem.GaussLegendre3D[2]].from_arrays(X, cells, theta)
    check_two_calls(q1, 0.02 * rng.standard_normal(q1.num_dofs), rng, scales=(0.5, 0.1))
    herm = fem.VolumetricFemEnergy[fem.NeoHookean, fem.HexHermiteBasis, fem.GaussLegendre3D[2]].from_arrays(
        X, cells, theta)
    check_two_calls(herm, 0.02 * rng.standard_normal(herm.num_dofs), rng, scales=(0.5, 0.1))


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


def test_noalloc_first_call_on_a_fresh_handle_allocates_nothing():
    w = workloads.deformed_box(5, seed=2)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    u = torch.as_tensor(w["u"], device="cuda")
    du = torch.as_tensor(np.random.default_rng(11).standard_normal(e.num_dofs), device="cuda")
    before = device_allocations()
    first = noalloc_step(e, u, du)
    second = noalloc_step(e, u, du)
    assert device_allocations() == before
    assert first == second
    # The allocating entry point, on the same fresh handle, does allocate its scratch (so the
    # count above would have seen an allocation), and agrees.
    expected = e.max_feasible_step(u, du)
    assert device_allocations() > before
    assert abs(first - expected) <= 1e-12 * max(expected, 1e-300)


def test_noalloc_rejects_host_pointers():
    w = workloads.deformed_box(3, seed=0)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    u_host = np.ascontiguousarray(w["u"])
    du_dev = torch.zeros(e.num_dofs, dtype=torch.float64, device="cuda")
    out = ctypes.c_double()
    code = N.lib.lpg_fem_feasible_step_noalloc(e.handle, N.dptr(u_host), N.vptr(du_dev), ctypes.byref(out))
    assert code == N.LPG_EINVAL and "device" in N.error_message()
    code = N.lib.lpg_fem_feasible_step_noalloc(e.handle, N.vptr(du_dev), N.dptr(u_host), ctypes.byref(out))
    assert code == N.LPG_EINVAL and "device" in N.error_message()
