"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances: FP64 results within 1e-12 relative (max-norm of the difference over the
max-norm of the oracle value); FP32 ("mixed") element arithmetic within the bounds stated
in each test; patterns bit-exact; repeated evaluations bitwise identical.
"""

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
from conftest import TWO_TET_CELLS, TWO_TET_THETA, TWO_TET_X, corner_chain, rel_err, two_tet_states
from litepgo_b200 import dof, energy, fem, mesh, workloads

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

Exact, Projected = energy.HessianKind.Exact, energy.HessianKind.Projected
TOL64 = 1e-12


@pytest.fixture(scope="module")
def cfg1():
    w = workloads.deformed_box(10, seed=0)
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    orc = oracle.OracleMesh(w["X"], w["tets"], w["theta"])
    return w, gpu, orc


def test_pattern_bit_exact(cfg1):
    _, gpu, orc = cfg1
    outer, inner = gpu.pattern_csc()
    o_ref, i_ref = orc.pattern()
    np.testing.assert_array_equal(outer, o_ref)
    np.testing.assert_array_equal(inner, i_ref)
    assert gpu.nnz == 136719 and gpu.nnzb == 15191


def test_f64_exact_parity(cfg1):
    w, gpu, orc = cfg1
    E, g, H = gpu.eval(w["u"], gradient=True, hessian=Exact)
    Er, gr, vr = orc.eval(w["u"], True, 1)
    assert abs(E - Er) <= TOL64 * abs(Er)
    assert rel_err(g, gr) <= TOL64
    assert rel_err(H.data, vr) <= TOL64


def test_element_energies_parity(cfg1):
    w, gpu, orc = cfg1
    eE = gpu.element_energies(w["u"])
    _, _, _, (eEr, _, _) = orc.eval(w["u"], False, 0, elements=True)
    assert rel_err(eE, eEr) <= TOL64


def test_f64_projected_parity(cfg1):
    w, gpu, orc = cfg1
    _, _, H = gpu.eval(w["u"], hessian=Projected)
    _, _, vr = orc.eval(w["u"], False, 2)
    assert rel_err(H.data, vr) <= 1e-11
    # The projection is PSD: x^T K x >= 0 up to rounding for random x.
    rng = np.random.default_rng(0)
    for _ in range(5):
        x = rng.standard_normal(gpu.num_dofs)
        assert x @ (H @ x) >= -1e-10 * np.abs(H.data).max() * (x @ x)


def test_projected_equals_exact_when_exact_is_psd():
    # Small uniform stretch: every element tangent is positive definite, so projection is the identity.
    X, tets = mesh.make_box(3)
    u = 0.05 * X.ravel()
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, np.array([1.4e5, 3.4e4]))
    _, _, He = gpu.eval(u, hessian=Exact)
    _, _, Hp = gpu.eval(u, hessian=Projected)
    assert rel_err(Hp.data, He.data) <= 1e-12


def test_hessian_is_bitwise_symmetric(cfg1):
    w, gpu, _ = cfg1
    _, _, H = gpu.eval(w["u"], hessian=Exact)
    D = (H - H.T).tocsc()
    D.eliminate_zeros()
    assert D.nnz == 0


def test_repeated_evaluations_are_bitwise_identical(cfg1):
    w, gpu, _ = cfg1
    a = gpu.eval(w["u"], gradient=True, hessian=Exact)
    b = gpu.eval(w["u"], gradient=True, hessian=Exact)
    assert a[0] == b[0]
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[2].data, b[2].data)


# tests/python/test_fem_batch_size.py:7-21: identical Hessians for batch sizes 1/16/64/256.
@pytest.mark.parametrize("batch_size", [1, 16, 64, 256])
def test_batch_size_invariance(batch_size):
    nodes = np.array([[0., 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    topology = mesh.TetTopology(4, np.tile(np.arange(4, dtype=np.int32), (17, 1)))
    mapping = dof.VertexDofMap(topology, 3)
    rest = [fem.InterpolatedResponse[fem.TetP1Basis](nodes) for _ in range(17)]
    Energy = fem.VolumetricFemEnergy[fem.NeoHookean, fem.TetP1Basis, fem.TetCentroidQuadrature]
    x = np.arange(12) * .001
    expected = Energy(mapping, rest, fem.constant_fields(np.eye(3), 17),
                      fem.constant_fields([2., 3.], 17)).eval_hessian(x).toarray()
    actual = Energy(mapping, rest, fem.constant_fields(np.eye(3), 17), fem.constant_fields([2., 3.], 17),
                    batch_size=batch_size).eval_hessian(x).toarray()
    np.testing.assert_array_equal(actual, expected)
    ref = oracle.OracleMesh(nodes, topology.cells, np.array([2.0, 3.0]))
    assert rel_err(actual, ref.hessian_csc(x).toarray()) <= TOL64


def test_mixed_precision_error_bounds(cfg1):
    """FP32 element arithmetic: errors against the FP64 oracle are stated here."""
    w, gpu, orc = cfg1
    E, g, H = gpu.eval(w["u"], gradient=True, hessian=Exact, precision="mixed")
    Er, gr, vr = orc.eval(w["u"], True, 1)
    assert abs(E - Er) <= 2e-6 * abs(Er)
    assert rel_err(g, gr) <= 2e-5
    assert rel_err(H.data, vr) <= 1e-5
    _, _, Hp = gpu.eval(w["u"], hessian=Projected, precision="mixed")
    _, _, vp = orc.eval(w["u"], False, 2)
    assert rel_err(Hp.data, vp) <= 1e-4


@pytest.mark.parametrize("state", [0, 1, 2])
def test_two_tet_matches_oracle_and_fd(state):
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA)
    orc = oracle.OracleMesh(TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA)
    x = two_tet_states()[state]
    E, g, H = gpu.eval(x, gradient=True, hessian=Exact)
    Er, gr, vr = orc.eval(x, True, 1)
    assert abs(E - Er) <= 1e-13 + TOL64 * abs(Er)
    assert rel_err(g, gr) <= TOL64 or np.abs(g - gr).max() < 1e-14
    assert rel_err(H.data, vr) <= TOL64
    Hd = H.toarray()
    for h in (1e-3, 1e-4):
        fd = np.zeros_like(Hd)
        for j in range(x.size):
            p, q = x.copy(), x.copy()
            p[j] += h
            q[j] -= h
            fd[:, j] = (gpu.eval_gradient(p) - gpu.eval_gradient(q)) / (2 * h)
        assert np.linalg.norm(Hd - fd) / (1 + np.linalg.norm(Hd)) < 10 * h * h + 1e-9


def test_feasible_step_constants_and_parity(cfg1):
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA)
    X = TWO_TET_X.ravel()
    zero = np.zeros_like(X)
    assert gpu.max_feasible_step(zero, zero) == 1
    d = zero.copy()
    d[0::3] = -4 * X[0::3]
    d[1::3] = -4 * X[1::3]
    assert abs(gpu.max_feasible_step(zero, d) - 0.225) < 1e-6
    d = zero.copy()
    d[14] = 16
    assert abs(gpu.max_feasible_step(zero, d) - 0.1125) < 1e-12
    with pytest.raises(ValueError):
        gpu.max_feasible_step(-X, zero)
    w, g1, orc = cfg1
    rng = np.random.default_rng(1)
    for scale in (0.05, 0.5, 3.0):
        du = scale * rng.standard_normal(g1.num_dofs)
        a, ar = g1.max_feasible_step(w["u"], du), orc.feasible_step(w["u"], du)
        assert abs(a - ar) <= 1e-12 * max(ar, 1e-300)


def test_force_vjp_parity(cfg1):
    w, gpu, orc = cfg1
    rng = np.random.default_rng(2)
    wt = rng.standard_normal(gpu.num_dofs)
    ref = orc.force_vjp_theta(w["u"], wt)
    topo = mesh.TetTopology(w["X"].shape[0], w["tets"])
    vm = dof.VertexDofMap(topo, 3)
    per = fem.VolumetricFemForceMaterialResponse[fem.NeoHookean, fem.TetP1Basis, fem.TetCentroidQuadrature](
        dof.ElementDofMap(topo, 2), vm, w["X"], w["u"], None)
    out = per.eval_vjp(np.tile(w["theta"], topo.num_cells), wt).reshape(-1, 2)
    assert rel_err(out, ref) <= TOL64
    shared = fem.VolumetricFemForceMaterialResponse[fem.NeoHookean, fem.TetP1Basis, fem.TetCentroidQuadrature](
        dof.ConstantDofMap(topo, 2), vm, w["X"], w["u"], None)
    s = shared.eval_vjp(w["theta"], wt)
    assert rel_err(s, ref.sum(axis=0)) <= 1e-11


def test_error_contract():
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(TWO_TET_X, TWO_TET_CELLS, np.array([2.0, 0.0]))
    with pytest.raises(ValueError, match="lambda >= 0 and mu > 0"):
        gpu.eval_value(np.zeros(15))
    good = fem.VolumetricFemEnergyTetP1.from_arrays(TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA)
    with pytest.raises(ValueError, match="det"):
        good.eval_value(-2 * TWO_TET_X.ravel())
    bad = np.zeros(15)
    bad[3] = np.nan
    with pytest.raises(ValueError, match="finite"):
        good.eval_value(bad)
    with pytest.raises(ValueError):
        good.eval_value(np.zeros(14))
    dev = torch.zeros(15, dtype=torch.float64, device="cuda")
    dev[4] = float("inf")
    with pytest.raises(ValueError):
        good.eval_device(dev)
    with pytest.raises(ValueError, match="invalid reference"):
        fem.VolumetricFemEnergyTetP1.from_arrays(0 * TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA)
    assert np.isfinite(good.eval_value(np.zeros(15)))  # the handle stays usable after errors


def test_device_resident_eval_matches_host(cfg1):
    w, gpu, _ = cfg1
    u = torch.as_tensor(w["u"], device="cuda")
    E, g, Hb = gpu.eval_device(u, gradient=True, hessian=Exact, layout="bsr")
    _, _, Hc = gpu.eval_device(u, gradient=False, hessian=Exact, layout="csc")
    Eh, gh, Hh = gpu.eval(w["u"], gradient=True, hessian=Exact)
    assert E == Eh
    np.testing.assert_array_equal(g.cpu().numpy(), gh)
    np.testing.assert_array_equal(Hc.cpu().numpy(), Hh.data)
    # BSR -> CSC by the documented permutation.
    row_ptr, col_idx = gpu.pattern_bsr()
    bsr = Hb.cpu().numpy().reshape(-1, 3, 3)
    v = 7
    blocks = bsr[row_ptr[v]:row_ptr[v + 1]]
    col = Hh[:, 3 * v + 1].toarray().ravel()
    rows = (3 * col_idx[row_ptr[v]:row_ptr[v + 1]][:, None] + np.arange(3)).ravel()
    np.testing.assert_array_equal(col[rows], blocks[:, 1, :].ravel())


def test_plastic_field_parity():
    X, tets = mesh.make_box(3)
    rng = np.random.default_rng(4)
    T = tets.shape[0]
    Fp = np.stack([np.eye(3) + 0.05 * rng.standard_normal((3, 3)) for _ in range(T)])
    Fpv = np.ascontiguousarray(Fp.transpose(0, 2, 1).reshape(T, 9))  # column-major
    theta = np.stack([1e3 * (1 + rng.random(T)), 5e2 * (1 + rng.random(T))], axis=1)
    u = 0.02 * rng.standard_normal(X.size)
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta, Fp=Fpv)
    orc = oracle.OracleMesh(X, tets, theta, Fp=Fpv)
    E, g, H = gpu.eval(u, gradient=True, hessian=Exact)
    Er, gr, vr = orc.eval(u, True, 1)
    assert abs(E - Er) <= 1e-11 * abs(Er)
    assert rel_err(g, gr) <= 1e-11
    assert rel_err(H.data, vr) <= 1e-11
    du = rng.standard_normal(X.size)
    assert abs(gpu.max_feasible_step(u, du) - orc.feasible_step(u, du)) <= 1e-10


def test_ragged_mesh_with_unused_vertices():
    X, t = mesh.make_box(4)
    keep = np.random.default_rng(5).random(t.shape[0]) < 0.6
    tets = t[keep]
    rng = np.random.default_rng(6)
    u = 0.01 * rng.standard_normal(X.size)
    theta = np.array([1.4e5, 3.4e4])
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta)
    orc = oracle.OracleMesh(X, tets, theta)
    E, g, H = gpu.eval(u, gradient=True, hessian=Projected)
    Er, gr, vr = orc.eval(u, True, 2)
    assert abs(E - Er) <= TOL64 * abs(Er)
    assert rel_err(g, gr) <= TOL64
    assert rel_err(H.data, vr) <= 1e-11
    unused = np.setdiff1d(np.arange(X.shape[0]), np.unique(tets))
    assert unused.size > 0 and np.all(g.reshape(-1, 3)[unused] == 0)


def test_valence_above_32():
    k = 40
    ang = np.linspace(0, 2 * np.pi, k, endpoint=False)
    ring = np.stack([np.cos(ang), np.sin(ang), np.zeros(k)], 1)
    X = np.vstack([[0, 0, 0], [0, 0, 1], ring])
    tets = np.array([[0, 2 + i, 2 + (i + 1) % k, 1] for i in range(k)], np.int32)
    theta = np.array([2.0, 3.0])
    u = 0.01 * np.random.default_rng(7).standard_normal(X.size)
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta)
    orc = oracle.OracleMesh(X, tets, theta)
    E, g, H = gpu.eval(u, gradient=True, hessian=Exact)
    Er, gr, vr = orc.eval(u, True, 1)
    assert abs(E - Er) <= TOL64 * abs(Er)
    assert rel_err(g, gr) <= TOL64
    assert rel_err(H.data, vr) <= TOL64


def test_full_clusters_corner_chain():
    """Assembly clusters at their 64-row limit (a chain of tets sharing corners): the diagonal
    items are summed by lane pairs there and by lane quads in the smaller clusters; Exact and
    Projected Hessians against the oracle."""
    X, tets = corner_chain(200)
    theta = np.array([1.4e5, 3.4e4])
    u = 0.01 * np.random.default_rng(8).standard_normal(X.size)
    gpu = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta)
    orc = oracle.OracleMesh(X, tets, theta)
    for kind, code, tol in ((Exact, 1, TOL64), (Projected, 2, 1e-11)):
        E, g, H = gpu.eval(u, gradient=True, hessian=kind)
        Er, gr, vr = orc.eval(u, True, code)
        assert abs(E - Er) <= TOL64 * abs(Er)
        assert rel_err(g, gr) <= TOL64
        assert rel_err(H.data, vr) <= tol


def sell_layout(e):
    import ctypes

    from litepgo_b200 import _native as N

    nslots, nch = ctypes.c_int64(), ctypes.c_int()
    N.check(N.lib.lpg_fem_solver_layout(e.handle, ctypes.byref(nslots), ctypes.byref(nch), None, None))
    ptr = np.empty(nch.value + 1, np.int32)
    rows = np.empty(32 * nch.value, np.int32)
    N.check(N.lib.lpg_fem_solver_layout(e.handle, None, None, N.iptr(ptr), N.iptr(rows)))
    return nslots.value, ptr, rows


def solver_values(e, u, hessian, precision, layout, nvalues):
    import ctypes

    from litepgo_b200 import _native as N

    dt = torch.float64 if precision == N.PRECISION_F64 else torch.float32
    hess = torch.full((nvalues,), float("nan"), dtype=dt, device="cuda")
    ud = torch.as_tensor(u, device="cuda")
    ma, me = ctypes.c_double(), ctypes.c_double()
    N.check(N.lib.lpg_fem_time_eval(e.handle, N.vptr(ud), None, int(hessian), precision, layout, N.vptr(hess), 1, 0,
                                    ctypes.byref(ma), ctypes.byref(me)))
    return hess.cpu().numpy()


@pytest.mark.parametrize("case", ["box", "ragged", "valence", "chain"])
def test_solver_sliced_ell_layout_holds_the_upper_bsr_blocks(case):
    """The Newton / adjoint solvers keep the upper triangle of the Hessian (blocks with column >=
    row, diagonal first) in sliced ELL (chunks of 32 rows sorted by block count within 128-row
    windows, slot-major); it must hold those BSR values bit for bit, and the BSR Hessian must be
    symmetric, so that the blocks it leaves out are the transposes of the ones it keeps."""
    from litepgo_b200 import _native as N

    rng = np.random.default_rng(12)
    if case == "box":
        w = workloads.deformed_box(5, seed=2)
        X, tets, theta, u = w["X"], w["tets"], w["theta"], w["u"]
    elif case == "ragged":
        X, t = mesh.make_box(4)
        tets = t[np.random.default_rng(5).random(t.shape[0]) < 0.6]
        theta, u = np.array([1.4e5, 3.4e4]), 0.01 * rng.standard_normal(X.size)
    elif case == "chain":
        X, tets = corner_chain(200)
        theta, u = np.array([1.4e5, 3.4e4]), 0.01 * rng.standard_normal(X.size)
    else:
        k = 40
        ang = np.linspace(0, 2 * np.pi, k, endpoint=False)
        X = np.vstack([[0, 0, 0], [0, 0, 1], np.stack([np.cos(ang), np.sin(ang), np.zeros(k)], 1)])
        tets = np.array([[0, 2 + i, 2 + (i + 1) % k, 1] for i in range(k)], np.int32)
        theta, u = np.array([2.0, 3.0]), 0.01 * rng.standard_normal(X.size)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta)
    row_ptr, col_idx = e.pattern_bsr()
    nb = np.diff(row_ptr)
    V = X.shape[0]
    rows_of = np.repeat(np.arange(V), nb)
    upper = col_idx >= rows_of
    own0 = np.array([row_ptr[v] + np.count_nonzero(col_idx[row_ptr[v]:row_ptr[v + 1]] < v) for v in range(V)])
    no = row_ptr[1:] - own0
    nslots, ptr, rows = sell_layout(e)
    # The layout's own rules: every row once, sorted by block count within 128-row windows,
    # each chunk as wide as its row with the most stored blocks.
    order = rows[rows >= 0]
    assert np.array_equal(np.sort(order), np.arange(V)) and np.all(rows[V:] == -1)
    for w0 in range(0, V, 128):
        win = order[w0:w0 + 128]
        assert np.array_equal(np.sort(win), np.arange(w0, min(V, w0 + 128)))
        assert np.all(np.diff(nb[win]) <= 0)
    for c in range(ptr.size - 1):
        rc = rows[32 * c:32 * c + 32]
        rc = rc[rc >= 0]
        assert ptr[c + 1] - ptr[c] == 32 * no[rc].max(initial=0)
    assert nslots == ptr[-1]
    bsr_at = []  # BSR entry positions of the stored blocks, and their sliced-ELL positions
    sell_at = []
    for c in range(ptr.size - 1):
        for lane in range(32):
            r = rows[32 * c + lane]
            if r < 0:
                continue
            q = np.arange(no[r])
            for t in range(9):
                bsr_at.append(9 * (own0[r] + q) + t)
                sell_at.append(9 * ptr[c] + 32 * (9 * q + t) + lane)
    bsr_at, sell_at = np.concatenate(bsr_at), np.concatenate(sell_at)
    assert np.unique(sell_at).size == sell_at.size and sell_at.max() < 9 * nslots
    assert bsr_at.size == 9 * np.count_nonzero(upper)
    for hk in (Exact, Projected):
        for prec in (N.PRECISION_F64, N.PRECISION_MIXED):
            bsr = solver_values(e, u, hk, prec, N.LAYOUT_BSR, 9 * e.nnzb)
            sell = solver_values(e, u, hk, prec, 2, 9 * nslots)
            assert np.array_equal(sell[sell_at], bsr[bsr_at])
            Hb = sp.bsr_matrix((bsr.reshape(-1, 3, 3), col_idx, row_ptr), shape=(3 * V, 3 * V)).toarray()
            if hk == Exact:
                assert np.array_equal(Hb, Hb.T)  # bitwise symmetric by construction
            else:
                assert np.abs(Hb - Hb.T).max() <= 1e-5 * np.abs(Hb).max()
