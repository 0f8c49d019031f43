"""Host-side logic on the CPU: mesh generator, block-CSR pattern, assembly plan, C ABI
exports and the argument validation of the Python mirror. No GPU is touched."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
from conftest import ROOT, TWO_TET_CELLS, TWO_TET_THETA, TWO_TET_X
from litepgo_b200 import _native as N
from litepgo_b200 import dof, energy, fem, mesh, solver, workloads


def bsr_pattern(X, tets):
    V = X.shape[0]
    tets = np.ascontiguousarray(tets, dtype=np.int32)
    nnzb = ctypes.c_int64()
    N.check(N.lib.lpg_mesh_pattern_bsr(V, tets.shape[0], N.iptr(tets), ctypes.byref(nnzb), None, None))
    row_ptr = np.empty(V + 1, np.int32)
    col_idx = np.empty(nnzb.value, np.int32)
    N.check(N.lib.lpg_mesh_pattern_bsr(V, tets.shape[0], N.iptr(tets), None, N.iptr(row_ptr), N.iptr(col_idx)))
    return row_ptr, col_idx


def bsr_to_csc_pattern(row_ptr, col_idx):
    """Column 3v + k lists rows 3w + i for the sorted block columns w of block row v."""
    V = row_ptr.size - 1
    outer = [0]
    inner = []
    for v in range(V):
        cols = col_idx[row_ptr[v]:row_ptr[v + 1]]
        rows = (3 * cols[:, None] + np.arange(3)).ravel()
        for _ in range(3):
            inner.append(rows)
            outer.append(outer[-1] + rows.size)
    return np.array(outer, np.int32), (np.concatenate(inner).astype(np.int32) if inner else np.zeros(0, np.int32))



@pytest.mark.parametrize("n", [1, 2, 3, 10, 64])
def test_box_counts_and_orientation(n):
    X, tets = mesh.make_box(n)
    V, T, nnzb = mesh.box_counts(n)
    assert X.shape == (V, 3) and tets.shape == (T, 4)
    vol = workloads.element_volumes(X, tets)
    assert np.all(vol > 0)
    assert abs(vol.sum() - 1.0) < 1e-11
    assert len({tuple(sorted(t)) for t in tets[: min(T, 5000)]}) == min(T, 5000)
    if n <= 10:
        rp, ci = bsr_pattern(X, tets)
        assert ci.size == nnzb


def test_published_sizes():
    # The five configurations' sizes (V, T, nnzb) of the structured five-tet boxes.
    assert mesh.box_counts(10) == (1331, 5000, 15191)
    assert mesh.box_counts(64) == (274625, 1310720, 3494465)
    assert mesh.box_counts(32) == (35937, 163840, 447777)
    assert mesh.box_counts(128) == (2146689, 10485760, 27608193)


@pytest.mark.parametrize("case", ["two_tet", "box3", "box10", "ragged"])
def test_bsr_pattern_expands_to_reference_csc_bit_exact(case):
    if case == "two_tet":
        X, tets, theta = TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA
    elif case == "ragged":
        # Uneven valences and unused vertices: a random subset of a box's tets.
        X, t = mesh.make_box(4)
        keep = np.random.default_rng(5).random(t.shape[0]) < 0.6
        X, tets, theta = X, t[keep], np.array([2.0, 3.0])
    else:
        n = 3 if case == "box3" else 10
        X, tets = mesh.make_box(n)
        theta = np.array([1.4e5, 3.4e4])
    m = oracle.OracleMesh(X, tets, theta)
    outer_ref, inner_ref = m.pattern()
    outer, inner = bsr_to_csc_pattern(*bsr_pattern(X, tets))
    np.testing.assert_array_equal(outer, outer_ref)
    np.testing.assert_array_equal(inner, inner_ref)


def test_plan_rejects_bad_connectivity():
    X, tets = mesh.make_box(2)
    bad = tets.copy()
    bad[3, 1] = bad[3, 0]
    with pytest.raises(ValueError, match="distinct"):
        cluster_summary(X, bad)
    bad = tets.copy()
    bad[0, 2] = X.shape[0]
    with pytest.raises(ValueError, match="outside"):
        cluster_summary(X, bad)


def test_plan_rejects_valence_above_the_cluster_capacity():
    # A fan of 230 tets around the axis (0, 1): both axis vertices have valence 230 > 224.
    k = 230
    ang = np.linspace(0, 2 * np.pi, k, endpoint=False)
    X = np.vstack([[0, 0, 0], [0, 0, 1], np.stack([np.cos(ang), np.sin(ang), np.zeros(k)], 1)])
    tets = np.array([[0, 2 + i, 2 + (i + 1) % k, 1] for i in range(k)], np.int32)
    with pytest.raises(ValueError, match="valence"):
        cluster_summary(X, tets)
    ok = tets[:200]
    assert cluster_summary(X, ok)[4] == 16 * 200


def cluster_summary(X, tets):
    out = np.zeros(5, np.int64)
    tets = np.ascontiguousarray(tets, dtype=np.int32)
    N.check(N.lib.lpg_mesh_cluster_summary(X.shape[0], tets.shape[0], N.iptr(tets), out.ctypes.data_as(N._i64p)))
    return out


def _fan(k):
    ang = np.linspace(0, 2 * np.pi, k, endpoint=False)
    X = np.vstack([[0, 0, 0], [0, 0, 1], np.stack([np.cos(ang), np.sin(ang), np.zeros(k)], 1)])
    return X, np.array([[0, 2 + i, 2 + (i + 1) % k, 1] for i in range(k)], np.int32)


@pytest.mark.parametrize("case", ["box2", "box10", "box24", "ragged", "fan40", "shuffled"])
def test_cluster_plan_invariants(case):
    """The element-once assembly's clusters: the library checks every invariant itself
    (ownership, energy counted once, exact and ordered contributor lists per block)."""
    rng = np.random.default_rng(4)
    if case.startswith("box"):
        X, tets = mesh.make_box(int(case[3:]))
    elif case == "ragged":
        X, t = mesh.make_box(6)
        tets = t[rng.random(t.shape[0]) < 0.6]
    elif case == "fan40":
        X, tets = _fan(40)
    else:  # vertex numbering with no locality
        X, t = mesh.make_box(8)
        perm = rng.permutation(X.shape[0])
        tets = perm[t].astype(np.int32)
    ncl, max_rows, max_els, evals, entries = cluster_summary(X, tets)
    T = tets.shape[0]
    assert entries == 16 * T
    assert 1 <= max_rows <= 24 and max_els <= 224
    assert T <= evals <= 4 * T  # each element once per cluster owning one of its vertices
    if case == "box24":
        assert evals <= 2.6 * T  # compact clusters on a structured box


def _header_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names.update(re.findall(r"\b(lpg_\w+)\s*\(", text))
    return names


def test_abi_exports_every_declared_symbol():
    declared = _header_functions()
    assert "lpg_fem_eval" in declared and "lpg_newton_solve" in declared
    for name in sorted(declared):
        assert hasattr(N.lib, name), f"{name} declared in include/ but not exported"
    assert declared == set(N.EXPORTED), "the ctypes binding must cover exactly the declared ABI"


def test_library_is_sm100a_and_reports_build():
    info = N.build_info()
    assert "sm_100a" in info and "12090" in info


def test_python_mirror_validation():
    topo = mesh.TetTopology(5, TWO_TET_CELLS)
    with pytest.raises(ValueError, match="distinct"):
        mesh.TetTopology(4, [[0, 1, 1, 2]])
    with pytest.raises(ValueError, match="outside"):
        mesh.TetTopology(3, [[0, 1, 2, 3]])
    with pytest.raises(ValueError, match="unique"):
        dof.DofReduction(6, [1, 1])
    with pytest.raises(ValueError, match="lie in"):
        dof.DofReduction(6, [6])
    red = dof.DofReduction(6, [4, 1])
    np.testing.assert_array_equal(red.free_dofs, [0, 2, 3, 5])
    assert red.free_index(4) == -1 and red.free_index(5) == 3
    full = np.zeros(6)
    red.expand(np.arange(4.0), full)
    np.testing.assert_array_equal(red.reduce(full), np.arange(4.0))
    m = dof.VertexDofMap(topo, 3)
    np.testing.assert_array_equal(m.dof_indices(1), [0, 1, 2, 6, 7, 8, 3, 4, 5, 12, 13, 14])
    Energy = fem.VolumetricFemEnergy[fem.NeoHookean, fem.TetP1Basis, fem.TetCentroidQuadrature]
    with pytest.raises(ValueError, match="batch size"):
        Energy(m, TWO_TET_X, None, TWO_TET_THETA, batch_size=0)
    with pytest.raises(ValueError, match="incompatible"):
        Energy(dof.VertexDofMap(topo, 2), TWO_TET_X, None, TWO_TET_THETA)
    with pytest.raises(TypeError, match="not instantiated"):
        fem.VolumetricFemEnergy[fem.NeoHookean, fem.TetP1Basis]
    opts = solver.NewtonOptions()
    assert np.isnan(opts.gradient_tolerance) and opts.max_iterations == 50
    assert opts.hessian == energy.HessianKind.Projected and opts.max_line_search_steps == 30
    assert opts.line_search_shrink == 0.5


def test_device_calls_fail_loudly_without_a_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    topo = mesh.TetTopology(5, TWO_TET_CELLS)
    Energy = fem.VolumetricFemEnergy[fem.NeoHookean, fem.TetP1Basis, fem.TetCentroidQuadrature]
    with pytest.raises(N.LitepgoError):
        Energy(dof.VertexDofMap(topo, 3), TWO_TET_X, None, TWO_TET_THETA)


def test_workloads_are_seeded_and_valid():
    a = workloads.deformed_box(3, seed=2)
    b = workloads.deformed_box(3, seed=2)
    np.testing.assert_array_equal(a["u"], b["u"])
    assert np.all(workloads.det_F(a["X"], a["tets"], a["u"]) > 0)
    g = workloads.gravity_box(4, seed=0)
    assert g["fixed"].size == 3 * 25
    assert abs(g["f"][2::3].sum() + 1000 * 9.8) < 1e-9  # total weight of the unit box
    assert np.all(g["theta"][:, 1] >= 1e3) and np.all(g["theta"][:, 1] <= 1e5)
    nu = g["theta"][:, 0] / (2 * (g["theta"][:, 0] + g["theta"][:, 1]))
    assert np.all((nu >= 0.3 - 1e-12) & (nu <= 0.45 + 1e-12))
    c = workloads.compressed_box(6, seed=0)
    d = workloads.det_F(c["X"], c["tets"], c["u"])
    assert d.min() >= 0.2 and d.max() <= 3.0


def cell_summary(X, cells, width):
    out = np.zeros(5, np.int64)
    cells = np.ascontiguousarray(cells, dtype=np.int32)
    N.check(N.lib.lpg_mesh_cluster_summary_cells(X.shape[0], cells.shape[0], N.iptr(cells), width,
                                                 out.ctypes.data_as(N._i64p)))
    return out


@pytest.mark.parametrize("case", ["hex4", "hex_ragged", "hex_shuffled"])
def test_hex_cluster_plan_invariants(case):
    """The assembly plan of 8-vertex cells: every invariant of the tet plan (ownership, energy once,
    exact ordered contributor lists) and of the solvers' layout, checked by the library itself."""
    rng = np.random.default_rng(9)
    X, cells = mesh.make_hex_box(4, 3, 5)
    if case == "hex_ragged":
        cells = cells[rng.random(cells.shape[0]) < 0.6]
    elif case == "hex_shuffled":
        perm = rng.permutation(X.shape[0])
        cells = perm[cells].astype(np.int32)
    ncl, max_rows, max_els, evals, entries = cell_summary(X, cells, 8)
    assert entries == 64 * cells.shape[0]
    assert 1 <= max_rows <= 24 and max_els <= 224
    assert cells.shape[0] <= evals <= 8 * cells.shape[0]
    with pytest.raises(ValueError):
        cell_summary(X, cells, 6)
    bad = cells.copy()
    bad[0, 3] = bad[0, 0]
    with pytest.raises(ValueError, match="distinct"):
        cell_summary(X, bad, 8)


def hermite_cells(cells):
    """The 64 nodes of each tricubic Hermite hex: node 8 v + slot for basis function
    8 corner + slot (v = cells[corner]), each node a 3-DOF row of the assembly plan."""
    cells = np.asarray(cells, dtype=np.int64)
    return (8 * cells[:, :, None] + np.arange(8)).reshape(-1, 64).astype(np.int32)


@pytest.mark.parametrize("shape,ragged", [((1, 1, 1), False), ((3, 2, 2), False), ((4, 3, 2), False),
                                          ((5, 4, 3), True)])
def test_hermite_cluster_plan_invariants(shape, ragged):
    """The assembly plan of 64-node cells (two 16-bit words per contributor, clusters of at most
    one vertex's eight rows): every invariant the library checks, and 64^2 contributors per cell;
    ragged: 40 % of the hexes removed (irregular valence, vertices of no cell)."""
    X, cells = mesh.make_hex_box(*shape)
    if ragged:
        cells = cells[np.random.default_rng(2).random(cells.shape[0]) < 0.6]
    nodes = hermite_cells(cells)
    ncl, max_rows, max_els, evals, entries = cell_summary(np.zeros((8 * X.shape[0], 3)), nodes, 64)
    assert entries == 64 * 64 * cells.shape[0]
    assert 1 <= max_rows <= 8 and max_els <= 224
    rng = np.random.default_rng(1)
    perm = rng.permutation(8 * X.shape[0])
    assert cell_summary(np.zeros((8 * X.shape[0], 3)), perm[nodes].astype(np.int32), 64)[4] == entries
