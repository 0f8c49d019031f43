"""VEG mesh files (mesh.read_veg / mesh.write_veg, src/core/mesh/io/veg.cpp), after the
reference's tests/python/test_mesh.py: exact round trips, 17-digit precision, *INCLUDE and its
cycle check, malformed files, and agreement with an independent text parse. The files are
generated here (structured boxes, a hex grid, hand-written records)."""

import numpy as np
import pytest

from conftest import ROOT  # noqa: F401  (puts the repository on sys.path)
from litepgo_b200 import mesh


def hex_grid(n):
    """n^3 unit-cube hexes (VEG CUBIC vertex order: bottom face, then top face)."""
    g = np.arange(n + 1) / n
    Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
    P = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    idx = lambda i, j, k: i + (n + 1) * (j + (n + 1) * k)  # noqa: E731
    cells = []
    for k in range(n):
        for j in range(n):
            for i in range(n):
                cells.append([idx(i, j, k), idx(i + 1, j, k), idx(i + 1, j + 1, k), idx(i, j + 1, k),
                              idx(i, j, k + 1), idx(i + 1, j, k + 1), idx(i + 1, j + 1, k + 1), idx(i, j + 1, k + 1)])
    return P, np.array(cells, np.int32)


def independent_parse(text):
    """The reference test's own reading of a VEG file (1-based ids, no *INCLUDE)."""
    lines = [ln.strip() for ln in text.splitlines() if ln.strip() and not ln.lstrip().startswith("#")]
    start = lines.index("*VERTICES")
    count = int(lines[start + 1].split()[0])
    vertices = [[float(x) for x in ln.split()[1:4]] for ln in lines[start + 2:start + 2 + count]]
    start = lines.index("*ELEMENTS")
    count = int(lines[start + 2].split()[0])
    cells = [[int(x) - 1 for x in ln.split()[1:]] for ln in lines[start + 3:start + 3 + count]]
    return np.array(vertices), np.array(cells)


@pytest.mark.parametrize("kind", ["tet", "hex"])
def test_round_trip_is_exact(tmp_path, kind):
    if kind == "tet":
        X, cells = mesh.make_box(4, 3, 2)
        X = X + 1e-3 * np.random.default_rng(0).standard_normal(X.shape)  # full-precision coordinates
        data = mesh.TetMesh(X, cells)
    else:
        X, cells = hex_grid(3)
        data = mesh.HexMesh(X, cells)
    path = tmp_path / f"{kind}.veg"
    mesh.write_veg(path, data)
    copy = mesh.read_veg(path)
    assert type(copy) is type(data)
    assert copy.positions.dtype == np.float64 and copy.cells.dtype == np.int32
    np.testing.assert_array_equal(copy.positions, data.positions)
    np.testing.assert_array_equal(copy.cells, data.cells)
    V, C = independent_parse(path.read_text())
    np.testing.assert_array_equal(copy.positions, V)
    np.testing.assert_array_equal(copy.cells, C)


def test_precision(tmp_path):
    positions = np.array([[0.12345678901234567, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    data = mesh.TetMesh(positions, np.array([[0, 1, 2, 3]], dtype=np.int32))
    path = tmp_path / "mesh.veg"
    mesh.write_veg(path, data)
    copy = mesh.read_veg(path)
    np.testing.assert_allclose(copy.positions, positions, rtol=0, atol=1e-16)
    np.testing.assert_array_equal(copy.cells, data.cells)


def test_include(tmp_path):
    (tmp_path / "vertices.inc").write_text("*VERTICES\n4 3 0 0\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n")
    path = tmp_path / "mesh.veg"
    path.write_text("*INCLUDE vertices.inc\n*ELEMENTS\nTET\n1 4 0\n1 1 2 3 4\n")
    np.testing.assert_array_equal(mesh.read_veg(path).cells, [[0, 1, 2, 3]])


def test_include_cycle(tmp_path):
    path = tmp_path / "cycle.veg"
    path.write_text("*INCLUDE cycle.veg\n")
    with pytest.raises(RuntimeError, match="cycle"):
        mesh.read_veg(path)


def test_zero_based_ids_commas_comments_and_other_records(tmp_path):
    path = tmp_path / "mesh.veg"
    path.write_text("# a comment\n\n*VERTICES\n4 3 0 0\n0, 0, 0, 0\n1\t1 0 0\n2 0 1 0\n3 0 0 1\n"
                    "*MATERIAL BODY\nENU, 1000, 1e6, 0.4\n*ELEMENTS\n  T E T \n1 4 0\n0 0 1 2 3\n*REGION\nall\n")
    data = mesh.read_veg(path)
    np.testing.assert_array_equal(data.positions, [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    np.testing.assert_array_equal(data.cells, [[0, 1, 2, 3]])


@pytest.mark.parametrize("text", [
    "*VERTICES\n1 3 0 0\n1 0 0 junk\n",                                  # malformed number (reference case)
    "*VERTICES\n2 3 0 0\n1 0 0 0\n",                                     # truncated (reference case)
    "*VERTICES\n2 3 0 0\n1 0 0 0\n3 1 0 0\n*ELEMENTS\nTET\n0 4 0\n",       # ids not consecutive
    "*VERTICES\n1 2 0 0\n1 0 0\n",                                       # not 3D
    "*VERTICES\n4 3 0 0\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n*ELEMENTS\nWEDGE\n1 6 0\n1 1 2 3 4 1 2\n",
    "*VERTICES\n4 3 0 0\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n*ELEMENTS\nTET\n1 8 0\n1 1 2 3 4\n",  # width mismatch
    "*VERTICES\n4 3 0 0\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n*ELEMENTS\nTET\n1 4 0\n1 1 2 3 5\n",  # index range
    "*VERTICES\n4 3 0 0\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n*ELEMENTS\nTET\n1 4 0\n1 1 2 3\n",    # short line
    "*VERTICES\n4 3 0 0\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n",                                    # no elements
    "*ELEMENTS\nTET\n0 4 0\n",                                                                     # no vertices
    "*VERTICES\n0 3 0 0\n*VERTICES\n0 3 0 0\n*ELEMENTS\nTET\n0 4 0\n",                              # duplicate
])
def test_bad_veg(tmp_path, text):
    path = tmp_path / "bad.veg"
    path.write_text(text)
    with pytest.raises(RuntimeError):
        mesh.read_veg(path)


def test_missing_file(tmp_path):
    with pytest.raises(RuntimeError, match="open"):
        mesh.read_veg(tmp_path / "absent.veg")


def test_invalid_meshes_raise_value_error(tmp_path):
    path = tmp_path / "dup.veg"
    path.write_text("*VERTICES\n4 3 0 0\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n*ELEMENTS\nTET\n1 4 0\n1 1 2 2 4\n")
    with pytest.raises(ValueError, match="distinct"):
        mesh.read_veg(path)
    with pytest.raises(ValueError):
        mesh.TetMesh(np.zeros((4, 3)), np.array([[0, 1, 2, 4]], dtype=np.int32))
    with pytest.raises(ValueError):
        mesh.TetMesh(np.full((4, 3), np.nan), np.array([[0, 1, 2, 3]], dtype=np.int32))
    with pytest.raises(ValueError):
        mesh.write_veg(tmp_path / "nan.veg", type("M", (), {"positions": np.full((4, 3), np.inf),
                                                             "cells": np.array([[0, 1, 2, 3]], np.int32)})())


def test_unstructured_mesh_round_trip_and_plan(tmp_path):
    """A Delaunay ball (unstructured, irregular valence) through VEG and the assembly plan's
    own invariant checks (clusters and the solvers' layout)."""
    import test_host

    X, tets = mesh.delaunay_ball(600, seed=3)
    path = tmp_path / "ball.veg"
    mesh.write_veg(path, mesh.TetMesh(X, tets))
    data = mesh.read_veg(path)
    np.testing.assert_array_equal(data.positions, X)
    np.testing.assert_array_equal(data.cells, tets)
    ncl, max_rows, max_els, evals, entries = test_host.cluster_summary(data.positions, data.cells)
    assert entries == 16 * tets.shape[0] and ncl >= 1 and max_rows <= 24 and max_els <= 224


def test_cubic_veg_feeds_the_hex_and_hermite_plans(tmp_path):
    """A CUBIC VEG file read back gives cells the Q1 (8-node) and tricubic Hermite (64-node)
    assembly plans accept with all their invariants (the reference's Hermite examples read
    assets/box-hex.veg the same way)."""
    import test_host

    X, cells = hex_grid(3)
    path = tmp_path / "grid.veg"
    mesh.write_veg(path, mesh.HexMesh(X, cells))
    data = mesh.read_veg(path)
    T = data.cells.shape[0]
    assert test_host.cell_summary(data.positions, data.cells, 8)[4] == 64 * T
    nodes = test_host.hermite_cells(data.cells)
    assert test_host.cell_summary(np.zeros((8 * data.positions.shape[0], 3)), nodes, 64)[4] == 64 * 64 * T
