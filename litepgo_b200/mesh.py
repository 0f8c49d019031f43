"""Tet connectivity and structured box meshes.

TetTopology mirrors litepgo's ``mesh.TetTopology(num_vertices, cells)``
(src/core/mesh/mesh_topology.hpp:18-68): fixed-arity connectivity whose cells hold
distinct vertex indices in [0, num_vertices); empty meshes and unused vertices
are allowed.

``make_box`` builds the structured five-tet box used by every synthetic workload:
each cube is split into one central tetrahedron and four corner tetrahedra, and the
split alternates with the cube parity (i + j + k) so that neighbouring cubes agree on
every face diagonal. The reference ships a six-tet generator
(benchmarks/contact_scaling.py:17-40); the five-tet split is this project's own.
"""

import numpy as np

__all__ = ["TetTopology", "HexTopology", "TetMesh", "HexMesh", "read_veg", "write_veg", "make_box", "box_counts",
           "delaunay_ball", "make_hex_box"]


class TetTopology:
    """Tetrahedral connectivity: ``num_vertices`` and an (T, 4) int32 cell array."""

    vertices_per_cell = 4

    def __init__(self, num_vertices, cells):
        k = self.vertices_per_cell
        num_vertices = int(num_vertices)
        cells = np.ascontiguousarray(np.asarray(cells, dtype=np.int64).reshape(-1, k))
        if num_vertices < 0:
            raise ValueError("MeshTopology requires a non-negative vertex count")
        if cells.shape[0] > np.iinfo(np.int32).max:
            raise ValueError("MeshTopology cell count exceeds the int index range")
        if cells.size:
            s = np.sort(cells, axis=1)
            bad = np.flatnonzero((s[:, 0] < 0) | (s[:, -1] >= num_vertices))
            if bad.size:
                raise ValueError(f"MeshTopology cell {int(bad[0])} has vertex indices outside [0, num_vertices)")
            dup = np.flatnonzero((s[:, 1:] == s[:, :-1]).any(axis=1))
            if dup.size:
                raise ValueError(f"MeshTopology cell {int(dup[0])} must contain distinct vertices")
        self._num_vertices = num_vertices
        self._cells = cells.astype(np.int32)

    @property
    def num_vertices(self):
        return self._num_vertices

    @property
    def num_cells(self):
        return int(self._cells.shape[0])

    @property
    def cells(self):
        return self._cells

    def cell_vertices(self, cell):
        if cell < 0 or cell >= self.num_cells:
            raise IndexError(f"MeshTopology::cell_vertices: cell {cell} is out of range")
        return self._cells[cell].copy()


class HexTopology(TetTopology):
    """Hexahedral connectivity (8 vertices per cell); read from and written to VEG files. The
    GPU energy path takes tets only."""

    vertices_per_cell = 8


class TetMesh:
    """Vertex positions (V, 3) with their tet connectivity: mesh.TetMesh(positions, cells)
    (src/core/mesh/mesh_data.hpp:10-21, src/binding/mesh/mesh_data.cpp). Coordinates must be
    finite (ValueError otherwise, as MeshData::validate)."""

    _topology_type = TetTopology

    def __init__(self, positions, cells):
        positions = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3))
        topology = cells if isinstance(cells, TetTopology) else self._topology_type(positions.shape[0], cells)
        if topology.num_vertices != positions.shape[0] or not np.all(np.isfinite(positions)):
            raise ValueError("MeshData requires three finite coordinates per vertex")
        self._positions = positions
        self._topology = topology

    @property
    def positions(self):
        return self._positions

    @property
    def cells(self):
        return self._topology.cells

    @property
    def topology(self):
        return self._topology


class HexMesh(TetMesh):
    """Vertex positions with hexahedral connectivity (mesh.HexMesh)."""

    _topology_type = HexTopology


def read_veg(path):
    """Reads a VEG volume mesh (mesh.read_veg, src/core/mesh/io/veg.cpp): a TetMesh for TET
    elements, a HexMesh for CUBIC ones. Parsed by the native library; file and format errors
    raise RuntimeError, an invalid mesh ValueError."""
    import ctypes

    from . import _native as N

    p = str(path).encode()
    V, T, W = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    N.check(N.lib.lpg_read_veg(p, ctypes.byref(V), ctypes.byref(T), ctypes.byref(W), None, None))
    pos = np.empty((V.value, 3), dtype=np.float64)
    cells = np.empty((T.value, W.value), dtype=np.int32)
    N.check(N.lib.lpg_read_veg(p, ctypes.byref(V), ctypes.byref(T), ctypes.byref(W), N.dptr(pos), N.iptr(cells)))
    return (TetMesh if W.value == 4 else HexMesh)(pos, cells)


def write_veg(path, mesh):
    """Writes a TetMesh or HexMesh as VEG (mesh.write_veg): 1-based ids, 17 significant
    digits, so read_veg(write_veg(m)) reproduces m exactly."""
    from . import _native as N

    pos = np.ascontiguousarray(mesh.positions, dtype=np.float64)
    cells = np.ascontiguousarray(mesh.cells, dtype=np.int32)
    N.check(N.lib.lpg_write_veg(str(path).encode(), pos.shape[0], N.dptr(pos), cells.shape[0], cells.shape[1],
                                N.iptr(cells)))


def delaunay_ball(n_points, seed=0, radius=1.0):
    """An unstructured tet mesh: the Delaunay tetrahedralisation (scipy.spatial) of n_points
    seeded points in a ball (a shell of surface points plus interior points), oriented so that
    every tet has det[X1-X0, X2-X0, X3-X0] > 0, with slivers (volume below 1e-3 of the mean)
    removed and unreferenced vertices dropped. Returns (X, tets)."""
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    n_shell = max(4, n_points // 4)
    d = rng.standard_normal((n_shell, 3))
    shell = radius * d / np.linalg.norm(d, axis=1, keepdims=True)
    inner = rng.standard_normal((n_points - n_shell, 3))
    inner = radius * 0.95 * inner / np.linalg.norm(inner, axis=1, keepdims=True) * rng.random((inner.shape[0], 1)) ** (1 / 3)
    P = np.vstack([shell, inner])
    tets = Delaunay(P).simplices.astype(np.int64)
    D = P[tets[:, 1:]] - P[tets[:, :1]]
    det = np.einsum("ij,ij->i", D[:, 0], np.cross(D[:, 1], D[:, 2]))
    flip = det < 0
    tets[flip, 2], tets[flip, 3] = tets[flip, 3].copy(), tets[flip, 2].copy()
    vol = np.abs(det) / 6
    tets = tets[vol > 1e-3 * vol.mean()]
    used = np.unique(tets)
    remap = np.full(P.shape[0], -1, np.int64)
    remap[used] = np.arange(used.size)
    return P[used], remap[tets].astype(np.int32)


# Local cube corners (dx, dy, dz); the tets of a cube with parity 0. Corner tets list the
# corner first, then its three edge neighbours.
_EVEN = [(0, 0, 0), (1, 1, 0), (1, 0, 1), (0, 1, 1)]
_ODD = [(1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 1)]


def _neighbours(c):
    return [tuple(c[k] ^ (1 if k == axis else 0) for k in range(3)) for axis in range(3)]


def _cube_tets(parity):
    centre, corners = (_EVEN, _ODD) if parity == 0 else (_ODD, _EVEN)
    return [list(centre)] + [[c] + _neighbours(c) for c in corners]


def box_counts(nx, ny=None, nz=None):
    """(V, T, nnzb) of the five-tet box: nnzb = V + 2 * (axis edges + one diagonal per face)."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    V = (nx + 1) * (ny + 1) * (nz + 1)
    T = 5 * nx * ny * nz
    axis = nx * (ny + 1) * (nz + 1) + (nx + 1) * ny * (nz + 1) + (nx + 1) * (ny + 1) * nz
    faces = nx * ny * (nz + 1) + nx * (ny + 1) * nz + (nx + 1) * ny * nz
    return V, T, V + 2 * (axis + faces)


def make_box(nx, ny=None, nz=None, size=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)):
    """Structured box of nx*ny*nz cubes, five positively oriented tets per cube.

    Returns (X, tets): X (V, 3) float64 rest positions with vertex index
    i + (nx+1) * (j + (ny+1) * k), tets (5*nx*ny*nz, 4) int32 in cube order
    (i fastest), central tet first in each cube.
    """
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    if min(nx, ny, nz) < 1:
        raise ValueError("make_box requires at least one cube per axis")
    xs = origin[0] + size[0] * np.arange(nx + 1) / nx
    ys = origin[1] + size[1] * np.arange(ny + 1) / ny
    zs = origin[2] + size[2] * np.arange(nz + 1) / nz
    Z, Y, Xg = np.meshgrid(zs, ys, xs, indexing="ij")
    X = np.stack([Xg.ravel(), Y.ravel(), Z.ravel()], axis=1)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    parity = (i + j + k) % 2
    sx, sy = nx + 1, (nx + 1) * (ny + 1)
    tets = np.empty((i.size, 5, 4), dtype=np.int64)
    for p in (0, 1):
        sel = parity == p
        for t, tet in enumerate(_cube_tets(p)):
            for slot, (dx, dy, dz) in enumerate(tet):
                tets[sel, t, slot] = (i[sel] + dx) + sx * (j[sel] + dy) + sy * (k[sel] + dz)
    tets = tets.reshape(-1, 4)
    # Orient every tet so that det[X1-X0, X2-X0, X3-X0] > 0 (swap the last two vertices otherwise).
    D = X[tets[:, 1:]] - X[tets[:, :1]]
    det = np.einsum("ij,ij->i", D[:, 0], np.cross(D[:, 1], D[:, 2]))
    flip = det < 0
    tets[flip, 2], tets[flip, 3] = tets[flip, 3].copy(), tets[flip, 2].copy()
    return X, tets.astype(np.int32)


def make_hex_box(nx, ny=None, nz=None, size=(1.0, 1.0, 1.0)):
    """Structured box of nx*ny*nz hexes on [0, size] (HexQ1Basis corner order, cells i fastest).
    Returns (X, cells): X (V, 3) with vertex index i + (nx+1) (j + (ny+1) k), cells (T, 8) int32."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    if min(nx, ny, nz) < 1:
        raise ValueError("make_hex_box requires at least one hex per axis")
    xs, ys, zs = (size[d] * np.arange(m + 1) / m for d, m in enumerate((nx, ny, nz)))
    Z, Y, Xg = np.meshgrid(zs, ys, xs, indexing="ij")
    X = np.stack([Xg.ravel(), Y.ravel(), Z.ravel()], axis=1)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    corners = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    cells = np.stack([(i + dx) + (nx + 1) * ((j + dy) + (ny + 1) * (k + dz)) for dx, dy, dz in corners], axis=1)
    return X, cells.astype(np.int32)


def concatenate(meshes):
    """Disjoint union of meshes [(X_m, tets_m), ...]: (X, tets, vertex_offsets,
    element_offsets), each mesh a contiguous vertex and element range (the layout
    solver.batch_newton_solve takes)."""
    Xs, Ts, voff, eoff = [], [], [0], [0]
    for X, tets in meshes:
        X = np.asarray(X, dtype=np.float64).reshape(-1, 3)
        tets = np.asarray(tets, dtype=np.int64)
        Ts.append(tets + voff[-1])
        Xs.append(X)
        voff.append(voff[-1] + X.shape[0])
        eoff.append(eoff[-1] + tets.shape[0])
    return (np.concatenate(Xs), np.concatenate(Ts).astype(np.int32), np.array(voff, np.int32),
            np.array(eoff, np.int32))
