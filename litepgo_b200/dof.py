"""DOF maps mirroring litepgo.dof for the volumetric FEM path.

VertexDofMap: src/core/dof/vertex_dof_map.hpp:16-72 (DOF = dofs_per_vertex * v + c).
DofReduction: src/core/dof/dof_reduction.hpp:13-53 / dof_reduction.cpp:13-78.
ConstantDofMap: src/core/dof/constant_dof_map.hpp (one shared parameter block).
ElementDofMap: src/core/dof/element_dof_map.hpp:9-47 (one block per element).
"""

import numpy as np

__all__ = ["VertexDofMap", "DofReduction", "ConstantDofMap", "ElementDofMap"]

_INT_MAX = np.iinfo(np.int32).max


class VertexDofMap:
    def __init__(self, topology, dofs_per_vertex):
        dofs_per_vertex = int(dofs_per_vertex)
        if dofs_per_vertex <= 0 or topology.num_vertices > _INT_MAX // dofs_per_vertex:
            raise ValueError("VertexDofMap requires positive width and total DOFs fitting in int")
        self._num_vertices = topology.num_vertices
        self._dpv = dofs_per_vertex
        self._cells = topology.cells.copy()

    @property
    def num_elements(self):
        return int(self._cells.shape[0])

    @property
    def num_dofs(self):
        return self._num_vertices * self._dpv

    @property
    def dofs_per_vertex(self):
        return self._dpv

    @property
    def num_vertices(self):
        return self._num_vertices

    @property
    def cells(self):
        return self._cells

    def _check(self, element):
        if element < 0 or element >= self.num_elements:
            raise IndexError("VertexDofMap: element out of range")

    def dof_indices(self, element):
        self._check(element)
        v = self._cells[element].astype(np.int64)
        return (v[:, None] * self._dpv + np.arange(self._dpv)).ravel().astype(np.int32)

    def gather(self, element, x):
        self._check(element)
        x = np.asarray(x, dtype=np.float64)
        if x.size != self.num_dofs:
            raise ValueError("VertexDofMap: incorrect global vector size")
        return x.reshape(-1, self._dpv)[self._cells[element]].copy()


class DofReduction:
    """Splits num_dofs indices into fixed and free ones; free DOFs in increasing order."""

    def __init__(self, num_dofs, fixed_dofs):
        num_dofs = int(num_dofs)
        if num_dofs < 0:
            raise ValueError("DofReduction requires a non-negative DOF count")
        fixed = np.sort(np.asarray(fixed_dofs, dtype=np.int64).ravel())
        if fixed.size and np.any(fixed[1:] == fixed[:-1]):
            raise ValueError("DofReduction fixed DOFs must be unique")
        if fixed.size and (fixed[0] < 0 or fixed[-1] >= num_dofs):
            raise ValueError("DofReduction fixed DOFs must lie in [0, num_dofs)")
        self._n = num_dofs
        self._fixed = fixed.astype(np.int32)
        mask = np.ones(num_dofs, dtype=bool)
        mask[self._fixed] = False
        self._free = np.flatnonzero(mask).astype(np.int32)
        self._free_index = np.full(num_dofs, -1, dtype=np.int32)
        self._free_index[self._free] = np.arange(self._free.size, dtype=np.int32)

    @property
    def num_dofs(self):
        return self._n

    @property
    def num_free(self):
        return int(self._free.size)

    @property
    def fixed_dofs(self):
        return self._fixed

    @property
    def free_dofs(self):
        return self._free

    def free_index(self, dof):
        if dof < 0 or dof >= self._n:
            raise IndexError(f"DofReduction::free_index: DOF {dof} is out of range")
        return int(self._free_index[dof])

    def reduce(self, full):
        full = np.asarray(full)
        if full.ndim == 1:
            if full.size != self._n:
                raise ValueError("DofReduction::reduce vector sizes must be num_dofs and num_free")
            return full[self._free].astype(np.float64)
        # A sparse matrix: principal submatrix on the free DOFs.
        import scipy.sparse as sp

        A = sp.csc_matrix(full)
        return A[self._free][:, self._free].tocsc()

    def expand(self, reduced, full):
        reduced = np.asarray(reduced, dtype=np.float64)
        if reduced.size != self.num_free or full.size != self._n:
            raise ValueError("DofReduction::expand vector sizes must be num_free and num_dofs")
        full[self._free] = reduced
        return full


class ConstantDofMap:
    def __init__(self, topology, num_dofs):
        num_dofs = int(num_dofs)
        if num_dofs <= 0:
            raise ValueError("ConstantDofMap: invalid DOF count")
        self._num_elements = topology.num_cells
        self._width = num_dofs

    @property
    def num_elements(self):
        return self._num_elements

    @property
    def num_dofs(self):
        return self._width

    def dof_indices(self, element):
        if element < 0 or element >= self._num_elements:
            raise IndexError("ConstantDofMap: element out of range")
        return np.arange(self._width, dtype=np.int32)


class ElementDofMap:
    def __init__(self, topology, dofs_per_element):
        dofs_per_element = int(dofs_per_element)
        if dofs_per_element <= 0 or topology.num_cells > _INT_MAX // dofs_per_element:
            raise ValueError("ElementDofMap: invalid DOF count")
        self._num_elements = topology.num_cells
        self._width = dofs_per_element

    @property
    def num_elements(self):
        return self._num_elements

    @property
    def num_dofs(self):
        return self._num_elements * self._width

    @property
    def dofs_per_element(self):
        return self._width

    def dof_indices(self, element):
        if element < 0 or element >= self._num_elements:
            raise IndexError("ElementDofMap: element out of range")
        return element * self._width + np.arange(self._width, dtype=np.int32)
