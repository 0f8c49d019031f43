"""Host-side validation of the hex and Hermite energies' constructors, which runs before any
native call (so it needs no GPU): the map width, the rest-position shape, element-constant
fields and the plastic field, each raising ValueError as the reference's invalid_argument does."""

import numpy as np
import pytest

from conftest import ROOT  # noqa: F401  (puts the repository on sys.path)
from litepgo_b200 import dof, fem, mesh
from litepgo_b200.energy import AffineResponse

X, CELLS = mesh.make_hex_box(2, 1, 1)
TOPO = mesh.HexTopology(X.shape[0], CELLS)
THETA = np.array([2.0, 3.0])


@pytest.mark.parametrize("basis,width", [(fem.HexQ1Basis, 3), (fem.HexHermiteBasis, 24)])
def test_constructor_validation(basis, width):
    cls = fem.VolumetricFemEnergy[fem.NeoHookean, basis, fem.GaussLegendre3D[2]]
    other = 24 if width == 3 else 3
    with pytest.raises(ValueError, match="incompatible map"):
        cls(dof.VertexDofMap(TOPO, other), X, None, THETA)
    with pytest.raises(ValueError, match="rest positions"):
        cls(dof.VertexDofMap(TOPO, width), X[:-1], None, THETA)
    varying = AffineResponse(np.array([[0.0, 0, 1.0], [0, 0, 0]]), THETA)
    with pytest.raises(ValueError, match="element-constant"):
        cls(dof.VertexDofMap(TOPO, width), X, None, [varying] * 2)
    with pytest.raises(ValueError, match="plastic"):
        cls(dof.VertexDofMap(TOPO, width), X, 1.1 * np.eye(3).ravel(), THETA)
    with pytest.raises(ValueError, match="batch size"):
        cls(dof.VertexDofMap(TOPO, width), X, None, THETA, batch_size=0)
