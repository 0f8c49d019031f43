"""Writes tests/golden/assets.npz: the reference's own mesh assets as arrays.

The reference feeds its examples and the unstructured-mesh path from VEG files in its assets
directory (box-tet.veg: 243 vertices, 827 tets; bunny-tet.veg: 6,171 vertices, 25,746 tets;
box-hex.veg: 125 vertices, 64 hexes; read by mesh.read_veg, src/core/mesh/io/veg.cpp). This
script reads them with this library's read_veg and stores positions and cells, so the GPU tests
run on the same meshes without the reference tree:

    box_tet_X, box_tet_cells, bunny_tet_X, bunny_tet_cells, box_hex_X, box_hex_cells

Run from the repository root with the reference checked out beside it:
    python tests/golden/make_assets.py /path/to/reference/assets
"""

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from litepgo_b200 import mesh  # noqa: E402


def main(assets):
    assets = Path(assets)
    out = {}
    for name in ("box-tet", "bunny-tet", "box-hex"):
        m = mesh.read_veg(assets / f"{name}.veg")
        key = name.replace("-", "_")
        out[key + "_X"] = np.ascontiguousarray(m.positions, dtype=np.float64)
        out[key + "_cells"] = np.ascontiguousarray(m.cells, dtype=np.int32)
    np.savez_compressed(HERE / "assets.npz", **out)
    for k, v in out.items():
        print(k, v.shape)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "assets")
