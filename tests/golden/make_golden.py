"""Writes the golden fixtures of this directory from the CPU oracle.

The reference cannot be built or imported here (its Eigen / oneTBB / nanobind dependencies are
fetched at configure time), so these vectors come from the oracle, which reproduces every
known-answer test the reference holds for this path (tests/test_oracle_known_answers.py,
tests/test_oracle_mesh.py). They pin the oracle against later changes and give the GPU tests
fixed expected values:

- two_tet.npz: the reference's two-tet mesh (volumetric_fem_energy_tet_p1_gtest.cpp:26-62),
  states u in {0, 0.1 X, 0.1 X + 0.02 sin(j + 0.3)}: E, gradient, Exact and Projected CSC values;
- box3.npz: a deformed 3^3 five-tet box (seed 0): the same outputs;
- box10.npz: the 10^3 config-1 box (seed 0): E, gradient, per-element energies and the column
  product H w with w = sin(j + 0.5) and the Frobenius norm of the Exact Hessian (the full values
  would make a large file; its column sums would be round-off, translations being in its null
  space).

Run from the repository root: python tests/golden/make_golden.py
"""

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import oracle  # noqa: E402
from conftest import TWO_TET_CELLS, TWO_TET_THETA, TWO_TET_X, two_tet_states  # noqa: E402
from litepgo_b200 import workloads  # noqa: E402


def full_case(X, tets, theta, states):
    m = oracle.OracleMesh(X, tets, theta)
    outer, inner = m.pattern()
    out = dict(X=X, tets=tets, theta=theta, outer=outer, inner=inner, u=np.stack(states))
    E, g, H1, H2 = [], [], [], []
    for u in states:
        e, gr, h1 = m.eval(u, True, 1)
        _, _, h2 = m.eval(u, False, 2)
        E.append(e)
        g.append(gr)
        H1.append(h1)
        H2.append(h2)
    out.update(E=np.array(E), g=np.stack(g), H_exact=np.stack(H1), H_projected=np.stack(H2))
    return out


def main():
    np.savez_compressed(HERE / "two_tet.npz", **full_case(TWO_TET_X, TWO_TET_CELLS, TWO_TET_THETA, two_tet_states()))
    w = workloads.deformed_box(3, seed=0)
    np.savez_compressed(HERE / "box3.npz", **full_case(w["X"], w["tets"], w["theta"], [w["u"]]))
    w = workloads.deformed_box(10, seed=0)
    m = oracle.OracleMesh(w["X"], w["tets"], w["theta"])
    outer, inner = m.pattern()
    E, g, H, (eE, _, _) = m.eval(w["u"], True, 1, elements=True)
    import scipy.sparse as sp

    n = w["u"].size
    Hw = sp.csc_matrix((H, inner, outer), shape=(n, n)) @ np.sin(np.arange(n) + 0.5)
    np.savez_compressed(HERE / "box10.npz", seed=w["seed"], u=w["u"], E=E, g=g, elem_E=eE, H_w=Hw,
                        H_fro=np.sqrt(np.sum(H * H)), nnz=H.size)
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
