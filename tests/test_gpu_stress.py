"""Large mixed-precision stress case: 128^3 cubes x 5 tets (10,485,760 tets), 0.6x axial
compression plus per-vertex noise 0.05 h N(0, 1) with every det F in [0.2, 3.0].

Per-result error of the mixed path (FP32 element arithmetic and Hessian, FP64 energy sum and
gradient output) against the FP64 path, with bounds written below; the FP64 path itself against
the oracle on the element energies of 2,000 sampled elements (1e-12 relative), since the
oracle's full assembly does not fit this size.
"""

import numpy as np
import pytest

import oracle
from litepgo_b200 import energy, fem, mesh, workloads

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def stress():
    w = workloads.compressed_box(128, seed=0)
    d = workloads.det_F(w["X"], w["tets"], w["u"])
    assert d.min() >= 0.2 and d.max() <= 3.0
    e = fem.VolumetricFemEnergyTetP1.from_arrays(w["X"], w["tets"], w["theta"])
    return w, e


def rel_max(a, b):
    return float((a - b).abs().max() / b.abs().max())


def test_stress_counts(stress):
    w, e = stress
    assert (e.num_vertices, e.num_elements, e.nnzb) == mesh.box_counts(128) == (2146689, 10485760, 27608193)


def test_stress_mixed_against_f64(stress):
    w, e = stress
    u = torch.as_tensor(w["u"], device="cuda")
    E64, g64, H64 = e.eval_device(u, gradient=True, hessian=energy.HessianKind.Exact, precision="f64")
    E32, g32, H32 = e.eval_device(u, gradient=True, hessian=energy.HessianKind.Exact, precision="mixed")
    errs = {"energy": abs(E32 - E64) / abs(E64), "gradient": rel_max(g32, g64),
            "hessian": rel_max(H32.double(), H64)}
    print("mixed vs FP64 at 128^3:", errs)
    assert errs["energy"] <= 1e-6 and errs["gradient"] <= 1e-5 and errs["hessian"] <= 1e-5


def test_stress_f64_element_energies_against_oracle(stress):
    w, e = stress
    u = torch.as_tensor(w["u"], device="cuda")
    got = e.element_energies(u).cpu().numpy()
    pick = np.sort(np.random.default_rng(0).choice(w["tets"].shape[0], 2000, replace=False))
    sub = w["tets"][pick]
    verts, local = np.unique(sub, return_inverse=True)
    orc = oracle.OracleMesh(w["X"][verts], local.reshape(-1, 4).astype(np.int32), w["theta"])
    uu = w["u"].reshape(-1, 3)[verts].ravel()
    _, _, _, (ref, _, _) = orc.eval(uu, False, 0, elements=True)
    assert np.max(np.abs(got[pick] - ref)) <= 1e-12 * np.max(np.abs(ref))
