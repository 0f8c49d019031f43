"""litepgo_b200: the litepgo volumetric neo-Hookean hot path on NVIDIA B200 (sm_100a).

Submodules mirror the reference's Python packages for this path:
``mesh`` (TetTopology, structured boxes), ``dof`` (VertexDofMap, DofReduction, ...),
``energy`` (HessianKind, QuadraticEnergy, WeightedSumEnergy), ``fem``
(VolumetricFemEnergy[NeoHookean, TetP1Basis, TetCentroidQuadrature], force response),
``solver`` (newton_solve, StaticEquilibriumResponse) and ``torch`` (energy / response
autograd adapters). All numerics run in the CUDA library liblpg_b200.so through its C ABI
(include/litepgo_b200.h).
"""

def build_info() -> dict:
    """Versions this build was compiled against."""
    from . import _native

    return {"version": "0.1.0", "cuda": _native.build_info(), "sparse_backends": ["BlockJacobiPCG"]}


__all__ = ["build_info"]
