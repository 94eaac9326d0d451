"""sumpy_b200: sumpy's FMM evaluation path on NVIDIA B200 (sm_100a).

The expansion wrangler (:mod:`sumpy_b200.fmm`) keeps sumpy's interface;
its stages run hand-written CUDA kernels behind the C-ABI in
``include/sumpy_b200.h``. Tree and interaction lists come from
:mod:`sumpy_b200.tree` (boxtree's role); :func:`drive_fmm` runs the stages in
boxtree's order. :mod:`sumpy_b200.qbx` holds the QBX layer potentials
(``LayerPotential`` and the matrix generators).
"""
from sumpy_b200.drive import drive_fmm
from sumpy_b200.expansion import (
    LinearPDEConformingVolumeTaylorLocalExpansion,
    LinearPDEConformingVolumeTaylorMultipoleExpansion,
    LineTaylorLocalExpansion,
    VolumeTaylorLocalExpansion,
)
from sumpy_b200.fmm import SumpyExpansionWrangler, SumpyTreeIndependentDataForWrangler
from sumpy_b200.kernel import (
    AxisSourceDerivative,
    AxisTargetDerivative,
    DirectionalSourceDerivative,
    HelmholtzKernel,
    LaplaceKernel,
)
from sumpy_b200.p2p import P2P, P2PMatrixGenerator, P2PMatrixSubsetGenerator
from sumpy_b200.qbx import (
    LayerPotential,
    LayerPotentialMatrixGenerator,
    LayerPotentialMatrixSubsetGenerator,
)

__all__ = [
    "AxisSourceDerivative",
    "AxisTargetDerivative",
    "DirectionalSourceDerivative",
    "LayerPotential",
    "LayerPotentialMatrixGenerator",
    "LayerPotentialMatrixSubsetGenerator",
    "LineTaylorLocalExpansion",
    "P2P",
    "P2PMatrixGenerator",
    "P2PMatrixSubsetGenerator",
    "HelmholtzKernel",
    "LaplaceKernel",
    "LinearPDEConformingVolumeTaylorLocalExpansion",
    "LinearPDEConformingVolumeTaylorMultipoleExpansion",
    "SumpyExpansionWrangler",
    "VolumeTaylorLocalExpansion",
    "SumpyTreeIndependentDataForWrangler",
    "drive_fmm",
]
