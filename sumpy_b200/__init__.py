"""sumpy_b200: sumpy's FMM evaluation path on NVIDIA B200 (sm_100a).

The expansion wrangler (:mod:`sumpy_b200.fmm`) keeps sumpy's interface;
its stages run hand-written CUDA kernels behind the C-ABI in
``include/sumpy_b200.h``. Tree and interaction lists come from
:mod:`sumpy_b200.tree` (boxtree's role); :func:`drive_fmm` runs the stages in
boxtree's order.
"""
from sumpy_b200.drive import drive_fmm
from sumpy_b200.expansion import (
    LinearPDEConformingVolumeTaylorLocalExpansion,
    LinearPDEConformingVolumeTaylorMultipoleExpansion,
)
from sumpy_b200.fmm import SumpyExpansionWrangler, SumpyTreeIndependentDataForWrangler
from sumpy_b200.kernel import HelmholtzKernel, LaplaceKernel
from sumpy_b200.p2p import P2P, P2PMatrixGenerator, P2PMatrixSubsetGenerator

__all__ = [
    "P2P",
    "P2PMatrixGenerator",
    "P2PMatrixSubsetGenerator",
    "HelmholtzKernel",
    "LaplaceKernel",
    "LinearPDEConformingVolumeTaylorLocalExpansion",
    "LinearPDEConformingVolumeTaylorMultipoleExpansion",
    "SumpyExpansionWrangler",
    "SumpyTreeIndependentDataForWrangler",
    "drive_fmm",
]
