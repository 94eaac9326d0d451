"""Kernel descriptors (sumpy/kernel.py): which Green's function an FMM uses.

Only what the B200 FMM path evaluates is provided: the 3D Laplace kernel
``1/|x|`` with scaling ``1/(4 pi)`` applied on point outputs
(``LaplaceKernel``, sumpy/kernel.py:639-691). The descriptors carry no
symbolic machinery; the expansion math they select is hand-written in the
CUDA kernels.
"""
from __future__ import annotations

import math
from dataclasses import dataclass


@dataclass(frozen=True)
class LaplaceKernel:
    """``sumpy.kernel.LaplaceKernel(dim)``; G(x) = 1/|x|, scaled by 1/(4 pi)."""
    dim: int

    def __post_init__(self):
        if self.dim != 3:
            raise NotImplementedError(
                f"sumpy_b200 evaluates the 3D Laplace kernel only (got dim={self.dim})")

    is_translation_invariant = True
    is_complex_valued = False

    def get_base_kernel(self):
        return self

    @property
    def global_scaling_const(self) -> float:
        return 1.0 / (4.0 * math.pi)

    def __str__(self):
        return f"LapKnl{self.dim}D"


def is_scale_invariant(kernel) -> bool:
    """Homogeneous kernels whose scaled translation operators depend on the
    level only through a scalar factor (1/r: derivatives scale as 1/rscale)."""
    return isinstance(kernel, LaplaceKernel)
