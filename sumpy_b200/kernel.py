"""Kernel descriptors (sumpy/kernel.py): which Green's function an FMM uses.

Only what the B200 FMM path evaluates is provided: the 3D Laplace kernel
``1/|x|`` (``LaplaceKernel``, sumpy/kernel.py:639-691) and the 3D Helmholtz
kernel ``exp(i k |x|)/|x|`` (``HelmholtzKernel``, sumpy/kernel.py:755-844),
both with scaling ``1/(4 pi)`` applied on point outputs. The descriptors
carry no symbolic machinery; the expansion math they select is hand-written
in the CUDA kernels. As in sumpy, the Helmholtz wave number is not part of
the kernel object: it is passed by name (``helmholtz_k_name``, default
``"k"``) in ``kernel_extra_kwargs`` / P2P keyword arguments.
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


@dataclass(frozen=True)
class HelmholtzKernel:
    """``sumpy.kernel.HelmholtzKernel(dim)``; G(x) = exp(i k |x|)/|x|,
    scaled by 1/(4 pi); complex valued; k real (no evanescent waves)."""
    dim: int
    helmholtz_k_name: str = "k"
    allow_evanescent: bool = False

    def __post_init__(self):
        if self.dim != 3:
            raise NotImplementedError(
                f"sumpy_b200 evaluates the 3D Helmholtz kernel only (got dim={self.dim})")
        if self.allow_evanescent:
            raise NotImplementedError("complex wave numbers are not supported")

    is_translation_invariant = True
    is_complex_valued = True

    def get_base_kernel(self):
        return self

    @property
    def global_scaling_const(self) -> float:
        return 1.0 / (4.0 * math.pi)

    def __str__(self):
        return f"HelmKnl{self.dim}D({self.helmholtz_k_name})"


def helmholtz_k(kernel, extra_kwargs) -> float:
    """The wave number of a Helmholtz kernel from the keyword arguments."""
    name = kernel.helmholtz_k_name
    if name not in extra_kwargs:
        raise TypeError(f"the Helmholtz kernel needs the wave number '{name}' "
                        "in kernel_extra_kwargs")
    k = complex(extra_kwargs[name])
    if k.imag != 0:
        raise NotImplementedError("complex wave numbers are not supported")
    return float(k.real)


def is_scale_invariant(kernel) -> bool:
    """Homogeneous kernels whose scaled translation operators depend on the
    level only through a scalar factor (1/r: derivatives scale as 1/rscale)."""
    return isinstance(kernel, LaplaceKernel)


# {{{ derivative wrappers (sumpy/kernel.py:2289-2386, directional source derivative)

@dataclass(frozen=True)
class AxisTargetDerivative:
    """``sumpy.kernel.AxisTargetDerivative(axis, inner_kernel)``: d/dt_axis."""
    axis: int
    inner_kernel: object

    def __post_init__(self):
        if self.axis not in (0, 1, 2):
            raise ValueError(f"axis must be 0, 1 or 2, got {self.axis}")

    def get_base_kernel(self):
        return self.inner_kernel.get_base_kernel()

    @property
    def global_scaling_const(self):
        return self.get_base_kernel().global_scaling_const

    @property
    def is_complex_valued(self):
        return self.get_base_kernel().is_complex_valued

    def __str__(self):
        return f"d/dx{self.axis} {self.inner_kernel}"


@dataclass(frozen=True)
class AxisSourceDerivative:
    """``sumpy.kernel.AxisSourceDerivative(axis, inner_kernel)``: d/ds_axis."""
    axis: int
    inner_kernel: object

    def __post_init__(self):
        if self.axis not in (0, 1, 2):
            raise ValueError(f"axis must be 0, 1 or 2, got {self.axis}")

    def get_base_kernel(self):
        return self.inner_kernel.get_base_kernel()

    @property
    def global_scaling_const(self):
        return self.get_base_kernel().global_scaling_const

    @property
    def is_complex_valued(self):
        return self.get_base_kernel().is_complex_valued

    def __str__(self):
        return f"d/dy{self.axis} {self.inner_kernel}"


@dataclass(frozen=True)
class DirectionalSourceDerivative:
    """``sumpy.kernel.DirectionalSourceDerivative(inner_kernel,
    dir_vec_name)``: n(s) . grad_s, with the per-source direction vectors
    passed by name (default ``"src_derivative_dir"``, shape (3, nsources));
    the double-layer kernel."""
    inner_kernel: object
    dir_vec_name: str = "src_derivative_dir"

    def get_base_kernel(self):
        return self.inner_kernel.get_base_kernel()

    @property
    def global_scaling_const(self):
        return self.get_base_kernel().global_scaling_const

    @property
    def is_complex_valued(self):
        return self.get_base_kernel().is_complex_valued

    def __str__(self):
        return f"{self.dir_vec_name} . grad_src {self.inner_kernel}"

# }}}
