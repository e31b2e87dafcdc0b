"""mydemcfd_b200 -- B200-native SMAC pressure projection (sm_100a).

divergence -> MG-PCG pressure Poisson solve -> velocity correction on the
staggered grid, with the VoF variable-density and IBM solid-mask variants,
behind the reference's pressure-solver seam.  The compute path is the native
library libsmac_b200.so (hand-written CUDA, C ABI in include/smac_b200.h).
"""
from . import _native  # noqa: F401
from ._native import (  # noqa: F401
    GMG_PCG, PRECISION_FP64, PRECISION_MIXED, PURENEUMANN_GMG_PCG, PURENEUMANN_STANDARD_PCG, STANDARD_PCG,
    STOP_REFERENCE, STOP_RELATIVE, SmacError,
)

__all__ = [
    "GMG_PCG", "PRECISION_FP64", "PRECISION_MIXED", "PURENEUMANN_GMG_PCG", "PURENEUMANN_STANDARD_PCG",
    "STANDARD_PCG", "STOP_REFERENCE", "STOP_RELATIVE", "SmacError",
]
