"""quantkernel_b200 -- B200-native batch Monte Carlo option pricing.

Python mirror of the Monte Carlo part of yluoc/Quant-Kernel's ``quantkernel``
package, backed by hand-written sm_100a CUDA kernels in libqk_b200.so.
"""

from ._abi import *  # noqa: F401,F403
from ._abi import ABI_MAJOR, ABI_MINOR, QK_CALL, QK_PUT
from .accelerator import QuantAccelerator
from .engine import (
    McPlan,
    QKBadSizeError,
    QKError,
    QKInvalidInputError,
    QKNullPointerError,
    QKRuntimeError,
    QuantKernel,
)

__all__ = [
    "ABI_MAJOR",
    "ABI_MINOR",
    "QK_CALL",
    "QK_PUT",
    "McPlan",
    "QuantAccelerator",
    "QKBadSizeError",
    "QKError",
    "QKInvalidInputError",
    "QKNullPointerError",
    "QKRuntimeError",
    "QuantKernel",
]
