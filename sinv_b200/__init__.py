"""sinv_b200 -- selected inversion of block-tridiagonal matrices on NVIDIA B200.

Drop-in for the serial path of Nano-TCAD/SINV: ``sinv_b200.algorithms.rgf.rgf``
replaces ``sinv.algorithms.rgf.rgf`` and ``sinv_b200.utils.matu`` replaces
``sinv.utils.matu``.  All arithmetic runs in the CUDA library
``libsinvb.so`` (C ABI in ``include/sinvb.h``).
"""

from . import algorithms, utils  # noqa: F401
from .algorithms.rgf import rgf, rgf_blocks  # noqa: F401
from .algorithms.batched import BatchPlan, rgf_batched  # noqa: F401

__all__ = ["algorithms", "utils", "rgf", "rgf_blocks", "rgf_batched", "BatchPlan"]
