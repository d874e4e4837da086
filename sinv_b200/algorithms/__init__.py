"""Selected-inversion algorithms, mirroring ``sinv.algorithms``
(``src/sinv/algorithms/__init__.py:3-9``): ``rgf`` is the RGF module
(``rgf.rgf(...)``) and ``bcr_s`` the BCR module (``bcr_s.bcr_serial(...)``).  ``rgf2s`` is the two-sided RGF
(``rgf2s.rgf2sided(...)``), both halves on one GPU; ``bcr_batched`` runs BCR over
a batch of matrices in one launch.  ``psr_s`` is the parallel Schur reduction
(``psr_s.psr_seqsolve(...)``), its partitions as teams of one launch;
``pdiv_lm`` the PDIV / pairwise algorithm (``pdiv_lm.pdiv(...)``,
``pdiv_lm.pdiv_localmap_all(...)``), all partitions in one schedule on one
GPU, with the partitioning helpers also reachable as ``pdiv_u``.  The
MPI-distributed bcr_parallel of the reference is not part of this library."""

from . import rgf  # noqa: F401
from . import rgf2sided as rgf2s  # noqa: F401
from . import bcr_serial  # noqa: F401
from . import bcr_serial as bcr_s  # noqa: F401
from .bcr_serial import BcrBatchPlan, bcr_batched  # noqa: F401
from . import psr_seqsolve  # noqa: F401
from . import psr_seqsolve as psr_s  # noqa: F401
from . import pdiv_localmap  # noqa: F401
from . import pdiv_localmap as pdiv_lm  # noqa: F401
from . import pdiv_localmap as pdiv_u  # noqa: F401
from . import batched  # noqa: F401
from .batched import BatchPlan, rgf_batched, rgf_batched_host  # noqa: F401
from . import adjoint  # noqa: F401
from .adjoint import RGFBatchFunction, RGFFunction, rgf_autograd, rgf_batched_autograd  # noqa: F401
from . import lesser  # noqa: F401
from .lesser import rgf_greater, rgf_greater_batched, rgf_lesser, rgf_lesser_batched  # noqa: F401
