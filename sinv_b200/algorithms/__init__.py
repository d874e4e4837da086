"""Selected-inversion algorithms, mirroring ``sinv.algorithms``
(``src/sinv/algorithms/__init__.py:3-9``): ``rgf`` is the RGF module
(``rgf.rgf(...)``).  The MPI-distributed algorithms of the reference
(rgf2sided, bcr_parallel, psr, pdiv) are not part of this library."""

from . import rgf  # noqa: F401
from . import batched  # noqa: F401
from .batched import BatchPlan, rgf_batched  # noqa: F401
