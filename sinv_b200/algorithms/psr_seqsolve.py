"""Parallel Schur reduction, mirroring ``sinv.algorithms.psr_s``
(``src/sinv/algorithms/psr/psr_seqsolve.py``).

The reference gives each of P MPI processes one partition of the block rows
(``psr_utils.py:61-100``), reduces the partitions in parallel, inverts the
reduced system of the 2(P-1) boundary rows on rank 0 and produces every
partition's blocks in parallel again (``psr_seqsolve.py:20-73``).  Here the P
partitions are P teams of CTAs of one launch (``sinvb_psr_z``), so one large
matrix runs chains of about n/P block steps at once.

``psr_seqsolve(A, blocksize, partitions=None)`` takes the dense matrix like the
reference and returns the dense block-tridiagonal part of the inverse; the
reference's number of processes becomes ``partitions`` (None: about
sqrt(n/2)).  ``psr_blocks`` is the block-array form.  The reference's limits
hold: at least 3 partitions and 3 block rows per partition
(``psr_utils.py:55-58``), raised as ``ValueError``.
"""

import numpy as np

from .. import _lib
from . import _device as dev


def partitions_for(n, partitions=None):
    """The number of partitions a call on n block rows uses (-1 when invalid)."""
    return int(_lib.load().sinvb_psr_partitions(int(n), int(partitions or 0)))


def psr_blocks(A_diag, A_upper, A_lower, partitions=None, check=True, stream=None):
    """``(A_diag, A_upper, A_lower) -> (G_diag, G_upper, G_lower)`` by PSR.

    complex128 and float64 run natively; complex64 / float32 are computed in
    FP64 and rounded back.  numpy inputs give numpy outputs; torch CUDA inputs
    stay on the device.  ``check`` synchronises and raises
    ``numpy.linalg.LinAlgError`` on a zero or non-finite pivot.
    """
    torch = dev._torch()
    lib = _lib.load()
    in_dt = dev.torch_dtype(A_diag)
    wide = {torch.complex64: torch.complex128, torch.float32: torch.float64}.get(in_dt, in_dt)
    code = _lib.dtype_code(wide)
    if code not in (_lib.C128, _lib.F64):
        raise TypeError("unsupported dtype %s" % in_dt)
    d = dev.to_device(A_diag, wide)
    if d.dim() != 3 or d.shape[1] != d.shape[2]:
        raise ValueError("A_diag must be (n, b, b), got %s" % (tuple(d.shape),))
    n, b = int(d.shape[0]), int(d.shape[1])
    P = partitions_for(n, partitions)
    if P < 0:
        raise ValueError("PSR needs 3 <= partitions <= 32 and at least 3 block rows per partition "
                         "(n=%d, partitions=%s)" % (n, partitions))
    u = dev.to_device(A_upper, wide)
    l = dev.to_device(A_lower, wide)
    for name, t in (("A_upper", u), ("A_lower", l)):
        if tuple(t.shape) != (n - 1, b, b):
            raise ValueError("%s must be (%d, %d, %d), got %s" % (name, n - 1, b, b, tuple(t.shape)))
    Gd = torch.empty((n, b, b), dtype=wide, device=d.device)
    Gu = torch.empty((n - 1, b, b), dtype=wide, device=d.device)
    Gl = torch.empty((n - 1, b, b), dtype=wide, device=d.device)
    with torch.cuda.device(d.device):
        ws = dev.workspace(lib.sinvb_psr_workspace_size(n, b, P, code, 0), d.device)
        fn = lib.sinvb_psr_z if code == _lib.C128 else lib.sinvb_psr_d
        rc = fn(dev.ptr(d), dev.ptr(u), dev.ptr(l), n, b, P, 0, dev.ptr(Gd), dev.ptr(Gu), dev.ptr(Gl), dev.ptr(ws),
                ws.numel(), dev.stream_handle(stream))
        _lib.check(rc, "sinvb_psr")
        if check:
            dev.raise_for_status(dev.read_status(lib, ws, stream), "psr_seqsolve")
    out = tuple(g.to(in_dt) if wide != in_dt else g for g in (Gd, Gu, Gl))
    return tuple(dev.to_output(g, A_diag) for g in out)


def psr_seqsolve(A, blocksize, partitions=None, **kw):
    """Drop-in for ``psr_seqsolve(A, blocksize)`` (``psr_seqsolve.py:20-45``):
    dense in, dense block-tridiagonal inverse out.  Unlike the reference, A is
    not overwritten."""
    from .bcr_serial import _dense_to_blocks, _blocks_to_dense
    An = A if dev.is_torch(A) else np.asarray(A)
    N = An.shape[0]
    b = int(blocksize)
    if An.shape[0] != An.shape[1] or b < 1 or N % b:   # psr_utils.py:45-50
        raise ValueError("A must be square with a size divisible by blocksize")
    G = psr_blocks(*_dense_to_blocks(An, b), partitions=partitions, **kw)
    return _blocks_to_dense(G, An)
