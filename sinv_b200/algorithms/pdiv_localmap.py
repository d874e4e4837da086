"""PDIV (pairwise) selected inversion, mirroring ``sinv.algorithms.pdiv_lm``
(``src/sinv/algorithms/pdiv/pdiv_localmap.py``) and the partitioning of
``sinv.algorithms.pdiv_u`` (``src/sinv/algorithms/pdiv/pdiv_utils.py``).

The reference runs one partition of the block rows per MPI process (a power
of two of them): each process inverts its partition, log2(P) reduction steps
merge neighbouring groups through the bridge blocks between partitions, and
each process produces its blocks of the inverse (``pdiv_localmap.py:27-91``).
Here every partition is worked on in one schedule on one GPU
(``sinvb_pdiv_z``): the partition inverses by RGF sweep pairs (first / last
block rows and columns and the tridiagonal blocks, never the dense inverse),
the map updates and the production as batches of b x b products.

* ``pdiv_blocks(A_diag, A_upper, A_lower, partitions)``: block arrays in,
  ``(G_diag, G_upper, G_lower)`` out, the bridges included;
* ``pdiv(A, blocksize, partitions)``: dense in, dense block-tridiagonal part
  of the inverse out;
* ``pdiv_localmap_all(K_i, Bu_i, Bl_i, blocksize)``: the inputs of every
  process as ``partition_subdomain`` makes them, and the list of every
  process's ``(X_diagblk, X_upperblk, X_lowerblk)`` (what ``pdiv_localmap``
  returns on that process: m diagonal blocks, m upper / lower blocks whose
  last is the bridge to the next partition, zero on the last process);
* ``check_multiprocessing``, ``check_input``, ``divide_matrix``,
  ``partition_subdomain``: the reference's host bookkeeping
  (``pdiv_utils.py:16-171``).

Limits as in the reference (``pdiv_utils.py:16-81``): a power-of-two number
of partitions, no more than the blocks (``ValueError``); at most 64 here.
"""

import math

import numpy as np

from .. import _lib
from . import _device as dev

MAX_PARTITIONS = 64


def check_partitions(n, partitions):
    """``pdiv_utils.py:16-36, :39-81``: the process count a power of two and
    no larger than the block count."""
    P = int(partitions)
    if P < 1 or not math.log2(P).is_integer():
        raise ValueError("The number of processes must be a power of 2.")
    if n < P:
        raise ValueError("The number of blocks must be greater than the number of processes.")
    if P > MAX_PARTITIONS:
        raise ValueError("at most %d partitions" % MAX_PARTITIONS)
    return P


def check_multiprocessing(comm_size):
    """``pdiv_utils.py:16-36``."""
    if comm_size < 1 or not math.log2(comm_size).is_integer():
        raise ValueError("The number of processes must be a power of 2.")


def check_input(A, blocksize, comm_size):
    """``pdiv_utils.py:39-81``, same checks and messages in the same order."""
    if A.shape[0] % blocksize != 0:
        raise ValueError("The matrix size must be a multiple of the blocksize.")
    if blocksize > A.shape[0]:
        raise ValueError("The blocksize must be smaller than the matrix size.")
    if blocksize < 1:
        raise ValueError("The blocksize must be greater than 0.")
    if A.shape[0] // blocksize < comm_size:
        raise ValueError("The number of blocks must be greater than the number of processes.")


def divide_matrix(A, n_partitions, blocksize):
    """``pdiv_utils.py:84-123``: first block row and block count of every
    partition (n // P each, the remainder in the first)."""
    nblocks = A.shape[0] // blocksize
    base = nblocks // n_partitions
    sizes = [nblocks - base * (n_partitions - 1)] + [base] * (n_partitions - 1)
    starts = [0]
    for s in sizes[:-1]:
        starts.append(starts[-1] + s)
    return starts, sizes


def partition_subdomain(A, l_start_blockrow, l_partitions_blocksizes, blocksize):
    """``pdiv_utils.py:126-171``: the dense partitions K_i and the upper /
    lower bridge blocks between consecutive partitions."""
    K_i, Bu_i, Bl_i = [], [], []
    for i, (s, m) in enumerate(zip(l_start_blockrow, l_partitions_blocksizes)):
        a, e = s * blocksize, (s + m) * blocksize
        K_i.append(A[a:e, a:e])
        if i < len(l_start_blockrow) - 1:
            Bu_i.append(A[e - blocksize:e, e:e + blocksize])
            Bl_i.append(A[e:e + blocksize, e - blocksize:e])
    return K_i, Bu_i, Bl_i


def pdiv_blocks(A_diag, A_upper, A_lower, partitions, check=True, stream=None):
    """``(A_diag, A_upper, A_lower) -> (G_diag, G_upper, G_lower)`` by PDIV over
    ``partitions`` partitions.

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
    P = check_partitions(n, partitions)
    u = dev.to_device(A_upper, wide)
    l = dev.to_device(A_lower, wide)
    for name, t in (("A_upper", u), ("A_lower", l)):
        if tuple(t.shape) != (n - 1, b, b):
            raise ValueError("%s must be (%d, %d, %d), got %s" % (name, n - 1, b, b, tuple(t.shape)))
    Gd = torch.empty((n, b, b), dtype=wide, device=d.device)
    Gu = torch.empty((n - 1, b, b), dtype=wide, device=d.device)
    Gl = torch.empty((n - 1, b, b), dtype=wide, device=d.device)
    with torch.cuda.device(d.device):
        ws = dev.workspace(lib.sinvb_pdiv_workspace_size(n, b, P, code, 0), d.device)
        fn = lib.sinvb_pdiv_z if code == _lib.C128 else lib.sinvb_pdiv_d
        rc = fn(dev.ptr(d), dev.ptr(u), dev.ptr(l), n, b, P, 0, dev.ptr(Gd), dev.ptr(Gu), dev.ptr(Gl), dev.ptr(ws),
                ws.numel(), dev.stream_handle(stream))
        _lib.check(rc, "sinvb_pdiv")
        if check:
            dev.raise_for_status(dev.read_status(lib, ws, stream), "pdiv")
    out = tuple(g.to(in_dt) if wide != in_dt else g for g in (Gd, Gu, Gl))
    return tuple(dev.to_output(g, A_diag) for g in out)


def pdiv(A, blocksize, partitions, **kw):
    """Dense in, dense block-tridiagonal part of the inverse out (the blocks
    the reference's processes return, assembled)."""
    from .bcr_serial import _dense_to_blocks, _blocks_to_dense
    An = A if dev.is_torch(A) else np.asarray(A)
    if An.shape[0] != An.shape[1]:
        raise ValueError("A must be square")
    check_multiprocessing(int(partitions))
    check_input(An, int(blocksize), int(partitions))
    G = pdiv_blocks(*_dense_to_blocks(An, int(blocksize)), partitions=partitions, **kw)
    return _blocks_to_dense(G, An)


def pdiv_localmap_all(K_i, Bu_i, Bl_i, blocksize, **kw):
    """What ``pdiv_localmap(K_local, l_upperbridges, l_lowerbridges,
    blocksize)`` returns on each of ``len(K_i)`` processes, all computed on
    this GPU: the list of ``(X_diagblk, X_upperblk, X_lowerblk)``, each
    ``(m, b, b)``; the last upper / lower block of a process is the bridge to
    the next partition (zero on the last process)."""
    b = int(blocksize)
    P = len(K_i)
    if len(Bu_i) != P - 1 or len(Bl_i) != P - 1:
        raise ValueError("P partitions need P - 1 upper and lower bridges")
    sizes = [int(K.shape[0]) // b for K in K_i]
    d, u, l = [], [], []
    for p, K in enumerate(K_i):
        K = np.asarray(K)
        m = sizes[p]
        for i in range(m):
            d.append(K[i * b:(i + 1) * b, i * b:(i + 1) * b])
            if i < m - 1:
                u.append(K[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b])
                l.append(K[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b])
        if p < P - 1:
            u.append(np.asarray(Bu_i[p]))
            l.append(np.asarray(Bl_i[p]))
    check_partitions(sum(sizes), P)
    base = sum(sizes) // P
    if sizes[1:] != [base] * (P - 1):
        raise ValueError("partitions must be those of divide_matrix")
    dtype = np.result_type(*d)
    Gd, Gu, Gl = pdiv_blocks(np.stack(d).astype(dtype), np.stack(u).astype(dtype) if u else
                             np.zeros((0, b, b), dtype), np.stack(l).astype(dtype) if l else
                             np.zeros((0, b, b), dtype), partitions=P, **kw)
    out, s = [], 0
    for p, m in enumerate(sizes):
        Xu = np.zeros((m, b, b), Gd.dtype)
        Xl = np.zeros((m, b, b), Gd.dtype)
        e = min(s + m, Gu.shape[0])
        Xu[:e - s] = Gu[s:e]
        Xl[:e - s] = Gl[s:e]
        out.append((Gd[s:s + m], Xu, Xl))
        s += m
    return out
