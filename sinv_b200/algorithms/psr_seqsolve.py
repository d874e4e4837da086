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

For one partition per GPU (the reference's one partition per process),
``PsrPart`` runs a partition on this GPU holding only its rows
(``local_blocks``), ``reduced_system`` / ``boundary_inverse`` do the host
bookkeeping of the exchange, and ``sinv_b200.distributed.psr_distributed``
drives them across ranks with one all-gather.
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


# --------------------------------------------------------------------------- one partition per GPU
def part_rows(n, P, part):
    """(first row t, last row B) of partition ``part`` (``psr_utils.py:61-100``)."""
    base = n // P
    s = 0 if part == 0 else n - base * (P - part)
    m = n - base * (P - 1) if part == 0 else base
    return s, s + m - 1


def reduced_rows(n, P):
    """Block rows of the reduced system: [B_0, t_1, B_1, ..., t_{P-1}]
    (``psr_seqsolve.py:336-384``)."""
    rows = [part_rows(n, P, 0)[1]]
    for p in range(1, P - 1):
        rows += list(part_rows(n, P, p))
    rows.append(part_rows(n, P, P - 1)[0])
    return rows


def local_blocks(A_diag, A_upper, A_lower, partitions, part):
    """The block arrays partition ``part`` holds: diag rows t..B and the
    couplings of rows t..B (one fewer for the last partition)."""
    n = A_diag.shape[0]
    t, B = part_rows(n, partitions, part)
    e = min(B + 1, n - 1)
    return A_diag[t:B + 1], A_upper[t:e], A_lower[t:e]


def reduced_system(boundaries, n, P):
    """The block tridiagonal reduced system from every partition's six boundary
    slots (in partition order): slots 0-3 its part of the reduced system, slots
    4-5 its couplings to the next partition.  Returns ``(R_diag, R_upper,
    R_lower)`` (host bookkeeping on tensors of any device)."""
    import torch
    diag = [boundaries[0][0]]
    for p in range(1, P - 1):
        diag += [boundaries[p][0], boundaries[p][1]]
    diag.append(boundaries[P - 1][0])
    upper, lower = [], []
    for x in range(2 * (P - 1) - 1):
        p = (x + 1) // 2
        if x % 2 == 0:  # B_p -> t_{p+1}: the input coupling sent by partition p
            upper.append(boundaries[x // 2][4])
            lower.append(boundaries[x // 2][5])
        else:           # t_p -> B_p of a central partition: its fill-in
            upper.append(boundaries[p][2])
            lower.append(boundaries[p][3])
    return torch.stack(diag), torch.stack(upper), torch.stack(lower)


def boundary_inverse(RG, part, P):
    """The four boundary slots partition ``part`` needs from the reduced
    system's inverse ``RG = (G_diag, G_upper, G_lower)``, and its coupling to
    the next partition ``(G[B,B+1], G[B+1,B])`` (None for the last)."""
    import torch
    Rd, Ru, Rl = RG
    zero = torch.zeros_like(Rd[0])
    if part == 0:
        slots = [Rd[0], zero, zero, zero]
    elif part == P - 1:
        slots = [Rd[-1], zero, zero, zero]
    else:
        x = 2 * part - 1
        slots = [Rd[x], Rd[x + 1], Ru[x], Rl[x]]
    link = (Ru[2 * part], Rl[2 * part]) if part < P - 1 else None
    return torch.stack(slots), link


class PsrPart:
    """Partition ``part`` of a ``partitions``-way PSR of an n-block matrix on
    this GPU (``sinvb_psr_part_*``), holding only the partition's rows
    (``local_blocks``).  ``reduce()`` returns the six boundary slots,
    ``produce(slots, link)`` returns the partition's ``(G_diag, G_upper,
    G_lower)`` with the shapes of its local arrays (the last element of
    G_upper / G_lower is the coupling to the next partition)."""

    def __init__(self, local_diag, local_upper, local_lower, n, partitions, part, device=None):
        torch = dev._torch()
        self.lib = _lib.load()
        self.in_dt = dev.torch_dtype(local_diag)
        self.wide = {torch.complex64: torch.complex128, torch.float32: torch.float64}.get(self.in_dt, self.in_dt)
        self.code = _lib.dtype_code(self.wide)
        if self.code not in (_lib.C128, _lib.F64):
            raise TypeError("unsupported dtype %s" % self.in_dt)
        self.n = int(n)
        self.P = partitions_for(self.n, partitions)
        if self.P < 0 or not 0 <= part < self.P:
            raise ValueError("PSR needs 3 <= partitions <= 32, 3 block rows per partition and 0 <= part < "
                             "partitions (n=%d, partitions=%s, part=%d)" % (self.n, partitions, part))
        self.part = part
        self.rows = part_rows(self.n, self.P, part)
        m = self.rows[1] - self.rows[0] + 1
        mc = m if part < self.P - 1 else m - 1
        with torch.cuda.device(device if device is not None else torch.cuda.current_device()):
            self.d = dev.to_device(local_diag, self.wide)
            self.u = dev.to_device(local_upper, self.wide)
            self.l = dev.to_device(local_lower, self.wide)
        self.b = int(self.d.shape[-1])
        b = self.b
        for name, t, k in (("diag", self.d, m), ("upper", self.u, mc), ("lower", self.l, mc)):
            if tuple(t.shape) != (k, b, b):
                raise ValueError("partition %d: local %s must be (%d, %d, %d), got %s"
                                 % (part, name, k, b, b, tuple(t.shape)))
        self.device = self.d.device
        self.G = tuple(torch.zeros((k, b, b), dtype=self.wide, device=self.device) for k in (m, mc, mc))
        self.slots = torch.zeros((6, b, b), dtype=self.wide, device=self.device)
        with torch.cuda.device(self.device):
            nbytes = self.lib.sinvb_psr_part_workspace_size(self.n, b, self.P, part, self.code)
            self.ws = dev.workspace(nbytes, self.device)

    def _stage(self, stage, stream=None):
        torch = dev._torch()
        fn = self.lib.sinvb_psr_part_z if self.code == _lib.C128 else self.lib.sinvb_psr_part_d
        with torch.cuda.device(self.device):
            rc = fn(dev.ptr(self.d), dev.ptr(self.u), dev.ptr(self.l), self.n, self.b, self.P, self.part, stage,
                    dev.ptr(self.slots), dev.ptr(self.G[0]), dev.ptr(self.G[1]), dev.ptr(self.G[2]),
                    dev.ptr(self.ws), self.ws.numel(), dev.stream_handle(stream))
            _lib.check(rc, "sinvb_psr_part")

    def reduce(self, stream=None):
        self._stage(0, stream)
        return self.slots

    def produce(self, slots, link=None, stream=None, check=True):
        self.slots[:4].copy_(slots[:4])
        self._stage(1, stream)
        if link is not None:
            self.G[1][-1].copy_(link[0])
            self.G[2][-1].copy_(link[1])
        if check:
            dev.raise_for_status(dev.read_status(self.lib, self.ws, stream), "psr part %d" % self.part)
        return self.G

    def solve_reduced(self, Rd, Ru, Rl):
        """Selected inverse of the reduced system (every rank solves it)."""
        from .rgf import rgf_blocks
        return rgf_blocks(Rd, Ru, Rl)
