"""Block cyclic reduction selected inversion on the GPU -- drop-in for the
reference's ``sinv.algorithms.bcr_s`` (``src/sinv/algorithms/bcr/bcr_serial.py``).

``bcr_serial(A, blocksize)`` takes the dense matrix like the reference
(``bcr_serial.py:19-62``) and returns a dense G holding the block-tridiagonal
part of the inverse (G_ii, G_{i,i+1}, G_{i+1,i}), zero elsewhere; the
reference's dense output additionally carries the intermediate blocks of its
production tree, which are not part of the selected inverse.
``bcr_blocks(A_diag, A_upper, A_lower)`` is the block-array form.

complex128 and float64 run natively; complex64 / float32 inputs are computed
in FP64 and rounded back.  Everything runs in ``libsinvb.so``.
"""

import numpy as np

from .. import _lib
from . import _device as dev


def bcr_blocks(A_diag, A_upper, A_lower, check=True, stream=None):
    """Selected inversion by BCR.  Returns ``(G_diag, G_upper, G_lower)``."""
    lib = _lib.load()
    torch = dev._torch()
    in_dt = dev.torch_dtype(A_diag)
    wide = {torch.complex64: torch.complex128, torch.float32: torch.float64}.get(in_dt, in_dt)
    code = _lib.dtype_code(wide)
    if code not in (_lib.C128, _lib.F64):
        raise TypeError("unsupported dtype %s" % in_dt)
    d = dev.to_device(A_diag, wide)
    if d.dim() != 3 or d.shape[1] != d.shape[2]:
        raise ValueError("A_diag must be (n, b, b), got %s" % (tuple(d.shape),))
    n, b = int(d.shape[0]), int(d.shape[1])
    if n > 1:
        u = dev.to_device(A_upper, wide)
        l = dev.to_device(A_lower, wide)
        for name, t in (("A_upper", u), ("A_lower", l)):
            if tuple(t.shape) != (n - 1, b, b):
                raise ValueError("%s must be (%d, %d, %d), got %s" % (name, n - 1, b, b, tuple(t.shape)))
    else:
        u = l = None
    Gd = torch.empty((n, b, b), dtype=wide, device=d.device)
    Gu = torch.empty((n - 1, b, b), dtype=wide, device=d.device)
    Gl = torch.empty((n - 1, b, b), dtype=wide, device=d.device)
    with torch.cuda.device(d.device):
        ws = dev.workspace(lib.sinvb_bcr_workspace_size(n, b, code, 0), d.device)
        fn = lib.sinvb_bcr_z if code == _lib.C128 else lib.sinvb_bcr_d
        rc = fn(dev.ptr(d), dev.ptr(u), dev.ptr(l), n, b, 0, dev.ptr(Gd), dev.ptr(Gu), dev.ptr(Gl), dev.ptr(ws),
                ws.numel(), dev.stream_handle(stream))
        _lib.check(rc, "sinvb_bcr")
        if check:
            dev.raise_for_status(dev.read_status(lib, ws, stream), "bcr_serial")
    out = tuple(g.to(in_dt) if wide != in_dt else g for g in (Gd, Gu, Gl))
    return tuple(dev.to_output(g, A_diag) for g in out)


class BcrBatchPlan:
    """Outputs, workspace and descriptors of one BCR batch, reusable across runs.

    The first ``run`` builds every matrix's schedule and uploads the merged op
    table (``sinvb_bcr_batched_*``); later runs relaunch it
    (``sinvb_bcr_batched_rerun_*``: two memsets and one launch).  Instances
    may differ in n and b and must share one dtype; complex64 / float32 inputs
    are computed in FP64 and rounded back by ``results``.
    """

    def __init__(self, instances):
        import ctypes
        self.lib = _lib.load()
        torch = dev._torch()
        if not instances:
            raise ValueError("empty batch")
        self.in_dt = dev.torch_dtype(instances[0][0])
        self.wide = {torch.complex64: torch.complex128, torch.float32: torch.float64}.get(self.in_dt, self.in_dt)
        self.code = _lib.dtype_code(self.wide)
        if self.code not in (_lib.C128, _lib.F64):
            raise TypeError("unsupported dtype %s" % self.in_dt)
        descs = (_lib.BatchDesc * len(instances))()
        self.inputs, self.outputs = [], []
        for k, (A_diag, A_upper, A_lower) in enumerate(instances):
            if dev.torch_dtype(A_diag) != self.in_dt:
                raise TypeError("instance %d: every instance must have dtype %s" % (k, self.in_dt))
            d = dev.to_device(A_diag, self.wide)
            if d.dim() != 3 or d.shape[1] != d.shape[2]:
                raise ValueError("instance %d: A_diag must be (n, b, b), got %s" % (k, tuple(d.shape)))
            n, b = int(d.shape[0]), int(d.shape[1])
            if n > 1:
                u = dev.to_device(A_upper, self.wide)
                l = dev.to_device(A_lower, self.wide)
                for name, t in (("A_upper", u), ("A_lower", l)):
                    if tuple(t.shape) != (n - 1, b, b):
                        raise ValueError("instance %d: %s must be (%d, %d, %d), got %s"
                                         % (k, name, n - 1, b, b, tuple(t.shape)))
            else:
                u = l = None
            G = tuple(torch.empty((m, b, b), dtype=self.wide, device=d.device) for m in (n, n - 1, n - 1))
            self.inputs.append((d, u, l))
            self.outputs.append(G)
            descs[k] = _lib.BatchDesc(*[t.data_ptr() if t is not None and t.numel() else None
                                        for t in (d, u, l) + G], n, b)
        self.descs = descs
        self.cdescs = ctypes.cast(descs, ctypes.c_void_p)
        self.device = self.inputs[0][0].device
        with torch.cuda.device(self.device):
            nbytes = self.lib.sinvb_bcr_batched_workspace_size(self.cdescs, len(descs), self.code, 0)
            self.ws = dev.workspace(nbytes, self.device)
            self.status_dev = torch.zeros(len(descs), dtype=torch.int32, device=self.device)
        self.uploaded = False

    def run(self, stream=None):
        """Enqueue the batch (the first run uploads the schedule, later runs only launch)."""
        torch = dev._torch()
        cz = self.code == _lib.C128
        with torch.cuda.device(self.device):
            if not self.uploaded:
                fn = self.lib.sinvb_bcr_batched_z if cz else self.lib.sinvb_bcr_batched_d
                rc = fn(self.cdescs, len(self.descs), 0, dev.ptr(self.ws), self.ws.numel(), dev.ptr(self.status_dev),
                        dev.stream_handle(stream))
                _lib.check(rc, "sinvb_bcr_batched")
                self.uploaded = True
            else:
                fn = self.lib.sinvb_bcr_batched_rerun_z if cz else self.lib.sinvb_bcr_batched_rerun_d
                rc = fn(self.cdescs, len(self.descs), dev.ptr(self.ws), dev.stream_handle(stream))
                _lib.check(rc, "sinvb_bcr_batched_rerun")

    def statuses(self):
        """Per-matrix device status (synchronises)."""
        return self.status_dev.cpu().numpy()

    def check(self):
        st = self.statuses()
        bad = np.nonzero(st)[0]
        if bad.size:
            j = int(bad[0])
            if st[j] == _lib.STATUS_PIVOT:
                raise np.linalg.LinAlgError(
                    "bcr_batched: zero or non-finite pivot in instance %d (%d instances failed)" % (j, bad.size))
            raise RuntimeError("bcr_batched: instance %d status %d" % (j, st[j]))

    def results(self, like=None):
        out = []
        for G in self.outputs:
            G = tuple(g.to(self.in_dt) if self.wide != self.in_dt else g for g in G)
            out.append(tuple(dev.to_output(g, like) for g in G) if like is not None else G)
        return out


def bcr_batched(instances, check=True, stream=None):
    """BCR selected inversion of every ``(A_diag, A_upper, A_lower)`` in ``instances``
    in one launch: phase k of every matrix's schedule runs between the same
    grid barriers.  Returns ``(G_diag, G_upper, G_lower)`` per instance in the
    input order, numpy when the inputs are numpy.  ``check`` synchronises and
    raises ``numpy.linalg.LinAlgError`` naming the first matrix with a zero or
    non-finite pivot.
    """
    if not instances:
        return []
    plan = BcrBatchPlan(instances)
    plan.run(stream)
    if check:
        plan.check()
    return plan.results(like=instances[0][0])


def _dense_to_blocks(A, b):
    """Tridiagonal blocks (diag, upper, lower) of a dense numpy or torch matrix."""
    n = A.shape[0] // b
    if dev.is_torch(A):
        blocks = A.reshape(n, b, n, b).permute(0, 2, 1, 3)
        d = blocks[range(n), range(n)].contiguous()
        u = blocks[range(n - 1), range(1, n)].contiguous() if n > 1 else None
        l = blocks[range(1, n), range(n - 1)].contiguous() if n > 1 else None
        return d, u, l
    An = np.asarray(A)
    blocks = An.reshape(n, b, n, b).transpose(0, 2, 1, 3)
    idx = np.arange(n)
    d = np.ascontiguousarray(blocks[idx, idx])
    u = np.ascontiguousarray(blocks[idx[:-1], idx[1:]]) if n > 1 else np.zeros((0, b, b), An.dtype)
    l = np.ascontiguousarray(blocks[idx[1:], idx[:-1]]) if n > 1 else np.zeros((0, b, b), An.dtype)
    return d, u, l


def _blocks_to_dense(G, like):
    """Dense matrix holding the blocks (G_diag, G_upper, G_lower), zero elsewhere,
    in the container type of ``like``."""
    Gd, Gu, Gl = G
    n, b = Gd.shape[0], Gd.shape[1]
    N = n * b
    if dev.is_torch(like):
        torch = dev._torch()
        out = torch.zeros((N, N), dtype=Gd.dtype, device=Gd.device)
        Gv = out.view(n, b, n, b).permute(0, 2, 1, 3)
        for i in range(n):
            Gv[i, i] = Gd[i]
            if i < n - 1:
                Gv[i, i + 1] = Gu[i]
                Gv[i + 1, i] = Gl[i]
        return out
    out = np.zeros((N, N), dtype=Gd.dtype)
    for i in range(n):
        out[i * b:(i + 1) * b, i * b:(i + 1) * b] = Gd[i]
        if i < n - 1:
            out[i * b:(i + 1) * b, (i + 1) * b:(i + 2) * b] = Gu[i]
            out[(i + 1) * b:(i + 2) * b, i * b:(i + 1) * b] = Gl[i]
    return out


def bcr_serial(A, blocksize, **kw):
    """Drop-in for ``bcr_serial(A, blocksize)`` (``bcr_serial.py:19-22``): dense in, dense out."""
    An = A if dev.is_torch(A) else np.asarray(A)
    N = An.shape[0]
    b = int(blocksize)
    if An.shape[0] != An.shape[1] or N % b:
        raise ValueError("A must be square with a size divisible by blocksize")
    return _blocks_to_dense(bcr_blocks(*_dense_to_blocks(An, b), **kw), An)
