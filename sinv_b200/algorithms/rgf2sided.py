"""Two-sided RGF, mirroring ``sinv.algorithms.rgf2s`` (``src/sinv/algorithms/rgf/rgf2sided.py``).

The reference splits the block chain over two MPI processes that sweep from
both ends towards the middle (``rgf2sided.py:18-274``).  Here both halves run
on one GPU as two teams of CTAs of one launch (``sinvb_rgf2s_z``), so a single
large matrix has a dependency chain of about n/2 block steps instead of n.
Results are those of ``rgf`` (same arrays, same NaN convention when
``save_off_diag=False``).
"""

from .. import _lib
from . import _device as dev


def rgf2sided(A_bloc_diag, A_bloc_upper, A_bloc_lower, sym_mat=False, save_off_diag=True, check=True,
              stream=None):
    """``(A_diag, A_upper, A_lower) -> (G_diag, G_upper, G_lower)`` (``rgf2sided.py:18-24``).

    numpy or torch inputs, complex128 or float64; numpy inputs give numpy
    outputs.  ``check`` synchronises and raises ``numpy.linalg.LinAlgError`` on
    a zero or non-finite pivot.
    """
    torch = dev._torch()
    lib = _lib.load()
    tdt = dev.torch_dtype(A_bloc_diag)
    code = _lib.dtype_code(tdt)
    if code not in (_lib.C128, _lib.F64):
        raise TypeError("rgf2sided takes complex128 or float64 blocks")
    d = dev.to_device(A_bloc_diag, tdt)
    if d.dim() != 3 or d.shape[1] != d.shape[2]:
        raise ValueError("A_bloc_diag must be (n, b, b), got %s" % (tuple(d.shape),))
    n, b = int(d.shape[0]), int(d.shape[1])
    if n > 1:
        u = dev.to_device(A_bloc_upper, tdt)
        l = dev.to_device(A_bloc_lower, tdt)
        for name, t in (("A_bloc_upper", u), ("A_bloc_lower", l)):
            if tuple(t.shape) != (n - 1, b, b):
                raise ValueError("%s must be (%d, %d, %d), got %s" % (name, n - 1, b, b, tuple(t.shape)))
    else:
        u = l = None
    # the halves keep their intermediate blocks in the off-diagonal outputs
    flags = (_lib.SYM if sym_mat else 0) | _lib.SAVE_OFFDIAG
    Gd = torch.empty((n, b, b), dtype=tdt, device=d.device)
    Gu = torch.empty((n - 1, b, b), dtype=tdt, device=d.device)
    Gl = torch.empty((n - 1, b, b), dtype=tdt, device=d.device)
    with torch.cuda.device(d.device):
        ws = dev.workspace(lib.sinvb_rgf2s_workspace_size(n, b, code, flags), d.device)
        fn = lib.sinvb_rgf2s_z if code == _lib.C128 else lib.sinvb_rgf2s_d
        rc = fn(dev.ptr(d), dev.ptr(u), dev.ptr(l), n, b, flags, dev.ptr(Gd), dev.ptr(Gu), dev.ptr(Gl),
                dev.ptr(ws), ws.numel(), dev.stream_handle(stream))
        _lib.check(rc, "sinvb_rgf2s")
        if not save_off_diag:
            Gu.fill_(float("nan"))
            Gl.fill_(float("nan"))
        if check:
            dev.raise_for_status(dev.read_status(lib, ws, stream), "rgf2sided")
    return dev.to_output(Gd, A_bloc_diag), dev.to_output(Gu, A_bloc_diag), dev.to_output(Gl, A_bloc_diag)
