"""Serial RGF selected inversion on the GPU -- drop-in for the reference's
``sinv.algorithms.rgf`` (``src/sinv/algorithms/rgf/rgf.py:17-64``).

``rgf(A, sym_mat=False, save_off_diag=True)`` accepts either

* the reference's block-sparse container (any object with ``.blockorder``,
  ``.blocks[i, j]``, ``.copy()`` and scalar ``*``, like ``quasi.bsparse``):
  the result is the same kind of container, off-selection blocks NaN exactly
  as ``rgf.py:41`` leaves them; or
* the three block arrays ``(A_diag[n,b,b], A_upper[n-1,b,b], A_lower[n-1,b,b])``
  of ``src/sinv/utils/matrices_utils.py:115-151`` (the signature of
  ``src/sinv/algorithms/rgf/rgf2sided.py:18-24``): the result is
  ``(G_diag, G_upper, G_lower)``.

Arrays may be numpy (results come back as numpy) or torch tensors (results
stay on the tensor's device).  The dtype follows the input (complex128,
float64, complex64, float32; single precision is computed in FP64 and rounded
on output).  Everything runs in ``libsinvb.so``; there is no CPU path.
"""

import numpy as np

from .. import _lib
from . import _device as dev


def _is_container(A):
    return hasattr(A, "blockorder") and hasattr(A, "blocks")


def rgf_blocks(A_diag, A_upper, A_lower, sym_mat=False, save_off_diag=True, check=True, stream=None,
               team=None, overwrite_a=False):
    """Block-array selected inversion.  Returns ``(G_diag, G_upper, G_lower)``.

    ``check`` synchronises and raises ``numpy.linalg.LinAlgError`` on a zero or
    non-finite pivot (the reference's ``np.linalg.inv`` failure mode).
    ``team`` forces the execution team: ``"cta"`` (one CTA walks the sweep) or
    ``"grid"`` (the whole GPU); by default the library picks from the block size.
    ``overwrite_a`` (torch CUDA complex128/float64 inputs, ``save_off_diag``)
    writes the results over the input tensors and returns them.
    """
    lib = _lib.load()
    tdt = dev.torch_dtype(A_diag)
    code = _lib.dtype_code(tdt)
    d = dev.to_device(A_diag, tdt)
    if d.dim() != 3 or d.shape[1] != d.shape[2]:
        raise ValueError("A_diag must be (n, b, b), got %s" % (tuple(d.shape),))
    n, b = int(d.shape[0]), int(d.shape[1])
    if n < 1 or b < 1:
        raise ValueError("empty matrix")
    torch = dev._torch()
    if n > 1:
        u = dev.to_device(A_upper, tdt)
        l = dev.to_device(A_lower, tdt)
        for name, t in (("A_upper", u), ("A_lower", l)):
            if tuple(t.shape) != (n - 1, b, b):
                raise ValueError("%s must be (%d, %d, %d), got %s" % (name, n - 1, b, b, tuple(t.shape)))
    else:
        u = l = None
    flags = (_lib.SYM if sym_mat else 0) | (_lib.SAVE_OFFDIAG if save_off_diag else 0)
    if team == "grid":
        flags |= _lib.FORCE_GRID
    elif team == "cta":
        flags |= _lib.FORCE_CTA
    elif team is not None:
        raise ValueError("team must be None, 'cta' or 'grid'")
    if overwrite_a:
        if not (dev.is_torch(A_diag) and A_diag.is_cuda and d.data_ptr() == A_diag.data_ptr()
                and (n == 1 or (u.data_ptr() == A_upper.data_ptr() and l.data_ptr() == A_lower.data_ptr()))):
            raise TypeError("overwrite_a takes contiguous torch CUDA tensors")
        if not save_off_diag or code not in (_lib.C128, _lib.F64):
            raise ValueError("overwrite_a needs save_off_diag=True and complex128 / float64")
        flags |= _lib.INPLACE
        Gd = d
        Gu = u if u is not None else d[:0]
        Gl = l if l is not None else d[:0]
    else:
        Gd = torch.empty((n, b, b), dtype=tdt, device=d.device)
        Gu = torch.empty((n - 1, b, b), dtype=tdt, device=d.device)
        Gl = torch.empty((n - 1, b, b), dtype=tdt, device=d.device)
    with torch.cuda.device(d.device):
        ws = dev.workspace(lib.sinvb_rgf_workspace_size(n, b, code, flags), d.device)
        fn = {_lib.C128: lib.sinvb_rgf_z, _lib.F64: lib.sinvb_rgf_d, _lib.C64: lib.sinvb_rgf_c,
              _lib.F32: lib.sinvb_rgf_s}[code]
        rc = fn(dev.ptr(d), dev.ptr(u), dev.ptr(l), n, b, flags, dev.ptr(Gd),
                dev.ptr(Gu) if save_off_diag else None, dev.ptr(Gl) if save_off_diag else None,
                dev.ptr(ws), ws.numel(), dev.stream_handle(stream))
        _lib.check(rc, "sinvb_rgf")
        if not save_off_diag:
            Gu.fill_(float("nan"))
            Gl.fill_(float("nan"))
        if check:
            dev.raise_for_status(dev.read_status(lib, ws, stream), "rgf")
    return dev.to_output(Gd, A_diag), dev.to_output(Gu, A_diag), dev.to_output(Gl, A_diag)


def rgf(A, *args, sym_mat=False, save_off_diag=True, **kw):
    """Drop-in for ``rgf(A, sym_mat=False, save_off_diag=True)`` (``rgf.py:17-21``).

    ``rgf(container[, sym_mat[, save_off_diag]])`` or
    ``rgf(A_diag, A_upper, A_lower[, sym_mat[, save_off_diag]])``.
    """
    if _is_container(A):
        if len(args) > 0:
            sym_mat = args[0]
        if len(args) > 1:
            save_off_diag = args[1]
        return _rgf_container(A, sym_mat, save_off_diag, **kw)
    if len(args) < 2:
        raise TypeError("rgf() takes a block-sparse container or (A_diag, A_upper, A_lower)")
    A_upper, A_lower = args[0], args[1]
    if len(args) > 2:
        sym_mat = args[2]
    if len(args) > 3:
        save_off_diag = args[3]
    return rgf_blocks(A, A_upper, A_lower, sym_mat, save_off_diag, **kw)


def _rgf_container(A, sym_mat, save_off_diag, **kw):
    n = A.blockorder
    d = np.stack([np.asarray(A.blocks[i, i]) for i in range(n)])
    b = d.shape[1]
    if n > 1:
        u = np.stack([np.asarray(A.blocks[i, i + 1]) for i in range(n - 1)])
        l = np.stack([np.asarray(A.blocks[i + 1, i]) for i in range(n - 1)])
    else:
        u = l = np.zeros((0, b, b), d.dtype)
    Gd, Gu, Gl = rgf_blocks(d, u, l, sym_mat, save_off_diag, **kw)
    G = A.copy() * np.nan                                   # rgf.py:41
    for i in range(n):
        G.blocks[i, i] = Gd[i]
    if save_off_diag:
        for i in range(n - 1):
            G.blocks[i + 1, i] = Gl[i]
            G.blocks[i, i + 1] = Gu[i]
    return G
