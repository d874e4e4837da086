"""Device plumbing shared by the algorithm modules: torch tensors as carriers
of device memory and streams, workspaces, status checks."""

import ctypes

import numpy as np

from .. import _lib


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise _lib.SinvbUnavailable("no CUDA device visible to torch")
    return torch


def is_torch(x):
    return type(x).__module__.startswith("torch")


def to_device(x, dtype=None):
    """numpy array / torch tensor -> contiguous CUDA tensor on the current device."""
    torch = _torch()
    if is_torch(x):
        t = x
    else:
        t = torch.from_numpy(np.ascontiguousarray(x))
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    if not t.is_cuda:
        t = t.to("cuda", non_blocking=False)
    return t.contiguous()


def torch_dtype(x):
    torch = _torch()
    if is_torch(x):
        return x.dtype
    return {np.dtype(np.complex128): torch.complex128, np.dtype(np.float64): torch.float64,
            np.dtype(np.complex64): torch.complex64, np.dtype(np.float32): torch.float32}.get(
        np.asarray(x).dtype) or _unsupported(np.asarray(x).dtype)


def _unsupported(dt):
    raise TypeError("unsupported dtype %s (complex128, float64, complex64, float32)" % dt)


def empty_blocks(count, b, dtype, device=None):
    torch = _torch()
    return torch.empty((count, b, b), dtype=dtype, device=device or "cuda")


def workspace(nbytes, device=None):
    """A 256-byte aligned device workspace (torch's allocator aligns to 512)."""
    torch = _torch()
    ws = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device or "cuda")
    assert ws.data_ptr() % 256 == 0
    return ws


def stream_handle(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else None


def read_status(lib, ws, stream=None):
    """Synchronise the stream and return the workspace's device status word."""
    st = ctypes.c_int(0)
    _lib.check(lib.sinvb_workspace_status(ptr(ws), stream_handle(stream), ctypes.byref(st)),
               "sinvb_workspace_status")
    return st.value


def raise_for_status(status, what):
    """Mirror the reference's failure mode: numpy.linalg.inv raises LinAlgError
    on a singular block (src/sinv/algorithms/rgf/rgf.py:44,48)."""
    if status == _lib.OK:
        return
    if status == _lib.STATUS_PIVOT:
        raise np.linalg.LinAlgError("%s: zero or non-finite pivot in a pivot-free block inversion" % what)
    raise RuntimeError("%s: device status %d (%s)" % (what, status, _lib.status_string(status)))


def to_output(t, like):
    """Return t as numpy when the caller passed numpy, else as the tensor."""
    if is_torch(like):
        return t if like.is_cuda else t.cpu()
    return t.cpu().numpy()
