"""Differentiable RGF: a ``torch.autograd.Function`` with a hand-written adjoint.

The reference has no gradients; this adds dL/dA on the tridiagonal pattern
for any real loss L of the selected blocks (for example the density of
states ``-Im Tr G_ii / pi``).  The forward pass is the ordinary RGF
(``src/sinv/algorithms/rgf/rgf.py:17-64``) that also saves checkpoints of the
left-connected blocks every ceil(sqrt(n)) block rows; the backward pass runs
both sweeps in reverse on the GPU, recomputing the left-connected blocks
between checkpoints instead of storing them.

Gradients follow torch's convention (dL/dA* for complex inputs).  complex128
and float64 run natively; complex64 / float32 are computed in FP64 and the
gradients rounded back.
"""

import ctypes

import torch

from .. import _lib
from . import _device as dev


def _checkpoints(lib, n):
    every, count = ctypes.c_int(0), ctypes.c_int(0)
    _lib.check(lib.sinvb_rgf_checkpoints(n, ctypes.byref(every), ctypes.byref(count)), "sinvb_rgf_checkpoints")
    return every.value, count.value


def _wide(torch, dt):
    return {torch.complex64: torch.complex128, torch.float32: torch.float64}.get(dt, dt)


def _forward(A_diag, A_upper, A_lower, sym_mat, team):
    torch = dev._torch()
    lib = _lib.load()
    dt = _wide(torch, A_diag.dtype)
    code = _lib.dtype_code(dt)
    d = A_diag.detach().to(dt).contiguous()
    n, b = int(d.shape[0]), int(d.shape[1])
    u = A_upper.detach().to(dt).contiguous()
    l = A_lower.detach().to(dt).contiguous()
    flags = _lib.SAVE_OFFDIAG | (_lib.SYM if sym_mat else 0) | {None: 0, "cta": _lib.FORCE_CTA,
                                                               "grid": _lib.FORCE_GRID}[team]
    every, count = _checkpoints(lib, n)
    Gd = torch.empty_like(d)
    Gu = torch.empty_like(u)
    Gl = torch.empty_like(l)
    ck = torch.empty((max(count, 1), b, b), dtype=dt, device=d.device)
    ws = dev.workspace(lib.sinvb_rgf_workspace_size(n, b, code, flags), d.device)
    fn = lib.sinvb_rgf_forward_ckpt_z if code == _lib.C128 else lib.sinvb_rgf_forward_ckpt_d
    rc = fn(dev.ptr(d), dev.ptr(u), dev.ptr(l), n, b, flags, dev.ptr(Gd), dev.ptr(Gu), dev.ptr(Gl),
            ck.data_ptr(), every, dev.ptr(ws), ws.numel(), dev.stream_handle())
    _lib.check(rc, "sinvb_rgf_forward_ckpt")
    dev.raise_for_status(dev.read_status(lib, ws), "rgf (autograd forward)")
    return d, u, l, Gd, Gu, Gl, ck, every, flags


def _adjoint(d, u, l, Gd, Gu, Gl, ck, every, flags, bGd, bGu, bGl):
    torch = dev._torch()
    lib = _lib.load()
    dt = d.dtype
    code = _lib.dtype_code(dt)
    n, b = int(d.shape[0]), int(d.shape[1])

    def prep(x, like):
        return torch.zeros_like(like) if x is None else x.to(dt).contiguous()

    bGd = prep(bGd, Gd)
    bGu = prep(bGu, Gu)
    bGl = prep(bGl, Gl)
    aD = torch.empty_like(d)
    aU = torch.empty_like(u)
    aL = torch.empty_like(l)
    ws = dev.workspace(lib.sinvb_rgf_adjoint_workspace_size(n, b, code, flags), d.device)
    fn = lib.sinvb_rgf_adjoint_z if code == _lib.C128 else lib.sinvb_rgf_adjoint_d
    rc = fn(dev.ptr(d), dev.ptr(u), dev.ptr(l), dev.ptr(Gd), dev.ptr(Gu), dev.ptr(Gl), dev.ptr(bGd), dev.ptr(bGu),
            dev.ptr(bGl), ck.data_ptr(), every, n, b, flags, dev.ptr(aD), dev.ptr(aU), dev.ptr(aL), dev.ptr(ws),
            ws.numel(), dev.stream_handle())
    _lib.check(rc, "sinvb_rgf_adjoint")
    dev.raise_for_status(dev.read_status(lib, ws), "rgf (adjoint)")
    return aD, aU, aL


class RGFFunction(torch.autograd.Function):
    """``(A_diag, A_upper, A_lower) -> (G_diag, G_upper, G_lower)`` with the GPU adjoint."""

    @staticmethod
    def forward(ctx, A_diag, A_upper, A_lower, sym_mat=False, team=None):
        d, u, l, Gd, Gu, Gl, ck, every, flags = _forward(A_diag, A_upper, A_lower, sym_mat, team)
        ctx.save_for_backward(d, u, l, Gd, Gu, Gl, ck)
        ctx.every, ctx.flags = every, flags
        ctx.in_dtypes = (A_diag.dtype, A_upper.dtype, A_lower.dtype)
        out_dt = A_diag.dtype
        return Gd.to(out_dt), Gu.to(out_dt), Gl.to(out_dt)

    @staticmethod
    def backward(ctx, bGd, bGu, bGl):
        d, u, l, Gd, Gu, Gl, ck = ctx.saved_tensors
        aD, aU, aL = _adjoint(d, u, l, Gd, Gu, Gl, ck, ctx.every, ctx.flags, bGd, bGu, bGl)
        dd, du, dl = ctx.in_dtypes
        return aD.to(dd), aU.to(du), aL.to(dl), None, None


def rgf_autograd(A_diag, A_upper, A_lower, sym_mat=False, team=None):
    """Differentiable selected inversion of torch CUDA tensors.

    Returns ``(G_diag, G_upper, G_lower)`` connected to the autograd graph of
    the inputs; ``backward`` runs the GPU adjoint.
    """
    return RGFFunction.apply(A_diag, A_upper, A_lower, sym_mat, team)
